"""The render decode kernel's two leaf paths, against the oracle bit for bit.

decode_leaf_kernel takes GRID4 and FINE6 leaves of the common shape (coarse resolution 4, fine 6,
FP16 keys that strictly increase and hold no NaN) through its specialised path whenever the
frames of a launch step by 0 or 1, and every other leaf, or any other frame list, through the
general path.  Here every launch shape the specialised path distinguishes -- 1 to 128 frames (one
or several frame batches, GRID4 frame parts of unequal length), repeated frames at the clamped
ends, boundary leaves with cropped extents, cache and dense outputs -- is checked against the
oracle on every frame, and frame lists that step back or skip (the general path) likewise.
"""
import os

import numpy as np
import pytest

from conftest import ASSETS, golden_asset

pytestmark = pytest.mark.gpu

FLAG_FINE, FLAG_SHELL, FLAG_OCC, FLAG_SORTED, FLAG_HALF = 1 << 11, 1 << 12, 1 << 13, 1 << 14, 1 << 15


def paths():
    out = [golden_asset(n) for n in ("tiny_density", "tiny_levelset")]
    for n in ("cfg1_blobs", "cfg4_sdf_small", "cfg2_plume", "mix_fire_temperature"):
        p = os.path.join(ASSETS, n + ".vbtp")
        if os.path.exists(p):
            out.append(p)
    return out


def fast_leaves(rows):
    """Active leaves the specialised path takes on a timeline (the kernel's fast_leaf_shape), and
    the active FINE6 leaves."""
    hdr, info = rows[:, 1], rows[:, 7]
    active = (info & (1 << 10)) != 0
    need = (info & (FLAG_SORTED | FLAG_HALF)) == (FLAG_SORTED | FLAG_HALF)
    no_shell = (info & (FLAG_OCC | FLAG_SHELL)) == 0
    coarse = (((hdr >> 6) & 7) == 4) & (((hdr >> 2) & 3) != 1)
    fine = (info & FLAG_FINE) != 0
    fine_ok = ~fine | ((((hdr >> 9) & 7) == 6) & (((hdr >> 4) & 3) != 1))
    return active & need & no_shell & coarse & fine_ok, active & fine


@pytest.fixture(scope="module")
def loaded(vbt, oracle):
    cache = {}

    def get(path):
        if path not in cache:
            cache[path] = (vbt.Asset(path), oracle.load(path))
        return cache[path]

    yield get
    for a, _ in cache.values():
        a.close()


def check_cache(cuda, a, f, frame_lists, what):
    n = max(a.active_count, 1)
    for frames in frame_lists:
        out = cuda.full((len(frames), n, 512), float("nan"), dtype=cuda.float32, device="cuda")
        a.decode_cache(frames, out)
        a.sync_status()
        got = out.cpu().numpy()
        for i, t in enumerate(frames):
            want = f.cache(t, threads=8)
            bad = np.flatnonzero(got[i, :a.active_count].reshape(-1).view(np.uint32) != want.reshape(-1).view(np.uint32))
            assert bad.size == 0, (what, len(frames), frames[0], t, bad[:8])


@pytest.mark.parametrize("path", paths(), ids=os.path.basename)
def test_timeline_launch_shapes(loaded, cuda, path):
    a, f = loaded(path)
    a.build_page_table()
    T = f.frames
    big = "cfg2" in path or "mix_fire" in path
    counts = [5, 48, 64, 96, 128] if big else [1, 2, 3, 4, 5, 9, 13, 17, 48, 64, 96, 128]
    lists = []
    for k in counts:
        for start in ([-1] if big else [-1, T // 3]):
            frames = list(range(start, min(start + k, T + 2)))
            if frames:
                lists.append(frames)
    lists.append([2, 2, 2, 3, 3, 4, 5, 5])                       # steps of 0 inside a timeline
    lists.append(list(range(T - 3, T + 4)))                      # clamped at the end
    check_cache(cuda, a, f, lists, os.path.basename(path))


@pytest.mark.parametrize("path", paths(), ids=os.path.basename)
def test_general_path_frame_lists(loaded, cuda, path):
    a, f = loaded(path)
    a.build_page_table()
    T = f.frames
    lists = [[T - 1, 0, T // 2], [0, 2, 4, 6], [T // 2, T // 2 - 1]]
    check_cache(cuda, a, f, lists, os.path.basename(path))


@pytest.mark.parametrize("path", [p for p in paths() if "cfg2" not in p and "mix_fire" not in p],
                         ids=os.path.basename)
def test_dense_timeline(loaded, cuda, path):
    a, f = loaded(path)
    X, Y, Z = f.dims
    frames = list(range(-1, f.frames + 1))
    out = cuda.empty((len(frames), Z, Y, X), dtype=cuda.float32, device="cuda")
    a.decode_frames(frames[:40], out[:min(40, len(frames))])
    if len(frames) > 40:
        a.decode_frames(frames[40:], out[40:])
    a.sync_status()
    got = out.cpu().numpy()
    for i, t in enumerate(frames):
        assert np.array_equal(got[i].view(np.uint32), f.frame(t, threads=8).view(np.uint32)), (path, t)


def test_bench_asset_takes_the_specialised_path(vbt):
    """Every active leaf of the benchmark plume (GRID4 and FINE6) is of the specialised shape, so
    the headline kernel time is that path's."""
    p = os.path.join(ASSETS, "cfg2_plume.vbtp")
    if not os.path.exists(p):
        pytest.skip("cfg2_plume not generated")
    a = vbt.Asset(p)
    rows = a.leaf_table()
    a.close()
    fast, fine = fast_leaves(rows)
    active = (rows[:, 7] & (1 << 10)) != 0
    assert fast.sum() == active.sum() and fine.sum() > 0


def test_leaves_larger_than_the_stage(vbt, cuda, oracle):
    """Leaves bigger than the shared-memory stage: FINE6 leaves of a noisy field over 120 frames
    (the fire's temperature recipe at 24 x 16 x 40, generated and encoded on the GPU), up to ~100 KB
    each; the specialised path reads those from global memory (and, when more than a quarter of
    the leaves are that big, every leaf).
    Timeline caches of several launch shapes and dense frames, bit for bit against the oracle."""
    import sys
    from conftest import GOLDEN
    sys.path.insert(0, GOLDEN)
    import gpu_fields as gf
    from vbt_b200.encode import encode_render_temporal, file_image
    fire = gf.Fire(cuda, (24, 16, 40), 120, 7, device="cuda")
    h, off, pay = encode_render_temporal(lambda z0, z1: fire.slab(2, z0, z1), (24, 16, 40))
    img = file_image(h, off, pay)
    a = vbt.Asset(data=img)
    f = oracle.load(image=img)
    try:
        rows = a.leaf_table()
        offs = f.offsets().astype(np.int64)
        windows = ((4 * offs[1:] + 15) & ~15) - ((4 * offs[:-1]) & ~15)
        fast, fine = fast_leaves(rows)
        stage_cap = 69632                                  # the stage's cap at two CTAs per SM
        assert fast.all() and fine.any()
        assert (windows > stage_cap).any(), windows.max()
        a.build_page_table()
        T = f.frames
        lists = [list(range(0, 48)), list(range(48, 112)), list(range(T - 5, T + 2)), [7], [T // 2, 3]]
        check_cache(cuda, a, f, lists, "large leaves")
        X, Y, Z = f.dims
        frames = [0, 1, 59, 118, 119]
        out = cuda.empty((len(frames), Z, Y, X), dtype=cuda.float32, device="cuda")
        a.decode_frames(frames, out)
        a.sync_status()
        got = out.cpu().numpy()
        for i, t in enumerate(frames):
            assert np.array_equal(got[i].view(np.uint32), f.frame(t, threads=8).view(np.uint32)), t
    finally:
        a.close()
