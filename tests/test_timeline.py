"""The batched cache timeline (vbt_decode_cache_timeline): every launch shape the autotuner can
choose (leaf per CTA or per warp, 1..64 frames per launch, one or two waves), eager and replayed
from a captured CUDA graph, writes exactly what vbt_decode_cache writes; replays stay exact after
an upload and across many replays (the work counters and page-table descriptors are cleared
inside the graph)."""
import os

import numpy as np
import pytest

from conftest import ASSETS, golden_asset

pytestmark = pytest.mark.gpu


def asset_paths():
    out = [golden_asset(n) for n in ("tiny_density", "tiny_levelset", "sci_small")]
    for n in ("cfg1_blobs", "cfg4_sdf_small"):
        p = os.path.join(ASSETS, n + ".vbtp")
        if os.path.exists(p):
            out.append(p)
    return out


def expected_cache(cuda, a, T):
    n = max(a.active_count, 1)
    ref = cuda.empty((T, n, 512), dtype=cuda.float32, device="cuda")
    for i in range(0, T, 32):
        ch = list(range(i, min(T, i + 32)))
        a.decode_cache(ch, ref[i], frame_stride=n * 512)
    a.sync_status()
    return ref


@pytest.mark.parametrize("path", asset_paths(), ids=os.path.basename)
def test_timeline_shapes_eager_and_graph(vbt, cuda, path):
    a = vbt.Asset(path)
    T = a.frames
    n = max(a.active_count, 1)
    ref = expected_cache(cuda, a, T)
    s = cuda.cuda.Stream()
    wave2 = 0
    for variant, fpl, grid in [(0, 48, 0), (0, 16, 0), (0, 64, 0), (0, 96, 0), (0, 128, 0), (1, 32, 0), (1, 16, 296), (0, 5, 0)]:
        a.set_tuning(variant, fpl, grid)
        out = cuda.full((T, n, 512), float("nan"), dtype=cuda.float32, device="cuda")
        a.decode_cache_timeline(0, T, out, graph=False)
        a.sync_status()
        assert cuda.equal(out.view(cuda.int32), ref.view(cuda.int32)), (variant, fpl, "eager")
        for rep in range(3):
            with cuda.cuda.stream(s):
                out.fill_(float("nan"))
                a.decode_cache_timeline(0, T, out, graph=True, stream=s)
            s.synchronize()
            a.sync_status(s)
            assert cuda.equal(out.view(cuda.int32), ref.view(cuda.int32)), (variant, fpl, "graph", rep)
    a.close()


def test_autotune_then_graph_replay_after_upload(vbt, cuda):
    path = os.path.join(ASSETS, "cfg1_blobs.vbtp")
    if not os.path.exists(path):
        path = golden_asset("tiny_density")
    a = vbt.Asset(path)
    T = a.frames
    n = max(a.active_count, 1)
    ref = expected_cache(cuda, a, T)
    out = cuda.empty((T, n, 512), dtype=cuda.float32, device="cuda")
    t = a.autotune(T, out)
    assert t.variant in (0, 1) and 1 <= t.frames_per_launch <= 128 and t.ms_per_frame > 0
    assert t.ms_per_frame <= t.ms_per_frame_default * 1.0001
    got = a.tuning()
    assert (got.variant, got.frames_per_launch, got.grid) == (t.variant, t.frames_per_launch, t.grid)
    s = cuda.cuda.Stream()
    img = cuda.from_numpy(np.fromfile(path, dtype=np.uint8)).pin_memory()
    for rep in range(4):
        if rep == 2:
            a.upload(img, s)          # same image: the leaf table is rebuilt under the graph
        with cuda.cuda.stream(s):
            out.zero_()
            a.decode_cache_timeline(0, T, out, graph=True, stream=s)
        s.synchronize()
        a.sync_status(s)
        assert cuda.equal(out.view(cuda.int32), ref.view(cuda.int32)), rep
    # a sub-range starting later, as its own graph
    part = cuda.empty((T // 2, n, 512), dtype=cuda.float32, device="cuda")
    with cuda.cuda.stream(s):
        a.decode_cache_timeline(T // 3, T // 2, part, graph=True, stream=s)
    s.synchronize()
    assert cuda.equal(part.view(cuda.int32), ref[T // 3:T // 3 + T // 2].view(cuda.int32))
    a.close()
