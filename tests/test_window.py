"""(d) Window decode of scientific leaves on the tensor cores (vbt_decode_window) and its FP64
error oracle (vbt_window_error).

The window path is not bit-exact by design (split-BF16 products, FP32 accumulation); the bar is
1e-6 of the field range against the FP64 oracle and against the exact per-frame decode.  The
oracle is checked to report a planted deviation of known size.
"""
import os

import numpy as np
import pytest

from conftest import ASSETS, golden_asset

pytestmark = pytest.mark.gpu

TOL = 1e-6   # relative to the field range


def sci_paths():
    out = [golden_asset(n) for n in ("sci_small", "sci_coarse", "sci_dense", "sci_dense_tb")]
    for n in ("sci_64", "mix_sci", "sci_modes"):
        p = os.path.join(ASSETS, n + ".vbtp")
        if os.path.exists(p):
            out.append(p)
    return out


def windows(T):
    w = [(0, min(T, 16)), (max(0, T - 7), min(T, 7)), (0, min(T, 64))]
    if T > 40:
        w.append((T // 2 - 20, 40))
    return w


@pytest.mark.parametrize("path", sci_paths(), ids=os.path.basename)
def test_window_matches_per_frame_and_oracle(vbt, cuda, path):
    a = vbt.Asset(path)
    T, L = a.frames, a.leaf_count
    assert a.active_count == L
    for t0, n in windows(T):
        exact = cuda.empty((n, L, 512), dtype=cuda.float32, device="cuda")
        a.decode_cache(list(range(t0, t0 + n)), exact, frame_stride=L * 512)
        win = cuda.full((n, L, 512), float("nan"), dtype=cuda.float32, device="cuda")
        a.decode_window(t0, n, win)
        a.sync_status()
        e = exact.cpu().numpy().astype(np.float64)
        w = win.cpu().numpy().astype(np.float64)
        assert np.isfinite(w).all()
        mx, rms, lo, hi = a.window_error(t0, n, win)
        mx_e, rms_e, lo_e, hi_e = a.window_error(t0, n, exact)
        assert (lo, hi) == (lo_e, hi_e)
        orng = hi - lo
        assert orng > 0
        diff = np.abs(w - e).max()
        assert diff <= TOL * orng, (t0, n, diff, orng)
        assert mx <= TOL * orng and mx_e <= TOL * orng, (mx, mx_e, orng)
    a.close()


def test_oracle_sees_a_perturbation(vbt, cuda):
    """The oracle's max error of the exact per-frame output is tiny; after moving one value by a
    known amount it reports that amount."""
    a = vbt.Asset(golden_asset("sci_small"))
    T, L = a.frames, a.leaf_count
    n = min(T, 16)
    exact = cuda.empty((n, L, 512), dtype=cuda.float32, device="cuda")
    a.decode_cache(list(range(n)), exact, frame_stride=L * 512)
    a.sync_status()
    mx, rms, lo, hi = a.window_error(0, n, exact)
    rng = hi - lo
    assert mx <= TOL * rng and rms <= mx
    bump = 1e-3 * rng
    exact[3, L // 2, 77] += bump
    mx2, _, lo2, hi2 = a.window_error(0, n, exact)
    assert (lo2, hi2) == (lo, hi)
    assert abs(mx2 - bump) <= 1e-6 * rng, (mx2, bump)
    a.close()


def test_window_rejects_long_windows(vbt, cuda):
    r = vbt.Asset(golden_asset("tiny_density"))
    out = cuda.empty(65 * r.leaf_count * 512, dtype=cuda.float32, device="cuda")
    r.build_page_table()
    for t0, n in ((0, 65), (r.frames - 2, 4), (0, 0)):
        with pytest.raises(vbt.VbtError) as ei:
            r.decode_window(t0, n, out, frame_stride=r.leaf_count * 512)
        assert ei.value.status == 40
    r.close()
    s = vbt.Asset(golden_asset("sci_small"))
    out = cuda.empty(65 * s.leaf_count * 512, dtype=cuda.float32, device="cuda")
    with pytest.raises(vbt.VbtError):
        s.decode_window(0, 65, out)
    with pytest.raises(vbt.VbtError):
        s.decode_window(s.frames - 2, 4, out)
    s.close()


# ---- render-temporal windows: exact voxels at the knots, hat-basis contraction on the tensor cores


def render_paths():
    out = [golden_asset("tiny_density"), golden_asset("tiny_levelset")]
    for n in ("cfg1_blobs", "mix_fire_density", "mix_fire_flames", "mix_fire_temperature", "cfg2_plume",
              "mix_sdf"):
        p = os.path.join(ASSETS, n + ".vbtp")
        if os.path.exists(p):
            out.append(p)
    return out


def render_windows(T):
    w = [(0, min(T, 16)), (max(0, T - 16), min(T, 16)), (T // 3, min(7, T - T // 3)), (0, 1), (0, min(T, 2)),
         (max(0, T - 3), min(T, 3)), (0, min(T, 64)), (max(0, T - 40), min(T, 40)), (1, min(T - 1, 17))]
    return sorted(set(w))


@pytest.mark.parametrize("path", render_paths(), ids=os.path.basename)
def test_render_window_matches_per_frame_and_oracle(vbt, cuda, path):
    a = vbt.Asset(path)
    a.build_page_table()
    T, A = a.frames, a.active_count
    stride = A * 512
    for t0, n in render_windows(T):
        exact = cuda.empty((n, A, 512), dtype=cuda.float32, device="cuda")
        a.decode_cache(list(range(t0, t0 + n)), exact, frame_stride=stride)
        win = cuda.full((n, A, 512), float("nan"), dtype=cuda.float32, device="cuda")
        a.decode_window(t0, n, win, frame_stride=stride)
        a.sync_status()
        e = exact.cpu().numpy().astype(np.float64)
        w = win.cpu().numpy().astype(np.float64)
        assert np.isfinite(w).all()
        mx, rms, lo, hi = a.window_error(t0, n, win, frame_stride=stride)
        mx_e, rms_e, lo_e, hi_e = a.window_error(t0, n, exact, frame_stride=stride)
        assert (lo, hi) == (lo_e, hi_e)
        rng = max(hi - lo, 1e-30)
        diff = np.abs(w - e).max() if w.size else 0.0
        assert diff <= TOL * rng, (t0, n, diff, rng)
        assert mx <= TOL * rng and mx_e <= TOL * rng, (t0, n, mx, mx_e, rng)
        assert rms <= mx + 1e-30
        # every 16-frame window's ends are knots: decoded exactly, bit for bit
        for j in sorted({*range(0, n, 16), *(min(n, j0 + 16) - 1 for j0 in range(0, n, 16))}):
            assert np.array_equal(w[j].view(np.uint32), e[j].view(np.uint32)), (t0, n, j)
    a.close()


def test_render_window_mode2_is_exact(vbt, cuda):
    """Mode2 leaves clamp negatives outside the occupancy (not linear in t), so every frame is a knot
    and the window equals the per-frame decode bit for bit on those leaves."""
    a = vbt.Asset(golden_asset("tiny_levelset"))
    a.build_page_table()
    T, A = a.frames, a.active_count
    compact, _ = a.page_table()
    modes = a.leaf_table()[:, 1] & 3   # header word: route tag in bits 0-1
    mode2_ranks = compact[(modes == 2) & (compact != 0xFFFFFFFF)].astype(np.int64)
    assert len(mode2_ranks) > 0
    n = min(T, 16)
    exact = cuda.empty((n, A, 512), dtype=cuda.float32, device="cuda")
    a.decode_cache(list(range(n)), exact, frame_stride=A * 512)
    win = cuda.empty((n, A, 512), dtype=cuda.float32, device="cuda")
    a.decode_window(0, n, win, frame_stride=A * 512)
    a.sync_status()
    e = exact.cpu().numpy()[:, mode2_ranks]
    w = win.cpu().numpy()[:, mode2_ranks]
    assert np.array_equal(e.view(np.uint32), w.view(np.uint32))
    a.close()


def test_render_oracle_sees_a_perturbation(vbt, cuda):
    a = vbt.Asset(golden_asset("tiny_density"))
    a.build_page_table()
    T, A = a.frames, a.active_count
    exact = cuda.empty((T, A, 512), dtype=cuda.float32, device="cuda")
    a.decode_cache(list(range(T)), exact, frame_stride=A * 512)
    a.sync_status()
    mx, rms, lo, hi = a.window_error(0, T, exact, frame_stride=A * 512)
    rng = hi - lo
    assert rng > 0 and mx <= TOL * rng
    bump = 1e-3 * rng
    exact[T // 2, A // 2, 300] += bump
    mx2, _, lo2, hi2 = a.window_error(0, T, exact, frame_stride=A * 512)
    assert (lo2, hi2) == (lo, hi)
    assert abs(mx2 - bump) <= 1e-6 * rng, (mx2, bump)
    a.close()
