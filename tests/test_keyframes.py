"""The encoder's per-voxel keyframe pass on the GPU (vbt_detect_keyframes) against the oracle
(oracle/vbt_keyframe_oracle.c, pinned on the reference's own detectDensityKeyFrames and
reconstructFromKeys): key sets, key counts, flags, reconstructions and squared errors bit for bit;
the pass's totals exactly (counts) and to 1e-12 relative (the squared-error sum, whose order
differs).  Also the golden series the reference itself produced, and every integer quotient the
pass forms."""
import ast
import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def run_gpu(vbt, cuda, frames, prof, series=None, with_totals=True):
    T, stride = frames.shape
    S = stride if series is None else series
    W = (T + 31) // 32
    d_v = cuda.from_numpy(np.ascontiguousarray(frames, np.float32)).cuda()
    mask = cuda.full((W, S), -1, dtype=cuda.int32, device="cuda")
    cnt = cuda.full((S,), -1, dtype=cuda.int32, device="cuda")
    flags = cuda.full((S,), 255, dtype=cuda.uint8, device="cuda")
    recon = cuda.full((T, stride), float("nan"), dtype=cuda.float32, device="cuda")
    err2 = cuda.full((S,), float("nan"), dtype=cuda.float64, device="cuda")
    tot = cuda.full((40,), 255, dtype=cuda.uint8, device="cuda") if with_totals else None
    vbt.detect_keyframes(d_v, prof, mask, cnt, flags, recon, err2, tot, series=S)
    cuda.cuda.synchronize()
    out = dict(key_mask=mask.cpu().numpy().view(np.uint32), key_count=cnt.cpu().numpy().view(np.uint32),
               flags=flags.cpu().numpy(), recon=recon.cpu().numpy(), err2=err2.cpu().numpy())
    if with_totals:
        out["totals"] = vbt.keyframe_totals(tot)
    return out


def oracle_prof(vbt_prof):
    from oracle.oracle import VoKeyframeProfile
    q = VoKeyframeProfile()
    for name, _ in VoKeyframeProfile._fields_:
        setattr(q, name, getattr(vbt_prof, name))
    return q


def compare(got, want, S, what):
    assert np.array_equal(got["key_mask"], want["key_mask"]), what
    assert np.array_equal(got["key_count"], want["key_count"]), what
    assert np.array_equal(got["flags"], want["flags"]), what
    assert np.array_equal(got["recon"][:, :S].view(np.uint32), want["recon"].view(np.uint32)), what
    assert np.array_equal(got["err2"].view(np.uint64), want["err2"].view(np.uint64)), what
    if "totals" in got:
        t = got["totals"]
        kc = want["key_count"].astype(np.int64)
        assert t.total_keys == kc.sum() and t.max_keys == kc.max(), what
        assert t.protected_series == int(((want["flags"] >> 1) & 1).sum()), what
        assert t.background_series == int((want["flags"] & 1).sum()), what
        assert abs(t.err2 - want["err2"].sum()) <= 1e-12 * max(1.0, want["err2"].sum()), what


def test_integer_division_exhaustive(vbt, cuda):
    assert vbt.selftest_keyframe_division(1024) == (0, 2 ** 64 - 1)


def test_golden_series(vbt, cuda):
    """The reference's own keys, flags and reconstructions (tests/golden/keyframes.npz)."""
    z = np.load(os.path.join(GOLDEN, "keyframes.npz"))
    profiles = [ast.literal_eval(str(p)) for p in z["profiles"]]
    groups = {}
    for T, kind, pi, voff, koff, nk, used in z["meta"]:
        groups.setdefault((int(T), int(pi)), []).append(
            (z["values"][voff:voff + T], z["keys"][koff:koff + nk], bool(used), z["recon"][voff:voff + T]))
    for (T, pi), cases in groups.items():
        prof = vbt.KeyframeProfile(bg_threshold=-1.0, **profiles[pi])
        frames = np.stack([c[0] for c in cases], axis=1)
        got = run_gpu(vbt, cuda, frames, prof, with_totals=False)
        for s, (v, keys, used, recon) in enumerate(cases):
            m = got["key_mask"][:, s]
            assert [t for t in range(T) if m[t // 32] >> (t % 32) & 1] == list(keys), (T, pi, s)
            assert got["key_count"][s] == len(keys) and got["flags"][s] == (2 if used else 0), (T, pi, s)
            assert np.array_equal(got["recon"][:, s].view(np.uint32), recon.view(np.uint32)), (T, pi, s)


def blob_frames(T, S, seed, bg_frac=0.3):
    rng = np.random.default_rng(seed)
    t = np.arange(T)[:, None]
    c = rng.uniform(-10, T + 10, S)
    w = rng.uniform(2, 15, S)
    amp = np.where(rng.random(S) < bg_frac, rng.uniform(0, 8e-5, S), rng.uniform(0.0, 1.0, S))
    noise = rng.normal(0, 1e-3, (T, S)) * (amp > 1e-4)
    f = amp * np.exp(-((t - c) / w) ** 2) + noise
    f[:, rng.random(S) < 0.05] = 0.0                      # exactly zero
    f[:, rng.random(S) < 0.05] = 0.25                     # constant
    return f.astype(np.float32)


@pytest.mark.parametrize("prof_kw", [{}, dict(iso_surface_protect=1, iso_band=0.05, iso_value=0.2),
                                     dict(gamma_delta=0.0, cutoff_temporal_protect=0, render_cutoff=-1.0)],
                         ids=["encoder", "iso", "plain"])
def test_volume_against_oracle(vbt, cuda, oracle, prof_kw):
    T, S = 96, 30000
    frames = blob_frames(T, S, seed=11)
    prof = vbt.KeyframeProfile(**prof_kw)
    got = run_gpu(vbt, cuda, frames, prof)
    want = oracle.keyframe_pass(frames, oracle_prof(prof))
    compare(got, want, S, prof_kw)
    assert (want["key_count"] > 2).sum() > 1000


@pytest.mark.parametrize("T", [1, 2, 3, 31, 32, 33, 120, 257, 700, 1024])
def test_frame_counts_and_padding(vbt, cuda, oracle, T):
    """Frame counts across the word and shared-memory limits (1024 frames takes the 32-series CTA);
    the series are the first columns of a padded frame stride."""
    S = 2000 if T <= 257 else 600
    stride = S + 37
    frames = np.zeros((T, stride), np.float32)
    frames[:, :S] = blob_frames(T, S, seed=T)
    prof = vbt.KeyframeProfile()
    got = run_gpu(vbt, cuda, frames, prof, series=S)
    want = oracle.keyframe_pass(np.ascontiguousarray(frames[:, :S]), oracle_prof(prof))
    compare(got, want, S, T)
    assert np.isnan(got["recon"][:, S:]).all()            # padding columns untouched


EDGE_PROFILES = [dict(eps_abs=0.0), dict(gamma_delta=0.0, eps_rel=0.001), dict(gamma_delta=5.0),
                 dict(render_cutoff=-1.0, iso_surface_protect=1, iso_value=0.5, iso_band=0.0),
                 dict(render_cutoff=-1.0, iso_surface_protect=1, iso_value=-2.0, iso_band=0.3, eps_rel=0.1),
                 dict(cutoff_band=0.0, render_cutoff=0.5), dict(eps_abs=1e-2, eps_rel=0.0)]


@pytest.mark.parametrize("pi", range(len(EDGE_PROFILES)))
def test_edge_profiles(vbt, cuda, oracle, pi):
    """Profiles away from the encoder's defaults over signed, piecewise-constant, oscillating and
    random-walk series at magnitudes from 1e-30 to 1e30."""
    rng = np.random.default_rng(100 + pi)
    T, S = 96, 4000
    t = np.arange(T)[:, None]
    kind = rng.integers(0, 4, S)
    walk = np.cumsum(rng.normal(0, 1, (T, S)), axis=0)
    osc = np.sin(t * rng.uniform(0.05, 0.6, S)) * 3.0 - 1.0
    steps = np.repeat(rng.normal(0, 1, (T // 3 + 1, S)), 3, axis=0)[:T]
    noise = rng.normal(0, 1, (T, S))
    f = np.choose(kind, [noise, osc, steps, walk])
    f = f * np.array([1e-30, 1e-6, 1.0, 1e3, 1e30])[rng.integers(0, 5, S)]
    frames = f.astype(np.float32)
    prof = vbt.KeyframeProfile(**EDGE_PROFILES[pi])
    got = run_gpu(vbt, cuda, frames, prof)
    want = oracle.keyframe_pass(frames, oracle_prof(prof))
    compare(got, want, S, EDGE_PROFILES[pi])


def test_time_fastest_layout(vbt, cuda, oracle):
    """RawVolume4D's time-fastest order: each series contiguous (rows padded past the frame count);
    the reconstruction comes back in the same layout."""
    T, S = 96, 5000
    frames = blob_frames(T, S, seed=21)
    rows = np.zeros((S, T + 5), np.float32)
    rows[:, :T] = frames.T
    d_v = cuda.from_numpy(rows).cuda()[:, :T]
    W = (T + 31) // 32
    mask = cuda.zeros((W, S), dtype=cuda.int32, device="cuda")
    cnt = cuda.zeros(S, dtype=cuda.int32, device="cuda")
    fl = cuda.zeros(S, dtype=cuda.uint8, device="cuda")
    recon_full = cuda.full((S, T + 5), float("nan"), dtype=cuda.float32, device="cuda")
    recon = recon_full[:, :T]
    err2 = cuda.zeros(S, dtype=cuda.float64, device="cuda")
    prof = vbt.KeyframeProfile()
    vbt.detect_keyframes(d_v, prof, mask, cnt, fl, recon, err2, time_fastest=True)
    cuda.cuda.synchronize()
    want = oracle.keyframe_pass(frames, oracle_prof(prof))
    got = dict(key_mask=mask.cpu().numpy().view(np.uint32), key_count=cnt.cpu().numpy().view(np.uint32),
               flags=fl.cpu().numpy(), recon=np.ascontiguousarray(recon.cpu().numpy().T), err2=err2.cpu().numpy())
    compare(got, want, S, "time fastest")
    assert np.isnan(recon_full.cpu().numpy()[:, T:]).all()


def test_rejects_bad_arguments(vbt, cuda):
    prof = vbt.KeyframeProfile()
    v = cuda.zeros((1025, 64), dtype=cuda.float32, device="cuda")
    mask = cuda.zeros((33, 64), dtype=cuda.int32, device="cuda")
    cnt = cuda.zeros(64, dtype=cuda.int32, device="cuda")
    fl = cuda.zeros(64, dtype=cuda.uint8, device="cuda")
    with pytest.raises(vbt.VbtError) as e:
        vbt.detect_keyframes(v, prof, mask, cnt, fl)
    assert e.value.status == 43                                           # VBT_STATUS_LIMIT: over 1024 frames
    with pytest.raises(vbt.VbtError) as e:
        vbt.detect_keyframes(v[:10], prof, mask, cnt, fl, series=65)      # series beyond the stride
    assert e.value.status == 40
    with pytest.raises(vbt.VbtError) as e:
        vbt.detect_keyframes(v[:0], prof, mask, cnt, fl)                  # no frames
    assert e.value.status == 40
