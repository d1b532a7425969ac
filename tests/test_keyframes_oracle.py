"""Pin the keyframe-pass restatement (oracle/vbt_keyframe_oracle.c) to the reference encoder.

CPU only.  The restatement must reproduce, bit for bit, what the reference's own
detectDensityKeyFrames and reconstructFromKeys (src/render_temporal_kf_probe_main.cpp:2080-2201)
produced on the golden series (tests/golden/make_keyframes.py): the keys, the usedCutoffProtect
flag and the reconstruction.  Where the compiled reference (oracle/_ref/libkfref.so) is present,
fresh seeded series and the whole per-voxel pass (key counts and squared errors of
:619-659) are compared with it directly.
"""
import ast
import os

import numpy as np
import pytest

from conftest import GOLDEN


def profile(kw):
    from oracle.oracle import VoKeyframeProfile
    return VoKeyframeProfile(**kw)


def golden_cases():
    z = np.load(os.path.join(GOLDEN, "keyframes.npz"))
    profiles = [ast.literal_eval(str(p)) for p in z["profiles"]]
    for T, kind, pi, voff, koff, nk, used in z["meta"]:
        yield (int(T), int(kind), profiles[int(pi)], z["values"][voff:voff + T], z["keys"][koff:koff + nk],
               bool(used), z["recon"][voff:voff + T])


def test_golden_keyframes(oracle):
    n = used_n = 0
    for T, kind, prof, v, keys, used, recon in golden_cases():
        k, u = oracle.detect_keyframes(v, profile(prof))
        assert np.array_equal(k, keys) and u == used, (T, kind, prof, k, keys)
        r = oracle.reconstruct(v, k)
        assert np.array_equal(r.view(np.uint32), recon.view(np.uint32)), (T, kind, prof)
        n += 1
        used_n += used
    assert n == 960 and 0 < used_n < n


def test_golden_pass_layout(oracle):
    """The batched pass (word-major key mask, counts, flags, reconstruction, squared error) agrees
    with the per-series functions on the golden series of each frame count."""
    from oracle.oracle import VoKeyframeProfile
    by_t = {}
    for T, kind, prof, v, keys, used, recon in golden_cases():
        if not prof:
            by_t.setdefault(T, []).append((v, keys, used, recon))
    for T, cases in by_t.items():
        frames = np.stack([c[0] for c in cases], axis=1)
        out = oracle.keyframe_pass(frames, VoKeyframeProfile(bg_threshold=-1.0), threads=2)
        for s, (v, keys, used, recon) in enumerate(cases):
            mask = out["key_mask"][:, s]
            got = [t for t in range(T) if mask[t // 32] >> (t % 32) & 1]
            assert got == list(keys)
            assert out["key_count"][s] == len(keys) and out["flags"][s] == (2 if used else 0)
            assert np.array_equal(out["recon"][:, s].view(np.uint32), recon.view(np.uint32))
            d = v.astype(np.float64) - recon.astype(np.float64)
            e2 = 0.0
            for x in d:
                e2 += x * x
            assert out["err2"][s] == e2


@pytest.fixture(scope="module")
def kfref():
    from oracle.oracle import KFREF_SO, KeyframeReference
    if not os.path.exists(KFREF_SO):
        pytest.skip("reference build (oracle/_ref/libkfref.so) not present")
    return KeyframeReference()


def test_random_series_against_reference(oracle, kfref):
    import sys
    sys.path.insert(0, GOLDEN)
    from make_keyframes import KINDS, PROFILES, series
    rng = np.random.default_rng(77)
    for it in range(3000):
        T = int(rng.choice([2, 4, 17, 48, 96, 150, 257]))
        v = series(rng, it % KINDS, T).astype(np.float32)
        p = profile(PROFILES[it % len(PROFILES)])
        k, u = oracle.detect_keyframes(v, p)
        k2, u2 = kfref.detect_keyframes(v, p)
        assert np.array_equal(k, k2) and u == u2, it


def test_pass_against_reference(oracle, kfref):
    """Background-zeroed and keyed series mixed, as the encoder's default background threshold
    (0.3 x cutoff) sees them: key counts equal and squared errors bit for bit."""
    from oracle.oracle import VoKeyframeProfile
    rng = np.random.default_rng(5)
    T, S = 96, 4000
    t = np.arange(T)[:, None]
    c = rng.uniform(0, T, S)
    amp = np.where(rng.random(S) < 0.3, 5e-5, rng.uniform(0.0, 1.0, S))
    frames = (amp * np.exp(-((t - c) / 6.0) ** 2) + rng.normal(0, 1e-3, (T, S)) * (amp > 1e-4)).astype(np.float32)
    p = VoKeyframeProfile()
    out = oracle.keyframe_pass(frames, p, threads=4)
    kc, e2 = kfref.temporal_pass(frames, p, threads=4)
    assert (out["flags"] & 1).sum() > 100
    assert np.array_equal(out["key_count"], kc)
    assert np.array_equal(out["err2"].view(np.uint64), e2.view(np.uint64))


def test_edge_profiles_against_reference(oracle, kfref):
    """Profiles and values away from the encoder's defaults: no absolute epsilon (the floor alone
    bounds it), no gamma, a large gamma, signed level-set values around a nonzero iso value with
    and without a band, huge and tiny magnitudes, and a cutoff band of zero."""
    rng = np.random.default_rng(91)
    profiles = [dict(eps_abs=0.0), dict(gamma_delta=0.0, eps_rel=0.001), dict(gamma_delta=5.0),
                dict(render_cutoff=-1.0, iso_surface_protect=1, iso_value=0.5, iso_band=0.0),
                dict(render_cutoff=-1.0, iso_surface_protect=1, iso_value=-2.0, iso_band=0.3, eps_rel=0.1),
                dict(cutoff_band=0.0, render_cutoff=0.5), dict(eps_abs=1e-2, eps_rel=0.0)]
    scales = [1e-30, 1e-6, 1.0, 1e3, 1e30]
    n = 0
    for it in range(2400):
        T = int(rng.choice([2, 3, 9, 40, 96, 200]))
        kind = it % 4
        t = np.arange(T)
        if kind == 0:
            v = rng.normal(0, 1, T)
        elif kind == 1:
            v = np.sin(t * rng.uniform(0.05, 0.6)) * 3.0 - 1.0
        elif kind == 2:
            v = np.repeat(rng.normal(0, 1, T // 3 + 1), 3)[:T]         # piecewise constant
        else:
            v = np.cumsum(rng.normal(0, 1, T))
        v = (v * scales[it % len(scales)]).astype(np.float32)
        p = profile(profiles[it % len(profiles)])
        k, u = oracle.detect_keyframes(v, p)
        k2, u2 = kfref.detect_keyframes(v, p)
        assert np.array_equal(k, k2) and u == u2, (it, T, profiles[it % len(profiles)])
        r = oracle.reconstruct(v, k)
        r2 = kfref.reconstruct(v, k2)
        assert np.array_equal(r.view(np.uint32), r2.view(np.uint32)), it
        n += 1
    assert n == 2400
