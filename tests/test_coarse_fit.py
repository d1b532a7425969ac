"""The encoder's coarse control fitting on the GPU (vbt_coarse_fit) after the GPU keyframe pass.

Config 1's field, regenerated from its seed, goes through vbt_detect_keyframes and vbt_coarse_fit on
the GPU: every leaf's coarse stream equals the one the reference encoder wrote into
assets/cfg1_blobs.vbtp (descriptors, bins, key frames, FP16 key values) and the oracle's fit
(oracle/vbt_keyframe_oracle.c: vo_coarse_fit, pinned on the reference in
tests/test_encoder_pipeline_oracle.py) bit for bit, float key values and fitted grid included.  A
volume with cropped boundary leaves checks the extents; an index outside the leaf grid is flagged.
"""
import os

import numpy as np
import pytest

from conftest import ASSETS, GOLDEN

pytestmark = pytest.mark.gpu
F32 = np.float32


def control_profile(cls):
    return cls(eps_abs=float(F32(1e-5) * F32(8)), eps_rel=float(F32(0.02) * F32(8)))


def gpu_fit(vbt, cuda, frames_tv, dims, leaves):
    T, V = frames_tv.shape
    d_v = cuda.from_numpy(np.ascontiguousarray(frames_tv, np.float32)).cuda()
    W = (T + 31) // 32
    mask = cuda.empty((W, V), dtype=cuda.int32, device="cuda")
    cnt = cuda.empty(V, dtype=cuda.int32, device="cuda")
    fl = cuda.empty(V, dtype=cuda.uint8, device="cuda")
    recon = cuda.empty_like(d_v)
    vbt.detect_keyframes(d_v, vbt.KeyframeProfile(), mask, cnt, fl, recon)
    n = len(leaves)
    d_leaves = cuda.tensor(np.asarray(leaves, np.int64).astype(np.int32), device="cuda")
    out = dict(desc=cuda.full((n, 64), -1, dtype=cuda.int32, device="cuda"),
               bins=cuda.full((n, 64, 8), 255, dtype=cuda.uint8, device="cuda"),
               key_frames=cuda.zeros((n, 64 * T), dtype=cuda.int16, device="cuda"),
               key_values=cuda.zeros((n, 64 * T), dtype=cuda.float32, device="cuda"),
               key_count=cuda.full((n,), -1, dtype=cuda.int32, device="cuda"),
               required=cuda.zeros(n, dtype=cuda.uint8, device="cuda"),
               grid=cuda.full((n, 64, T), float("nan"), dtype=cuda.float32, device="cuda"))
    vbt.coarse_fit(recon, dims, d_leaves, control_profile(vbt.KeyframeProfile), out["desc"], out["bins"],
                   out["key_frames"], out["key_values"], out["key_count"], out["required"], out["grid"])
    cuda.cuda.synchronize()
    res = {k: v.cpu().numpy() for k, v in out.items()}
    res["recon"] = recon.cpu().numpy()
    return res


def oracle_fit(oracle, recon_tv, dims, leaf):
    X, Y, Z = dims
    T = recon_tv.shape[0]
    lcx, lcy = (X + 7) // 8, (Y + 7) // 8
    bx, by, bz = leaf % lcx, (leaf // lcx) % lcy, leaf // (lcx * lcy)
    vol = recon_tv.reshape(T, Z, Y, X)
    sub = vol[:, 8 * bz:8 * bz + 8, 8 * by:8 * by + 8, 8 * bx:8 * bx + 8]
    w, h, d = sub.shape[3], sub.shape[2], sub.shape[1]
    lt = np.zeros((T, 8, 8, 8), np.float32)
    lt[:, :d, :h, :w] = sub
    from oracle.oracle import VoKeyframeProfile
    return oracle.coarse_fit(np.ascontiguousarray(lt.reshape(T, 512).T), (w, h, d), control_profile(VoKeyframeProfile))


def check_leaf(got, i, want, T):
    n = int(got["key_count"][i])
    assert n == want["key_frames"].size, i
    assert np.array_equal(got["desc"][i].view(np.uint32), want["desc"]), i
    assert np.array_equal(got["bins"][i], want["bins"]), i
    assert np.array_equal(got["key_frames"][i, :n].view(np.uint16), want["key_frames"]), i
    assert np.array_equal(got["key_values"][i, :n].view(np.uint32), want["key_values"].view(np.uint32)), i
    assert int(got["required"][i]) == want["required_max_local"], i
    assert np.array_equal(got["grid"][i].view(np.uint32), want["grid"].view(np.uint32)), i


def test_config1_coarse_streams(vbt, cuda, oracle):
    import sys
    sys.path.insert(0, GOLDEN)
    from make_assets import blobs
    raw = blobs((64, 64, 64), 24, 6, 1)
    T = raw.shape[0]
    frames = raw.reshape(T, -1)
    leaves = list(range(512))
    got = gpu_fit(vbt, cuda, frames, (64, 64, 64), leaves)
    for li in leaves:
        check_leaf(got, li, oracle_fit(oracle, got["recon"], (64, 64, 64), li), T)
    path = os.path.join(ASSETS, "cfg1_blobs.vbtp")
    if not os.path.exists(path):
        return
    from leafstreams import streams_from_file
    fl, arr, _ = streams_from_file(path)
    for li in leaves:
        l = fl[li]
        if int(l["header"]) & 3 == 0:
            continue
        c0, k0, nk = int(l["coarse_control"]), int(l["coarse_key"]), int(l["coarse_kf"])
        assert int(got["key_count"][li]) == nk, li
        assert np.array_equal(got["desc"][li].view(np.uint32), arr["descriptors"][c0:c0 + 64]), li
        assert np.array_equal(got["bins"][li], arr["bins"].reshape(-1, 8)[c0:c0 + 64]), li
        assert np.array_equal(got["key_frames"][li, :nk].view(np.uint16), arr["key_frames"][k0:k0 + nk]), li
        want = arr["key_values"][k0:k0 + nk].astype(np.float16).view(np.uint16)
        assert np.array_equal(oracle.float_to_half(got["key_values"][li, :nk]), want), li


def test_cropped_leaves_and_bad_index(vbt, cuda, oracle):
    rng = np.random.default_rng(12)
    X, Y, Z, T = 20, 12, 17, 30
    t = np.arange(T)[:, None]
    V = X * Y * Z
    c = rng.uniform(0, T, V)
    amp = rng.uniform(0.0, 1.0, V)
    frames = (amp * np.exp(-((t - c) / rng.uniform(2, 8, V)) ** 2) + rng.normal(0, 2e-3, (T, V))).astype(np.float32)
    n_leaves = 3 * 2 * 3
    leaves = list(range(n_leaves)) + [n_leaves + 5]
    got = gpu_fit(vbt, cuda, frames, (X, Y, Z), leaves)
    for li in range(n_leaves):
        check_leaf(got, li, oracle_fit(oracle, got["recon"], (X, Y, Z), li), T)
    assert int(got["key_count"][n_leaves]) == -1                  # 0xFFFFFFFF: outside the leaf grid
