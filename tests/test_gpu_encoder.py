"""The render-temporal encoder on the GPU (vbt_b200.encode): whole VBTPACK4 files from their raw
fields, byte for byte the files the reference encoder wrote.

The fields are regenerated from their seeds (tests/golden/make_assets.py), uploaded, and encoded by
the chain of this library's kernels: keyframe pass, EMPTY test, coarse fit, then the FINE6 fit and
the density route, or the Mode2 shell stage for a level set, and the leaf packer.  Each file is
compared with the asset on disk where it is present, else with the SHA-256 of the reference's file
(tests/golden/asset_digests.json), and then saved under assets/ for the tests that read it.  The chain is also run slab by slab from a field function and in
groups of one leaf layer, which must not change a byte.  The stages themselves are checked against
the oracle's restatements (vo_fine6_fit, vo_shell_fit and the route of
tests/test_encoder_pipeline_oracle.py, which are pinned there on the reference) on seeded leaves.
"""
import hashlib
import json
import os
import sys

import numpy as np
import pytest

from conftest import ASSETS, GOLDEN

pytestmark = pytest.mark.gpu
F32 = np.float32

sys.path.insert(0, GOLDEN)


def reference_file(name):
    """(bytes or None, digest entry or None) of the reference encoder's file for an asset."""
    for d in (os.path.join(GOLDEN, "assets"), ASSETS):
        p = os.path.join(d, name + ".vbtp")
        if os.path.exists(p):
            return open(p, "rb").read(), None
    with open(os.path.join(GOLDEN, "asset_digests.json")) as fh:
        return None, json.load(fh).get(name)


def first_difference(a, b):
    """Where two file images part: the header, the offsets, or the first leaf whose bytes differ."""
    if a[:52] != b[:52]:
        return "header"
    L = int(np.frombuffer(a[40:44], "<u4")[0])
    oa = np.frombuffer(a[52:56 + 4 * L], "<u4")
    ob = np.frombuffer(b[52:56 + 4 * L], "<u4") if len(b) >= 56 + 4 * L else None
    pa = 56 + 4 * L
    for i in range(L):
        la = a[pa + 4 * int(oa[i]):pa + 4 * int(oa[i + 1])]
        lb = b[pa + 4 * int(ob[i]):pa + 4 * int(ob[i + 1])] if ob is not None else b""
        if la != lb:
            return f"leaf {i}: mode {la[0] & 3 if la else None} vs {lb[0] & 3 if lb else None}, {len(la)} vs {len(lb)} bytes"
    return "the offsets"


def check_image(name, img):
    want, digest = reference_file(name)
    if want is None and digest is None:
        pytest.skip(f"neither asset {name} nor its digest present")
    if want is not None:
        assert img == want, (name, first_difference(img, want))
    else:
        assert len(img) == digest["bytes"], (name, len(img), digest["bytes"])
        assert hashlib.sha256(img).hexdigest() == digest["sha256"], name


@pytest.mark.parametrize("name", ["tiny_density", "tiny_levelset", "cfg1_blobs", "cfg4_sdf_small",
                                  "mix_fire_temperature", "mix_sdf"])
def test_file_encoded_on_the_gpu(vbt, cuda, name):
    import make_assets
    from vbt_b200.encode import encode_render_temporal, file_image
    raw, dims, levelset = make_assets.field_of(name)
    T = raw.shape[0]
    d_raw = cuda.from_numpy(np.ascontiguousarray(raw.reshape(T, -1))).cuda()
    h, off, pay = encode_render_temporal(d_raw, dims, levelset=levelset)
    img = file_image(h, off, pay).numpy().tobytes()
    check_image(name, img)
    path = os.path.join(ASSETS, name + ".vbtp")
    if not os.path.exists(path) and os.path.isdir(ASSETS):
        # the reference's file, regenerated here (its digest matched): the later tests can use it
        with open(path + ".tmp", "wb") as fh:
            fh.write(img)
        os.replace(path + ".tmp", path)


@pytest.mark.parametrize("name", ["tiny_density", "cfg4_sdf_small"])
def test_slabs_and_groups_change_nothing(vbt, cuda, name):
    """The field given as a function of z-planes, one leaf layer per group, the value range given:
    the same bytes."""
    import make_assets
    from vbt_b200.encode import encode_render_temporal, file_image
    raw, dims, levelset = make_assets.field_of(name)
    X, Y, Z = dims
    T = raw.shape[0]
    d_raw = cuda.from_numpy(np.ascontiguousarray(raw)).cuda()          # [T, Z, Y, X]
    calls = []

    def slab(z0, z1):
        calls.append((z0, z1))
        return d_raw[:, z0:z1].reshape(T, -1)

    rng = (float(raw.min()), float(raw.max()))
    h, off, pay = encode_render_temporal(slab, dims, levelset=levelset, batch=1, value_range=rng)
    assert calls == [(z, min(Z, z + 8)) for z in range(0, Z, 8)]
    check_image(name, file_image(h, off, pay).numpy().tobytes())


def _leaf_series(recon, dims, li):
    X, Y, Z = dims
    T = recon.shape[0]
    lcx, lcy = (X + 7) // 8, (Y + 7) // 8
    bx, by, bz = li % lcx, (li // lcx) % lcy, li // (lcx * lcy)
    sub = recon.reshape(T, Z, Y, X)[:, 8 * bz:8 * bz + 8, 8 * by:8 * by + 8, 8 * bx:8 * bx + 8]
    d, h, w = sub.shape[1:]
    lt = np.zeros((T, 8, 8, 8), np.float32)
    lt[:, :d, :h, :w] = sub
    return np.ascontiguousarray(lt.reshape(T, 512).T), (w, h, d), (8 * bx, 8 * by, 8 * bz)


def _seeded_field(rng, dims, T, levelset):
    X, Y, Z = dims
    zz, yy, xx = np.meshgrid(np.arange(Z), np.arange(Y), np.arange(X), indexing="ij")
    out = np.empty((T, Z, Y, X), np.float32)
    c = rng.uniform(0, 1, (3, 3)) * np.array([X, Y, Z])
    for t in range(T):
        if levelset:
            phi = zz - (Z * 0.4 + 1.5 * np.sin(0.3 * xx + 0.2 * t))
            for s in range(3):
                p = c[s] + np.array([0.3, -0.2, 0.1]) * t
                phi = np.minimum(phi, np.sqrt((xx - p[0]) ** 2 + (yy - p[1]) ** 2 + (zz - p[2]) ** 2) - 3.0)
            out[t] = phi
        else:
            v = np.zeros_like(out[t])
            for s in range(3):
                p = c[s] + np.array([0.4, 0.2, -0.3]) * t
                v += rng.uniform(0.2, 1.0) * np.exp(-((xx - p[0]) ** 2 + (yy - p[1]) ** 2 + (zz - p[2]) ** 2) / 30.0)
            out[t] = v + rng.normal(0, 0.01, v.shape)
    return out


@pytest.mark.parametrize("levelset", [False, True])
def test_stages_against_the_oracle(vbt, cuda, oracle, levelset):
    """FINE6 fit + route (density) or the shell stage (level set) per leaf, against the oracle,
    on a seeded field with cropped boundary leaves: streams, fitted grids, occupancy, counts."""
    from vbt_b200.encode import COARSE_RES, profiles
    import test_encoder_pipeline_oracle as pipe
    rng = np.random.default_rng(31 + levelset)
    dims, T = (20, 13, 18), 17
    X, Y, Z = dims
    raw = _seeded_field(rng, dims, T, levelset)
    prof, cprof = profiles(levelset)
    d_raw = cuda.from_numpy(raw.reshape(T, -1).copy()).cuda()
    V = X * Y * Z
    recon = cuda.empty_like(d_raw)
    vbt.detect_keyframes(d_raw, prof, cuda.empty(((T + 31) // 32, V), dtype=cuda.int32, device="cuda"),
                         cuda.empty(V, dtype=cuda.int32, device="cuda"), cuda.empty(V, dtype=cuda.uint8, device="cuda"),
                         recon)
    L = ((X + 7) // 8) * ((Y + 7) // 8) * ((Z + 7) // 8)
    leaves = cuda.arange(L, dtype=cuda.int32, device="cuda")
    C = COARSE_RES ** 3
    z = lambda *s, dt=cuda.int32: cuda.zeros(s, dtype=dt, device="cuda")  # noqa: E731
    co = [z(L, C), z(L, C, 8, dt=cuda.uint8), z(L, C * T, dt=cuda.int16), z(L, C * T, dt=cuda.float32), z(L),
          z(L, dt=cuda.uint8), z(L, C, T, dt=cuda.float32)]
    vbt.coarse_fit(recon, dims, leaves, cprof, *co)
    rh = recon.cpu().numpy()
    ocp = pipe.levelset_profiles()[1] if levelset else pipe.control_profile()
    peak = float(max(F32(1e-6), F32(F32(raw.max()) - F32(raw.min()))))
    if levelset:
        F = 512
        fi = [z(L, 80, dt=cuda.uint8), z(L, F), z(L, F, 8, dt=cuda.uint8), z(L, F * T, dt=cuda.int16),
              z(L, F * T, dt=cuda.float32), z(L), z(L), z(L, dt=cuda.uint8)]
        vbt.shell_fit(recon, dims, leaves, cprof, co[6], True, 3.0, 1.5, float(F32(0.1) * F32(1.0)), 0.0, *fi)
        occ, desc, bins, kf, kv, cnt, act, req = (t.cpu().numpy() for t in fi)
        shells = 0
        for li in range(L):
            lt, ext, _ = _leaf_series(rh, dims, li)
            fit = oracle.coarse_fit(lt, ext, ocp)
            sh = oracle.shell_fit(lt, ext, ocp, fit["grid"], True, 3.0, 1.5, float(F32(0.1) * F32(1.0)), 0.0)
            a = int(sh["active"])
            assert int(act[li]) == a, li
            if a == 0:
                continue
            shells += 1
            n = int(cnt[li])
            assert np.array_equal(occ[li], np.asarray(sh["occupancy"], np.uint8)), li
            assert np.array_equal(desc[li, :a].view(np.uint32), sh["desc"]), li
            assert np.array_equal(bins[li, :a, :4], sh["bins"][:, :4]), li
            assert n == sh["key_frames"].size, li
            assert np.array_equal(kf[li, :n].view(np.uint16), sh["key_frames"]), li
            assert np.array_equal(kv[li, :n].view(np.uint32), sh["key_values"].view(np.uint32)), li
            assert int(req[li]) == sh["required_max_local"], li
        assert shells >= 4
    else:
        F = 216
        fi = [z(L, F), z(L, F, 8, dt=cuda.uint8), z(L, F * T, dt=cuda.int16), z(L, F * T, dt=cuda.float32), z(L),
              z(L, dt=cuda.uint8), z(L, F, T, dt=cuda.float32)]
        vbt.fine6_fit(recon, dims, leaves, cprof, co[6], *fi)
        md = z(L, dt=cuda.uint8)
        cut, band = F32(prof.render_cutoff), F32(prof.cutoff_band)
        vbt.route_density(d_raw, dims, leaves, co[6], fi[6], peak, float(F32(cut - band)), float(F32(cut + band)), md)
        desc, bins, kf, kv, cnt, req, grid = (t.cpu().numpy() for t in fi)
        mode = md.cpu().numpy()
        for li in range(L):
            lt, ext, base = _leaf_series(rh, dims, li)
            fit = oracle.coarse_fit(lt, ext, ocp)
            f6 = oracle.fine6_fit(lt, ext, ocp, fit["grid"])
            n = int(cnt[li])
            assert np.array_equal(desc[li].view(np.uint32), f6["desc"]), li
            assert np.array_equal(bins[li], f6["bins"]), li
            assert n == f6["key_frames"].size, li
            assert np.array_equal(kf[li, :n].view(np.uint16), f6["key_frames"]), li
            assert np.array_equal(kv[li, :n].view(np.uint32), f6["key_values"].view(np.uint32)), li
            assert int(req[li]) == f6["required_max_local"], li
            assert np.array_equal(grid[li].view(np.uint32), f6["grid"].view(np.uint32)), li
            assert int(mode[li]) == pipe.route_leaf(raw, base, fit["grid"], f6["grid"], peak), li
