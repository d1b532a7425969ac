#!/usr/bin/env python3
"""Generate the golden fixtures under tests/golden/ from the reference decoder itself.

Runs in the development container only (it needs oracle/_ref/libvbtref.so, which
oracle/Makefile builds from the reference sources).  The fixtures restate the known-answer
constructions of the reference's own tests and record the reference's outputs on them:

  streams.npz      control streams built as tests/temporal_decode_tests.cpp:17-38 (makeStream)
                   builds them (values sin(0.19 t), FP16 pre-rounded for codec 0, keys at every
                   frame or at t = 0, T-1 and t % 13 == 7), for codecs {0, 1}, bins {4, 8}, a
                   spread of frame counts, bin hints {built, 0, 255}; packed by the reference's
                   packRenderTemporalControlStream; decoded by the reference at t = -2 .. T+2; and
                   the brute-force lower_bound + lerp expectation of :40-50.
  shell_leaf.npz   the Mode2 leaf of tests/temporal_decode_tests.cpp:68-101 (64-control coarse
                   stream, FP32 residual stream on voxels {0, 63, 64, 255, 511}) built by the
                   reference's buildRenderTemporalPackedLeafBytes, and the reference's
                   decodeRenderTemporalLeafShellVoxelValue for all 512 voxels x t = -1 .. 101.
  payload_cases.npz  the Mode2 leaf of tests/render_temporal_payload_tests.cpp:39-63 and its four
                   corruptions (:81-114) with the reference parser's verdicts.
  reader/*.vbtp    the files of tests/vbt_file_tests.cpp:86-131 and the expected message fragments
                   (reader/cases.json).
  assets/*.vbtp    six small synthetic assets (tests/golden/make_assets.py; the three sci_* beyond
                   sci_small hold the CoarseOnly, DenseGrid3/4 and temporal-basis leaf modes) and
  assets/*.npz     the reference decoder's frames for every frame index -1 .. T.
"""
import json
import os
import shutil
import struct
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.oracle import Reference  # noqa: E402

FRAME_SET = [1, 2, 3, 4, 5, 7, 8, 9, 13, 14, 16, 24, 31, 33, 64, 96, 100, 101, 120, 127, 128, 200, 254, 255]


def make_stream(ref, frames, bins, codec, dense):
    """tests/temporal_decode_tests.cpp:17-38."""
    keys_f, keys_v = [], []
    for t in range(frames):
        if dense or t == 0 or t == frames - 1 or t % 13 == 7:
            v = np.float32(np.sin(np.float32(t) * np.float32(0.19)))
            if codec == 0:
                v = np.float32(ref.lib.vr_half_to_float(ref.lib.vr_float_to_half(float(v))))
            keys_f.append(t)
            keys_v.append(v)
    bin_index = []
    for b in range(bins):
        boundary = b * frames // bins
        idx = 0
        while idx < len(keys_f) and keys_f[idx] < boundary:
            idx += 1
        bin_index.append(0 if idx == 0 else idx - 1)
    return np.array(keys_f, np.uint32), np.array(keys_v, np.float32), np.array(bin_index, np.uint8)


def brute(keys_f, keys_v, frames, t):
    """tests/temporal_decode_tests.cpp:40-50 (lower_bound + lerp), in float32."""
    t = min(max(t, 0), frames - 1)
    hi = int(np.searchsorted(keys_f, t, side="left"))
    if hi == len(keys_f):
        return np.float32(keys_v[-1])
    if hi == 0 or keys_f[hi] == t:
        return np.float32(keys_v[hi])
    lo = hi - 1
    alpha = np.float32(np.float32(t - keys_f[lo]) / np.float32(keys_f[hi] - keys_f[lo]))
    return np.float32(keys_v[lo] * (np.float32(1) - alpha) + keys_v[hi] * alpha)


def gen_streams(ref):
    blobs, meta, ts, ref_vals, brute_vals = [], [], [], [], []
    for codec in (0, 1):
        for bins in (4, 8):
            for frames in FRAME_SET:
                for dense, hint in ((True, -1), (False, -1), (False, 0), (False, 255)):
                    kf, kv, bi = make_stream(ref, frames, bins, codec, dense)
                    if hint >= 0:
                        bi[:] = hint
                    desc = np.array([[0, len(kf), 1]], np.uint32)
                    packed = ref.pack_stream(codec, desc, bi, kf, kv, bins, max_local=255)
                    tt = np.arange(-2, frames + 3, dtype=np.int32)
                    rv = np.zeros(tt.size, np.float32)
                    for i, t in enumerate(tt):
                        err, v = ref.decode_control(packed, codec, 1, bins, len(kf), packed.size, frames, 0, int(t))
                        assert err is None, err
                        rv[i] = v
                    bv = np.array([brute(kf, kv, frames, int(t)) for t in tt], np.float32)
                    assert np.all(np.abs(rv - bv) <= 2e-6), (codec, bins, frames, dense, hint)
                    meta.append([codec, bins, frames, len(kf), packed.size, len(blobs and np.concatenate(blobs)) if blobs else 0, tt.size])
                    blobs.append(packed)
                    ts.append(tt)
                    ref_vals.append(rv)
                    brute_vals.append(bv)
    offs = np.cumsum([0] + [b.size for b in blobs])
    meta = np.array([[m[0], m[1], m[2], m[3], m[4], offs[i], m[6]] for i, m in enumerate(meta)], np.int64)
    np.savez_compressed(os.path.join(HERE, "streams.npz"), meta=meta, bytes=np.concatenate(blobs),
                        t=np.concatenate(ts), ref=np.concatenate(ref_vals), brute=np.concatenate(brute_vals))
    print("streams.npz:", len(blobs), "streams")


def gen_shell(ref):
    """tests/temporal_decode_tests.cpp:68-101."""
    frames = 101
    kf, kv, bi = make_stream(ref, frames, 8, 0, False)
    desc = np.tile(np.array([[0, len(kf), 1]], np.uint32), (64, 1))
    coarse = ref.pack_stream(0, desc, np.tile(bi, 64), kf, kv, 8, max_local=255)
    rkf, rkv, rbi = make_stream(ref, frames, 4, 1, True)
    voxels = [0, 63, 64, 255, 511]
    rdesc = np.tile(np.array([[0, len(rkf), 1]], np.uint32), (len(voxels), 1))
    residual = ref.pack_stream(1, rdesc, np.tile(rbi, len(voxels)), rkf, rkv, 4, max_local=255)
    mask = [0] * 8
    for v in voxels:
        mask[v // 64] |= 1 << (v % 64)
    prefix = [sum(1 for v in voxels if v < g * 64) for g in range(8)]
    occ = np.frombuffer(struct.pack("<8Q8H", *mask, *prefix), np.uint8)
    header = 2 | (0 << 2) | (1 << 4) | (4 << 6) | (0 << 9)   # Mode2, coarse FP16, fine FP32, coarse res 4
    leaf = ref.build_leaf(header, len(kf), len(rkf), coarse, residual, occ)
    tt = np.arange(-1, frames + 1, dtype=np.int32)
    vals = np.zeros((tt.size, 512), np.float32)
    for i, t in enumerate(tt):
        for v in range(512):
            err, x = ref.shell_voxel(leaf, frames, v, int(t))
            assert err is None, err
            vals[i, v] = x
    expect = np.zeros_like(vals)
    for i, t in enumerate(tt):
        b = brute(rkf, rkv, frames, int(t))
        for v in voxels:
            expect[i, v] = b
    assert np.all(np.abs(vals - expect) <= 2e-6)
    # the full leaf decode (coarse + residual, Mode2 clamp) at a few frames, 8^3 extent
    full = np.zeros((tt.size, 512), np.float32)
    for i, t in enumerate(tt):
        err, full[i] = ref.decode_leaf(leaf, frames, int(t))
        assert err is None, err
    np.savez_compressed(os.path.join(HERE, "shell_leaf.npz"), leaf=leaf, t=tt, values=vals, expect=expect,
                        full=full, frames=frames)
    print("shell_leaf.npz:", leaf.size, "bytes")


def gen_payload_cases(ref):
    """tests/render_temporal_payload_tests.cpp:39-114."""
    header = 2 | (0 << 2) | (0 << 4) | (1 << 6) | (0 << 9)   # Mode2, FP16/FP16, coarse res 1, fine res 0
    # coarse stream for res 1 and 0 keyframes: desc 4 + bins 8 + keys 0
    coarse = np.zeros(12, np.uint8)
    occ = np.frombuffer(struct.pack("<8Q8H", 1, 0, 1 << 5, 0, 0, 0, 0, 0, 0, 1, 1, 2, 2, 2, 2, 2), np.uint8)
    residual = np.zeros(2 * 4 + 2 * 4 + 8, np.uint8)
    valid = ref.build_leaf(header, 0, 2, coarse, residual, occ)
    err, view = ref.parse_leaf(valid)
    assert err is None and view[12] == 2 and view[13] + view[14] == valid.size
    occ_off = int(view[9])   # layout.fineOffset == occupancy offset
    cases = {"valid": valid}
    bad = valid.copy()
    bad[occ_off + 64 + 2: occ_off + 64 + 4] = 0
    cases["bad_prefix"] = bad
    cases["truncated"] = valid[:-4].copy()
    cases["trailing"] = np.concatenate([valid, np.zeros(4, np.uint8)])
    none = valid.copy()
    none[occ_off: occ_off + 80] = 0
    cases["no_active"] = none
    verdicts = {}
    for k, b in cases.items():
        err, v = ref.parse_leaf(b)
        verdicts[k] = {"error": err, "view": [int(x) for x in v]}
    np.savez(os.path.join(HERE, "payload_cases.npz"), **cases)
    with open(os.path.join(HERE, "payload_cases.json"), "w") as fh:
        json.dump(verdicts, fh, indent=1)
    print("payload_cases:", {k: v["error"] for k, v in verdicts.items()})


def write_vbt(path, width=8, height=8, depth=8, frames=4, version=4, leaf_count=1, offsets=(0, 1), payload=(0,),
              trailing=False):
    """tests/vbt_file_tests.cpp:33-63 writeFile."""
    with open(path, "wb") as fh:
        fh.write(b"VBTPACK4")
        fh.write(struct.pack("<11I", version, width, height, depth, frames, 8, 4, 0, leaf_count, 1, 0))
        fh.write(struct.pack(f"<{len(offsets)}I", *offsets))
        if payload:
            fh.write(struct.pack(f"<{len(payload)}I", *payload))
        if trailing:
            fh.write(b"\0")


def gen_reader_cases():
    d = os.path.join(HERE, "reader")
    os.makedirs(d, exist_ok=True)
    cases = {
        "valid": ({}, None),
        "bad_version": ({"version": 3}, "Unsupported VBTPACK4 version"),
        "bad_leaf_count": ({"width": 16}, "leafCount does not match"),
        "non_monotonic": ({"width": 16, "leaf_count": 2, "offsets": (0, 2, 1)}, "strictly increasing"),
        "empty_leaf": ({"offsets": (0, 0), "payload": ()}, "strictly increasing"),
        "trailing": ({"trailing": True}, "trailing bytes"),
        "truncated": ({"offsets": (0, 2)}, "truncated"),
    }
    for name, (kw, _) in cases.items():
        write_vbt(os.path.join(d, name + ".vbtp"), **kw)
    with open(os.path.join(d, "cases.json"), "w") as fh:
        json.dump({k: v[1] for k, v in cases.items()}, fh, indent=1)
    print("reader cases:", len(cases))


GOLDEN_ASSETS = ("tiny_density", "tiny_levelset", "sci_small", "sci_coarse", "sci_dense", "sci_dense_tb")


def gen_assets(ref, names=GOLDEN_ASSETS):
    d = os.path.join(HERE, "assets")
    os.makedirs(d, exist_ok=True)
    for name in names:
        src = os.path.join(ROOT, "assets", name + ".vbtp")
        if not os.path.exists(src):
            import subprocess
            subprocess.check_call([sys.executable, os.path.join(HERE, "make_assets.py"), name])
        dst = os.path.join(d, name + ".vbtp")
        shutil.copyfile(src, dst)
        raw = open(dst, "rb").read()
        dims = struct.unpack("<4I", raw[12:28])
        X, Y, Z, T = dims
        profile = struct.unpack("<I", raw[44:48])[0]
        h = ref.load(dst)
        ts = list(range(0, T)) if profile == 2 else list(range(-1, T + 1))
        frames = np.stack([ref.frame(h, (X, Y, Z), t, profile) for t in ts])
        ref.free(h)
        np.savez_compressed(os.path.join(d, name + ".npz"), t=np.array(ts, np.int32), frames=frames)
        print(name, os.path.getsize(dst), "bytes;", frames.shape)


QUERY_DIMS = [(20, 12, 17, 9), (256, 256, 256, 96), (1, 1, 1, 1), (8, 8, 8, 4), (100, 37, 64, 33)]
QUERY_SEEDS = [0, 7, 12345]
QUERY_COUNT = 513
DCT_LENGTHS = [1, 2, 3, 7, 24, 96, 128]


def gen_host_api(ref):
    """host_api.npz: the reference's generateQueries/fillLeafIndices/sortQueriesByLeaf
    (render/src/query_patterns.cpp:29-101) and dctEncodeKeep[Weighted]/dctDecodeAt
    (src/dct_codec.cpp:63-122) on seeded inputs."""
    qmeta, qgen, qsorted = [], [], []
    for dims in QUERY_DIMS:
        for pattern in range(4):
            for seed in QUERY_SEEDS:
                g, s = ref.generate_queries(dims, pattern, QUERY_COUNT, seed)
                qmeta.append(list(dims) + [pattern, seed, QUERY_COUNT])
                qgen.append(g)
                qsorted.append(s)
    rng = np.random.default_rng(5)
    dmeta, series, weights, coeffs, decoded = [], [], [], [], []
    for n in DCT_LENGTHS:
        for keep in sorted({1, 3, n, n + 2}):
            for weighted in (0, 1):
                s = (rng.standard_normal(n) * 3.0 + 1.0).astype(np.float32)
                w = rng.uniform(0.0, 2.0, n).astype(np.float32)
                w[rng.uniform(size=n) < 0.2] = 0.0
                c, d = ref.dct(s, keep, w if weighted else None)
                dmeta.append([n, keep, weighted, c.size])
                series.append(s)
                weights.append(w)
                coeffs.append(c)
                decoded.append(d)
    np.savez_compressed(os.path.join(HERE, "host_api.npz"), qmeta=np.array(qmeta, np.uint32),
                        qgen=np.concatenate(qgen), qsorted=np.concatenate(qsorted),
                        dmeta=np.array(dmeta, np.int32), series=np.concatenate(series),
                        weights=np.concatenate(weights), coeffs=np.concatenate(coeffs),
                        decoded=np.concatenate(decoded))
    print("host api cases:", len(qmeta), "query sets,", len(dmeta), "dct cases")


if __name__ == "__main__":
    r = Reference()
    if len(sys.argv) > 1:
        for name in sys.argv[1:]:
            globals()["gen_" + name](r) if name != "reader_cases" else gen_reader_cases()
        sys.exit(0)
    gen_streams(r)
    gen_shell(r)
    gen_payload_cases(r)
    gen_reader_cases()
    gen_assets(r)
    gen_host_api(r)
