"""Pin the oracle (the C restatement in oracle/vbt_oracle.c) to the reference.

CPU only.  The oracle must reproduce, bit for bit, every output the reference produced on the
golden fixtures (tests/golden/make_golden.py): the known-answer constructions of the reference's
own tests/temporal_decode_tests.cpp, tests/render_temporal_payload_tests.cpp and
tests/vbt_file_tests.cpp, and the reference's frames of three small synthetic assets.  Where the
compiled reference (oracle/_ref) is present it is also compared directly on every asset.
"""
import json
import os

import numpy as np
import pytest

from conftest import ASSETS, GOLDEN, golden_asset

ERRORS = {
    1: "render temporal leaf bytes too small", 2: "render temporal leaf prefix missing",
    3: "render temporal leaf shorter than computed layout", 4: "render temporal shell occupancy is out of bounds",
    5: "render temporal shell group prefix is inconsistent", 6: "render temporal shell mode contains no active voxels",
    7: "render temporal shell residual stream is out of bounds", 8: "render temporal shell leaf contains trailing bytes",
}


def load_streams():
    z = np.load(os.path.join(GOLDEN, "streams.npz"))
    meta, blob, ts, ref, brute = z["meta"], z["bytes"], z["t"], z["ref"], z["brute"]
    pos = 0
    for codec, bins, frames, kf, nbytes, off, nt in meta:
        yield (int(codec), int(bins), int(frames), int(kf), blob[off:off + nbytes], ts[pos:pos + nt],
               ref[pos:pos + nt], brute[pos:pos + nt])
        pos += nt


def test_streams_match_reference_bit_exact(oracle):
    """tests/temporal_decode_tests.cpp: both codecs, 4/8 bins, dense/sparse keys, corrupted hints,
    t from -2 to T+2; the oracle equals the reference's decoded value bit for bit and the
    brute-force lower_bound + lerp within the reference test's 2e-6."""
    n = 0
    for codec, bins, frames, kf, stream, ts, ref, brute in load_streams():
        got = np.array([oracle.decode_control(stream, codec, 1, bins, kf, stream.size, frames, 0, int(t))[1]
                        for t in ts], np.float32)
        assert np.array_equal(got.view(np.uint32), ref.view(np.uint32)), (codec, bins, frames)
        assert np.all(np.abs(got - brute) <= 2e-6)
        n += 1
    assert n == 384


def test_shell_leaf_matches_reference(oracle):
    """tests/temporal_decode_tests.cpp:68-101: Mode2 residual on voxels {0,63,64,255,511}."""
    z = np.load(os.path.join(GOLDEN, "shell_leaf.npz"))
    leaf, ts, vals, frames = z["leaf"], z["t"], z["values"], int(z["frames"])
    for i, t in enumerate(ts):
        for v in range(512):
            st, x = oracle.shell_voxel(leaf, frames, v, int(t))
            assert st == 0
            assert np.float32(x).view(np.uint32) == vals[i, v].view(np.uint32)
        st, full = oracle.decode_leaf(leaf, frames, int(t))
        assert st == 0 and np.array_equal(full.view(np.uint32), z["full"][i].view(np.uint32))


def test_payload_cases_match_reference(oracle):
    """tests/render_temporal_payload_tests.cpp:65-114: voxel stride, Mode2 parse, corruptions."""
    cases = np.load(os.path.join(GOLDEN, "payload_cases.npz"))
    verdicts = json.load(open(os.path.join(GOLDEN, "payload_cases.json")))
    for name, want in verdicts.items():
        st, view = oracle.parse_leaf(cases[name])
        if want["error"] is None:
            assert st == 0
            assert view.shell_active == want["view"][12]
            assert view.shell_residual_off == want["view"][13]
            assert view.shell_residual_bytes == want["view"][14]
            assert view.total == want["view"][11]
        else:
            assert st != 0 and ERRORS[st] == want["error"], (name, st)
    # voxel index keeps the fixed 8^3 stride (:67-70): (lz*8 + ly)*8 + lx
    assert (1 * 8 + 0) * 8 + 0 == 64 and (1 * 8 + 2) * 8 + 2 == 82


def test_reader_cases(oracle):
    """tests/vbt_file_tests.cpp:86-131, by message fragment."""
    cases = json.load(open(os.path.join(GOLDEN, "reader", "cases.json")))
    for name, frag in cases.items():
        path = os.path.join(GOLDEN, "reader", name + ".vbtp")
        if frag is None:
            f = oracle.load(path)
            assert f.leaf_count == 1 and list(f.offsets()) == [0, 1] and list(f.payload()) == [0]
        else:
            with pytest.raises(RuntimeError, match=frag):
                oracle.load(path)


GOLDEN_NAMES = ["tiny_density", "tiny_levelset", "sci_small", "sci_coarse", "sci_dense", "sci_dense_tb"]


@pytest.mark.parametrize("name", GOLDEN_NAMES)
def test_golden_asset_frames(oracle, name):
    """Frames of six small synthetic assets (odd sizes: cropped boundary leaves; Mode2;
    scientific SparseEvents, CoarseOnly, DenseGrid3/4 with the per-frame BFP residual and with
    the DCT temporal-basis residual) equal the reference's frames bit for bit."""
    f = oracle.load(golden_asset(name))
    z = np.load(os.path.join(GOLDEN, "assets", name + ".npz"))
    for t, want in zip(z["t"], z["frames"]):
        got = f.frame(int(t))
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), (name, int(t))


def _asset_paths():
    out = [golden_asset(n) for n in GOLDEN_NAMES]
    for n in ("cfg1_blobs", "cfg4_sdf_small", "sci_64", "sci_modes"):
        p = os.path.join(ASSETS, n + ".vbtp")
        if os.path.exists(p):
            out.append(p)
    return out


@pytest.mark.parametrize("path", _asset_paths(), ids=lambda p: os.path.basename(p))
def test_oracle_equals_compiled_reference(oracle, reference, path):
    """The oracle against the reference decoder compiled from its own sources, every frame."""
    f = oracle.load(path)
    h = reference.load(path)
    try:
        ts = range(f.frames) if f.profile == 2 else range(-1, f.frames + 1)
        for t in ts:
            a = f.frame(t, threads=8)
            b = reference.frame(h, f.dims, t, f.profile, threads=8)
            assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), (path, t)
        if f.profile == 2:
            rng = np.random.default_rng(3)
            q = np.stack([rng.integers(0, d, 4096) for d in f.dims] + [rng.integers(0, f.frames, 4096)], 1)
            assert np.array_equal(f.query(q).view(np.uint32), reference.sci_query(h, q).view(np.uint32))
    finally:
        reference.free(h)


def test_page_table_rank_is_ascending(oracle):
    """Canonical page table: ascending exclusive rank of non-EMPTY leaves, 0xFFFFFFFF for EMPTY
    (VBTStudio/frontend/shaders/vbt_active_index.comp:28-57 without its atomic ordering)."""
    f = oracle.load(golden_asset("tiny_levelset"))
    compact, n = f.page_table()
    off, pay = f.offsets(), f.payload()
    active = (pay[off[:-1]] & 3) != 0
    assert n == int(active.sum())
    assert np.array_equal(compact[active], np.arange(n, dtype=np.uint32))
    assert np.all(compact[~active] == 0xFFFFFFFF)


def test_corrupted_leaves_statuses(oracle, reference):
    """Byte-flip fuzz on a Mode2 + Grid4 asset: the oracle's verdict (error or not) and decoded
    values equal the reference's on every corrupted leaf."""
    f = oracle.load(golden_asset("tiny_levelset"))
    off, pay = f.offsets(), f.payload()
    raw = pay.view(np.uint8)
    rng = np.random.default_rng(7)
    ERR = {v: k for k, v in ERRORS.items()}
    checked = 0
    for leaf in range(f.leaf_count):
        b0, b1 = 4 * int(off[leaf]), 4 * int(off[leaf + 1])
        for _ in range(6):
            leaf_bytes = raw[b0:b1].copy()
            k = int(rng.integers(0, leaf_bytes.size))
            leaf_bytes[k] ^= np.uint8(1 << int(rng.integers(0, 8)))
            for t in (0, 5, 11):
                err, want = reference.decode_leaf(leaf_bytes, f.frames, t)
                st, got = oracle.decode_leaf(leaf_bytes, f.frames, t)
                if err is None:
                    assert st == 0 and np.array_equal(got.view(np.uint32), want.view(np.uint32))
                else:
                    assert st != 0
                    if err in ERR:
                        assert st == ERR[err]
                checked += 1
    assert checked > 100


def test_pack_payload_restatement_rebuilds_reference_files():
    """oracle.pack_payload (writeRenderTemporalProbeFile's payload loop) reproduces the payload and
    offsets of files the reference encoder wrote."""
    from oracle.oracle import pack_payload
    for name in ("tiny_density", "tiny_levelset"):
        raw = open(os.path.join(GOLDEN, "assets", name + ".vbtp"), "rb").read()
        h = np.frombuffer(raw[8:52], np.uint32)
        leaf_count, scale_count = int(h[8]), int(h[10])
        off_at = 52 + 4 * scale_count
        offsets = np.frombuffer(raw[off_at:off_at + 4 * (leaf_count + 1)], np.uint32)
        pay_at = off_at + 4 * (leaf_count + 1)
        blocks = [raw[pay_at + 4 * int(offsets[i]):pay_at + 4 * int(offsets[i + 1])] for i in range(leaf_count)]
        off, pay = pack_payload(blocks)
        assert raw[:off_at] + off.tobytes() + pay.tobytes() == raw
