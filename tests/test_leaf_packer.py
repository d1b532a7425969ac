"""VBTPACK4 leaves packed on the GPU from their control streams (vbt_pack_leaves).

Every leaf of reference-written assets, unpacked into control streams (tests/leafstreams.py, pinned
on the reference's own packer by tests/test_leaf_packer_oracle.py), is packed again on the GPU:
the offsets and the payload must equal the file's, word for word.  Seeded random leaves of every
mode with both keyframe codecs are compared with the reference packer (oracle/_ref), and the
reference's rejections (invalid stream, FP16 frame above 255) and the call's own checks are
exercised.
"""
import os

import numpy as np
import pytest

from conftest import ASSETS, golden_asset
from leafstreams import LEAF_DTYPE, streams_from_file

pytestmark = pytest.mark.gpu


def gpu_pack(vbt, cuda, leaves, arr, capacity=None):
    t = lambda a, dt: cuda.from_numpy(np.ascontiguousarray(a).view(dt)).cuda() if a.size else None  # noqa: E731
    d_leaves = cuda.from_numpy(leaves.view(np.uint8).copy()).cuda()
    n = leaves.shape[0]
    d_off = cuda.full((n + 1,), -1, dtype=cuda.int32, device="cuda")
    # an upper bound: header, prefix, occupancy and section padding per leaf, plus the rows
    words = int(capacity if capacity is not None else 16 + 28 * n + arr["descriptors"].size + arr["bins"].size // 4 +
                2 * arr["key_frames"].size)
    d_pay = cuda.full((max(words, 1),), -1, dtype=cuda.int32, device="cuda")
    total = vbt.pack_leaves(d_leaves, t(arr["descriptors"], np.int32), t(arr["bins"], np.uint8),
                            t(arr["key_frames"], np.int16), t(arr["key_values"], np.float32),
                            t(arr["occupancy"], np.uint8), d_off, d_pay)
    return d_off.cpu().numpy().view(np.uint32), d_pay.cpu().numpy().view(np.uint32)[:total]


def render_assets():
    out = [golden_asset("tiny_density"), golden_asset("tiny_levelset")]
    for n in ("cfg1_blobs", "cfg4_sdf_small", "cfg2_plume", "mix_sdf", "mix_fire_density"):
        p = os.path.join(ASSETS, n + ".vbtp")
        if os.path.exists(p):
            out.append(p)
    return out


@pytest.mark.parametrize("path", render_assets(), ids=os.path.basename)
def test_rebuild_asset_payload(vbt, cuda, oracle, path):
    leaves, arr, blocks = streams_from_file(path, oracle)
    off, pay = gpu_pack(vbt, cuda, leaves, arr)
    raw = open(path, "rb").read()
    h = np.frombuffer(raw[8:52], np.uint32)
    off_at = 52 + 4 * int(h[10])
    want_off = np.frombuffer(raw[off_at:off_at + 4 * (int(h[8]) + 1)], np.uint32)
    want_pay = np.frombuffer(raw[off_at + 4 * (int(h[8]) + 1):], np.uint32)
    assert np.array_equal(off, want_off)
    assert np.array_equal(pay, want_pay)


def random_leaves(rng, n):
    """Seeded leaves of every mode, both codecs, valid streams."""
    leaves = np.zeros(n, LEAF_DTYPE)
    desc, bins, frames, values, occ = [], [], [], [], []
    nc = nk = 0

    def stream(controls, nbins, keys, codec, max_local):
        nonlocal nc, nk
        start = rng.integers(0, max(keys, 1), controls)
        count = np.minimum(rng.integers(0, nbins * max_local + 1, controls), keys - start)
        count = np.where(keys == 0, 0, count)
        start = np.where(keys == 0, 0, start)
        reserved = rng.integers(0, max_local + 1, controls)
        desc.append((start | (count << 16) | (reserved << 24)).astype(np.uint32))
        b = np.zeros((controls, 8), np.uint8)
        b[:, :nbins] = rng.integers(0, 256, (controls, nbins))
        bins.append(b)
        hi = 65535 if codec == 1 else 255
        frames.append(rng.integers(0, hi + 1, keys).astype(np.uint16))
        v = rng.normal(0, 1, keys) * 10.0 ** rng.integers(-9, 6, keys)
        values.append(v.astype(np.float32))
        first = (nc, nk)
        nc += controls
        nk += keys
        return first

    for i in range(n):
        mode = int(rng.integers(0, 4))
        cc, fc = int(rng.integers(0, 2)), int(rng.integers(0, 2))
        word = mode | (cc << 2) | (fc << 4) | (4 << 6) | ((6 if mode == 3 else 0) << 9)
        leaves[i]["header"] = word
        if mode == 0:
            continue
        ckf, fkf = int(rng.integers(0, 200)), int(rng.integers(0, 200)) if mode != 1 else 0
        ml = int(rng.integers(1, 6))
        leaves[i]["coarse_kf"], leaves[i]["fine_kf"] = ckf, fkf
        leaves[i]["coarse_control"], leaves[i]["coarse_key"] = stream(64, 8, ckf, cc, ml)
        leaves[i]["coarse_max_local"] = ml
        if mode == 3:
            leaves[i]["fine_control"], leaves[i]["fine_key"] = stream(216, 8, fkf, fc, ml)
            leaves[i]["fine_max_local"] = ml
        elif mode == 2:
            mask = (rng.random(512) < rng.uniform(0.02, 0.5)).astype(np.uint8)
            mask[int(rng.integers(0, 512))] = 1
            sec = np.zeros(80, np.uint8)
            sec[:64] = np.packbits(mask, bitorder="little")
            leaves[i]["occupancy"] = len(occ)
            occ.append(sec)
            leaves[i]["fine_control"], leaves[i]["fine_key"] = stream(int(mask.sum()), 4, fkf, fc, ml)
            leaves[i]["fine_max_local"] = ml
    arr = dict(descriptors=np.concatenate(desc), bins=np.concatenate(bins).reshape(-1),
               key_frames=np.concatenate(frames), key_values=np.concatenate(values),
               occupancy=np.concatenate(occ) if occ else np.zeros(0, np.uint8))
    return leaves, arr


def test_random_leaves_against_reference(vbt, cuda, reference):
    from oracle.oracle import pack_payload
    from test_leaf_packer_oracle import ref_build, ref_stream
    rng = np.random.default_rng(8)
    leaves, arr = random_leaves(rng, 600)
    blocks = []
    for l in leaves:
        word = int(l["header"])
        mode = word & 3
        if mode == 0:
            blocks.append(ref_build(reference, word, 0, 0, b"", b"", None))
            continue
        coarse = ref_stream(reference, arr, int(l["coarse_control"]), 64, 8, int(l["coarse_key"]), int(l["coarse_kf"]),
                            (word >> 2) & 3, int(l["coarse_max_local"]))
        fine, occ = b"", None
        if mode == 3:
            fine = ref_stream(reference, arr, int(l["fine_control"]), 216, 8, int(l["fine_key"]), int(l["fine_kf"]),
                              (word >> 4) & 3, int(l["fine_max_local"]))
        elif mode == 2:
            occ = arr["occupancy"][80 * int(l["occupancy"]):80 * int(l["occupancy"]) + 80].tobytes()
            act = int(np.unpackbits(np.frombuffer(occ[:64], np.uint8)).sum())
            fine = ref_stream(reference, arr, int(l["fine_control"]), act, 4, int(l["fine_key"]), int(l["fine_kf"]),
                              (word >> 4) & 3, int(l["fine_max_local"]))
        blocks.append(ref_build(reference, word, int(l["coarse_kf"]), int(l["fine_kf"]), coarse, fine, occ))
    want_off, want_pay = pack_payload(blocks)
    off, pay = gpu_pack(vbt, cuda, leaves, arr)
    assert np.array_equal(off, want_off) and np.array_equal(pay, want_pay)
    assert {int(w) & 3 for w in leaves["header"]} == {0, 1, 2, 3}


def test_rejections(vbt, cuda):
    rng = np.random.default_rng(3)
    leaves, arr = random_leaves(rng, 40)
    k = int(np.flatnonzero((leaves["header"] & 3) == 1)[0])

    def expect(lv, a, fragment, status=40):
        with pytest.raises(vbt.VbtError) as e:
            gpu_pack(vbt, cuda, lv, a)
        assert e.value.status == status and fragment in str(e.value), str(e.value)

    bad = {key: v.copy() for key, v in arr.items()}
    c0 = int(leaves[k]["coarse_control"])
    bad["descriptors"][c0] = 0xFFFF | (1 << 16)                 # keyStart + keyCount beyond the keys
    expect(leaves, bad, "invalid render temporal control stream")
    lv = leaves.copy()
    lv[k]["header"] = (int(lv[k]["header"]) & ~0xC)             # FP16 coarse keys
    bad = {key: v.copy() for key, v in arr.items()}
    if lv[k]["coarse_kf"] > 0:
        bad["key_frames"][int(lv[k]["coarse_key"])] = 300
        expect(lv, bad, "fp16 keyframe frame exceeds uint8 range")
    lv = leaves.copy()
    lv[k]["coarse_control"] = arr["descriptors"].size            # rows beyond the arrays
    expect(lv, arr, "stream rows outside")
    with pytest.raises(vbt.VbtError) as e:                       # payload buffer too small
        gpu_pack(vbt, cuda, leaves, arr, capacity=8)
    assert e.value.status == 43
