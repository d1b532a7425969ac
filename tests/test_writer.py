"""The VBTPACK4 writer's payload half on the GPU (vbt_pack_payload) against the restatement of
writeRenderTemporalProbeFile's loop (oracle.pack_payload): word offsets and zero-padded payload,
bit for bit.  Each asset is also rebuilt from its own leaf blocks into the identical file."""
import os

import numpy as np
import pytest

from conftest import ASSETS, golden_asset

pytestmark = pytest.mark.gpu


def gpu_pack(vbt, cuda, blocks):
    lens = np.array([len(b) for b in blocks], np.int64)
    boff = np.zeros(len(blocks) + 1, np.int64)
    boff[1:] = np.cumsum(lens)
    flat = np.frombuffer(b"".join(bytes(b) for b in blocks) or b"\0", np.uint8)
    d_blocks = cuda.from_numpy(flat.copy()).cuda()
    d_boff = cuda.from_numpy(boff).cuda()
    d_off = cuda.zeros(len(blocks) + 1, dtype=cuda.int32, device="cuda")
    cap = int((boff[-1] + 3 * len(blocks)) // 4 + 1)
    d_pay = cuda.full((cap,), -1, dtype=cuda.int32, device="cuda")
    total = vbt.pack_payload(d_blocks, d_boff, d_off, d_pay)
    return d_off.cpu().numpy().view(np.uint32), d_pay.cpu().numpy().view(np.uint32)[:total]


def test_random_blocks(vbt, cuda):
    from oracle.oracle import pack_payload
    rng = np.random.default_rng(4)
    for n in (1, 7, 1000, 20000):
        lens = rng.integers(0, 90, n)
        lens[rng.random(n) < 0.1] = 0                       # EMPTY-like zero-length blocks
        blocks = [rng.integers(0, 256, int(k), dtype=np.uint8).tobytes() for k in lens]
        off, pay = gpu_pack(vbt, cuda, blocks)
        want_off, want_pay = pack_payload(blocks)
        assert np.array_equal(off, want_off) and np.array_equal(pay, want_pay), n


def asset_paths():
    out = [golden_asset(n) for n in ("tiny_density", "tiny_levelset", "sci_small")]
    for n in ("cfg1_blobs", "cfg4_sdf_small", "cfg2_plume"):
        p = os.path.join(ASSETS, n + ".vbtp")
        if os.path.exists(p):
            out.append(p)
    return out


@pytest.mark.parametrize("path", asset_paths(), ids=os.path.basename)
def test_rebuild_asset(vbt, cuda, path):
    raw = open(path, "rb").read()
    h = np.frombuffer(raw[8:52], np.uint32)
    leaf_count, scale_count = int(h[8]), int(h[10])
    off_at = 52 + 4 * scale_count
    offsets = np.frombuffer(raw[off_at:off_at + 4 * (leaf_count + 1)], np.uint32)
    pay_at = off_at + 4 * (leaf_count + 1)
    blocks = [raw[pay_at + 4 * int(offsets[i]):pay_at + 4 * int(offsets[i + 1])] for i in range(leaf_count)]
    off, pay = gpu_pack(vbt, cuda, blocks)
    rebuilt = raw[:off_at] + off.tobytes() + pay.tobytes()
    assert rebuilt == raw


def test_capacity_is_checked(vbt, cuda):
    d_blocks = cuda.zeros(64, dtype=cuda.uint8, device="cuda")
    d_boff = cuda.tensor([0, 30, 64], dtype=cuda.int64, device="cuda")
    d_off = cuda.zeros(3, dtype=cuda.int32, device="cuda")
    small = cuda.zeros(4, dtype=cuda.int32, device="cuda")
    with pytest.raises(vbt.VbtError) as ei:
        vbt.pack_payload(d_blocks, d_boff, d_off, small)
    assert ei.value.status == 43
