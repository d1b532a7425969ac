"""The allocation-free page table (vbt_build_page_table_noalloc), checked against the regular
entry point (vbt_build_page_table through an asset) on two calls in a row.

The allocation-free variant exists for callers that may not let the library allocate device
memory -- hosts that hand out every buffer from their own pool, or frame loops that cannot afford
cudaMalloc's device synchronisation -- so here the test itself owns every buffer: the offsets and
payload of the file image, the outputs, and nothing else is created by the library.  This file is
collected last on purpose.
"""
import os
import struct

import numpy as np
import pytest

from conftest import ASSETS, golden_asset

pytestmark = pytest.mark.gpu


def image_parts(path):
    raw = open(path, "rb").read()
    hdr = struct.unpack("<11I", raw[8:52])
    leaf_count, profile, scale_count = hdr[8], hdr[9], hdr[10]
    off0 = 52 + 4 * scale_count
    offsets = np.frombuffer(raw, np.uint32, leaf_count + 1, off0)
    payload = np.frombuffer(raw, np.uint32, offset=off0 + 4 * (leaf_count + 1))
    return offsets, payload, leaf_count, profile


def paths():
    out = [golden_asset(n) for n in ("tiny_density", "tiny_levelset", "sci_small")]
    for n in ("cfg1_blobs", "cfg4_sdf_small", "cfg2_plume"):
        p = os.path.join(ASSETS, n + ".vbtp")
        if os.path.exists(p):
            out.append(p)
    return out


def expected(vbt, path):
    a = vbt.Asset(path)
    compact, n = a.page_table()
    a.close()
    active = np.zeros(n, np.uint32)
    ranked = compact != 0xFFFFFFFF
    active[compact[ranked]] = np.flatnonzero(ranked).astype(np.uint32)
    return compact, n, active


@pytest.mark.parametrize("path", paths(), ids=os.path.basename)
def test_noalloc_page_table_matches_regular_entry_point(vbt, cuda, path):
    offsets, payload, leaf_count, profile = image_parts(path)
    want_compact, want_n, want_active = expected(vbt, path)
    d_off = cuda.from_numpy(offsets.view(np.int32).copy()).cuda()
    d_pay = cuda.from_numpy(payload.view(np.int32).copy()).cuda()
    d_compact = cuda.empty(leaf_count, dtype=cuda.int32, device="cuda")
    d_active = cuda.empty(leaf_count, dtype=cuda.int32, device="cuda")
    d_count = cuda.empty(1, dtype=cuda.int32, device="cuda")
    for call in range(2):
        d_compact.fill_(-7)
        d_active.fill_(-7)
        d_count.fill_(-7)
        vbt.build_page_table_noalloc(d_off, d_pay, payload.size, leaf_count, profile, d_compact, d_active, d_count)
        cuda.cuda.synchronize()
        n = int(d_count.cpu().numpy().view(np.uint32)[0])
        assert n == want_n, (call, n, want_n)
        assert np.array_equal(d_compact.cpu().numpy().view(np.uint32), want_compact), call
        assert np.array_equal(d_active.cpu().numpy().view(np.uint32)[:n], want_active), call


def test_noalloc_rejects_too_many_leaves(vbt, cuda):
    d = cuda.zeros(16, dtype=cuda.int32, device="cuda")
    with pytest.raises(vbt.VbtError) as ei:
        vbt.build_page_table_noalloc(d, d, 16, (1 << 24) + 1, 1, d, d, d)
    assert ei.value.status == 43 and "16777216" in ei.value.message


def test_noalloc_rejects_unknown_profile(vbt, cuda):
    d = cuda.zeros(16, dtype=cuda.int32, device="cuda")
    for profile in (3, 7):
        with pytest.raises(vbt.VbtError) as ei:
            vbt.build_page_table_noalloc(d, d, 16, 4, profile, d, d, d)
        assert ei.value.status == 40 and "profile type" in ei.value.message
