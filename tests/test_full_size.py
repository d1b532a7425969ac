"""Configurations 3 and 4 at their stated sizes, decoded on the GPU and checked against the oracle.

The raw fields (36-64 GB of float32 each) are generated on the GPU from their seeds
(tests/golden/gpu_fields.py) and encoded there by the library's encoder chain (vbt_b200.encode,
byte-exact against the reference encoder in tests/test_gpu_encoder.py); the file image comes back
to the host, where the oracle (oracle/vbt_oracle.c) loads it from memory.

  config 4, the liquid level set, 512^3 x 120 with Mode2 shell leaves: the page table, and dense
            full frames at the first, a middle and the last frame bit for bit -- values and the
            signs of phi;
  config 3, the fire's density (EMPTY leaves outside the growing sphere) and temperature (the
            largest of the three fields: noise in every leaf), 384 x 384 x 512 x 120: the page
            table, the cache of three frames bit for bit, and a 16-frame tensor-core window within
            1e-6 of the field's range of the FP64 oracle.
"""
import os
import sys

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu
sys.path.insert(0, GOLDEN)


def encode(torch, slab, dims, levelset):
    from vbt_b200.encode import encode_render_temporal, file_image
    h, off, pay = encode_render_temporal(slab, dims, levelset=levelset)
    img = file_image(h, off, pay, pinned=True)
    del off, pay
    torch.cuda.empty_cache()
    return img


def test_config4_levelset_full_size(vbt, cuda, oracle):
    import gpu_fields as gf
    torch = cuda
    lv = gf.LevelSet(torch, **gf.LEVELSET_FULL, device="cuda")
    X, Y, Z = gf.LEVELSET_FULL["shape_xyz"]
    img = encode(torch, lv.slab, (X, Y, Z), True)
    a = vbt.Asset(data=img)
    of = oracle.load(image=img)
    assert (a.leaf_count, a.frames) == (262144, 120)
    a.build_page_table()
    compact, n = a.page_table()
    want_c, want_n = of.page_table()
    assert n == want_n == a.leaf_count                     # a level set has no EMPTY leaf
    assert np.array_equal(compact, want_c)
    modes = np.bincount(a.leaf_table()[:, 1] & 3, minlength=4)
    assert modes[2] > 0 and modes[0] == 0
    out = torch.empty((1, X * Y * Z), dtype=torch.float32, device="cuda")
    for t in (0, 61, 119):
        a.decode_frames([t], out)
        torch.cuda.synchronize()
        a.sync_status()
        got = out[0].cpu().numpy()
        want = of.frame(t).reshape(-1)
        assert np.array_equal(np.signbit(got), np.signbit(want)), t
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), t
    a.close()


@pytest.mark.parametrize("field", [0, 2], ids=["density", "temperature"])
def test_config3_fire_full_size(vbt, cuda, oracle, field):
    import gpu_fields as gf
    torch = cuda
    fire = gf.Fire(torch, **gf.FIRE_FULL, device="cuda")
    dims = gf.FIRE_FULL["shape_xyz"]
    img = encode(torch, lambda z0, z1: fire.slab(field, z0, z1), dims, False)
    del fire
    torch.cuda.empty_cache()
    a = vbt.Asset(data=img)
    of = oracle.load(image=img)
    assert (a.leaf_count, a.frames) == (147456, 120)
    a.build_page_table()
    compact, n = a.page_table()
    want_c, want_n = of.page_table()
    assert n == want_n and np.array_equal(compact, want_c)
    cache = torch.empty((1, n, 512), dtype=torch.float32, device="cuda")
    for t in (0, 57, 119):
        a.decode_cache([t], cache, frame_stride=n * 512)
        torch.cuda.synchronize()
        a.sync_status()
        got = cache[0].cpu().numpy()
        want = of.cache(t)
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), t
    W = 16
    win = torch.empty((W, n, 512), dtype=torch.float32, device="cuda")
    a.decode_window(48, W, win, frame_stride=n * 512)
    mx, rms, lo, hi = a.window_error(48, W, win, frame_stride=n * 512)
    a.sync_status()
    assert mx / (hi - lo) <= 1e-6, (mx, lo, hi)
    a.close()
