"""C-ABI host checks that need no GPU: the library loads, exports every declared entry point,
and its host-side VBTPACK4 reader validation follows tests/vbt_file_tests.cpp."""
import ctypes as C
import json
import os
import re

import pytest

from conftest import GOLDEN, ROOT


def declared_symbols():
    out = []
    for name in os.listdir(os.path.join(ROOT, "include")):
        if name.endswith(".h"):
            text = open(os.path.join(ROOT, "include", name)).read()
            out += re.findall(r"^\s*(?:const\s+)?\w+\**\s+\**(vbt_\w+)\s*\(", text, re.M)
    return sorted(set(out))


def test_library_exports_every_declared_symbol(vbt):
    syms = declared_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(vbt.lib(), s), s
    assert set(vbt.EXPORTS) <= set(syms)


def test_reader_validation_matches_reference_cases(vbt):
    cases = json.load(open(os.path.join(GOLDEN, "reader", "cases.json")))
    for name, frag in cases.items():
        data = open(os.path.join(GOLDEN, "reader", name + ".vbtp"), "rb").read()
        if frag is None:
            h = vbt.validate_file_image(data)
            assert h.version == 4 and h.leaf_count == 1
        else:
            with pytest.raises(vbt.VbtError) as ei:
                vbt.validate_file_image(data)
            assert ei.value.status == 41 and frag in ei.value.message, (name, ei.value.message)


def test_reader_validation_on_assets(vbt):
    for n in ("tiny_density", "tiny_levelset", "sci_small"):
        data = open(os.path.join(GOLDEN, "assets", n + ".vbtp"), "rb").read()
        h = vbt.validate_file_image(data)
        assert h.leaf_size == 8 and h.version == 4


def test_status_strings_match_reference_messages(vbt):
    assert vbt.status_string(5) == "render temporal shell group prefix is inconsistent"
    assert vbt.status_string(12) == "render temporal keyframe range out of bounds"


def test_no_gpu_fails_loudly(vbt):
    """Without a usable device, loading an asset reports VBT_STATUS_CUDA (there is no CPU path)."""
    if vbt.device_count() > 0:
        pytest.skip("a GPU is present")
    with pytest.raises(vbt.VbtError) as ei:
        vbt.Asset(os.path.join(GOLDEN, "assets", "tiny_density.vbtp"))
    assert ei.value.status == 42


def test_encoder_and_writer_argument_checks(vbt):
    """The keyframe pass, coarse fit, leaf packer and samplers reject bad scalar arguments on the host,
    before any device work (the pointers below are never dereferenced)."""
    L = vbt.lib()
    fake = C.c_void_p(0x10000)
    prof = vbt.KeyframeProfile()
    z = C.c_void_p(None)

    def kf(series, frames, fstride, sstride):
        return L.vbt_detect_keyframes(fake, series, frames, fstride, sstride, C.byref(prof), fake, fake, fake, z, z,
                                      z, z)
    assert kf(10, 0, 10, 1) == 40                      # no frames
    assert kf(10, 1025, 10, 1) == 43                   # above 1024 frames
    assert kf(10, 8, 5, 1) == 40                       # frame-major stride shorter than the series
    assert kf(10, 8, 1, 7) == 40                       # time-fastest stride shorter than the frames
    assert kf(10, 8, 2, 3) == 40                       # neither layout
    assert L.vbt_detect_keyframes(fake, 10, 8, 10, 1, None, fake, fake, fake, z, z, z, z) == 40

    def cf(frames, fstride, dims=(16, 16, 16)):
        return L.vbt_coarse_fit(fake, *dims, frames, fstride, fake, 4, C.byref(prof), fake, fake, fake, fake, fake,
                                fake, z, z)
    assert cf(0, 4096) == 40
    assert cf(2000, 4096) == 43
    assert cf(8, 100) == 40                            # frame stride shorter than the volume
    assert cf(8, 4096, (0, 16, 16)) == 40

    total = C.c_uint64()
    assert L.vbt_pack_leaves(fake, 4, fake, fake, 8, fake, fake, 8, z, 0, None, fake, 64, C.byref(total), z) == 40
    assert L.vbt_pack_leaves(fake, 4, None, fake, 8, fake, fake, 8, z, 0, fake, fake, 64, C.byref(total), z) == 40
    assert L.vbt_pack_leaves(fake, 4, fake, C.c_void_p(0x10001), 8, fake, fake, 8, z, 0, fake, fake, 64,
                             C.byref(total), z) == 40   # bin rows not 4-byte aligned
    assert L.vbt_pack_payload(fake, None, 4, fake, fake, 64, C.byref(total), z) == 40

    sp = vbt.SampleParams()
    assert L.vbt_smoke_sample_rays(None, C.byref(sp), fake, 4, fake, z) == 40
    assert L.vbt_sample_rays(None, fake, C.byref(sp), fake, 4, fake, z) == 40
    res = (C.c_uint64 * 2)()
    assert L.vbt_selftest_keyframe_division(0, res, 0) == 40
    assert L.vbt_selftest_keyframe_division(70000, res, 0) == 40
