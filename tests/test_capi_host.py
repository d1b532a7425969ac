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
