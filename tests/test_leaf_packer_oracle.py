"""The leaf packer's inputs, pinned on the reference (CPU).

Every leaf of reference-written assets is unpacked into control streams (tests/leafstreams.py) and
packed again by the reference's own packRenderTemporalControlStream and
buildRenderTemporalPackedLeafBytes (oracle/_ref/libvbtref.so): the bytes must equal the leaf the
encoder wrote.  This pins the stream arrays that tests/test_leaf_packer.py hands to the GPU packer,
and the reference semantics it restates (FP16 re-encoding of the widened values included).
"""
import os

import numpy as np
import pytest

from conftest import ASSETS, golden_asset
from leafstreams import streams_from_file


def render_assets():
    out = [golden_asset("tiny_density"), golden_asset("tiny_levelset")]
    for n in ("cfg1_blobs", "cfg4_sdf_small"):
        p = os.path.join(ASSETS, n + ".vbtp")
        if os.path.exists(p):
            out.append(p)
    return out


def ref_stream(ref, arr, first_c, controls, bins, first_k, keys, codec, max_local):
    d = arr["descriptors"][first_c:first_c + controls]
    triples = np.stack([d & 0xFFFF, (d >> 16) & 0xFF, d >> 24], axis=1).astype(np.uint32).reshape(-1)
    b = arr["bins"].reshape(-1, 8)[first_c:first_c + controls, :bins].reshape(-1).copy()
    fr = arr["key_frames"][first_k:first_k + keys].astype(np.uint32)
    va = arr["key_values"][first_k:first_k + keys].copy()
    return ref.pack_stream(codec, triples, b, fr, va, bins, max_local=max_local).tobytes()


@pytest.mark.parametrize("path", render_assets(), ids=os.path.basename)
def test_reference_packer_rebuilds_every_leaf(oracle, reference, path):
    leaves, arr, blocks = streams_from_file(path, oracle)
    for i, l in enumerate(leaves):
        word = int(l["header"])
        mode, cres, fres = word & 3, (word >> 6) & 7, (word >> 9) & 7
        if mode == 0:
            got = ref_build(reference, word, 0, 0, b"", b"", None)
        else:
            coarse = ref_stream(reference, arr, int(l["coarse_control"]), cres ** 3, 8, int(l["coarse_key"]),
                                int(l["coarse_kf"]), (word >> 2) & 3, int(l["coarse_max_local"]))
            fine, occ = b"", None
            if mode == 3:
                fine = ref_stream(reference, arr, int(l["fine_control"]), fres ** 3, 8, int(l["fine_key"]),
                                  int(l["fine_kf"]), (word >> 4) & 3, int(l["fine_max_local"]))
            elif mode == 2:
                occ = arr["occupancy"][80 * int(l["occupancy"]):80 * int(l["occupancy"]) + 80].tobytes()
                act = int(np.unpackbits(np.frombuffer(occ[:64], np.uint8)).sum())
                fine = ref_stream(reference, arr, int(l["fine_control"]), act, 4, int(l["fine_key"]),
                                  int(l["fine_kf"]), (word >> 4) & 3, int(l["fine_max_local"]))
            got = ref_build(reference, word, int(l["coarse_kf"]), int(l["fine_kf"]), coarse, fine, occ)
        assert got == blocks[i], (os.path.basename(path), i, mode)


def ref_build(ref, word, ckf, fkf, coarse, fine, occ):
    occ = None if occ is None else np.frombuffer(occ, np.uint8)
    return ref.build_leaf(word, ckf, fkf, np.frombuffer(coarse, np.uint8), np.frombuffer(fine, np.uint8), occ).tobytes()
