"""The encoder's coarse control fitting, restated (oracle/vbt_keyframe_oracle.c: vo_coarse_fit), pinned
on the reference (CPU).

1. Against the reference's own sampleLeafBufferAtFractional, detectDensityKeyFrames,
   appendControlSequenceToStream and reconstructFromKeys (oracle/_ref/libkfref.so) on seeded leaves
   of full and cropped extents: descriptors, bin rows, keyframes, requiredMaxBinLocalKeys and the
   fitted grid, bit for bit.
2. End to end against a file the reference encoder wrote: config 1's blob field regenerated from its
   seed (tests/golden/make_assets.py), the per-voxel keyframe pass with the encoder's defaults, each
   leaf's reconstruction fitted with the control profile (epsilons x 8, the formal default
   controlEpsScale) -- every leaf's coarse stream equals the one in assets/cfg1_blobs.vbtp
   (descriptors, bins, key frames, FP16 key values), and the EMPTY leaves are the leaves whose
   reconstruction stays under the background threshold.
"""
import os
import sys

import numpy as np
import pytest

from conftest import ASSETS, GOLDEN

F32 = np.float32


def control_profile():
    from oracle.oracle import VoKeyframeProfile
    return VoKeyframeProfile(eps_abs=float(F32(1e-5) * F32(8)), eps_rel=float(F32(0.02) * F32(8)))


@pytest.fixture(scope="module")
def kfref():
    from oracle.oracle import KFREF_SO, KeyframeReference
    if not os.path.exists(KFREF_SO):
        pytest.skip("reference build (oracle/_ref/libkfref.so) not present")
    return KeyframeReference()


def test_coarse_fit_against_reference(oracle, kfref):
    rng = np.random.default_rng(0)
    prof = control_profile()
    for it in range(200):
        T = int(rng.choice([1, 2, 5, 24, 96]))
        ext = tuple(int(x) for x in rng.choice([8, 8, 8, 3, 5, 1], 3))
        t = np.arange(T)[None, :]
        c = rng.uniform(0, T, (512, 1))
        amp = rng.uniform(0, 1, (512, 1))
        lt = (amp * np.exp(-((t - c) / rng.uniform(2, 9)) ** 2) + rng.normal(0, 1e-3, (512, T)) * (it % 2))
        lt = lt.astype(np.float32)
        a, b = oracle.coarse_fit(lt, ext, prof), kfref.coarse_fit(lt, ext, prof)
        for k in ("desc", "bins", "key_frames", "key_values", "grid"):
            assert np.array_equal(np.asarray(a[k]).view(np.uint8), np.asarray(b[k]).view(np.uint8)), (it, k)
        assert a["required_max_local"] == b["required_max_local"], it


def test_config1_coarse_streams_equal_the_encoders(oracle):
    path = os.path.join(ASSETS, "cfg1_blobs.vbtp")
    if not os.path.exists(path):
        pytest.skip("asset cfg1_blobs not generated (python tests/golden/make_assets.py cfg1_blobs)")
    from oracle.oracle import VoKeyframeProfile
    sys.path.insert(0, GOLDEN)
    from make_assets import blobs
    from leafstreams import streams_from_file
    raw = blobs((64, 64, 64), 24, 6, 1)                     # the config-1 field, [T, Z, Y, X]
    T = raw.shape[0]
    prof = VoKeyframeProfile()
    recon = oracle.keyframe_pass(raw.reshape(T, -1), prof)["recon"].reshape(T, 64, 64, 64)
    leaves, arr, _ = streams_from_file(path)
    cprof = control_profile()
    fitted = 0
    for li in range(leaves.shape[0]):
        bz, by, bx = li // 64, (li // 8) % 8, li % 8
        sub = recon[:, 8 * bz:8 * bz + 8, 8 * by:8 * by + 8, 8 * bx:8 * bx + 8]
        empty = max(0.0, float(sub.max())) < prof.bg_threshold
        mode = int(leaves[li]["header"]) & 3
        assert (mode == 0) == empty, li
        if mode == 0:
            continue
        fit = oracle.coarse_fit(np.ascontiguousarray(sub.reshape(T, 512).T), (8, 8, 8), cprof)
        l = leaves[li]
        c0, k0, nk = int(l["coarse_control"]), int(l["coarse_key"]), int(l["coarse_kf"])
        assert np.array_equal(fit["desc"], arr["descriptors"][c0:c0 + 64]), li
        assert np.array_equal(fit["bins"], arr["bins"].reshape(-1, 8)[c0:c0 + 64]), li
        assert np.array_equal(fit["key_frames"], arr["key_frames"][k0:k0 + nk]), li
        want = arr["key_values"][k0:k0 + nk].astype(np.float16).view(np.uint16)
        assert np.array_equal(oracle.float_to_half(fit["key_values"]), want), li
        fitted += 1
    assert fitted > 400


def test_config1_leaves_rebuilt_from_the_raw_field(oracle, reference):
    """The encoder chain (keyframe pass -> coarse fit -> FINE6 residual fit -> leaf packer), here
    through the oracle and the reference packer: every GRID4 and every FINE6 leaf of cfg1_blobs.vbtp
    is rebuilt byte for byte from the raw field, with each fit's requiredMaxBinLocalKeys as its
    stream's maxBinLocalKeys (the FINE6 stream: the residual of the reconstruction over the fitted
    coarse grid, vo_fine6_fit)."""
    path = os.path.join(ASSETS, "cfg1_blobs.vbtp")
    if not os.path.exists(path):
        pytest.skip("asset cfg1_blobs not generated (python tests/golden/make_assets.py cfg1_blobs)")
    from oracle.oracle import VoKeyframeProfile
    sys.path.insert(0, GOLDEN)
    from make_assets import blobs
    from leafstreams import streams_from_file
    raw = blobs((64, 64, 64), 24, 6, 1)
    T = raw.shape[0]
    recon = oracle.keyframe_pass(raw.reshape(T, -1), VoKeyframeProfile())["recon"].reshape(T, 64, 64, 64)
    leaves, _, blocks = streams_from_file(path)
    cprof = control_profile()
    def pack(fit, codec):
        d = fit["desc"]
        triples = np.stack([d & 0xFFFF, (d >> 16) & 0xFF, d >> 24], axis=1).astype(np.uint32).reshape(-1)
        return reference.pack_stream(codec, triples, fit["bins"].reshape(-1), fit["key_frames"].astype(np.uint32),
                                     fit["key_values"], 8, max_local=fit["required_max_local"])

    rebuilt = {1: 0, 3: 0}
    for li in range(leaves.shape[0]):
        word = int(leaves[li]["header"])
        mode = word & 3
        if mode not in (1, 3):
            continue
        bz, by, bx = li // 64, (li // 8) % 8, li % 8
        sub = recon[:, 8 * bz:8 * bz + 8, 8 * by:8 * by + 8, 8 * bx:8 * bx + 8]
        lt = np.ascontiguousarray(sub.reshape(T, 512).T)
        fit = oracle.coarse_fit(lt, (8, 8, 8), cprof)
        coarse = pack(fit, (word >> 2) & 3)
        fine, nf = np.zeros(0, np.uint8), 0
        if mode == 3:
            f6 = oracle.fine6_fit(lt, (8, 8, 8), cprof, fit["grid"])
            fine, nf = pack(f6, (word >> 4) & 3), f6["key_frames"].size
        leaf = reference.build_leaf(word, fit["key_frames"].size, nf, coarse, fine)
        assert leaf.tobytes() == blocks[li], (li, mode)
        rebuilt[mode] += 1
    assert rebuilt[1] > 400 and rebuilt[3] > 20, rebuilt


def levelset_profiles():
    """The encoder's temporal and control profiles for a level set (render_temporal_kf_probe_main.cpp:
    430-445 and runRenderTemporalMainline): no cutoff, iso-surface protection at 0 with a band of
    0.1 voxel in the pass, none in the control fitting."""
    from oracle.oracle import VoKeyframeProfile
    common = dict(render_cutoff=0.0, cutoff_band=0.0, cutoff_temporal_protect=0, bg_threshold=-1.0)
    temporal = VoKeyframeProfile(iso_surface_protect=1, iso_value=0.0, iso_band=float(F32(0.1) * F32(1.0)), **common)
    control = VoKeyframeProfile(eps_abs=float(F32(1e-5) * F32(8)), eps_rel=float(F32(0.02) * F32(8)), **common)
    return temporal, control


CASES = {   # name: (field recipe of tests/golden/make_assets.py, dims, level set)
    "tiny_density": (("blobs", ((20, 12, 17), 9, 3, 11)), (20, 12, 17), False),
    "tiny_levelset": (("sdf_scene", ((24, 20, 28), 12, 12.0, 2.0, 0.3, 3, 2.0, 5.0, 12)), (24, 20, 28), True),
    "cfg4_sdf_small": (("sdf_scene", ((64, 64, 64), 24, 24.0, 2.0, 0.2, 6, 3.0, 8.0, 4)), (64, 64, 64), True),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_coarse_streams_of_more_files(oracle, name):
    """As the config-1 check, on a density field with cropped boundary leaves and on two level sets
    (iso-surface protection in the pass, Mode2 shell leaves in the file: their coarse streams)."""
    (fn, args), (X, Y, Z), levelset = CASES[name]
    path = os.path.join(GOLDEN, "assets", name + ".vbtp")
    if not os.path.exists(path):
        path = os.path.join(ASSETS, name + ".vbtp")
    if not os.path.exists(path):
        pytest.skip(f"asset {name} not generated")
    from oracle.oracle import VoKeyframeProfile
    sys.path.insert(0, GOLDEN)
    import make_assets
    from leafstreams import streams_from_file
    raw = getattr(make_assets, fn)(*args)
    T = raw.shape[0]
    temporal, control = levelset_profiles() if levelset else (VoKeyframeProfile(), control_profile())
    recon = oracle.keyframe_pass(raw.reshape(T, -1), temporal)["recon"].reshape(T, Z, Y, X)
    leaves, arr, _ = streams_from_file(path)
    lcx, lcy = (X + 7) // 8, (Y + 7) // 8
    fitted = 0
    for li in range(leaves.shape[0]):
        if int(leaves[li]["header"]) & 3 == 0:
            continue
        bx, by, bz = li % lcx, (li // lcx) % lcy, li // (lcx * lcy)
        sub = recon[:, 8 * bz:8 * bz + 8, 8 * by:8 * by + 8, 8 * bx:8 * bx + 8]
        d, h, w = sub.shape[1:]
        lt = np.zeros((T, 8, 8, 8), np.float32)
        lt[:, :d, :h, :w] = sub
        fit = oracle.coarse_fit(np.ascontiguousarray(lt.reshape(T, 512).T), (w, h, d), control)
        l = leaves[li]
        c0, k0, nk = int(l["coarse_control"]), int(l["coarse_key"]), int(l["coarse_kf"])
        assert np.array_equal(fit["desc"], arr["descriptors"][c0:c0 + 64]), li
        assert np.array_equal(fit["bins"], arr["bins"].reshape(-1, 8)[c0:c0 + 64]), li
        assert np.array_equal(fit["key_frames"], arr["key_frames"][k0:k0 + nk]), li
        want = arr["key_values"][k0:k0 + nk].astype(np.float16).view(np.uint16)
        assert np.array_equal(oracle.float_to_half(fit["key_values"]), want), li
        fitted += 1
    assert fitted >= 10


def route_leaf(raw, base, grid_coarse, grid_fine, peak, step=8, cutoff=F32(0.0003), band=F32(0.0001)):
    """The density route (src/render_temporal_kf_probe_main.cpp:1105-1245 with routeRenderTemporalLeaf,
    src/render_temporal_route.cpp:27-66, and the thresholds of makeRenderTemporalRouteDefaults): the
    points of the leaf on the encoder's sampling lattice (every `step`-th frame and voxel; sampleStep
    8), their truth against the coarse prediction and the coarse + FINE6 prediction sampled from the
    fitted grids; FINE6 when the coarse fit is too rough, the points are visible and the fine fit gains
    enough, else GRID4.  Points sit at multiples of 8, so each is a leaf's voxel (0, 0, 0): control 0
    of either grid."""
    T = raw.shape[0]
    bx, by, bz = base
    lo, hi = float(F32(cutoff - band)), float(F32(cutoff + band))
    n = vis = bnd = 0
    ce2 = fe2 = cpk = 0.0
    for t in range(0, T, step):
        if bx % step or by % step or bz % step:
            continue
        truth = float(raw[t, bz, by, bx])
        cp, fp = F32(grid_coarse[0, t]), F32(grid_fine[0, t])
        n += 1
        vis += truth >= lo
        bnd += lo <= truth <= hi
        cd, fd = truth - float(cp), truth - float(F32(cp + fp))
        ce2 += cd * cd
        fe2 += fd * fd
        cpk = max(cpk, abs(cd) / peak)
    cnt = float(max(1, n))
    crm, frm = np.sqrt(ce2 / cnt) / peak, np.sqrt(fe2 / cnt) / peak
    rough = crm > float(F32(0.008)) or cpk > float(F32(0.03))
    sensitive = vis / cnt >= float(F32(0.005)) or bnd / cnt >= float(F32(0.005))
    gain = (crm - frm) / max(crm, 1e-12)
    return 3 if rough and sensitive and gain >= float(F32(0.05)) else 1


FILES = {   # name: (field recipe of tests/golden/make_assets.py, dims, level set)
    "cfg2_plume": (("plume", (256, 96, 2)), (256, 256, 256), False),   # ~2 minutes, 14 GB of host memory
    "cfg1_blobs": (("blobs", ((64, 64, 64), 24, 6, 1)), (64, 64, 64), False),
    "tiny_density": (("blobs", ((20, 12, 17), 9, 3, 11)), (20, 12, 17), False),
    "tiny_levelset": (("sdf_scene", ((24, 20, 28), 12, 12.0, 2.0, 0.3, 3, 2.0, 5.0, 12)), (24, 20, 28), True),
    "cfg4_sdf_small": (("sdf_scene", ((64, 64, 64), 24, 24.0, 2.0, 0.2, 6, 3.0, 8.0, 4)), (64, 64, 64), True),
    "mix_fire_temperature": (("fire", ((128, 128, 192), 40, 7), 2), (128, 128, 192), False),   # 300-1800 K
    "mix_sdf": (("sdf_scene", ((128, 128, 128), 48, 50.0, 12.0, 0.05, 20, 3.0, 12.0, 9)), (128, 128, 128), True),
}


@pytest.mark.parametrize("name", sorted(FILES))
def test_file_regenerated_from_the_raw_field(oracle, reference, name):
    """A whole VBTPACK4 file from its raw field, byte for byte the file the reference encoder wrote:
    the per-voxel pass, the EMPTY test, the coarse fit, then per leaf either (density) the FINE6 fit
    and the route between GRID4 and FINE6, or (level set: shell width 3 voxels, coarse guard band
    1.5, temporal band 0.1) the Mode2 shell stage (vo_shell_fit), a Mode2 leaf wherever it finds shell
    voxels; leaf packing by the reference packer and the file layout (52-byte header, word offsets,
    payload).  The config-2 plume (256^3 x 96, 88 % EMPTY leaves, 72 MB), config 1, the fire's
    temperature field, a small density field with cropped boundary leaves, and three level sets."""
    recipe, (X, Y, Z), levelset = FILES[name]
    path = os.path.join(GOLDEN, "assets", name + ".vbtp")
    if not os.path.exists(path):
        path = os.path.join(ASSETS, name + ".vbtp")
    if not os.path.exists(path):
        pytest.skip(f"asset {name} not generated")
    import struct
    from oracle.oracle import VoKeyframeProfile, pack_payload
    sys.path.insert(0, GOLDEN)
    import make_assets
    raw = getattr(make_assets, recipe[0])(*recipe[1])
    if len(recipe) > 2:                                     # one field of a multi-field recipe
        raw = raw[recipe[2]]
    T = raw.shape[0]
    peak = float(max(F32(1e-6), F32(F32(raw.max()) - F32(raw.min()))))
    prof, cprof = levelset_profiles() if levelset else (VoKeyframeProfile(), control_profile())
    recon = oracle.keyframe_pass(raw.reshape(T, -1), prof)["recon"].reshape(T, Z, Y, X)

    def pack(fit, codec, bins=8):
        d = fit["desc"]
        triples = np.stack([d & 0xFFFF, (d >> 16) & 0xFF, d >> 24], axis=1).astype(np.uint32).reshape(-1)
        return reference.pack_stream(codec, triples, fit["bins"][:, :bins].reshape(-1),
                                     fit["key_frames"].astype(np.uint32), fit["key_values"], bins,
                                     max_local=fit["required_max_local"])

    lcx, lcy, lcz = (X + 7) // 8, (Y + 7) // 8, (Z + 7) // 8
    none = np.zeros(0, np.uint8)
    blocks = []
    for li in range(lcx * lcy * lcz):
        bx, by, bz = li % lcx, (li // lcx) % lcy, li // (lcx * lcy)
        sub = recon[:, 8 * bz:8 * bz + 8, 8 * by:8 * by + 8, 8 * bx:8 * bx + 8]
        if prof.bg_threshold >= 0 and max(0.0, float(sub.max())) < prof.bg_threshold:
            blocks.append(reference.build_leaf(4 << 6, 0, 0, none, none).tobytes())   # EMPTY, default header
            continue
        d, h, w = sub.shape[1:]
        lt = np.zeros((T, 8, 8, 8), np.float32)
        lt[:, :d, :h, :w] = sub
        lt = np.ascontiguousarray(lt.reshape(T, 512).T)
        fit = oracle.coarse_fit(lt, (w, h, d), cprof)
        coarse = pack(fit, 0)
        if levelset:
            sh = oracle.shell_fit(lt, (w, h, d), cprof, fit["grid"], True, 3.0, 1.5, float(F32(0.1) * F32(1.0)), 0.0)
            if sh["active"] > 0:
                leaf = reference.build_leaf(2 | (4 << 6), fit["key_frames"].size, sh["key_frames"].size, coarse,
                                            pack(sh, 0, bins=4), sh["occupancy"])
            else:
                leaf = reference.build_leaf(1 | (4 << 6), fit["key_frames"].size, 0, coarse, none)
        else:
            f6 = oracle.fine6_fit(lt, (w, h, d), cprof, fit["grid"])
            mode = route_leaf(raw, (8 * bx, 8 * by, 8 * bz), fit["grid"], f6["grid"], peak)
            word = mode | (4 << 6) | ((6 if mode == 3 else 0) << 9)          # FP16 keyframes in both streams
            fine, nf = (pack(f6, 0), f6["key_frames"].size) if mode == 3 else (none, 0)
            leaf = reference.build_leaf(word, fit["key_frames"].size, nf, coarse, fine)
        blocks.append(leaf.tobytes())
    offsets, payload = pack_payload(blocks)
    header = b"VBTPACK4" + struct.pack("<11I", 4, X, Y, Z, T, 8, 4, 0, len(blocks), 1, 0)
    assert header + offsets.tobytes() + payload.tobytes() == open(path, "rb").read()
