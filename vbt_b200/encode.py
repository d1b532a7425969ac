"""The render-temporal encoder on the GPU: a frame-major float32 field to a VBTPACK4 file image, with
the stages of the reference's temporal-first encoder (src/render_temporal_kf_probe_main.cpp) run as
this library's kernels:

  1. the per-voxel keyframe pass and reconstruction (vbt_detect_keyframes; the leaf loop's body,
     :619-659), under the density profile or, for a level set, with iso-surface protection at 0;
  2. the EMPTY test per leaf (density: the reconstruction's maximum over the leaf below
     bgZeroRatio x cutoff, :477, :664);
  3. the coarse control fitting (vbt_coarse_fit, :705-729);
  4. density fields: the FINE6 residual fitting (vbt_fine6_fit, :815-850) and the route between
     GRID4 and FINE6 (vbt_route_density, :1105-1245); level sets: the Mode2 shell stage
     (vbt_shell_fit, :930-1025), a Mode2 leaf wherever a shell voxel exists, else GRID4;
  5. the leaves packed straight into the payload (vbt_pack_leaves) and the file layout of
     writeRenderTemporalProbeFile (:2561-2606): 52-byte header, word offsets, payload.

FP16 keyframes in every stream, coarse resolution 4, fine resolution 6, 8 time bins (4 for the
Mode2 residual stream): the encoder's defaults.  Every stage is local to a leaf and its frames (the
route reads the raw field at the leaf's own voxels), so the volume is encoded one layer of leaves
(8 z-planes) at a time, or a few layers together: the field may be given whole or as a function
that produces the z-planes of a layer, and the device memory held beyond the finished payload is
that of one group of layers.  PyTorch is used for device buffers and for the small reductions
between the stages (leaf maxima, field range, offsets of the groups).
"""
import struct

import numpy as np

from . import KeyframeProfile, coarse_fit, detect_keyframes, fine6_fit, pack_leaves, route_density, shell_fit

LEAF_DTYPE = np.dtype([("header", "<u4"), ("coarse_kf", "<u2"), ("fine_kf", "<u2"), ("coarse_control", "<u4"),
                       ("coarse_key", "<u4"), ("fine_control", "<u4"), ("fine_key", "<u4"), ("occupancy", "<u4"),
                       ("coarse_max_local", "u1"), ("fine_max_local", "u1"), ("pad", "u1", (2,))])
COARSE_RES, FINE_RES, SHELL_ROWS = 4, 6, 512
SHELL_WIDTH, GUARD_BAND = 3.0, 1.5          # shell half-width in voxels, coarse guard band


def _f32(x):
    return float(np.float32(x))


def profiles(levelset):
    """(temporal, control) keyframe profiles of the encoder: the density profile (defaults) with the
    control fitting's epsilons x 8; for a level set (conversion_mode levelset, :430-445) no cutoff,
    iso-surface protection at 0 with a band of 0.1 voxel in the pass, none in the control fitting."""
    ctrl_eps = dict(eps_abs=_f32(np.float32(1e-5) * np.float32(8)), eps_rel=_f32(np.float32(0.02) * np.float32(8)))
    if not levelset:
        return KeyframeProfile(), KeyframeProfile(**ctrl_eps)
    common = dict(render_cutoff=0.0, cutoff_band=0.0, cutoff_temporal_protect=0, bg_threshold=-1.0)
    temporal = KeyframeProfile(iso_surface_protect=1, iso_value=0.0, iso_band=_f32(np.float32(0.1) * np.float32(1.0)),
                               **common)
    return temporal, KeyframeProfile(**ctrl_eps, **common)


def _leaf_max(torch, recon, X, Y, zs):
    """Per leaf of a slab of zs z-planes, the maximum of the reconstruction over the leaf's voxels
    and all frames."""
    T = recon.shape[0]
    lcx, lcy, lcz = (X + 7) // 8, (Y + 7) // 8, (zs + 7) // 8
    v = recon[:, :X * Y * zs].view(T, zs, Y, X)
    out = torch.empty((lcz, lcy, lcx), dtype=torch.float32, device=recon.device)
    pad = torch.full((lcy * 8, lcx * 8), float("-inf"), dtype=torch.float32, device=recon.device)
    for bz in range(lcz):
        pad[:Y, :X] = v[:, 8 * bz:8 * bz + 8].amax(dim=(0, 1))
        out[bz] = pad.view(lcy, 8, lcx, 8).amax(dim=(1, 3))
    return out.reshape(-1)


class _Field:
    """The field as slabs of z-planes: a frame-major device tensor [frames, >= X*Y*Z] or a function
    (z0, z1) -> device tensor [frames, (z1 - z0) * X * Y]."""

    def __init__(self, field, dims):
        self.field, self.dims = field, dims
        X, Y, Z = dims
        if not callable(field) and (field.dim() != 2 or field.shape[1] < X * Y * Z):
            raise ValueError("the field must be [frames, >= X*Y*Z]")

    def slab(self, z0, z1):
        X, Y, _ = self.dims
        if callable(self.field):
            s = self.field(z0, z1)
            if s.dim() != 2 or s.shape[1] != (z1 - z0) * X * Y:
                raise ValueError("a slab must be [frames, (z1 - z0) * X * Y]")
            return s.contiguous()
        return self.field[:, z0 * X * Y:z1 * X * Y].contiguous()

    def value_range(self, step):
        X, Y, Z = self.dims
        if not callable(self.field):
            v = self.field[:, :X * Y * Z]
            return float(v.min()), float(v.max())
        lo, hi = float("inf"), float("-inf")
        for z0 in range(0, Z, step):
            s = self.slab(z0, min(Z, z0 + step))
            lo, hi = min(lo, float(s.min())), max(hi, float(s.max()))
            del s
        return lo, hi


def encode_render_temporal(field, dims, levelset=False, batch=4096, value_range=None, stream=None):
    """Encode a float32 field of the volume dims = (X, Y, Z) as the reference's temporal-first
    encoder does with its default density settings, or with conversion_mode levelset and a 3-voxel
    shell.  field: a frame-major device tensor [frames, >= X*Y*Z], or a function (z0, z1) returning
    the device tensor [frames, (z1 - z0) * X * Y] of z-planes z0..z1-1 (called with multiples of 8).
    value_range: the field's (min, max), which the density route needs; found with a first pass over
    the field when not given.  Leaves are fitted in groups of whole leaf layers of about `batch`
    leaves.  Returns (header, offsets, payload): the 52-byte header as bytes, and int32 device
    tensors of the leaf_count + 1 word offsets and the payload words."""
    import torch
    X, Y, Z = dims
    src = _Field(field, dims)
    lcx, lcy, lcz = (X + 7) // 8, (Y + 7) // 8, (Z + 7) // 8
    layer, L = lcx * lcy, lcx * lcy * lcz
    group = max(1, batch // layer)
    prof, cprof = profiles(levelset)
    if not levelset:
        lo_v, hi_v = value_range if value_range is not None else src.value_range(8 * group)
        peak = max(_f32(1e-6), _f32(np.float32(hi_v) - np.float32(lo_v)))
        cut, band = np.float32(prof.render_cutoff), np.float32(prof.cutoff_band)
        vis_lo, vis_hi = _f32(cut - band), _f32(cut + band)
    dev = offsets = T = None
    pieces, words = [], 0
    for bz0 in range(0, lcz, group):
        bz1 = min(lcz, bz0 + group)
        z0, z1 = 8 * bz0, min(Z, 8 * bz1)
        raw = src.slab(z0, z1)
        if dev is None:
            dev, T = raw.device, raw.shape[0]
            offsets = torch.empty(L + 1, dtype=torch.int32, device=dev)
            offsets[0] = 0
        elif raw.shape[0] != T:
            raise ValueError("every slab must hold the same frames")
        zs, V = z1 - z0, (z1 - z0) * X * Y
        slab_dims = (X, Y, zs)
        recon = torch.empty((T, V), dtype=torch.float32, device=dev)
        mask = torch.empty(((T + 31) // 32, V), dtype=torch.int32, device=dev)
        cnt = torch.empty(V, dtype=torch.int32, device=dev)
        flags = torch.empty(V, dtype=torch.uint8, device=dev)
        detect_keyframes(raw, prof, mask, cnt, flags, recon, stream=stream)
        del mask, cnt, flags
        nl = (bz1 - bz0) * layer
        if prof.bg_threshold >= 0:
            torch.cuda.synchronize(dev)
            empty = (torch.clamp(_leaf_max(torch, recon, X, Y, zs), min=0.0) < prof.bg_threshold).cpu().numpy()
        else:
            empty = np.zeros(nl, bool)
        fit_idx = np.flatnonzero(~empty)
        nb = fit_idx.size
        rec = np.zeros(nl, LEAF_DTYPE)
        rec["header"] = COARSE_RES << 6                        # EMPTY leaves: the default header word
        arrays = dict(desc=torch.zeros(1, dtype=torch.int32, device=dev),
                      bins=torch.zeros(8, dtype=torch.uint8, device=dev),
                      kf=torch.zeros(1, dtype=torch.int16, device=dev),
                      kv=torch.zeros(1, dtype=torch.float32, device=dev), occ=None)
        rows = keys = 0
        if nb:
            leaves = torch.from_numpy(fit_idx.astype(np.int32)).to(dev)
            C = COARSE_RES ** 3
            co = dict(desc=torch.empty((nb, C), dtype=torch.int32, device=dev),
                      bins=torch.empty((nb, C, 8), dtype=torch.uint8, device=dev),
                      kf=torch.empty((nb, C * T), dtype=torch.int16, device=dev),
                      kv=torch.empty((nb, C * T), dtype=torch.float32, device=dev),
                      cnt=torch.empty(nb, dtype=torch.int32, device=dev),
                      req=torch.empty(nb, dtype=torch.uint8, device=dev),
                      grid=torch.empty((nb, C, T), dtype=torch.float32, device=dev))
            coarse_fit(recon, slab_dims, leaves, cprof, co["desc"], co["bins"], co["kf"], co["kv"], co["cnt"],
                       co["req"], co["grid"], stream=stream)
            if levelset:
                F = SHELL_ROWS
                fi = dict(occ=torch.zeros((nb, 80), dtype=torch.uint8, device=dev),
                          desc=torch.zeros((nb, F), dtype=torch.int32, device=dev),
                          bins=torch.zeros((nb, F, 8), dtype=torch.uint8, device=dev),
                          kf=torch.zeros((nb, F * T), dtype=torch.int16, device=dev),
                          kv=torch.zeros((nb, F * T), dtype=torch.float32, device=dev),
                          cnt=torch.empty(nb, dtype=torch.int32, device=dev),
                          act=torch.empty(nb, dtype=torch.int32, device=dev),
                          req=torch.empty(nb, dtype=torch.uint8, device=dev))
                shell_fit(recon, slab_dims, leaves, cprof, co["grid"], True, SHELL_WIDTH, GUARD_BAND,
                          _f32(np.float32(0.1) * np.float32(1.0)), 0.0, fi["occ"], fi["desc"], fi["bins"], fi["kf"],
                          fi["kv"], fi["cnt"], fi["act"], fi["req"], stream=stream)
                torch.cuda.synchronize(dev)
                act = fi["act"].cpu().numpy().astype(np.int64)
                mode = np.where(act > 0, 2, 1)
                rows = int(act.sum())
            else:
                F = FINE_RES ** 3
                fi = dict(desc=torch.empty((nb, F), dtype=torch.int32, device=dev),
                          bins=torch.empty((nb, F, 8), dtype=torch.uint8, device=dev),
                          kf=torch.empty((nb, F * T), dtype=torch.int16, device=dev),
                          kv=torch.empty((nb, F * T), dtype=torch.float32, device=dev),
                          cnt=torch.empty(nb, dtype=torch.int32, device=dev),
                          req=torch.empty(nb, dtype=torch.uint8, device=dev),
                          grid=torch.empty((nb, F, T), dtype=torch.float32, device=dev))
                fine6_fit(recon, slab_dims, leaves, cprof, co["grid"], fi["desc"], fi["bins"], fi["kf"], fi["kv"],
                          fi["cnt"], fi["req"], fi["grid"], stream=stream)
                md = torch.empty(nb, dtype=torch.uint8, device=dev)
                route_density(raw, slab_dims, leaves, co["grid"], fi["grid"], peak, vis_lo, vis_hi, md, stream=stream)
                torch.cuda.synchronize(dev)
                mode = md.cpu().numpy().astype(np.int64)
                rows = int((mode == 3).sum()) * F
            ccnt, creq = co["cnt"].cpu().numpy(), co["req"].cpu().numpy()
            fcnt, freq = fi["cnt"].cpu().numpy(), fi["req"].cpu().numpy()
            has_fine = mode != 1
            r = rec[fit_idx]
            r["header"] = mode | (COARSE_RES << 6) | (np.where(mode == 3, FINE_RES, 0) << 9)
            r["coarse_kf"] = ccnt
            r["coarse_control"] = np.arange(nb) * C
            r["coarse_key"] = np.arange(nb) * C * T
            r["coarse_max_local"] = creq
            r["fine_kf"] = np.where(has_fine, fcnt, 0)
            r["fine_control"] = nb * C + np.arange(nb) * F
            r["fine_key"] = nb * C * T + np.arange(nb) * F * T
            r["fine_max_local"] = np.where(has_fine, freq, 0)
            r["occupancy"] = np.arange(nb)
            rec[fit_idx] = r
            keys = int(ccnt.sum()) + int(np.where(has_fine, fcnt, 0).sum())
            rows += nb * C
            arrays = dict(desc=torch.cat([co["desc"].reshape(-1), fi["desc"].reshape(-1)]),
                          bins=torch.cat([co["bins"].reshape(-1), fi["bins"].reshape(-1)]),
                          kf=torch.cat([co["kf"].reshape(-1), fi["kf"].reshape(-1)]),
                          kv=torch.cat([co["kv"].reshape(-1), fi["kv"].reshape(-1)]),
                          occ=fi["occ"].reshape(-1) if levelset else None)
            del co, fi
        del recon, raw
        d_rec = torch.from_numpy(rec.view(np.uint8).copy()).to(dev)
        g_off = torch.empty(nl + 1, dtype=torch.int32, device=dev)
        # a leaf: 2 header words, 3 words per control row (descriptor + 8 bin bytes), 3 bytes per
        # FP16 key, the 80-byte occupancy and the alignment of each section
        cap = 32 * nl + 3 * rows + (3 * keys) // 4 + 1024
        g_pay = torch.empty(cap, dtype=torch.int32, device=dev)
        n_words = pack_leaves(d_rec, arrays["desc"], arrays["bins"], arrays["kf"], arrays["kv"], arrays["occ"],
                              g_off, g_pay, stream=stream)
        offsets[bz0 * layer + 1:bz0 * layer + nl + 1] = g_off[1:] + words
        pieces.append(g_pay[:n_words].clone())
        words += n_words
        del arrays, g_pay, g_off, d_rec
    payload = torch.cat(pieces) if len(pieces) > 1 else pieces[0]
    header = b"VBTPACK4" + struct.pack("<11I", 4, X, Y, Z, T, 8, COARSE_RES, 0, L, 1, 0)
    return header, offsets, payload


def file_image(header, offsets, payload, pinned=False):
    """The whole VBTPACK4 file image (header, offsets, payload) as a host uint8 tensor, page-locked
    when pinned; the device tensors are copied straight into it."""
    import torch
    n_off, n_pay = offsets.numel(), payload.numel()
    img = torch.empty(len(header) + 4 * (n_off + n_pay), dtype=torch.uint8, pin_memory=pinned)
    a = len(header)
    img[:a] = torch.frombuffer(bytearray(header), dtype=torch.uint8)
    img[a:a + 4 * n_off].view(torch.int32).copy_(offsets)
    img[a + 4 * n_off:].view(torch.int32).copy_(payload)
    return img
