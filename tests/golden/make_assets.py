#!/usr/bin/env python3
"""Build the seeded synthetic VBTPACK4 assets used by the tests and the benchmark.

Each asset is a float32 field generated here with numpy from a fixed seed, written as a
RAW file plus the metadata JSON the reference encoder reads (src/frame_metadata.h), then
encoded by the reference encoder ``vbt_spatialfirst_probe`` (built from the reference
sources into oracle/_ref/ by oracle/Makefile).  Outputs go to assets/<name>.vbtp
(git-ignored; they travel to the GPU host with the working tree).  The encoder is
deterministic, so the same seed gives byte-identical assets.

Field recipes (shapes are X x Y x Z x T):
  cfg1_blobs      64^3 x 24, 6 Gaussian blobs (sigma U(4,10), amplitude U(0.2,1)) moving on
                  linear paths at <=1 voxel/frame, plus N(0, 0.01) noise; density profile.
  cfg2_plume      256^3 x 96, buoyant plume: 4-octave fBm value noise inside a cone rising at
                  1.5 voxels/frame, clamped to [0, 1], exactly 0 outside; density profile.
  cfg4_sdf_small  64^3 x 24 level set (a scaled-down config-4 scene): sloshing plane
                  z = 24 + 2 sin(0.2 x + 0.1 t) united with 6 ballistic spheres; Mode2 shell.
  tiny_*          small, odd-sized fields (boundary leaves with cropped extents).
  sci_small/_64   scientific (generic profile, time-fastest RAW) Gaussian random fields with a
                  k^-5/3 spectrum, phase drift, and 0.1% spikes of 10 sigma (SparseEvents leaves).
  sci_coarse      smooth drifting blobs: every leaf CoarseOnly.
  sci_dense       blobs + a large-scale pattern with white-noise amplitude: DenseGrid3/4 leaves with
                  the per-frame BFP residual.
  sci_dense_tb    blobs + the pattern modulated by DCT frequencies 4..7, encoded with
                  --generic-dense-temporal-basis --generic-dense-temporal-keep 8: CoarseOnly and
                  DenseGrid leaves of both residual subtypes (per-frame BFP and DCT temporal basis).
  sci_modes       64^3 x 32 with regions of each kind: all four generic modes and both dense
                  subtypes in one asset.
  cfg5_sci        the config-5 scientific field at its stated size, 512^3 x 64 (generated to disk
                  frame by frame and encoded from there).
  mix_fire_*      the config-3 fire (density, flames, temperature = 300 + 1500 flames + N(0, 20))
                  at 128 x 128 x 192 x 40: fBm inside a sphere of radius 20 + 2.5 t.
  mix_sdf         the config-4 liquid level set at 128^3 x 48 (sloshing plane, 20 ballistic spheres
                  under gravity 0.05 voxels/frame^2); Mode2 shell.
  mix_sci         the config-5 scientific field at 128^3 x 64, time fastest.
  The mix_* assets, cfg2_plume, cfg1_blobs and cfg4_sdf_small are the serving mix (MIX).

Usage: python tests/golden/make_assets.py [names...]   (default: the small set + cfg1 + cfg2;
       the name "digests" writes tests/golden/asset_digests.json for the assets present)
"""
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
ASSETS = os.path.join(ROOT, "assets")
ENCODER = os.path.join(ROOT, "oracle", "_ref", "vbt_spatialfirst_probe")


# ----------------------------------------------------------------------------- fields
def blobs(shape_xyz, frames, n_blobs, seed, noise=0.01):
    rng = np.random.default_rng(seed)
    X, Y, Z = shape_xyz
    sig = rng.uniform(4.0, 10.0, n_blobs)
    amp = rng.uniform(0.2, 1.0, n_blobs)
    c0 = rng.uniform(0.2, 0.8, (n_blobs, 3)) * np.array([X, Y, Z])
    d = rng.normal(size=(n_blobs, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    vel = d * rng.uniform(0.0, 1.0, (n_blobs, 1))
    zz, yy, xx = np.meshgrid(np.arange(Z), np.arange(Y), np.arange(X), indexing="ij")
    out = np.empty((frames, Z, Y, X), np.float32)
    for t in range(frames):
        f = np.zeros((Z, Y, X), np.float64)
        for b in range(n_blobs):
            c = c0[b] + vel[b] * t
            r2 = (xx - c[0]) ** 2 + (yy - c[1]) ** 2 + (zz - c[2]) ** 2
            f += amp[b] * np.exp(-r2 / (2.0 * sig[b] ** 2))
        f += rng.normal(0.0, noise, f.shape)
        out[t] = f.astype(np.float32)
    return out


def fbm_volume(shape_zyx, octaves, base_cell, seed):
    """4-octave fBm of trilinearly interpolated value noise on a lattice, in [0, 1]."""
    from scipy.ndimage import zoom
    rng = np.random.default_rng(seed)
    Z, Y, X = shape_zyx
    acc = np.zeros(shape_zyx, np.float32)
    amp, norm = 1.0, 0.0
    for o in range(octaves):
        cell = max(1, base_cell >> o)
        lat = rng.random((Z // cell + 2, Y // cell + 2, X // cell + 2)).astype(np.float32)
        up = zoom(lat, cell, order=1, prefilter=False)[:Z, :Y, :X]
        acc += amp * up
        norm += amp
        amp *= 0.5
    return acc / norm


def plume(size, frames, seed):
    """Cone-shaped plume rising at 1.5 voxels/frame.  The fBm is advected upward by sampling
    a static noise volume built at half-voxel z spacing (1.5 voxels = 3 half-voxel slices)."""
    S = size
    zpad = 3 * (frames - 1)
    noise = fbm_volume((2 * S + zpad, S, S), 4, 32, seed)   # half-voxel z spacing
    zz, yy, xx = np.meshgrid(np.arange(S), np.arange(S), np.arange(S), indexing="ij")
    cx = cy = S / 2.0
    r_xy = np.sqrt((xx - cx) ** 2 + (yy - cy) ** 2)
    z0 = S * 0.04
    out = np.empty((frames, S, S, S), np.float32)
    for t in range(frames):
        top = z0 + S * 0.25 + 1.5 * t                      # front of the rising plume
        radius = 0.06 * S + 0.30 * (zz - z0)               # cone opening upward (~12% of leaves)
        inside = (zz >= z0) & (zz <= top) & (r_xy <= radius)
        idx = 2 * zz - 3 * t + zpad                        # z - 1.5 t in half-voxel units
        n = noise[idx, yy, xx]
        edge = np.clip((radius - r_xy) / 6.0, 0.0, 1.0) * np.clip((top - zz) / 8.0, 0.0, 1.0)
        val = np.clip((n - 0.35) * 2.5 * edge, 0.0, 1.0)
        val[~inside] = 0.0
        out[t] = val.astype(np.float32)
    return out


_FIRE = {}


def fire(shape_xyz, frames, seed):
    """Three aligned fields (density, flames, temperature) of an expanding fireball: fBm inside a
    sphere of radius 20 + 2.5 t at the volume's lower centre, the noise advected upward at one
    voxel per frame; flames = the fBm of a second seed in the sphere's outer band; temperature
    = 300 + 1500 * flames + N(0, 20).  Cached, so the three encodes share one generation."""
    key = (tuple(shape_xyz), frames, seed)
    if key in _FIRE:
        return _FIRE[key]
    rng = np.random.default_rng(seed + 1000)
    X, Y, Z = shape_xyz
    n1 = fbm_volume((Z + frames, Y, X), 4, 32, seed)
    n2 = fbm_volume((Z + frames, Y, X), 4, 16, seed + 1)
    zz, yy, xx = np.meshgrid(np.arange(Z), np.arange(Y), np.arange(X), indexing="ij")
    r = np.sqrt((xx - X / 2.0) ** 2 + (yy - Y / 2.0) ** 2 + (zz - Z * 0.3) ** 2)
    den = np.empty((frames, Z, Y, X), np.float32)
    fl = np.empty((frames, Z, Y, X), np.float32)
    tmp = np.empty((frames, Z, Y, X), np.float32)
    for t in range(frames):
        R = 20.0 + 2.5 * t
        inside = r <= R
        sl = slice(frames - t, frames - t + Z)           # advect upward one voxel per frame
        d = np.clip((n1[sl] - 0.3) * 2.0, 0.0, 1.0) * np.clip((R - r) / 4.0, 0.0, 1.0)
        band = np.clip(1.0 - np.abs(r - 0.8 * R) / (0.25 * R + 1e-6), 0.0, 1.0)
        f = np.clip((n2[sl] - 0.4) * 3.0, 0.0, 1.0) * band
        d[~inside] = 0.0
        f[~inside] = 0.0
        den[t] = d
        fl[t] = f
        tmp[t] = (300.0 + 1500.0 * f + rng.normal(0.0, 20.0, f.shape)).astype(np.float32)
    _FIRE[key] = (den, fl, tmp)
    return _FIRE[key]


def sdf_scene(shape_xyz, frames, plane_z, plane_amp, kx, n_spheres, rmin, rmax, seed, g=0.05):
    rng = np.random.default_rng(seed)
    X, Y, Z = shape_xyz
    c0 = np.stack([rng.uniform(0, X, n_spheres), rng.uniform(0, Y, n_spheres),
                   rng.uniform(plane_z, Z * 0.9, n_spheres)], axis=1)
    v0 = np.stack([rng.uniform(-0.5, 0.5, n_spheres), rng.uniform(-0.5, 0.5, n_spheres),
                   rng.uniform(0.0, 1.0, n_spheres)], axis=1)
    rad = rng.uniform(rmin, rmax, n_spheres)
    zz, yy, xx = np.meshgrid(np.arange(Z), np.arange(Y), np.arange(X), indexing="ij")
    out = np.empty((frames, Z, Y, X), np.float32)
    for t in range(frames):
        phi = zz - (plane_z + plane_amp * np.sin(kx * xx + 0.1 * t))
        for s in range(n_spheres):
            c = c0[s] + v0[s] * t + np.array([0.0, 0.0, -0.5 * g * t * t])
            d = np.sqrt((xx - c[0]) ** 2 + (yy - c[1]) ** 2 + (zz - c[2]) ** 2) - rad[s]
            phi = np.minimum(phi, d)
        out[t] = phi.astype(np.float32)
    return out


def grf_scientific(shape_xyz, frames, seed, spike_frac=0.001, spike_sigma=10.0):
    """Gaussian random field, k^-5/3 power spectrum, evolved by a per-mode phase drift."""
    rng = np.random.default_rng(seed)
    X, Y, Z = shape_xyz
    kz = np.fft.fftfreq(Z)[:, None, None]
    ky = np.fft.fftfreq(Y)[None, :, None]
    kx = np.fft.fftfreq(X)[None, None, :]
    k = np.sqrt(kx ** 2 + ky ** 2 + kz ** 2)
    k[0, 0, 0] = 1.0
    amp = k ** (-5.0 / 6.0)                                  # |F|^2 ~ k^-5/3
    amp[0, 0, 0] = 0.0
    phase0 = rng.uniform(0, 2 * np.pi, k.shape)
    omega = rng.normal(0.0, 0.08, k.shape)
    out = np.empty((Z, Y, X, frames), np.float32)           # time fastest
    for t in range(frames):
        spec = amp * np.exp(1j * (phase0 + omega * t))
        f = np.real(np.fft.ifftn(spec))
        out[..., t] = f.astype(np.float32)
    sigma = float(out.std())
    out /= max(sigma, 1e-12)
    n_spk = max(1, int(spike_frac * out.size))
    idx = rng.choice(out.size, n_spk, replace=False)
    out.reshape(-1)[idx] += np.float32(spike_sigma) * np.sign(rng.normal(size=n_spk)).astype(np.float32)
    return out


def grf_scientific_to_file(shape_xyz, frames, seed, raw_path, spike_frac=0.001, spike_sigma=10.0):
    """grf_scientific's recipe for fields too large to hold in memory (configuration 5: 512^3 x 64
    float32, 34 GB), written straight to a time-fastest RAW file ([Z, Y, X, T]).  Frames are made
    one at a time by a float32 inverse FFT into a frame-major scratch file beside raw_path, then
    transposed slab by slab; the field is divided by its standard deviation over all frames and
    0.1% of its values get spikes of +-10 sigma, as in grf_scientific (the random draws differ, so
    the field is not grf_scientific's for the same seed).  Returns the field's min and max."""
    import scipy.fft
    rng = np.random.default_rng(seed)
    X, Y, Z = shape_xyz
    kz = np.fft.fftfreq(Z).astype(np.float32)[:, None, None]
    ky = np.fft.fftfreq(Y).astype(np.float32)[None, :, None]
    kx = np.fft.fftfreq(X).astype(np.float32)[None, None, :]
    k = np.sqrt(kx ** 2 + ky ** 2 + kz ** 2)
    k[0, 0, 0] = 1.0
    amp = (k ** np.float32(-5.0 / 6.0)).astype(np.float32)
    amp[0, 0, 0] = 0.0
    del k
    phase0 = rng.uniform(0, 2 * np.pi, amp.shape).astype(np.float32)
    omega = rng.normal(0.0, 0.08, amp.shape).astype(np.float32)
    scratch = raw_path + ".frames"
    fm = np.memmap(scratch, np.float32, "w+", shape=(frames, Z, Y, X))
    sq = 0.0
    for t in range(frames):
        spec = amp * np.exp(1j * (phase0 + omega * np.float32(t))).astype(np.complex64)
        f = scipy.fft.ifftn(spec, workers=os.cpu_count()).real.astype(np.float32)
        del spec
        fm[t] = f
        sq += float(np.square(f, dtype=np.float64).sum())
        del f
    fm.flush()
    del amp, phase0, omega
    n = frames * X * Y * Z
    sigma = np.float32(max(np.sqrt(sq / n), 1e-12))
    n_spk = max(1, int(spike_frac * n))
    idx = np.sort(rng.choice(n, n_spk, replace=False))
    sgn = np.sign(rng.normal(size=n_spk)).astype(np.float32)
    out = np.memmap(raw_path, np.float32, "w+", shape=(Z, Y, X, frames))
    slab = max(1, (256 << 20) // (Y * X * frames * 4))
    lo_v, hi_v = float("inf"), float("-inf")
    for z0 in range(0, Z, slab):
        z1 = min(Z, z0 + slab)
        block = np.ascontiguousarray(np.moveaxis(np.asarray(fm[:, z0:z1]), 0, -1)) / sigma
        lo, hi = np.searchsorted(idx, [z0 * Y * X * frames, z1 * Y * X * frames])
        flat = block.reshape(-1)
        flat[idx[lo:hi] - z0 * Y * X * frames] += np.float32(spike_sigma) * sgn[lo:hi]
        out[z0:z1] = block
        lo_v, hi_v = min(lo_v, float(block.min())), max(hi_v, float(block.max()))
    out.flush()
    del fm, out
    os.remove(scratch)
    return lo_v, hi_v


def _drifting_blobs(shape_xyz, frames, rng, n, sigma_lo, sigma_hi):
    """[Z, Y, X, T] sum of n Gaussian blobs (amplitude U(0.5, 1.5)) drifting at N(0, 0.3) voxels
    per frame, and the voxel coordinate grids."""
    X, Y, Z = shape_xyz
    zz, yy, xx = np.meshgrid(np.arange(Z), np.arange(Y), np.arange(X), indexing="ij")
    c0 = rng.uniform(0, 1, (n, 3)) * np.array([X, Y, Z])
    v = rng.normal(0.0, 0.3, (n, 3))
    s = rng.uniform(sigma_lo, sigma_hi, n)
    a = rng.uniform(0.5, 1.5, n)
    out = np.empty((Z, Y, X, frames), np.float64)
    for t in range(frames):
        f = np.zeros((Z, Y, X))
        for b in range(n):
            c = c0[b] + v[b] * t
            f += a[b] * np.exp(-((xx - c[0]) ** 2 + (yy - c[1]) ** 2 + (zz - c[2]) ** 2) / (2.0 * s[b] ** 2))
        out[..., t] = f
    return out, (xx, yy, zz)


def sci_flicker(shape_xyz, frames, seed, amp, kind):
    """Scientific fields that steer the generic encoder's leaf modes (time fastest, [Z, Y, X, T]):
    smooth drifting blobs (every leaf CoarseOnly), plus a large-scale spatial pattern
    sin(0.35 x + 0.2 y) cos(0.3 z) whose amplitude changes over time -- white noise per frame
    (kind "white": the DenseGrid per-frame BFP residual) or a sum of the DCT-II frequencies 4..7
    (kind "mid": with --generic-dense-temporal-basis, also the temporal-basis residual)."""
    rng = np.random.default_rng(seed)
    out, (xx, yy, zz) = _drifting_blobs(shape_xyz, frames, rng, 4, 6.0, 12.0)
    if kind != "none":
        t = np.arange(frames)
        if kind == "white":
            sig = rng.normal(0.0, 1.0, frames)
        else:
            sig = sum(rng.normal(0.0, 1.0) * np.cos(np.pi / frames * (t + 0.5) * k) for k in range(4, 8))
        pat = np.sin(0.35 * xx + 0.2 * yy) * np.cos(0.3 * zz)
        out += amp * pat[..., None] * sig[None, None, None, :]
    return out.astype(np.float32)


def sci_modes(shape_xyz, frames, seed):
    """A scientific field whose leaves take all four generic modes: smooth drifting blobs
    everywhere; x in the middle third adds the pattern of sci_flicker modulated by DCT-II
    frequencies 4..7 (amplitude 1), the last third by white noise per frame (amplitude 2.5); the
    upper half of the first third carries 0.2 % spikes of +-4 (SparseEvents), its lower half
    stays smooth (CoarseOnly).  Time fastest, [Z, Y, X, T]."""
    X, Y, Z = shape_xyz
    rng = np.random.default_rng(seed)
    out, (xx, yy, zz) = _drifting_blobs(shape_xyz, frames, rng, 6, 8.0, 16.0)
    pat = np.sin(0.35 * xx + 0.2 * yy) * np.cos(0.3 * zz)
    t = np.arange(frames)
    mid = sum(rng.normal(0.0, 1.0) * np.cos(np.pi / frames * (t + 0.5) * k) for k in range(4, 8))
    white = rng.normal(0.0, 1.0, frames)
    region = (xx * 3) // X
    out += np.where(region == 1, 1.0 * pat, 0.0)[..., None] * mid[None, None, None, :]
    out += np.where(region == 2, 2.5 * pat, 0.0)[..., None] * white[None, None, None, :]
    n = int(0.002 * out.size)
    idx = rng.choice(out.size, n, replace=False)
    zi, yi, xi, ti = np.unravel_index(idx, out.shape)
    keep = (xi < X // 3) & (zi >= Z // 2)
    out[zi[keep], yi[keep], xi[keep], ti[keep]] += 4.0 * np.sign(rng.normal(size=int(keep.sum())))
    return out.astype(np.float32)


# ----------------------------------------------------------------------------- encode
def encode(name, data, xyzt, profile, extra_meta=None, time_fastest=False, args=()):
    os.makedirs(ASSETS, exist_ok=True)
    if not os.path.exists(ENCODER):
        sys.path.insert(0, ROOT)
        from oracle.oracle import build
        build(ref=True)
    X, Y, Z, T = xyzt
    with tempfile.TemporaryDirectory(dir=os.environ.get("VBT_ASSET_TMP")) as td:
        raw = os.path.join(td, name + ".raw")
        meta = os.path.join(td, name + ".metadata.json")
        data.astype(np.float32).tofile(raw)
        m = {"dimensions": [X, Y, Z, T], "axis_order": ["X", "Y", "Z", "T"],
             "time_is_fastest_dimension": bool(time_fastest), "data_type": "float32",
             "data_min": float(data.min()), "data_max": float(data.max())}
        if extra_meta:
            m.update(extra_meta)
        with open(meta, "w") as fh:
            json.dump(m, fh)
        out = os.path.join(ASSETS, name + ".vbtp")
        cmd = [ENCODER, "--input-raw", raw, "--metadata", meta, "--profile", profile,
               "--save-vbt", out, "--report", os.path.join(td, "report.md"), "--omp-threads", "8"] + list(args)
        subprocess.check_call(cmd, stdout=subprocess.DEVNULL)
    print(f"{name}: {os.path.getsize(out)} bytes")
    return out


def encode_large_scientific(name, shape_xyz, frames, seed):
    """A scientific field written to disk by grf_scientific_to_file and encoded from there (the
    encoder reads the RAW file itself); the scratch files go under VBT_ASSET_TMP (default: the
    system temporary directory) and need about twice the RAW size."""
    os.makedirs(ASSETS, exist_ok=True)
    if not os.path.exists(ENCODER):
        sys.path.insert(0, ROOT)
        from oracle.oracle import build
        build(ref=True)
    X, Y, Z = shape_xyz
    with tempfile.TemporaryDirectory(dir=os.environ.get("VBT_ASSET_TMP")) as td:
        raw = os.path.join(td, name + ".raw")
        lo, hi = grf_scientific_to_file(shape_xyz, frames, seed, raw)
        meta = os.path.join(td, name + ".metadata.json")
        with open(meta, "w") as fh:
            json.dump({"dimensions": [X, Y, Z, frames], "axis_order": ["X", "Y", "Z", "T"],
                       "time_is_fastest_dimension": True, "data_type": "float32", "data_min": lo,
                       "data_max": hi}, fh)
        out = os.path.join(ASSETS, name + ".vbtp")
        cmd = [ENCODER, "--input-raw", raw, "--metadata", meta, "--profile", "generic", "--save-vbt", out,
               "--report", os.path.join(td, "report.md"), "--omp-threads", str(os.cpu_count())]
        subprocess.check_call(cmd, stdout=subprocess.DEVNULL)
    print(f"{name}: {os.path.getsize(out)} bytes")
    return out


LEVELSET = {"conversion_mode": "levelset", "shell_width_voxels": 3.0, "voxel_size": 1.0}

RECIPES = {
    "tiny_density": lambda: encode("tiny_density", blobs((20, 12, 17), 9, 3, 11), (20, 12, 17, 9), "density"),
    "tiny_levelset": lambda: encode("tiny_levelset", sdf_scene((24, 20, 28), 12, 12.0, 2.0, 0.3, 3, 2.0, 5.0, 12),
                                    (24, 20, 28, 12), "density", LEVELSET),
    "cfg1_blobs": lambda: encode("cfg1_blobs", blobs((64, 64, 64), 24, 6, 1), (64, 64, 64, 24), "density"),
    "cfg4_sdf_small": lambda: encode("cfg4_sdf_small", sdf_scene((64, 64, 64), 24, 24.0, 2.0, 0.2, 6, 3.0, 8.0, 4),
                                     (64, 64, 64, 24), "density", LEVELSET),
    "sci_small": lambda: encode("sci_small", grf_scientific((24, 16, 20), 16, 5), (24, 16, 20, 16), "generic",
                                time_fastest=True),
    "sci_64": lambda: encode("sci_64", grf_scientific((64, 64, 64), 32, 6), (64, 64, 64, 32), "generic",
                             time_fastest=True),
    "cfg2_plume": lambda: encode("cfg2_plume", plume(256, 96, 2), (256, 256, 256, 96), "density"),
    # scientific leaf modes beyond SparseEvents (generic profile): CoarseOnly, DenseGrid3/4 with the
    # per-frame BFP residual, and the DCT temporal-basis residual
    "sci_coarse": lambda: encode("sci_coarse", sci_flicker((24, 16, 20), 16, 3, 0.0, "none"), (24, 16, 20, 16),
                                 "generic", time_fastest=True),
    "sci_dense": lambda: encode("sci_dense", sci_flicker((24, 16, 20), 16, 3, 1.0, "white"), (24, 16, 20, 16),
                                "generic", time_fastest=True),
    "sci_dense_tb": lambda: encode("sci_dense_tb", sci_flicker((24, 16, 20), 16, 3, 0.3, "mid"), (24, 16, 20, 16),
                                   "generic", time_fastest=True,
                                   args=("--generic-dense-temporal-basis", "--generic-dense-temporal-keep", "8")),
    # configuration 5's scientific field at its stated size (512^3 x 64, time fastest, 34 GB of RAW)
    "cfg5_sci": lambda: encode_large_scientific("cfg5_sci", (512, 512, 512), 64, 8),
    "sci_modes": lambda: encode("sci_modes", sci_modes((64, 64, 64), 32, 21), (64, 64, 64, 32), "generic",
                                time_fastest=True,
                                args=("--generic-dense-temporal-basis", "--generic-dense-temporal-keep", "8")),
    # serving-mix assets: the config-3/4/5 scenes at reduced sizes (the full sizes need 36-64 GB
    # of raw float32 input per field, more than this machine's memory, and the encoded fields
    # must stay small enough to travel with the working tree)
    "mix_fire_density": lambda: encode("mix_fire_density", fire((128, 128, 192), 40, 7)[0], (128, 128, 192, 40),
                                       "density"),
    "mix_fire_flames": lambda: encode("mix_fire_flames", fire((128, 128, 192), 40, 7)[1], (128, 128, 192, 40),
                                      "density"),
    "mix_fire_temperature": lambda: encode("mix_fire_temperature", fire((128, 128, 192), 40, 7)[2],
                                           (128, 128, 192, 40), "density"),
    "mix_sdf": lambda: encode("mix_sdf", sdf_scene((128, 128, 128), 48, 50.0, 12.0, 0.05, 20, 3.0, 12.0, 9),
                              (128, 128, 128, 48), "density", LEVELSET),
    "mix_sci": lambda: encode("mix_sci", grf_scientific((128, 128, 128), 64, 8), (128, 128, 128, 64), "generic",
                              time_fastest=True),
}
MIX = ["cfg2_plume", "mix_fire_density", "mix_fire_flames", "mix_fire_temperature", "mix_sdf",
       "cfg1_blobs", "cfg4_sdf_small", "mix_sci"]
DEFAULT = ["tiny_density", "tiny_levelset", "sci_small", "cfg1_blobs", "cfg4_sdf_small", "sci_64", "cfg2_plume",
           "sci_modes"]

# the raw fields of the render-temporal assets: name -> (recipe, arguments, field of a multi-field
# recipe or None, (X, Y, Z), level set)
FIELDS = {
    "tiny_density": ("blobs", ((20, 12, 17), 9, 3, 11), None, (20, 12, 17), False),
    "tiny_levelset": ("sdf_scene", ((24, 20, 28), 12, 12.0, 2.0, 0.3, 3, 2.0, 5.0, 12), None, (24, 20, 28), True),
    "cfg1_blobs": ("blobs", ((64, 64, 64), 24, 6, 1), None, (64, 64, 64), False),
    "cfg4_sdf_small": ("sdf_scene", ((64, 64, 64), 24, 24.0, 2.0, 0.2, 6, 3.0, 8.0, 4), None, (64, 64, 64), True),
    "cfg2_plume": ("plume", (256, 96, 2), None, (256, 256, 256), False),
    "mix_fire_density": ("fire", ((128, 128, 192), 40, 7), 0, (128, 128, 192), False),
    "mix_fire_flames": ("fire", ((128, 128, 192), 40, 7), 1, (128, 128, 192), False),
    "mix_fire_temperature": ("fire", ((128, 128, 192), 40, 7), 2, (128, 128, 192), False),
    "mix_sdf": ("sdf_scene", ((128, 128, 128), 48, 50.0, 12.0, 0.05, 20, 3.0, 12.0, 9), None, (128, 128, 128), True),
}


def field_of(name):
    """(raw [T, Z, Y, X] float32, (X, Y, Z), level set) of a render-temporal asset's field."""
    fn, args, index, dims, levelset = FIELDS[name]
    raw = globals()[fn](*args)
    return (raw if index is None else raw[index]), dims, levelset


DIGESTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "asset_digests.json")


def write_digests():
    """SHA-256 and size of every asset present, so a machine that holds only some of the files can
    still check a file regenerated there against the one the reference encoder wrote."""
    import hashlib
    out = {}
    for f in sorted(os.listdir(ASSETS)):
        if f.endswith(".vbtp"):
            data = open(os.path.join(ASSETS, f), "rb").read()
            out[f[:-5]] = {"sha256": hashlib.sha256(data).hexdigest(), "bytes": len(data)}
    with open(DIGESTS, "w") as fh:
        json.dump(out, fh, indent=1, sort_keys=True)
        fh.write("\n")


if __name__ == "__main__":
    names = sys.argv[1:] or DEFAULT
    for n in names:
        if n == "digests":
            write_digests()
        else:
            RECIPES[n]()
