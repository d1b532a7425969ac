"""Seeded synthetic fields generated on the GPU, slab by slab (test and benchmark input only).

The fire and liquid scenes of make_assets.py at sizes whose raw float32 field (36-64 GB per field)
would not fit in host memory or travel as a file: the random draws that fix a scene (the value-noise
lattices, the sphere parameters) come from the same numpy generators and seeds as make_assets.py,
and the per-voxel arithmetic runs on the GPU with PyTorch, one group of z-planes at a time, so a
field is never held whole.  A slab function returns the frame-major [frames, (z1 - z0) * Y * X]
float32 tensor of the z-planes z0..z1-1, the layout vbt_b200.encode reads.

The values follow make_assets.py's recipes but are not bit-identical to its numpy fields (trilinear
upsampling and float32 arithmetic on the GPU); parity is checked on the files encoded from them,
against the oracle's decode of the same files.
"""
import numpy as np


def fbm_volume(torch, shape_zyx, octaves, base_cell, seed, device):
    """make_assets.fbm_volume on the GPU: value-noise lattices of the same seed, upsampled by the
    cell size with linear interpolation along each axis and the lattice corners on the output
    corners (scipy's zoom of order 1), summed over octaves with halving amplitude and normalised
    to [0, 1].  The interpolation is separable: bilinear in (y, x) on each lattice plane, then
    linear in z, a chunk of output planes at a time."""
    import torch.nn.functional as Fn
    rng = np.random.default_rng(seed)
    Z, Y, X = shape_zyx
    acc = torch.zeros(shape_zyx, dtype=torch.float32, device=device)
    amp, norm = 1.0, 0.0
    for o in range(octaves):
        cell = max(1, base_cell >> o)
        lat = rng.random((Z // cell + 2, Y // cell + 2, X // cell + 2)).astype(np.float32)
        nz, ny, nx = lat.shape
        t = torch.from_numpy(lat).to(device)[:, None]
        xy = Fn.interpolate(t, size=(ny * cell, nx * cell), mode="bilinear", align_corners=True)[:, 0, :Y, :X]
        scale = (nz - 1) / (nz * cell - 1)
        for z0 in range(0, Z, 64):
            zc = torch.arange(z0, min(Z, z0 + 64), device=device, dtype=torch.float64) * scale
            i0 = torch.clamp(zc.floor().long(), max=nz - 2)
            w = (zc - i0).float()[:, None, None]
            acc[z0:z0 + zc.numel()] += amp * (xy[i0] * (1.0 - w) + xy[i0 + 1] * w)
        norm += amp
        amp *= 0.5
    return acc / norm


class Fire:
    """make_assets.fire on the GPU: density, flames and temperature of an expanding fireball (fBm
    inside a sphere of radius 20 + 2.5 t at the lower centre, advected up one voxel per frame;
    flames from a second fBm in the sphere's outer band; temperature = 300 + 1500 flames +
    N(0, 20), the noise of each z-plane drawn from its own seeded generator so that a plane's
    values do not depend on the slab it is produced in)."""

    def __init__(self, torch, shape_xyz, frames, seed, device="cuda"):
        self.torch, self.dims, self.frames, self.seed, self.device = torch, tuple(shape_xyz), frames, seed, device
        X, Y, Z = shape_xyz
        self.n1 = fbm_volume(torch, (Z + frames, Y, X), 4, 32, seed, device)
        self.n2 = fbm_volume(torch, (Z + frames, Y, X), 4, 16, seed + 1, device)

    def slab(self, field, z0, z1):
        """field 0 density, 1 flames, 2 temperature: [frames, (z1 - z0) * Y * X] float32."""
        torch = self.torch
        X, Y, Z = self.dims
        T = self.frames
        dev = self.device
        zz = torch.arange(z0, z1, device=dev, dtype=torch.float32)[:, None, None]
        yy = torch.arange(Y, device=dev, dtype=torch.float32)[None, :, None]
        xx = torch.arange(X, device=dev, dtype=torch.float32)[None, None, :]
        r = torch.sqrt((xx - X / 2.0) ** 2 + (yy - Y / 2.0) ** 2 + (zz - Z * 0.3) ** 2)
        out = torch.empty((T, z1 - z0, Y, X), dtype=torch.float32, device=dev)
        for t in range(T):
            R = 20.0 + 2.5 * t
            inside = r <= R
            lo = T - t + z0
            if field == 0:
                v = torch.clamp((self.n1[lo:lo + z1 - z0] - 0.3) * 2.0, 0.0, 1.0) * torch.clamp((R - r) / 4.0, 0.0, 1.0)
            else:
                band = torch.clamp(1.0 - torch.abs(r - 0.8 * R) / (0.25 * R + 1e-6), 0.0, 1.0)
                v = torch.clamp((self.n2[lo:lo + z1 - z0] - 0.4) * 3.0, 0.0, 1.0) * band
            out[t] = torch.where(inside, v, torch.zeros_like(v))
        if field == 2:
            g = torch.Generator(device=dev)
            for z in range(z0, z1):
                g.manual_seed(self.seed * 1000003 + z)
                out[:, z - z0] = 300.0 + 1500.0 * out[:, z - z0] + 20.0 * torch.randn((T, Y, X), generator=g,
                                                                                      device=dev)
        return out.reshape(T, -1)


class LevelSet:
    """make_assets.sdf_scene on the GPU: the signed distance to the union of a sloshing plane
    z = plane_z + plane_amp sin(kx x + 0.1 t) and n_spheres spheres on ballistic paths under
    gravity g, evaluated in float64 and rounded to float32 as the numpy recipe does."""

    def __init__(self, torch, shape_xyz, frames, plane_z, plane_amp, kx, n_spheres, rmin, rmax, seed, g=0.05,
                 device="cuda"):
        self.torch, self.dims, self.frames, self.device = torch, tuple(shape_xyz), frames, device
        rng = np.random.default_rng(seed)
        X, Y, Z = shape_xyz
        self.c0 = np.stack([rng.uniform(0, X, n_spheres), rng.uniform(0, Y, n_spheres),
                            rng.uniform(plane_z, Z * 0.9, n_spheres)], axis=1)
        self.v0 = np.stack([rng.uniform(-0.5, 0.5, n_spheres), rng.uniform(-0.5, 0.5, n_spheres),
                            rng.uniform(0.0, 1.0, n_spheres)], axis=1)
        self.rad = rng.uniform(rmin, rmax, n_spheres)
        self.plane_z, self.plane_amp, self.kx, self.g = plane_z, plane_amp, kx, g

    def slab(self, z0, z1):
        torch = self.torch
        X, Y, Z = self.dims
        T = self.frames
        dev = self.device
        zz = torch.arange(z0, z1, device=dev, dtype=torch.float64)[:, None, None]
        yy = torch.arange(Y, device=dev, dtype=torch.float64)[None, :, None]
        xx = torch.arange(X, device=dev, dtype=torch.float64)[None, None, :]
        out = torch.empty((T, z1 - z0, Y, X), dtype=torch.float32, device=dev)
        for t in range(T):
            phi = zz - (self.plane_z + self.plane_amp * torch.sin(self.kx * xx + 0.1 * t))
            for s in range(self.c0.shape[0]):
                c = self.c0[s] + self.v0[s] * t + np.array([0.0, 0.0, -0.5 * self.g * t * t])
                d = torch.sqrt((xx - c[0]) ** 2 + (yy - c[1]) ** 2 + (zz - c[2]) ** 2) - self.rad[s]
                phi = torch.minimum(phi, d)
            out[t] = phi.float()
        return out.reshape(T, -1)


# the stated sizes of the fire and liquid configurations
FIRE_FULL = dict(shape_xyz=(384, 384, 512), frames=120, seed=7)
LEVELSET_FULL = dict(shape_xyz=(512, 512, 512), frames=120, plane_z=200.0, plane_amp=12.0, kx=0.05, n_spheres=40,
                     rmin=3.0, rmax=12.0, seed=9)
