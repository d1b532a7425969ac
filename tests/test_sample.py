"""Ray sampling from the control cache (vbt_sample_rays): the Studio's sampler
(VBTStudio/frontend/shaders/vbt_sample.comp) as plain CUDA, against the oracle's C restatement of
the same shader arithmetic, bit for bit, on every output of every ray.

Density accumulation (plain and into 8 depth bins) runs on the blob fields; the level-set surface
(hit, normal, thickness, floor shadow) on the Mode2 level sets.  Rays are seeded: they aim at
random points of the volume from outside it, so they cross EMPTY leaves, boundary leaves and the
background.
"""
import os

import numpy as np
import pytest

from conftest import ASSETS, golden_asset

pytestmark = pytest.mark.gpu


def make_rays(dims, n, seed, bbox_min=(0.0, 0.0, 0.0)):
    rng = np.random.default_rng(seed)
    X, Y, Z = dims
    target = rng.uniform([0, 0, 0], [X - 1, Y - 1, Z - 1], (n, 3)) + np.array(bbox_min)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    span = float(np.linalg.norm([X, Y, Z]))
    origin = target - d * span
    rays = np.zeros((n, 8), np.float32)
    rays[:, 0:3] = origin
    rays[:, 3] = rng.uniform(0.0, 2.0, n)          # t_min
    rays[:, 4:7] = d
    rays[:, 7] = 2.0 * span                          # t_max
    return rays


def params(vbt, **kw):
    p = vbt.SampleParams()
    p.step_count = kw.get("step_count", 64)
    p.frame_index = kw.get("frame_index", 0)
    for i, b in enumerate(kw.get("bbox_min", (0.0, 0.0, 0.0))):
        p.bbox_min[i] = b
    p.render_mode = kw.get("render_mode", 0)
    p.voxel_size = kw.get("voxel_size", 1.0)
    p.background_value = kw.get("background_value", 0.0)
    p.surface_iso = kw.get("surface_iso", 0.0)
    p.surface_epsilon_voxels = kw.get("surface_epsilon_voxels", 0.5)
    p.surface_normal_step = kw.get("surface_normal_step", 1.0)
    p.max_step_voxels = kw.get("max_step_voxels", 4.0)
    p.surface_model = kw.get("surface_model", 0)
    p.floor_height = kw.get("floor_height", 1.5)
    p.shadow_steps = kw.get("shadow_steps", 48)
    p.up_axis = kw.get("up_axis", 2)
    return p


def to_oracle_params(p):
    from oracle.oracle import VoSampleParams
    q = VoSampleParams()
    for name, _ in VoSampleParams._fields_:
        if name == "bbox_min":
            for i in range(3):
                q.bbox_min[i] = p.bbox_min[i]
        else:
            setattr(q, name, getattr(p, name))
    return q


def run_both(vbt, cuda, oracle, path, p, rays):
    a = vbt.Asset(path)
    f = oracle.load(path)
    a.build_page_table()
    compact, n = a.page_table()
    ctrl = cuda.zeros((1, max(n, 1), 576), dtype=cuda.float32, device="cuda")
    a.decode_control_cache([p.frame_index], ctrl, frame_stride=max(n, 1) * 576)
    want_ctrl = f.control_cache(p.frame_index, compact)
    assert np.array_equal(ctrl.cpu().numpy()[0, :n].view(np.uint32), want_ctrl.view(np.uint32))
    d_rays = cuda.from_numpy(rays).cuda()
    out = cuda.full((rays.shape[0], 8), float("nan"), dtype=cuda.float32, device="cuda")
    a.sample_rays(ctrl, p, d_rays, out)
    a.sync_status()
    got = out.cpu().numpy()
    want = f.sample_rays(want_ctrl, compact, to_oracle_params(p), rays)
    a.close()
    return got, want


def check(got, want, what):
    bad = np.flatnonzero((got.view(np.uint32) != want.view(np.uint32)).any(axis=1))
    assert bad.size == 0, (what, bad[:5], got[bad[:2]], want[bad[:2]])


def density_paths():
    out = [golden_asset("tiny_density")]
    for n in ("cfg1_blobs", "mix_fire_density"):
        p = os.path.join(ASSETS, n + ".vbtp")
        if os.path.exists(p):
            out.append(p)
    return out


def levelset_paths():
    out = [golden_asset("tiny_levelset")]
    for n in ("cfg4_sdf_small", "mix_sdf"):
        p = os.path.join(ASSETS, n + ".vbtp")
        if os.path.exists(p):
            out.append(p)
    return out


@pytest.mark.parametrize("path", density_paths(), ids=os.path.basename)
@pytest.mark.parametrize("bins", [0, 1], ids=["sum", "8bins"])
def test_density_rays(vbt, cuda, oracle, path, bins):
    a = vbt.Asset(path)
    dims, T = a.dims, a.frames
    a.close()
    rays = make_rays(dims, 3000, seed=5)
    for frame in (0, T // 2, T + 3):
        p = params(vbt, render_mode=0, step_count=72, frame_index=frame, surface_model=bins)
        got, want = run_both(vbt, cuda, oracle, path, p, rays)
        check(got, want, (os.path.basename(path), frame))
        assert np.abs(want).max() > 0         # the rays see the field


@pytest.mark.parametrize("path", levelset_paths(), ids=os.path.basename)
def test_level_set_rays(vbt, cuda, oracle, path):
    a = vbt.Asset(path)
    dims, T = a.dims, a.frames
    a.close()
    rays = make_rays(dims, 2000, seed=9, bbox_min=(-3.0, 2.0, 0.5))
    for frame, model in ((0, 1), (T - 1, 0)):
        p = params(vbt, render_mode=1, step_count=96, frame_index=frame, surface_model=model,
                   bbox_min=(-3.0, 2.0, 0.5), background_value=1.0, floor_height=1.0)
        got, want = run_both(vbt, cuda, oracle, path, p, rays)
        check(got, want, (os.path.basename(path), frame))
        assert (want[:, 3] >= 0).any()        # some rays hit the surface


def test_sampler_rejects_bad_arguments(vbt, cuda):
    a = vbt.Asset(golden_asset("sci_small"))
    ctrl = cuda.zeros(576, dtype=cuda.float32, device="cuda")
    rays = cuda.zeros((4, 8), dtype=cuda.float32, device="cuda")
    out = cuda.zeros((4, 8), dtype=cuda.float32, device="cuda")
    with pytest.raises(vbt.VbtError):
        a.sample_rays(ctrl, params(vbt), rays, out)     # scientific asset
    a.close()
    a = vbt.Asset(golden_asset("tiny_density"))
    with pytest.raises(vbt.VbtError):
        a.sample_rays(ctrl, params(vbt, render_mode=2), rays, out)
    a.close()


def smoke_paths():
    out = [golden_asset("tiny_density"), golden_asset("tiny_levelset")]
    for n in ("cfg1_blobs", "mix_fire_density", "mix_sdf"):
        p = os.path.join(ASSETS, n + ".vbtp")
        if os.path.exists(p):
            out.append(p)
    return out


@pytest.mark.parametrize("path", smoke_paths(), ids=os.path.basename)
def test_smoke_sampler(vbt, cuda, oracle, path):
    """render/shaders/vbt_smoke_sample.comp (density summed straight from the payload) against the
    oracle's C restatement, bit for bit, at the first, a middle and a clamped frame; FINE6 and
    Mode2 leaves included (Mode2 contributes its coarse stream, as in the shader)."""
    a = vbt.Asset(path)
    f = oracle.load(path)
    dims, T = a.dims, a.frames
    rays = make_rays(dims, 3000, seed=13, bbox_min=(1.5, -2.0, 0.25))
    d_rays = cuda.from_numpy(rays).cuda()
    out = cuda.full((rays.shape[0],), float("nan"), dtype=cuda.float32, device="cuda")
    for frame, steps in ((0, 48), (T // 2, 96), (T + 4, 33)):
        p = params(vbt, step_count=steps, frame_index=frame, bbox_min=(1.5, -2.0, 0.25))
        a.smoke_sample_rays(p, d_rays, out)
        cuda.cuda.synchronize()
        got = out.cpu().numpy()
        want = f.smoke_sample_rays(to_oracle_params(p), rays)
        bad = np.flatnonzero(got.view(np.uint32) != want.view(np.uint32))
        assert bad.size == 0, (os.path.basename(path), frame, bad[:5], got[bad[:3]], want[bad[:3]])
        assert (want != 0).sum() > 100                      # the rays see the field
    a.close()


def test_smoke_sampler_rejects_scientific(vbt, cuda):
    a = vbt.Asset(golden_asset("sci_small"))
    rays = cuda.zeros((4, 8), dtype=cuda.float32, device="cuda")
    out = cuda.zeros(4, dtype=cuda.float32, device="cuda")
    with pytest.raises(vbt.VbtError):
        a.smoke_sample_rays(params(vbt), rays, out)
    a.close()
