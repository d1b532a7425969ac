// sample.cu -- the Studio's ray sampler over the current-frame control cache
// (VBTStudio/frontend/shaders/vbt_sample.comp), one thread per ray, as plain CUDA with a device
// buffer for its results (vbt_sample_rays); and the render tree's smoke sampler that sums density
// straight from the payload (render/shaders/vbt_smoke_sample.comp, vbt_smoke_sample_rays).
//
// The arithmetic follows the shader operation by operation in single precision with every
// operation rounded on its own (the library is built without FMA contraction): GLSL mix(a, b, t)
// is a*(1 - t) + b*t, round() rounds halves away from zero, normalize(v) is v / length(v), dot
// products sum x, y, z in that order, and min / max / clamp select as GLSL defines them.  A
// control value read straight from the payload (coarse grids above 64 controls, which the cache
// does not hold) is the reference CPU decoder's, as the cache's values are.
#include <cuda_runtime.h>

#include <string>

#include "asset.h"
#include "kernels.cuh"
#include "rt_search.cuh"

namespace vbtb {
int set_last_error(int status, const std::string& msg);

namespace {

constexpr uint32_t kCacheStride = 576u, kCoarseSlots = 64u;

struct Sampler {
    const DeviceAsset& a;
    const float* __restrict__ cache;
    const vbt_sample_params& p;
    int frame;              // clamped frame index
    uint32_t bin8;          // its 8-bin time bin
};

__device__ __forceinline__ uint32_t rd_byte(const uint32_t* __restrict__ pw, uint32_t bw, uint32_t o)
{
    return (__ldg(pw + bw + (o >> 2)) >> ((o & 3u) * 8u)) & 0xFFu;
}
__device__ __forceinline__ uint32_t rd_u16(const uint32_t* pw, uint32_t bw, uint32_t o)
{
    return rd_byte(pw, bw, o) | (rd_byte(pw, bw, o + 1u) << 8);
}
__device__ __forceinline__ uint32_t rd_u32(const uint32_t* pw, uint32_t bw, uint32_t o)
{
    return rd_byte(pw, bw, o) | (rd_byte(pw, bw, o + 1u) << 8) | (rd_byte(pw, bw, o + 2u) << 16) |
           (rd_byte(pw, bw, o + 3u) << 24);
}
__device__ __forceinline__ float mixf(float a, float b, float t)
{
    return __fadd_rn(__fmul_rn(a, __fsub_rn(1.0f, t)), __fmul_rn(b, t));
}
// GLSL min / max / clamp: min(x, y) = y < x ? y : x, max(x, y) = x < y ? y : x, clamp = min(max())
__device__ __forceinline__ float gmin(float x, float y) { return y < x ? y : x; }
__device__ __forceinline__ float gmax(float x, float y) { return x < y ? y : x; }
__device__ __forceinline__ float clampf(float x, float lo, float hi) { return gmin(gmax(x, lo), hi); }
__device__ __forceinline__ float along(float o, float d, float t) { return __fadd_rn(o, __fmul_rn(d, t)); }

// vbt_sample.comp:191-206
__device__ __forceinline__ float control_coord(uint32_t index, uint32_t res)
{
    if (res <= 1u) return 0.0f;
    return __fmul_rn((float)index, __fdiv_rn(7.0f, (float)(res - 1u)));
}
__device__ __forceinline__ void locate_coord(float pos, uint32_t extent, uint32_t res, uint32_t& i0, uint32_t& i1,
                                             float& w)
{
    const float c = clampf(pos, 0.0f, gmax(__fsub_rn((float)extent, 1.0f), 0.0f));
    uint32_t j1 = 1u;
    while (j1 < res - 1u && control_coord(j1, res) < c) ++j1;
    i0 = (int)j1 - 1 > 0 ? j1 - 1u : 0u;
    i1 = j1;
    const float c0 = control_coord(i0, res), c1 = control_coord(j1, res);
    w = c1 > c0 ? __fdiv_rn(__fsub_rn(c, c0), __fsub_rn(c1, c0)) : 0.0f;
}

// vbt_sample.comp:213-268 (currentFrameControl, sampleControlStream)
__device__ float sample_stream(const Sampler& S, uint32_t cl, uint32_t slot_base, uint32_t wb, uint32_t stream_base,
                               uint32_t codec, uint32_t res, uint32_t kf, uint32_t w, uint32_t h, uint32_t d, float lx,
                               float ly, float lz)
{
    if (res == 0u) return 0.0f;   // no controls (locateCoord would count to 2^32)
    uint32_t x0, x1, y0, y1, z0, z1;
    float tx, ty, tz;
    locate_coord(lx, w, res, x0, x1, tx);
    locate_coord(ly, h, res, y0, y1, ty);
    locate_coord(lz, d, res, z0, z1, tz);
    const uint32_t cc = res * res * res;
    const bool direct = slot_base == 0u && cc > kCoarseSlots;
    const StreamRef st{4ull * wb + stream_base, cc, 8u, kf, codec};
    const float* row = S.cache + (uint64_t)cl * kCacheStride + slot_base;
    auto ctrl = [&](uint32_t x, uint32_t y, uint32_t z) -> float {
        const uint32_t ci = (z * res + y) * res + x;
        return direct ? decode_control(S.a.payload, st, ci, S.frame, S.bin8) : __ldg(row + ci);
    };
    const float v000 = ctrl(x0, y0, z0), v100 = ctrl(x1, y0, z0), v010 = ctrl(x0, y1, z0), v110 = ctrl(x1, y1, z0);
    const float v001 = ctrl(x0, y0, z1), v101 = ctrl(x1, y0, z1), v011 = ctrl(x0, y1, z1), v111 = ctrl(x1, y1, z1);
    const float c00 = mixf(v000, v100, tx), c10 = mixf(v010, v110, tx);
    const float c01 = mixf(v001, v101, tx), c11 = mixf(v011, v111, tx);
    return mixf(mixf(c00, c10, ty), mixf(c01, c11, ty), tz);
}

// vbt_sample.comp:298-320 (sampleShellResidual)
__device__ float sample_shell(const Sampler& S, uint32_t wb, uint32_t occ_base, uint32_t cl, uint32_t voxel,
                              bool& occupied)
{
    const uint32_t* pw = S.a.payload;
    const uint32_t group = voxel >> 6, bit = voxel & 63u, wig = bit >> 5, lb = bit & 31u;
    const uint32_t mask_word = rd_u32(pw, wb, occ_base + group * 8u + wig * 4u);
    occupied = ((mask_word >> lb) & 1u) != 0u;
    if (!occupied) return 0.0f;
    const uint32_t prefix = rd_u16(pw, wb, occ_base + 64u + group * 2u);
    const uint32_t low_word = rd_u32(pw, wb, occ_base + group * 8u);
    uint32_t di = prefix;
    if (wig != 0u) di += (uint32_t)__popc(low_word);
    const uint32_t before = lb == 0u ? 0u : (0xFFFFFFFFu >> (32u - lb));
    di += (uint32_t)__popc(mask_word & before);
    if (di >= kCacheStride - kCoarseSlots) return 0.0f;   // past the cache row (a malformed leaf)
    return __ldg(S.cache + (uint64_t)cl * kCacheStride + kCoarseSlots + di);
}

// vbt_sample.comp:322-415 (sampleVbtValue)
__device__ float sample_value(const Sampler& S, float wx, float wy, float wz, bool preserve_interior)
{
    const DeviceAsset& a = S.a;
    const vbt_sample_params& p = S.p;
    const float bg = p.render_mode == 1u ? p.background_value : 0.0f;
    const float px = __fsub_rn(wx, p.bbox_min[0]), py = __fsub_rn(wy, p.bbox_min[1]), pz = __fsub_rn(wz, p.bbox_min[2]);
    if (px < 0.0f || py < 0.0f || pz < 0.0f || px > (float)(a.g.width - 1u) || py > (float)(a.g.height - 1u) ||
        pz > (float)(a.g.depth - 1u))
        return bg;
    const uint32_t x = min(a.g.width - 1u, (uint32_t)floorf(px)), y = min(a.g.height - 1u, (uint32_t)floorf(py)),
                   z = min(a.g.depth - 1u, (uint32_t)floorf(pz));
    const uint32_t bx = min(a.g.lcx - 1u, x / 8u), by = min(a.g.lcy - 1u, y / 8u), bz = min(a.g.lcz - 1u, z / 8u);
    const uint32_t leaf = (bz * a.g.lcy + by) * a.g.lcx + bx;
    const uint32_t wb = __ldg(a.offsets + leaf), we = __ldg(a.offsets + leaf + 1);
    if (we <= wb) return bg;
    const uint32_t* pw = a.payload;
    const uint32_t hdr = __ldg(pw + wb), mode = hdr & 3u;
    if (mode == kModeEmpty) return bg;
    if (entry_status(a.entries[leaf]) != kOk) return bg;   // a leaf the walker rejected is not read
    const uint32_t cl = __ldg(a.compact + leaf);
    const uint32_t ccodec = (hdr >> 2) & 3u, fcodec = (hdr >> 4) & 3u;
    const uint32_t cres = (hdr >> 6) & 7u, fres = (hdr >> 9) & 7u;
    const uint32_t ckf = rd_u16(pw, wb, 4u), fkf = rd_u16(pw, wb, 6u);
    const uint32_t cc = cres * cres * cres;
    const uint32_t cbase = 8u;
    const uint32_t fbase = cbase + cc * 4u + align4(cc * 8u) + align4(ckf * (ccodec == 1u ? 8u : 3u));
    const uint32_t gx = bx * 8u, gy = by * 8u, gz = bz * 8u;
    const uint32_t w = min(8u, a.g.width - gx), h = min(8u, a.g.height - gy), d = min(8u, a.g.depth - gz);
    const float lx = __fsub_rn(px, (float)gx), ly = __fsub_rn(py, (float)gy), lz = __fsub_rn(pz, (float)gz);
    float value = sample_stream(S, cl, 0u, wb, cbase, ccodec, cres, ckf, w, h, d, lx, ly, lz);
    if (mode == kModeFine6 && fres > 0u) {
        value = __fadd_rn(value, sample_stream(S, cl, kCoarseSlots, wb, fbase, fcodec, fres, fkf, w, h, d, lx, ly, lz));
    } else if (mode == kModeFineCompact) {
        const uint32_t ux = (uint32_t)clampf(roundf(lx), 0.0f, 7.0f);
        const uint32_t uy = (uint32_t)clampf(roundf(ly), 0.0f, 7.0f);
        const uint32_t uz = (uint32_t)clampf(roundf(lz), 0.0f, 7.0f);
        bool occupied = false;
        value = __fadd_rn(value, sample_shell(S, wb, fbase, cl, (uz * 8u + uy) * 8u + ux, occupied));
        if (!preserve_interior && !occupied && value < 0.0f) value = bg;
    }
    return value;
}

__device__ __forceinline__ float sample_at(const Sampler& S, const float* o, const float* dir, float t, bool keep)
{
    return sample_value(S, along(o[0], dir[0], t), along(o[1], dir[1], t), along(o[2], dir[2], t), keep);
}

// vbt_sample.comp:417-431 (intersectWorldBox)
__device__ bool intersect_box(const Sampler& S, const float* o, const float* dir, float& near_t, float& far_t)
{
    const vbt_sample_params& p = S.p;
    const float mx[3] = {__fadd_rn(p.bbox_min[0], (float)(S.a.g.width - 1u)),
                         __fadd_rn(p.bbox_min[1], (float)(S.a.g.height - 1u)),
                         __fadd_rn(p.bbox_min[2], (float)(S.a.g.depth - 1u))};
    float lo[3], hi[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float inv = __fdiv_rn(1.0f, dir[k]);
        const float c0 = __fmul_rn(__fsub_rn(p.bbox_min[k], o[k]), inv), c1 = __fmul_rn(__fsub_rn(mx[k], o[k]), inv);
        lo[k] = gmin(c0, c1);
        hi[k] = gmax(c0, c1);
    }
    near_t = gmax(0.0f, gmax(lo[0], gmax(lo[1], lo[2])));
    far_t = gmin(hi[0], gmin(hi[1], hi[2]));
    return far_t > near_t;
}

__device__ __forceinline__ float phi_step(float phi, float voxel, float scale, float lo, float hi)
{
    return clampf(__fmul_rn(__fdiv_rn(fabsf(phi), gmax(voxel, 1e-6f)), scale), lo, hi);
}

// vbt_sample.comp:433-455 (traceShadow)
__device__ float trace_shadow(const Sampler& S, const float* o, const float* dir)
{
    const vbt_sample_params& p = S.p;
    float near_t, far_t;
    if (!intersect_box(S, o, dir, near_t, far_t)) return 0.0f;
    const float eps = gmax(__fmul_rn(p.surface_epsilon_voxels, p.voxel_size), 1e-5f);
    float t = near_t;
    float prev = __fsub_rn(sample_at(S, o, dir, t, false), p.surface_iso);
    for (uint32_t it = 0; it < p.shadow_steps; ++it) {
        const float nt = gmin(__fadd_rn(t, phi_step(prev, p.voxel_size, 0.8f, 0.35f, 5.0f)), far_t);
        const float np = __fsub_rn(sample_at(S, o, dir, nt, false), p.surface_iso);
        if ((prev < 0.0f) != (np < 0.0f)) {
            const bool next_inside = np < 0.0f;
            const float neg = next_inside ? np : prev;
            const float st = next_inside ? gmin(__fadd_rn(nt, 0.35f), far_t) : gmax(__fsub_rn(t, 0.35f), near_t);
            const float sp = __fsub_rn(sample_at(S, o, dir, st, false), p.surface_iso);
            if (neg <= __fmul_rn(-eps, 0.5f) || sp <= __fmul_rn(-eps, 0.25f)) return 1.0f;
        }
        if (nt >= far_t) break;
        t = nt;
        prev = fabsf(np) <= eps ? eps : np;
    }
    return 0.0f;
}

// vbt_sample.comp:457-476 (estimateThickness)
__device__ float estimate_thickness(const Sampler& S, const float* ray, float hit_t)
{
    const vbt_sample_params& p = S.p;
    const float* o = ray;
    const float* dir = ray + 4;
    const float tmax = ray[7];
    const float eps = gmax(__fmul_rn(p.surface_epsilon_voxels, p.voxel_size), 1e-5f);
    float t = gmin(__fadd_rn(hit_t, 0.35f), tmax);
    float prev = __fsub_rn(sample_at(S, o, dir, t, true), p.surface_iso);
    bool entered = prev < __fmul_rn(-0.25f, eps);
    const uint32_t limit = min(p.step_count, 160u);
    for (uint32_t it = 0; it < limit; ++it) {
        const float nt = gmin(__fadd_rn(t, phi_step(prev, p.voxel_size, 0.7f, 0.3f, 3.0f)), tmax);
        const float np = __fsub_rn(sample_at(S, o, dir, nt, true), p.surface_iso);
        entered = entered || np < __fmul_rn(-0.25f, eps);
        if (entered && prev < 0.0f && np >= 0.0f)
            return gmax(__fmul_rn(__fsub_rn(nt, hit_t), p.voxel_size), __fmul_rn(p.voxel_size, 0.25f));
        if (nt >= tmax) break;
        t = nt;
        prev = np;
    }
    return __fmul_rn(p.voxel_size, 6.0f);
}

__device__ __forceinline__ float len3(float x, float y, float z)
{
    return __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(x, x), __fmul_rn(y, y)), __fmul_rn(z, z)));
}

// vbt_sample.comp:478-546 (traceLevelSet)
__device__ void trace_level_set(const Sampler& S, const float* ray, float* res)
{
    const vbt_sample_params& p = S.p;
    const float* o = ray;
    const float* dir = ray + 4;
    const float tmax = ray[7];
    res[0] = res[1] = res[2] = 0.0f;
    res[3] = -1.0f;
    res[4] = res[5] = res[6] = res[7] = 0.0f;
    if (tmax <= 0.0f) return;
    const float eps = gmax(__fmul_rn(p.surface_epsilon_voxels, p.voxel_size), 1e-5f);
    float prev_t = 0.0f;
    float prev = __fsub_rn(sample_value(S, o[0], o[1], o[2], false), p.surface_iso);
    float hit_t = -1.0f;
    for (uint32_t it = 0; it < p.step_count; ++it) {
        const float step = phi_step(prev, p.voxel_size, 0.8f, 0.2f, gmax(p.max_step_voxels, 0.2f));
        const float cur_t = gmin(__fadd_rn(prev_t, step), tmax);
        const float cur = __fsub_rn(sample_at(S, o, dir, cur_t, false), p.surface_iso);
        if ((prev < 0.0f) != (cur < 0.0f)) {
            const bool cur_inside = cur < 0.0f;
            const float neg = cur_inside ? cur : prev;
            const float st = cur_inside ? gmin(__fadd_rn(cur_t, 0.35f), tmax) : gmax(__fsub_rn(prev_t, 0.35f), 0.0f);
            const float sp = __fsub_rn(sample_at(S, o, dir, st, false), p.surface_iso);
            const bool support = neg <= __fmul_rn(-eps, 0.5f) || sp <= __fmul_rn(-eps, 0.25f);
            if (!support) {
                if (cur_t >= tmax) break;
                prev_t = cur_t;
                prev = gmax(cur, eps);
                continue;
            }
            float low = prev_t, high = cur_t, low_phi = prev;
            for (int r = 0; r < 5; ++r) {
                const float mid = __fmul_rn(0.5f, __fadd_rn(low, high));
                const float mid_phi = __fsub_rn(sample_at(S, o, dir, mid, false), p.surface_iso);
                if ((low_phi < 0.0f) != (mid_phi < 0.0f)) {
                    high = mid;
                } else {
                    low = mid;
                    low_phi = mid_phi;
                }
            }
            hit_t = __fmul_rn(0.5f, __fadd_rn(low, high));
            break;
        }
        if (cur_t >= tmax) break;
        prev_t = cur_t;
        prev = cur;
    }
    if (hit_t < 0.0f) return;
    const float hx = along(o[0], dir[0], hit_t), hy = along(o[1], dir[1], hit_t), hz = along(o[2], dir[2], hit_t);
    const float ns = gmax(p.surface_normal_step, 0.25f);
    const float gx = __fsub_rn(sample_value(S, __fadd_rn(hx, ns), hy, hz, false), sample_value(S, __fsub_rn(hx, ns), hy, hz, false));
    const float gy = __fsub_rn(sample_value(S, hx, __fadd_rn(hy, ns), hz, false), sample_value(S, hx, __fsub_rn(hy, ns), hz, false));
    const float gz = __fsub_rn(sample_value(S, hx, hy, __fadd_rn(hz, ns), false), sample_value(S, hx, hy, __fsub_rn(hz, ns), false));
    const float gl = len3(gx, gy, gz);
    float nx, ny, nz;
    if (gl > 1e-6f) {
        nx = __fdiv_rn(gx, gl);
        ny = __fdiv_rn(gy, gl);
        nz = __fdiv_rn(gz, gl);
    } else {
        nx = -dir[0];
        ny = -dir[1];
        nz = -dir[2];
    }
    res[0] = nx;
    res[1] = ny;
    res[2] = nz;
    res[3] = hit_t;
    res[4] = p.surface_model != 0u ? estimate_thickness(S, ray, hit_t) : 0.0f;
    res[7] = fabsf(__fadd_rn(__fadd_rn(__fmul_rn(nx, -dir[0]), __fmul_rn(ny, -dir[1])), __fmul_rn(nz, -dir[2])));
}

// vbt_sample.comp:548-622 (main)
__global__ void __launch_bounds__(128) sample_rays_kernel(DeviceAsset a, const float* __restrict__ cache,
                                                          vbt_sample_params p, const float4* __restrict__ rays,
                                                          uint32_t n, float4* __restrict__ out)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int frame = clamp_frame(p.frame_index, (int)a.g.frames);
    const Sampler S{a, cache, p, frame, time_bin(frame, 8u, a.g.frames)};
    const float4 r0 = rays[2 * i], r1 = rays[2 * i + 1];
    const float ray[8] = {r0.x, r0.y, r0.z, r0.w, r1.x, r1.y, r1.z, r1.w};
    const float* o = ray;
    const float* dir = ray + 4;
    float res[8];
    if (p.render_mode == 1u) {
        trace_level_set(S, ray, res);
        const float fdir = p.up_axis == 2u ? dir[2] : dir[1];
        const float forg = p.up_axis == 2u ? o[2] : o[1];
        if (p.surface_model != 0u && res[3] < 0.0f && fdir < -1e-5f) {
            const float ft = __fdiv_rn(__fsub_rn(p.floor_height, forg), fdir);
            if (ft > 0.0f) {
                const float fx = along(o[0], dir[0], ft), fy = along(o[1], dir[1], ft), fz = along(o[2], dir[2], ft);
                float kx = -0.55f, ky = p.up_axis == 2u ? 0.42f : 0.72f, kz = p.up_axis == 2u ? 0.72f : 0.42f;
                const float kl = len3(kx, ky, kz);
                kx = __fdiv_rn(kx, kl);
                ky = __fdiv_rn(ky, kl);
                kz = __fdiv_rn(kz, kl);
                const float so[3] = {along(fx, kx, 0.5f), along(fy, ky, 0.5f), along(fz, kz, 0.5f)};
                const float sd[3] = {kx, ky, kz};
                res[5] = 1.0f;
                res[6] = trace_shadow(S, so, sd);
            }
        }
    } else {
        const float dt = __fdiv_rn(ray[7], gmax((float)p.step_count, 1.0f));
        float t = __fadd_rn(ray[3], __fmul_rn(0.5f, dt));
#pragma unroll
        for (int k = 0; k < 8; ++k) res[k] = 0.0f;
        if (p.surface_model != 0u) {
            const uint32_t sc = max(p.step_count, 1u);
            for (uint32_t s = 0; s < p.step_count; ++s) {
                const float v = sample_at(S, o, dir, t, false);
                const uint32_t bin = min((s * 8u) / sc, 7u);
                res[bin] = __fadd_rn(res[bin], v);
                t = __fadd_rn(t, dt);
            }
        } else {
            float acc = 0.0f;
            for (uint32_t s = 0; s < p.step_count; ++s) {
                acc = __fadd_rn(acc, sample_at(S, o, dir, t, false));
                t = __fadd_rn(t, dt);
            }
            res[0] = acc;
        }
    }
    out[2 * i] = make_float4(res[0], res[1], res[2], res[3]);
    out[2 * i + 1] = make_float4(res[4], res[5], res[6], res[7]);
}

// ---- render/shaders/vbt_smoke_sample.comp: density summed straight from the payload -----------
// Every sample decodes the eight corner controls of the coarse stream (and of the FINE6 stream)
// with the shader's own decodeTemporalControlValue: the reference search, but the lerp is
// mix(previous, next, w) with w = float(frame - f0) / float(f1 - f0) (IEEE division).  Mode2
// leaves contribute their coarse stream only, as in the shader.  Leaves the walker rejected, and
// streams of resolution 0 (where the shader's locateCoord would count to 2^32), contribute 0.

struct SmokeSampler {
    const DeviceAsset& a;
    uint32_t frame, bin;    // clamped frame and its 8-bin time bin
};

__device__ __forceinline__ uint32_t smoke_key_frame(const uint32_t* pw, uint32_t wb, uint32_t kb, uint32_t codec,
                                                    uint32_t i)
{
    return codec == 1u ? rd_u16(pw, wb, kb + i * 8u) : rd_byte(pw, wb, kb + i * 3u);
}
__device__ __forceinline__ float smoke_key_value(const uint32_t* pw, uint32_t wb, uint32_t kb, uint32_t codec,
                                                 uint32_t i)
{
    if (codec == 1u) return __uint_as_float(rd_u32(pw, wb, kb + i * 8u + 4u));
    return half_bits_to_float(rd_u16(pw, wb, kb + i * 3u + 1u));
}

// vbt_smoke_sample.comp:124-171 (decodeTemporalControlValue)
__device__ float smoke_control(const SmokeSampler& S, uint32_t wb, uint32_t sb, uint32_t codec, uint32_t cc,
                               uint32_t kf, uint32_t ci)
{
    if (ci >= cc) return 0.0f;
    const uint32_t* pw = S.a.payload;
    const uint32_t kb = sb + cc * 4u + align4(cc * 8u);
    const uint32_t start = rd_u16(pw, wb, sb + ci * 4u), count = rd_byte(pw, wb, sb + ci * 4u + 2u);
    if (count == 0u || start + count > kf) return 0.0f;
    const uint32_t frame = S.frame, bins = sb + cc * 4u + ci * 8u;
    uint32_t lo = min(rd_byte(pw, wb, bins + S.bin), count - 1u);
    uint32_t f0 = smoke_key_frame(pw, wb, kb, codec, start + lo);
    if (f0 > frame) {
        lo = 0u;
        f0 = smoke_key_frame(pw, wb, kb, codec, start);
    }
    if (f0 >= frame || lo + 1u >= count) return smoke_key_value(pw, wb, kb, codec, start + lo);
    uint32_t hi = S.bin + 1u < 8u ? min(count - 1u, rd_byte(pw, wb, bins + S.bin + 1u) + 1u) : count - 1u;
    hi = max(hi, lo + 1u);
    uint32_t f1 = smoke_key_frame(pw, wb, kb, codec, start + hi);
    if (f1 < frame) {
        hi = count - 1u;
        f1 = smoke_key_frame(pw, wb, kb, codec, start + hi);
    }
    if (f1 <= frame) return smoke_key_value(pw, wb, kb, codec, start + hi);
    while (hi > lo + 1u) {
        const uint32_t mid = lo + (hi - lo) / 2u;
        const uint32_t fm = smoke_key_frame(pw, wb, kb, codec, start + mid);
        if (fm < frame) {
            lo = mid;
            f0 = fm;
        } else {
            hi = mid;
            f1 = fm;
        }
    }
    const float next = smoke_key_value(pw, wb, kb, codec, start + hi);
    if (f1 == frame) return next;
    const float prev = smoke_key_value(pw, wb, kb, codec, start + lo);
    return mixf(prev, next, __fdiv_rn((float)(frame - f0), (float)(f1 - f0)));
}

// vbt_smoke_sample.comp:195-232 (sampleControlStream)
__device__ float smoke_stream(const SmokeSampler& S, uint32_t wb, uint32_t sb, uint32_t codec, uint32_t res,
                              uint32_t kf, uint32_t w, uint32_t h, uint32_t d, float lx, float ly, float lz)
{
    if (res == 0u) return 0.0f;
    uint32_t x0, x1, y0, y1, z0, z1;
    float tx, ty, tz;
    locate_coord(lx, w, res, x0, x1, tx);
    locate_coord(ly, h, res, y0, y1, ty);
    locate_coord(lz, d, res, z0, z1, tz);
    const uint32_t cc = res * res * res;
    auto ctrl = [&](uint32_t x, uint32_t y, uint32_t z) {
        return smoke_control(S, wb, sb, codec, cc, kf, (z * res + y) * res + x);
    };
    const float v000 = ctrl(x0, y0, z0), v100 = ctrl(x1, y0, z0), v010 = ctrl(x0, y1, z0), v110 = ctrl(x1, y1, z0);
    const float v001 = ctrl(x0, y0, z1), v101 = ctrl(x1, y0, z1), v011 = ctrl(x0, y1, z1), v111 = ctrl(x1, y1, z1);
    const float c00 = mixf(v000, v100, tx), c10 = mixf(v010, v110, tx);
    const float c01 = mixf(v001, v101, tx), c11 = mixf(v011, v111, tx);
    return mixf(mixf(c00, c10, ty), mixf(c01, c11, ty), tz);
}

// vbt_smoke_sample.comp:234-305 (sampleVbtDensity)
__device__ float smoke_density(const SmokeSampler& S, const vbt_sample_params& p, float wx, float wy, float wz)
{
    const DeviceAsset& a = S.a;
    const float px = __fsub_rn(wx, p.bbox_min[0]), py = __fsub_rn(wy, p.bbox_min[1]), pz = __fsub_rn(wz, p.bbox_min[2]);
    if (px < 0.0f || py < 0.0f || pz < 0.0f || px > (float)(a.g.width - 1u) || py > (float)(a.g.height - 1u) ||
        pz > (float)(a.g.depth - 1u))
        return 0.0f;
    const uint32_t x = min(a.g.width - 1u, (uint32_t)floorf(px)), y = min(a.g.height - 1u, (uint32_t)floorf(py)),
                   z = min(a.g.depth - 1u, (uint32_t)floorf(pz));
    const uint32_t bx = min(a.g.lcx - 1u, x / 8u), by = min(a.g.lcy - 1u, y / 8u), bz = min(a.g.lcz - 1u, z / 8u);
    const uint32_t leaf = (bz * a.g.lcy + by) * a.g.lcx + bx;
    const uint32_t wb = __ldg(a.offsets + leaf), we = __ldg(a.offsets + leaf + 1);
    if (we <= wb) return 0.0f;
    const uint32_t hdr = __ldg(a.payload + wb), mode = hdr & 3u;
    if (mode == kModeEmpty) return 0.0f;
    if (entry_status(a.entries[leaf]) != kOk) return 0.0f;   // a leaf the walker rejected is not read
    const uint32_t ccodec = (hdr >> 2) & 3u, fcodec = (hdr >> 4) & 3u;
    const uint32_t cres = (hdr >> 6) & 7u, fres = (hdr >> 9) & 7u;
    const uint32_t ckf = rd_u16(a.payload, wb, 4u), fkf = rd_u16(a.payload, wb, 6u);
    const uint32_t cc = cres * cres * cres;
    const uint32_t fbase = 8u + cc * 4u + align4(cc * 8u) + align4(ckf * (ccodec == 1u ? 8u : 3u));
    const uint32_t gx = bx * 8u, gy = by * 8u, gz = bz * 8u;
    const uint32_t w = min(8u, a.g.width - gx), h = min(8u, a.g.height - gy), d = min(8u, a.g.depth - gz);
    const float lx = __fsub_rn(px, (float)gx), ly = __fsub_rn(py, (float)gy), lz = __fsub_rn(pz, (float)gz);
    float value = smoke_stream(S, wb, 8u, ccodec, cres, ckf, w, h, d, lx, ly, lz);
    if (mode == kModeFine6 && fres > 0u)
        value = __fadd_rn(value, smoke_stream(S, wb, fbase, fcodec, fres, fkf, w, h, d, lx, ly, lz));
    return value;
}

// vbt_smoke_sample.comp:307-336 (main): one thread per ray, the sum of step_count samples.
__global__ void __launch_bounds__(128) smoke_sample_kernel(DeviceAsset a, vbt_sample_params p,
                                                           const float4* __restrict__ rays, uint32_t n,
                                                           float* __restrict__ out)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int frame = clamp_frame(p.frame_index, (int)a.g.frames);
    const SmokeSampler S{a, (uint32_t)frame, time_bin(frame, 8u, a.g.frames)};
    const float4 r0 = rays[2 * i], r1 = rays[2 * i + 1];
    const float dt = __fdiv_rn(r1.w, gmax((float)p.step_count, 1.0f));
    float t = __fadd_rn(r0.w, __fmul_rn(0.5f, dt));
    float acc = 0.0f;
    for (uint32_t s = 0; s < p.step_count; ++s) {
        acc = __fadd_rn(acc, smoke_density(S, p, along(r0.x, r1.x, t), along(r0.y, r1.y, t), along(r0.z, r1.z, t)));
        t = __fadd_rn(t, dt);
    }
    out[i] = acc;
}

}  // namespace
}  // namespace vbtb

using namespace vbtb;

extern "C" int vbt_sample_rays(vbt_asset* a, const float* d_controls, const vbt_sample_params* params,
                               const vbt_ray* d_rays, uint32_t n, vbt_sample_result* d_out, void* stream)
{
    if (!a || !params || (n && (!d_controls || !d_rays || !d_out)))
        return set_last_error(VBT_STATUS_INVALID_ARGUMENT, "null argument");
    if (a->hdr.profile_type == 2u) return set_last_error(VBT_STATUS_INVALID_ARGUMENT, "the sampler covers render-temporal assets");
    if (params->render_mode > 1u) return set_last_error(VBT_STATUS_INVALID_ARGUMENT, "render_mode must be 0 or 1");
    if ((reinterpret_cast<uintptr_t>(d_rays) & 15u) != 0u || (reinterpret_cast<uintptr_t>(d_out) & 15u) != 0u)
        return set_last_error(VBT_STATUS_INVALID_ARGUMENT, "rays and results must be 16-byte aligned");
    if (n == 0) return VBT_STATUS_OK;
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != a->device) cudaSetDevice(a->device);
    sample_rays_kernel<<<(n + 127u) / 128u, 128, 0, static_cast<cudaStream_t>(stream)>>>(
        a->dev, d_controls, *params, reinterpret_cast<const float4*>(d_rays), n, reinterpret_cast<float4*>(d_out));
    const cudaError_t e = cudaGetLastError();
    if (prev >= 0 && prev != a->device) cudaSetDevice(prev);
    return e == cudaSuccess ? VBT_STATUS_OK
                            : set_last_error(VBT_STATUS_CUDA, std::string("sample_rays_kernel: ") + cudaGetErrorString(e));
}

extern "C" int vbt_smoke_sample_rays(vbt_asset* a, const vbt_sample_params* params, const vbt_ray* d_rays, uint32_t n,
                                     float* d_out, void* stream)
{
    if (!a || !params || (n && (!d_rays || !d_out))) return set_last_error(VBT_STATUS_INVALID_ARGUMENT, "null argument");
    if (a->hdr.profile_type == 2u) return set_last_error(VBT_STATUS_INVALID_ARGUMENT, "the sampler covers render-temporal assets");
    if ((reinterpret_cast<uintptr_t>(d_rays) & 15u) != 0u || (reinterpret_cast<uintptr_t>(d_out) & 3u) != 0u)
        return set_last_error(VBT_STATUS_INVALID_ARGUMENT, "rays must be 16-byte and results 4-byte aligned");
    if (n == 0) return VBT_STATUS_OK;
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != a->device) cudaSetDevice(a->device);
    smoke_sample_kernel<<<(n + 127u) / 128u, 128, 0, static_cast<cudaStream_t>(stream)>>>(
        a->dev, *params, reinterpret_cast<const float4*>(d_rays), n, d_out);
    const cudaError_t e = cudaGetLastError();
    if (prev >= 0 && prev != a->device) cudaSetDevice(prev);
    return e == cudaSuccess ? VBT_STATUS_OK
                            : set_last_error(VBT_STATUS_CUDA, std::string("smoke_sample_kernel: ") + cudaGetErrorString(e));
}
