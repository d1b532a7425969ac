/*
 * vbt_sample_oracle.c -- CPU restatement of the Studio's ray sampler over the current-frame
 * control cache (VBTStudio/frontend/shaders/vbt_cache.comp and vbt_sample.comp).
 *
 * TEST INFRASTRUCTURE ONLY: the parity checker of vbt_b200's ray sampler.  The shaders cannot run
 * here (no graphics stack); this file restates their arithmetic in C, operation by operation, in
 * single precision with no contraction (-ffp-contract=off), so that the CUDA kernel can be checked
 * bit for bit.  Choices shared with the CUDA kernel where GLSL leaves room: mix(a, b, t) is
 * a*(1 - t) + b*t with every operation rounded, round() rounds halves away from zero,
 * normalize(v) is v / length(v), and a control value decoded straight from the
 * payload (coarse grids above 64 controls, vbt_sample.comp:230-249) is the reference CPU
 * decoder's (vo_decode_control) rather than the shader's mix().
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "vbt_oracle.h"

#define CACHE_STRIDE 576u
#define COARSE_CACHE_COUNT 64u

static uint32_t rd_byte(const vo_file* f, uint32_t base_word, uint32_t byte_off)
{
    const uint32_t w = f->payload[base_word + (byte_off >> 2)];
    return (w >> ((byte_off & 3u) * 8u)) & 0xFFu;
}
static uint32_t rd_u16(const vo_file* f, uint32_t bw, uint32_t o) { return rd_byte(f, bw, o) | (rd_byte(f, bw, o + 1u) << 8); }
static uint32_t rd_u32(const vo_file* f, uint32_t bw, uint32_t o)
{
    return rd_byte(f, bw, o) | (rd_byte(f, bw, o + 1u) << 8) | (rd_byte(f, bw, o + 2u) << 16) | (rd_byte(f, bw, o + 3u) << 24);
}
static uint32_t align4u(uint32_t b) { return (b + 3u) & ~3u; }
static float mixf(float a, float b, float t) { return a * (1.0f - t) + b * t; }
/* GLSL min / max / clamp: min(x, y) = y < x ? y : x, max(x, y) = x < y ? y : x, clamp = min(max()) */
static float minf(float x, float y) { return y < x ? y : x; }
static float maxf(float x, float y) { return x < y ? y : x; }
static float clampf(float x, float a, float b) { return minf(maxf(x, a), b); }

/* vbt_cache.comp:168-236 -- 576 slots per active leaf; slot values from the reference decoder. */
int vo_control_cache(const vo_file* f, int frame, const uint32_t* compact, float* cache)
{
    const uint8_t* base = (const uint8_t*)f->payload;
    int status = VO_OK;
    for (uint32_t leaf = 0; leaf < f->leaf_count; ++leaf) {
        if (compact[leaf] == 0xFFFFFFFFu) continue;
        float* dst = cache + (uint64_t)compact[leaf] * CACHE_STRIDE;
        memset(dst, 0, CACHE_STRIDE * sizeof(float));
        const uint32_t wb = f->offsets[leaf], we = f->offsets[leaf + 1];
        const uint8_t* blk = base + 4ull * wb;
        vo_leaf_view v;
        int st = vo_parse_leaf(blk, 4ull * (we - wb), 1, &v);
        if (st) {
            status = st;
            continue;
        }
        const uint32_t cc = v.header.coarse_res * v.header.coarse_res * v.header.coarse_res;
        for (uint32_t s = 0; s < COARSE_CACHE_COUNT && s < cc; ++s)
            vo_decode_control(blk + v.coarse_off, v.header.coarse_codec, cc, 8u, v.coarse_kf, v.coarse.total, 1,
                              (int)f->frames, s, frame, &dst[s]);
        if (v.header.mode == 3u) {
            const uint32_t cf = v.header.fine_res * v.header.fine_res * v.header.fine_res;
            for (uint32_t s = 0; s < 512u && s < cf; ++s)
                vo_decode_control(blk + v.fine_off, v.header.fine_codec, cf, 8u, v.fine_kf, v.fine.total, 1,
                                  (int)f->frames, s, frame, &dst[COARSE_CACHE_COUNT + s]);
        } else if (v.header.mode == 2u) {
            for (uint32_t s = 0; s < 512u && s < v.shell_active; ++s)
                vo_decode_control(blk + v.shell_residual_off, v.header.fine_codec, v.shell_active, 4u, v.fine_kf,
                                  v.shell_residual_bytes, 1, (int)f->frames, s, frame, &dst[COARSE_CACHE_COUNT + s]);
        }
    }
    return status;
}

typedef struct {
    const vo_file* f;
    const float* cache;
    const uint32_t* compact;
    const vo_sample_params* p;
    uint32_t lcx, lcy;
    const uint8_t* bad;   /* per leaf: the parser rejects it (such leaves sample as background) */
} sampler;

/* vbt_sample.comp:191-206 */
static float control_coord(uint32_t index, uint32_t res)
{
    if (res <= 1u) return 0.0f;
    return (float)index * (7.0f / (float)(res - 1u));
}
static void locate_coord(float p, uint32_t extent, uint32_t res, uint32_t* i0, uint32_t* i1, float* w)
{
    const float max_p = maxf((float)extent - 1.0f, 0.0f);
    const float c = clampf(p, 0.0f, max_p);
    uint32_t j1 = 1u;
    while (j1 < res - 1u && control_coord(j1, res) < c) ++j1;
    const int j0 = (int)j1 - 1;
    *i0 = (uint32_t)(j0 > 0 ? j0 : 0);
    *i1 = j1;
    const float c0 = control_coord(*i0, res), c1 = control_coord(j1, res);
    *w = c1 > c0 ? (c - c0) / (c1 - c0) : 0.0f;
}

/* vbt_sample.comp:213-230 (currentFrameControl) */
static float current_control(const sampler* S, uint32_t compact_leaf, uint32_t slot_base, uint32_t word_begin,
                             uint32_t stream_base, uint32_t codec, uint32_t control_count, uint32_t kf,
                             uint32_t stream_bytes, uint32_t ci)
{
    if (slot_base == 0u && control_count > COARSE_CACHE_COUNT) {
        float out = 0.0f;
        const uint8_t* blk = (const uint8_t*)(S->f->payload + word_begin);
        vo_decode_control(blk + stream_base, codec, control_count, 8u, kf, stream_bytes, 1, (int)S->f->frames, ci,
                          S->p->frame_index, &out);
        return out;
    }
    return S->cache[(uint64_t)compact_leaf * CACHE_STRIDE + slot_base + ci];
}

/* vbt_sample.comp:232-268 (sampleControlStream) */
static float sample_stream(const sampler* S, uint32_t compact_leaf, uint32_t slot_base, uint32_t word_begin,
                           uint32_t stream_base, uint32_t codec, uint32_t res, uint32_t kf, uint32_t stream_bytes,
                           uint32_t w, uint32_t h, uint32_t d, float lx, float ly, float lz)
{
    if (res == 0u) return 0.0f;   /* no controls (locateCoord would count to 2^32) */
    uint32_t x0, x1, y0, y1, z0, z1;
    float tx, ty, tz;
    locate_coord(lx, w, res, &x0, &x1, &tx);
    locate_coord(ly, h, res, &y0, &y1, &ty);
    locate_coord(lz, d, res, &z0, &z1, &tz);
    const uint32_t cc = res * res * res;
#define CTRL(x, y, z) current_control(S, compact_leaf, slot_base, word_begin, stream_base, codec, cc, kf, stream_bytes, ((z) * res + (y)) * res + (x))
    const float v000 = CTRL(x0, y0, z0), v100 = CTRL(x1, y0, z0), v010 = CTRL(x0, y1, z0), v110 = CTRL(x1, y1, z0);
    const float v001 = CTRL(x0, y0, z1), v101 = CTRL(x1, y0, z1), v011 = CTRL(x0, y1, z1), v111 = CTRL(x1, y1, z1);
#undef CTRL
    const float c00 = mixf(v000, v100, tx), c10 = mixf(v010, v110, tx);
    const float c01 = mixf(v001, v101, tx), c11 = mixf(v011, v111, tx);
    const float c0 = mixf(c00, c10, ty), c1 = mixf(c01, c11, ty);
    return mixf(c0, c1, tz);
}

/* vbt_sample.comp:298-320 (sampleShellResidual) */
static float sample_shell(const sampler* S, uint32_t word_begin, uint32_t occ_base, uint32_t compact_leaf,
                          uint32_t voxel, int* occupied)
{
    const uint32_t group = voxel >> 6, bit = voxel & 63u, word_in_group = bit >> 5, local_bit = bit & 31u;
    const uint32_t mask_word = rd_u32(S->f, word_begin, occ_base + group * 8u + word_in_group * 4u);
    *occupied = ((mask_word >> local_bit) & 1u) != 0u;
    if (!*occupied) return 0.0f;
    const uint32_t prefix = rd_u16(S->f, word_begin, occ_base + 64u + group * 2u);
    const uint32_t low_word = rd_u32(S->f, word_begin, occ_base + group * 8u);
    uint32_t di = prefix;
    if (word_in_group != 0u) di += (uint32_t)__builtin_popcount(low_word);
    const uint32_t before = local_bit == 0u ? 0u : (0xFFFFFFFFu >> (32u - local_bit));
    di += (uint32_t)__builtin_popcount(mask_word & before);
    if (di >= CACHE_STRIDE - COARSE_CACHE_COUNT) return 0.0f;
    return S->cache[(uint64_t)compact_leaf * CACHE_STRIDE + COARSE_CACHE_COUNT + di];
}

/* vbt_sample.comp:322-415 (sampleVbtValue) */
static float sample_value(const sampler* S, float wx, float wy, float wz, int preserve_interior)
{
    const vo_sample_params* p = S->p;
    const vo_file* f = S->f;
    const float bg = p->render_mode == 1u ? p->background_value : 0.0f;
    const float px = wx - p->bbox_min[0], py = wy - p->bbox_min[1], pz = wz - p->bbox_min[2];
    if (px < 0.0f || py < 0.0f || pz < 0.0f || px > (float)(f->width - 1u) || py > (float)(f->height - 1u) ||
        pz > (float)(f->depth - 1u))
        return bg;
    uint32_t x = (uint32_t)floorf(px), y = (uint32_t)floorf(py), z = (uint32_t)floorf(pz);
    if (x > f->width - 1u) x = f->width - 1u;
    if (y > f->height - 1u) y = f->height - 1u;
    if (z > f->depth - 1u) z = f->depth - 1u;
    const uint32_t lcz = (f->depth + 7u) / 8u;
    uint32_t bx = x / 8u, by = y / 8u, bz = z / 8u;
    if (bx > S->lcx - 1u) bx = S->lcx - 1u;
    if (by > S->lcy - 1u) by = S->lcy - 1u;
    if (bz > lcz - 1u) bz = lcz - 1u;
    const uint32_t leaf = (bz * S->lcy + by) * S->lcx + bx;
    const uint32_t wb = f->offsets[leaf], we = f->offsets[leaf + 1];
    if (we <= wb) return bg;
    const uint32_t hdr = f->payload[wb], mode = hdr & 3u;
    if (mode == 0u) return bg;
    if (S->bad[leaf]) return bg;
    const uint32_t cl = S->compact[leaf];
    const uint32_t ccodec = (hdr >> 2) & 3u, fcodec = (hdr >> 4) & 3u;
    const uint32_t cres = (hdr >> 6) & 7u, fres = (hdr >> 9) & 7u;
    const uint32_t ckf = rd_u16(f, wb, 4u), fkf = rd_u16(f, wb, 6u);
    const uint32_t cc = cres * cres * cres;
    const uint32_t ckey_bytes = align4u(ckf * (ccodec == 1u ? 8u : 3u));
    const uint32_t cbase = 8u;
    const uint32_t fbase = cbase + cc * 4u + align4u(cc * 8u) + ckey_bytes;
    const uint32_t gx = bx * 8u, gy = by * 8u, gz = bz * 8u;
    const uint32_t w = f->width - gx < 8u ? f->width - gx : 8u;
    const uint32_t h = f->height - gy < 8u ? f->height - gy : 8u;
    const uint32_t d = f->depth - gz < 8u ? f->depth - gz : 8u;
    const float lx = px - (float)gx, ly = py - (float)gy, lz = pz - (float)gz;
    float value = sample_stream(S, cl, 0u, wb, cbase, ccodec, cres, ckf, fbase - cbase, w, h, d, lx, ly, lz);
    if (mode == 3u && fres > 0u) {
        const uint32_t cf = fres * fres * fres;
        const uint32_t fbytes = cf * 4u + align4u(cf * 8u) + align4u(fkf * (fcodec == 1u ? 8u : 3u));
        value = value + sample_stream(S, cl, COARSE_CACHE_COUNT, wb, fbase, fcodec, fres, fkf, fbytes, w, h, d, lx, ly, lz);
    } else if (mode == 2u) {
        const uint32_t ux = (uint32_t)clampf(roundf(lx), 0.0f, 7.0f);
        const uint32_t uy = (uint32_t)clampf(roundf(ly), 0.0f, 7.0f);
        const uint32_t uz = (uint32_t)clampf(roundf(lz), 0.0f, 7.0f);
        int occupied = 0;
        value = value + sample_shell(S, wb, fbase, cl, (uz * 8u + uy) * 8u + ux, &occupied);
        if (!preserve_interior && !occupied && value < 0.0f) value = bg;
    }
    return value;
}

static float sample_at(const sampler* S, const float* o, const float* dir, float t, int keep)
{
    return sample_value(S, o[0] + dir[0] * t, o[1] + dir[1] * t, o[2] + dir[2] * t, keep);
}

/* vbt_sample.comp:417-431 (intersectWorldBox) */
static int intersect_box(const sampler* S, const float* o, const float* dir, float* near_t, float* far_t)
{
    const vo_sample_params* p = S->p;
    const float mn[3] = {p->bbox_min[0], p->bbox_min[1], p->bbox_min[2]};
    const float mx[3] = {mn[0] + (float)(S->f->width - 1u), mn[1] + (float)(S->f->height - 1u),
                         mn[2] + (float)(S->f->depth - 1u)};
    float lo[3], hi[3];
    for (int k = 0; k < 3; ++k) {
        const float inv = 1.0f / dir[k];
        const float a = (mn[k] - o[k]) * inv, b = (mx[k] - o[k]) * inv;
        lo[k] = minf(a, b);
        hi[k] = maxf(a, b);
    }
    *near_t = maxf(0.0f, maxf(lo[0], maxf(lo[1], lo[2])));
    *far_t = minf(hi[0], minf(hi[1], hi[2]));
    return *far_t > *near_t;
}

/* vbt_sample.comp:433-455 (traceShadow) */
static float trace_shadow(const sampler* S, const float* o, const float* dir)
{
    const vo_sample_params* p = S->p;
    float near_t, far_t;
    if (!intersect_box(S, o, dir, &near_t, &far_t)) return 0.0f;
    const float eps = maxf(p->surface_epsilon_voxels * p->voxel_size, 1e-5f);
    float t = near_t;
    float prev = sample_at(S, o, dir, t, 0) - p->surface_iso;
    for (uint32_t it = 0; it < p->shadow_steps; ++it) {
        const float step = clampf(fabsf(prev) / maxf(p->voxel_size, 1e-6f) * 0.8f, 0.35f, 5.0f);
        const float nt = minf(t + step, far_t);
        const float np = sample_at(S, o, dir, nt, 0) - p->surface_iso;
        if ((prev < 0.0f) != (np < 0.0f)) {
            const int next_inside = np < 0.0f;
            const float neg = next_inside ? np : prev;
            const float st = next_inside ? minf(nt + 0.35f, far_t) : maxf(t - 0.35f, near_t);
            const float sp = sample_at(S, o, dir, st, 0) - p->surface_iso;
            if (neg <= -eps * 0.5f || sp <= -eps * 0.25f) return 1.0f;
        }
        if (nt >= far_t) break;
        t = nt;
        prev = fabsf(np) <= eps ? eps : np;
    }
    return 0.0f;
}

/* vbt_sample.comp:457-476 (estimateThickness) */
static float estimate_thickness(const sampler* S, const float* ray, float hit_t)
{
    const vo_sample_params* p = S->p;
    const float* o = ray;
    const float* dir = ray + 4;
    const float tmax = ray[7];
    const float eps = maxf(p->surface_epsilon_voxels * p->voxel_size, 1e-5f);
    float t = minf(hit_t + 0.35f, tmax);
    float prev = sample_at(S, o, dir, t, 1) - p->surface_iso;
    int entered = prev < -0.25f * eps;
    const uint32_t limit = p->step_count < 160u ? p->step_count : 160u;
    for (uint32_t it = 0; it < limit; ++it) {
        const float step = clampf(fabsf(prev) / maxf(p->voxel_size, 1e-6f) * 0.7f, 0.3f, 3.0f);
        const float nt = minf(t + step, tmax);
        const float np = sample_at(S, o, dir, nt, 1) - p->surface_iso;
        entered = entered || np < -0.25f * eps;
        if (entered && prev < 0.0f && np >= 0.0f) return maxf((nt - hit_t) * p->voxel_size, p->voxel_size * 0.25f);
        if (nt >= tmax) break;
        t = nt;
        prev = np;
    }
    return p->voxel_size * 6.0f;
}

static float len3(float x, float y, float z) { return sqrtf(x * x + y * y + z * z); }

/* vbt_sample.comp:478-546 (traceLevelSet) */
static void trace_level_set(const sampler* S, const float* ray, float* res)
{
    const vo_sample_params* p = S->p;
    const float* o = ray;
    const float* dir = ray + 4;
    const float tmax = ray[7];
    res[0] = res[1] = res[2] = 0.0f;
    res[3] = -1.0f;
    res[4] = res[5] = res[6] = res[7] = 0.0f;
    if (tmax <= 0.0f) return;
    const float eps = maxf(p->surface_epsilon_voxels * p->voxel_size, 1e-5f);
    float prev_t = 0.0f;
    float prev = sample_value(S, o[0], o[1], o[2], 0) - p->surface_iso;
    float hit_t = -1.0f;
    for (uint32_t it = 0; it < p->step_count; ++it) {
        const float step = clampf(fabsf(prev) / maxf(p->voxel_size, 1e-6f) * 0.8f, 0.2f, maxf(p->max_step_voxels, 0.2f));
        const float cur_t = minf(prev_t + step, tmax);
        const float cur = sample_at(S, o, dir, cur_t, 0) - p->surface_iso;
        if ((prev < 0.0f) != (cur < 0.0f)) {
            const int cur_inside = cur < 0.0f;
            const float neg = cur_inside ? cur : prev;
            const float st = cur_inside ? minf(cur_t + 0.35f, tmax) : maxf(prev_t - 0.35f, 0.0f);
            const float sp = sample_at(S, o, dir, st, 0) - p->surface_iso;
            const int support = neg <= -eps * 0.5f || sp <= -eps * 0.25f;
            if (!support) {
                if (cur_t >= tmax) break;
                prev_t = cur_t;
                prev = maxf(cur, eps);
                continue;
            }
            float low = prev_t, high = cur_t, low_phi = prev;
            for (uint32_t r = 0; r < 5u; ++r) {
                const float mid = 0.5f * (low + high);
                const float mid_phi = sample_at(S, o, dir, mid, 0) - p->surface_iso;
                if ((low_phi < 0.0f) != (mid_phi < 0.0f)) {
                    high = mid;
                } else {
                    low = mid;
                    low_phi = mid_phi;
                }
            }
            hit_t = 0.5f * (low + high);
            break;
        }
        if (cur_t >= tmax) break;
        prev_t = cur_t;
        prev = cur;
    }
    if (hit_t < 0.0f) return;
    const float hx = o[0] + dir[0] * hit_t, hy = o[1] + dir[1] * hit_t, hz = o[2] + dir[2] * hit_t;
    const float ns = maxf(p->surface_normal_step, 0.25f);
    const float gx = sample_value(S, hx + ns, hy, hz, 0) - sample_value(S, hx - ns, hy, hz, 0);
    const float gy = sample_value(S, hx, hy + ns, hz, 0) - sample_value(S, hx, hy - ns, hz, 0);
    const float gz = sample_value(S, hx, hy, hz + ns, 0) - sample_value(S, hx, hy, hz - ns, 0);
    const float gl = len3(gx, gy, gz);
    float nx, ny, nz;
    if (gl > 1e-6f) {
        nx = gx / gl;
        ny = gy / gl;
        nz = gz / gl;
    } else {
        nx = -dir[0];
        ny = -dir[1];
        nz = -dir[2];
    }
    res[0] = nx;
    res[1] = ny;
    res[2] = nz;
    res[3] = hit_t;
    res[4] = p->surface_model != 0u ? estimate_thickness(S, ray, hit_t) : 0.0f;
    res[7] = fabsf(nx * (-dir[0]) + ny * (-dir[1]) + nz * (-dir[2]));
}

/* vbt_sample.comp:548-622 (main), one ray */
static void sample_ray(const sampler* S, const float* ray, float* res)
{
    const vo_sample_params* p = S->p;
    const float* o = ray;
    const float* dir = ray + 4;
    if (p->render_mode == 1u) {
        trace_level_set(S, ray, res);
        const float fdir = p->up_axis == 2u ? dir[2] : dir[1];
        const float forg = p->up_axis == 2u ? o[2] : o[1];
        if (p->surface_model != 0u && res[3] < 0.0f && fdir < -1e-5f) {
            const float ft = (p->floor_height - forg) / fdir;
            if (ft > 0.0f) {
                const float fx = o[0] + dir[0] * ft, fy = o[1] + dir[1] * ft, fz = o[2] + dir[2] * ft;
                float kx = -0.55f, ky = p->up_axis == 2u ? 0.42f : 0.72f, kz = p->up_axis == 2u ? 0.72f : 0.42f;
                const float kl = len3(kx, ky, kz);
                kx = kx / kl;
                ky = ky / kl;
                kz = kz / kl;
                const float so[3] = {fx + kx * 0.5f, fy + ky * 0.5f, fz + kz * 0.5f};
                const float sd[3] = {kx, ky, kz};
                res[5] = 1.0f;
                res[6] = trace_shadow(S, so, sd);
            }
        }
        return;
    }
    const float dt = ray[7] / maxf((float)p->step_count, 1.0f);
    float t = ray[3] + 0.5f * dt;
    for (int k = 0; k < 8; ++k) res[k] = 0.0f;
    if (p->surface_model != 0u) {
        const uint32_t sc = p->step_count > 1u ? p->step_count : 1u;
        for (uint32_t i = 0; i < p->step_count; ++i) {
            const float v = sample_at(S, o, dir, t, 0);
            uint32_t bin = (i * 8u) / sc;
            if (bin > 7u) bin = 7u;
            res[bin] = res[bin] + v;
            t = t + dt;
        }
        return;
    }
    float acc = 0.0f;
    for (uint32_t i = 0; i < p->step_count; ++i) {
        acc = acc + sample_at(S, o, dir, t, 0);
        t = t + dt;
    }
    res[0] = acc;
}

/* Rays are [origin.xyz, tmin, dir.xyz, tmax] (8 floats); results [primary.xyzw, auxiliary.xyzw]. */
void vo_sample_rays(const vo_file* f, const float* cache, const uint32_t* compact, const vo_sample_params* p,
                    const float* rays, uint32_t n, float* results)
{
    uint8_t* bad = (uint8_t*)calloc(f->leaf_count, 1);
    for (uint32_t leaf = 0; leaf < f->leaf_count; ++leaf) {
        const uint32_t wb = f->offsets[leaf], we = f->offsets[leaf + 1];
        vo_leaf_view v;
        if (we > wb && (f->payload[wb] & 3u) != 0u)
            bad[leaf] = vo_parse_leaf((const uint8_t*)(f->payload + wb), 4ull * (we - wb), 1, &v) != VO_OK;
    }
    sampler S = {f, cache, compact, p, (f->width + 7u) / 8u, (f->height + 7u) / 8u, bad};
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 64)
#endif
    for (int64_t i = 0; i < (int64_t)n; ++i) sample_ray(&S, rays + 8 * i, results + 8 * i);
    free(bad);
}

/* ---- render/shaders/vbt_smoke_sample.comp: density accumulated straight from the payload ------
 * Each sample decodes the eight corner controls of the coarse stream (and of the FINE6 stream) with
 * the shader's own decodeTemporalControlValue, whose lerp is mix(previous, next, w) with
 * w = float(frame - f0) / float(f1 - f0) (divided with IEEE rounding); Mode2 leaves contribute
 * their coarse stream only, as in the shader.  A leaf whose walker status is bad, and a stream of
 * resolution 0 (where the shader's locateCoord would count to 2^32), contribute 0. */

/* vbt_smoke_sample.comp:118-122 readPackedKeyframeFrame, :94-116 readPackedKeyframeValue */
static uint32_t smoke_key_frame(const vo_file* f, uint32_t bw, uint32_t key_base, uint32_t codec, uint32_t i)
{
    return codec == 1u ? rd_u16(f, bw, key_base + i * 8u) : rd_byte(f, bw, key_base + i * 3u);
}
static float smoke_key_value(const vo_file* f, uint32_t bw, uint32_t key_base, uint32_t codec, uint32_t i)
{
    if (codec == 1u) {
        const uint32_t bits = rd_u32(f, bw, key_base + i * 8u + 4u);
        float v;
        memcpy(&v, &bits, 4);
        return v;
    }
    return vo_half_to_float((uint16_t)rd_u16(f, bw, key_base + i * 3u + 1u));
}

/* vbt_smoke_sample.comp:124-171 decodeTemporalControlValue */
static float smoke_control(const vo_file* f, uint32_t bw, uint32_t stream_base, uint32_t codec, uint32_t cc,
                           uint32_t kf, uint32_t ci, int total, int frame_index)
{
    const uint32_t bins_n = 8u;
    if (ci >= cc) return 0.0f;
    const uint32_t desc_bytes = cc * 4u;
    const uint32_t key_base = stream_base + desc_bytes + align4u(cc * bins_n);
    const uint32_t desc = stream_base + ci * 4u;
    const uint32_t start = rd_u16(f, bw, desc), count = rd_byte(f, bw, desc + 2u);
    if (count == 0u || start + count > kf) return 0.0f;
    const int hi_frame = total - 1 > 0 ? total - 1 : 0;
    const uint32_t frame = (uint32_t)(frame_index < 0 ? 0 : (frame_index > hi_frame ? hi_frame : frame_index));
    const uint32_t tb = frame * bins_n / (uint32_t)(total > 1 ? total : 1);
    const uint32_t bin = tb < bins_n - 1u ? tb : bins_n - 1u;
    const uint32_t bins = stream_base + desc_bytes + ci * bins_n;
    uint32_t lo = rd_byte(f, bw, bins + bin);
    if (lo > count - 1u) lo = count - 1u;
    uint32_t f0 = smoke_key_frame(f, bw, key_base, codec, start + lo);
    if (f0 > frame) {
        lo = 0u;
        f0 = smoke_key_frame(f, bw, key_base, codec, start);
    }
    if (f0 >= frame || lo + 1u >= count) return smoke_key_value(f, bw, key_base, codec, start + lo);
    uint32_t hi = count - 1u;
    if (bin + 1u < bins_n) {
        const uint32_t nb = rd_byte(f, bw, bins + bin + 1u) + 1u;
        hi = nb < count - 1u ? nb : count - 1u;
    }
    if (hi < lo + 1u) hi = lo + 1u;
    uint32_t f1 = smoke_key_frame(f, bw, key_base, codec, start + hi);
    if (f1 < frame) {
        hi = count - 1u;
        f1 = smoke_key_frame(f, bw, key_base, codec, start + hi);
    }
    if (f1 <= frame) return smoke_key_value(f, bw, key_base, codec, start + hi);
    while (hi > lo + 1u) {
        const uint32_t mid = lo + (hi - lo) / 2u;
        const uint32_t fm = smoke_key_frame(f, bw, key_base, codec, start + mid);
        if (fm < frame) {
            lo = mid;
            f0 = fm;
        } else {
            hi = mid;
            f1 = fm;
        }
    }
    const float next = smoke_key_value(f, bw, key_base, codec, start + hi);
    if (f1 == frame) return next;
    const float prev = smoke_key_value(f, bw, key_base, codec, start + lo);
    return mixf(prev, next, (float)(frame - f0) / (float)(f1 - f0));
}

/* vbt_smoke_sample.comp:195-232 sampleControlStream */
static float smoke_stream(const vo_file* f, const vo_sample_params* p, uint32_t bw, uint32_t stream_base,
                          uint32_t codec, uint32_t res, uint32_t kf, uint32_t w, uint32_t h, uint32_t d, float lx,
                          float ly, float lz)
{
    if (res == 0u) return 0.0f;
    uint32_t x0, x1, y0, y1, z0, z1;
    float tx, ty, tz;
    locate_coord(lx, w, res, &x0, &x1, &tx);
    locate_coord(ly, h, res, &y0, &y1, &ty);
    locate_coord(lz, d, res, &z0, &z1, &tz);
    const uint32_t cc = res * res * res;
    const int T = (int)f->frames;
#define SCTRL(x, y, z) smoke_control(f, bw, stream_base, codec, cc, kf, ((z) * res + (y)) * res + (x), T, p->frame_index)
    const float v000 = SCTRL(x0, y0, z0), v100 = SCTRL(x1, y0, z0), v010 = SCTRL(x0, y1, z0), v110 = SCTRL(x1, y1, z0);
    const float v001 = SCTRL(x0, y0, z1), v101 = SCTRL(x1, y0, z1), v011 = SCTRL(x0, y1, z1), v111 = SCTRL(x1, y1, z1);
#undef SCTRL
    const float c00 = mixf(v000, v100, tx), c10 = mixf(v010, v110, tx);
    const float c01 = mixf(v001, v101, tx), c11 = mixf(v011, v111, tx);
    return mixf(mixf(c00, c10, ty), mixf(c01, c11, ty), tz);
}

/* vbt_smoke_sample.comp:234-305 sampleVbtDensity */
static float smoke_density(const vo_file* f, const vo_sample_params* p, const uint8_t* bad, float wx, float wy,
                           float wz)
{
    const float px = wx - p->bbox_min[0], py = wy - p->bbox_min[1], pz = wz - p->bbox_min[2];
    if (px < 0.0f || py < 0.0f || pz < 0.0f || px > (float)(f->width - 1u) || py > (float)(f->height - 1u) ||
        pz > (float)(f->depth - 1u))
        return 0.0f;
    const uint32_t lcx = (f->width + 7u) / 8u, lcy = (f->height + 7u) / 8u, lcz = (f->depth + 7u) / 8u;
    uint32_t x = (uint32_t)floorf(px), y = (uint32_t)floorf(py), z = (uint32_t)floorf(pz);
    if (x > f->width - 1u) x = f->width - 1u;
    if (y > f->height - 1u) y = f->height - 1u;
    if (z > f->depth - 1u) z = f->depth - 1u;
    const uint32_t bx = x / 8u < lcx - 1u ? x / 8u : lcx - 1u, by = y / 8u < lcy - 1u ? y / 8u : lcy - 1u,
                   bz = z / 8u < lcz - 1u ? z / 8u : lcz - 1u;
    const uint32_t leaf = (bz * lcy + by) * lcx + bx;
    const uint32_t wb = f->offsets[leaf], we = f->offsets[leaf + 1];
    if (we <= wb) return 0.0f;
    const uint32_t hdr = f->payload[wb], mode = hdr & 3u;
    if (mode == 0u || bad[leaf]) return 0.0f;
    const uint32_t ccodec = (hdr >> 2) & 3u, fcodec = (hdr >> 4) & 3u, cres = (hdr >> 6) & 7u, fres = (hdr >> 9) & 7u;
    const uint32_t ckf = rd_u16(f, wb, 4u), fkf = rd_u16(f, wb, 6u);
    const uint32_t cc = cres * cres * cres;
    const uint32_t fbase = 8u + cc * 4u + align4u(cc * 8u) + align4u(ckf * (ccodec == 1u ? 8u : 3u));
    const uint32_t gx = bx * 8u, gy = by * 8u, gz = bz * 8u;
    const uint32_t w = f->width - gx < 8u ? f->width - gx : 8u, h = f->height - gy < 8u ? f->height - gy : 8u,
                   d = f->depth - gz < 8u ? f->depth - gz : 8u;
    const float lx = px - (float)gx, ly = py - (float)gy, lz = pz - (float)gz;
    float value = smoke_stream(f, p, wb, 8u, ccodec, cres, ckf, w, h, d, lx, ly, lz);
    if (mode == 3u && fres > 0u) value += smoke_stream(f, p, wb, fbase, fcodec, fres, fkf, w, h, d, lx, ly, lz);
    return value;
}

/* vbt_smoke_sample.comp:307-336 main: results[ray] = sum over step_count samples */
void vo_smoke_sample_rays(const vo_file* f, const vo_sample_params* p, const float* rays, uint32_t n, float* out)
{
    uint8_t* bad = (uint8_t*)calloc(f->leaf_count ? f->leaf_count : 1u, 1);
    for (uint32_t leaf = 0; leaf < f->leaf_count; ++leaf) {
        const uint32_t wb = f->offsets[leaf], we = f->offsets[leaf + 1];
        vo_leaf_view v;
        if (we > wb && vo_parse_leaf((const uint8_t*)(f->payload + wb), (size_t)(we - wb) * 4u, 1, &v) != VO_OK)
            bad[leaf] = 1;
    }
#pragma omp parallel for schedule(dynamic, 256)
    for (long long i = 0; i < (long long)n; ++i) {
        const float* r = rays + 8 * i;
        const float dt = r[7] / maxf((float)p->step_count, 1.0f);
        float t = r[3] + 0.5f * dt;
        float acc = 0.0f;
        for (uint32_t s = 0; s < p->step_count; ++s) {
            acc += smoke_density(f, p, bad, r[0] + r[4] * t, r[1] + r[5] * t, r[2] + r[6] * t);
            t += dt;
        }
        out[i] = acc;
    }
    free(bad);
}
