/*
 * vbt_keyframe_oracle.c -- CPU restatement of the encoder's per-voxel keyframe pass.
 *
 * TEST INFRASTRUCTURE ONLY: the parity checker for vbt_detect_keyframes (vbt_b200/csrc/
 * keyframes.cu).  Pinned against the reference itself: oracle/_ref/libkfref.so runs the
 * reference's own detectDensityKeyFrames and reconstructFromKeys, and tests/golden/keyframes.npz
 * holds their outputs on seeded series (tests/golden/make_keyframes.py).
 *
 * Follows src/render_temporal_kf_probe_main.cpp:
 *   computeStats             :200-225   mean, stddev, 90th-percentile |delta|
 *   cutoffState              :227-233
 *   epsilonAt                :235-247
 *   dpRecurse                :249-276   split at the largest normalised error, recurse
 *   addIsoSurfaceKeyFrames   :2051-2078
 *   detectDensityKeyFrames   :2080-2167
 *   reconstructFromKeys      :2169-2201
 *   per-voxel leaf loop      :619-659   background test, keys, reconstruction, squared error
 *   coarse control fitting   :705-729   controlCoords (:189-198), sampleLeafBufferAtFractional
 *                                       (:2203-2237), buildBinIndexFromKeys (:2288-2305),
 *                                       appendControlSequenceToStream (:2361-2399)
 * Floating point is kept in the reference's types (float where it computes in float, double
 * where it promotes), with no contraction (built with -ffp-contract=off).  Values are finite.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "vbt_oracle.h"

/* std::max / std::min: the first argument unless the comparison says otherwise. */
static float fmax_r(float a, float b) { return a < b ? b : a; }
static double dmax_r(double a, double b) { return a < b ? b : a; }

typedef struct {
    float mean, stddev, delta_scale;
} kf_stats;

static int cmp_f32(const void* a, const void* b)
{
    const float x = *(const float*)a, y = *(const float*)b;
    return (x > y) - (x < y);
}

/* computeStats (:200-225). */
static kf_stats kf_compute_stats(const float* v, int n, float* scratch)
{
    kf_stats s = {0.0f, 0.0f, 1.0f};
    if (n == 0) return s;
    double sum = 0.0, sum2 = 0.0;
    for (int i = 0; i < n; ++i) {
        sum += v[i];
        sum2 += (double)v[i] * v[i];
    }
    s.mean = (float)(sum / (double)n);
    const double var = dmax_r(0.0, sum2 / (double)n - (double)s.mean * s.mean);
    s.stddev = (float)sqrt(var);
    if (n >= 2) {
        const int m = n - 1;
        for (int i = 1; i < n; ++i) scratch[i - 1] = fabsf(v[i] - v[i - 1]);
        qsort(scratch, (size_t)m, sizeof(float), cmp_f32);
        const int idx = (m - 1) < (m * 9) / 10 ? (m - 1) : (m * 9) / 10;
        s.delta_scale = fmax_r(1e-6f, scratch[idx]);
    }
    return s;
}

/* cutoffState (:227-233). */
static int kf_cutoff_state(float v, float cutoff, float band)
{
    if (cutoff <= 0.0f) return 1;
    if (v < cutoff - band) return 0;
    if (v > cutoff + band) return 2;
    return 1;
}

/* epsilonAt (:235-247). */
static float kf_epsilon_at(const float* v, int t, const vo_keyframe_profile* p, const kf_stats* st)
{
    float eps = p->eps_abs + p->eps_rel * fmax_r(fabsf(v[t]), st->stddev);
    if (p->gamma_delta > 0.0f && t > 0) {
        const float delta = fabsf(v[t] - v[t - 1]) / fmax_r(1e-6f, st->delta_scale);
        eps /= (1.0f + p->gamma_delta * delta);
    }
    return fmax_r(eps, fmax_r(1e-6f, p->eps_abs * 0.1f));
}

/* dpRecurse (:249-276): marks the split frames in `key`, counts them in *splits. */
static void kf_split(const float* v, int a, int b, const vo_keyframe_profile* p, const kf_stats* st,
                     uint8_t* key, int* splits)
{
    if (b - a <= 1) return;
    const double v0 = v[a], v1 = v[b];
    double best = 0.0;
    int split = -1;
    for (int t = a + 1; t < b; ++t) {
        const double alpha = (double)(t - a) / (double)(b - a);
        const double pred = v0 + alpha * (v1 - v0);
        const double eps = kf_epsilon_at(v, t, p, st);
        const double e = fabs((double)v[t] - pred) / eps;
        if (e > best) {
            best = e;
            split = t;
        }
    }
    if (best > 1.0 && split != -1) {
        key[split] = 1;
        ++*splits;
        kf_split(v, a, split, p, st, key, splits);
        kf_split(v, split, b, p, st, key, splits);
    }
}

static void kf_push(uint8_t* key, int t, long* pushes)
{
    key[t] = 1;
    ++*pushes;
}

/* detectDensityKeyFrames (:2080-2167) without the validation-experiment switches (they are
 * compiled out of the reference unless VBT_VALIDATION_EXPERIMENTS is defined). */
int vo_detect_keyframes(const float* values, int n, const vo_keyframe_profile* p, int* keys, int* used_protect)
{
    if (used_protect) *used_protect = 0;
    if (n <= 0) return 0;
    if (n == 1) {
        keys[0] = 0;
        return 1;
    }
    float* scratch = (float*)malloc((size_t)n * sizeof(float));
    uint8_t* key = (uint8_t*)calloc((size_t)n, 1);
    const kf_stats st = kf_compute_stats(values, n, scratch);
    const float eps_floor = fmax_r(1e-6f, p->eps_abs * 0.1f);
    double sum = 0.0, sum2 = 0.0;
    for (int i = 0; i < n; ++i) {
        sum += values[i];
        sum2 += (double)values[i] * values[i];
    }
    const double mean = sum / (double)n;
    const double var = dmax_r(0.0, sum2 / (double)n - mean * mean);
    if (var < (double)eps_floor * eps_floor) {
        free(scratch);
        free(key);
        keys[0] = 0;
        return 1;
    }
    long pushes = 2;
    int splits = 0;
    key[0] = key[n - 1] = 1;
    kf_split(values, 0, n - 1, p, &st, key, &splits);
    pushes += splits;
    int used = 0;
    if (p->cutoff_temporal_protect && p->render_cutoff > 0.0f && p->cutoff_band >= 0.0f) {
        const float cutoff = p->render_cutoff, band = p->cutoff_band;
        for (int t = 0; t < n; ++t) {
            const int s = kf_cutoff_state(values[t], cutoff, band);
            if (s == 1) {
                kf_push(key, t, &pushes);
                if (t > 0) kf_push(key, t - 1, &pushes);
                if (t + 1 < n) kf_push(key, t + 1, &pushes);
                used = 1;
            }
            if (t > 0 && kf_cutoff_state(values[t - 1], cutoff, band) != s) {
                kf_push(key, t - 1, &pushes);
                kf_push(key, t, &pushes);
                if (t + 1 < n) kf_push(key, t + 1, &pushes);
                used = 1;
            }
        }
    }
    if (p->iso_surface_protect) {
        /* addIsoSurfaceKeyFrames (:2051-2078); it sorts and de-duplicates the whole key list, so
         * "keys were added" compares the distinct count after it with the pushes before it. */
        const long before = pushes;
        const float band = fmax_r(0.0f, p->iso_band);
        for (int t = 0; t < n; ++t) {
            const float cur = values[t] - p->iso_value;
            if (fabsf(cur) <= band) {
                if (t > 0) key[t - 1] = 1;
                key[t] = 1;
                if (t + 1 < n) key[t + 1] = 1;
            }
            if (t > 0) {
                const float prev = values[t - 1] - p->iso_value;
                if ((prev >= 0.0f) != (cur >= 0.0f)) {
                    for (int u = t - 2; u <= t + 1; ++u)
                        if (u >= 0 && u < n) key[u] = 1;
                }
            }
        }
        long distinct = 0;
        for (int t = 0; t < n; ++t) distinct += key[t];
        used = used || distinct > before;
    }
    int k = 0;
    for (int t = 0; t < n; ++t)
        if (key[t]) keys[k++] = t;
    free(scratch);
    free(key);
    if (used_protect) *used_protect = used;
    return k;
}

/* reconstructFromKeys (:2169-2201). */
void vo_reconstruct(const float* values, int n, const int* keys, int key_count, float* out)
{
    if (n <= 0) return;
    if (key_count == 0) {
        memcpy(out, values, (size_t)n * sizeof(float));
        return;
    }
    if (key_count == 1) {
        for (int t = 0; t < n; ++t) out[t] = values[keys[0]];
        return;
    }
    int seg = 0;
    for (int t = 0; t < n; ++t) {
        while (seg + 1 < key_count && t > keys[seg + 1]) ++seg;
        if (seg + 1 >= key_count) {
            out[t] = values[keys[key_count - 1]];
            continue;
        }
        const int a = keys[seg], b = keys[seg + 1];
        if (t <= a) {
            out[t] = values[a];
            continue;
        }
        const double alpha = (double)(t - a) / (double)(b - a);
        out[t] = (float)((double)values[a] + alpha * (double)(values[b] - values[a]));
    }
}

/* The per-voxel body of the encoder's leaf loop (:619-659) over independent series; series s at
 * values[t * frame_stride + s].  key_mask is word-major: bit t%32 of key_mask[(t/32) * series + s].
 * flags: bit 0 background-zeroed (no keys, counted as 1, reconstruction 0), bit 1 protected keys
 * added.  recon (optional) uses the input's layout; err2 (optional) is the series' squared error. */
void vo_keyframe_pass(const float* values, uint64_t series, int frames, uint64_t frame_stride,
                      const vo_keyframe_profile* p, uint32_t* key_mask, uint32_t* key_count, uint8_t* flags,
                      float* recon, double* err2, int threads)
{
    const int words = (frames + 31) / 32;
#pragma omp parallel num_threads(threads > 0 ? threads : 1) if (threads != 1)
    {
        float* v = (float*)malloc((size_t)frames * sizeof(float));
        float* r = (float*)malloc((size_t)frames * sizeof(float));
        int* keys = (int*)malloc((size_t)frames * sizeof(int));
#pragma omp for schedule(dynamic, 256)
        for (long long s = 0; s < (long long)series; ++s) {
            float vmax = 0.0f;
            for (int t = 0; t < frames; ++t) {
                v[t] = values[(uint64_t)t * frame_stride + (uint64_t)s];
                vmax = fmax_r(vmax, v[t]);
            }
            for (int w = 0; w < words; ++w) key_mask[(uint64_t)w * series + (uint64_t)s] = 0u;
            double e2 = 0.0;
            if (p->bg_threshold >= 0.0 && (double)vmax < p->bg_threshold) {
                for (int t = 0; t < frames; ++t) {
                    const double d = (double)v[t];
                    e2 += d * d;
                    r[t] = 0.0f;
                }
                key_count[s] = 1;
                flags[s] = 1;
            } else {
                int used = 0;
                const int k = vo_detect_keyframes(v, frames, p, keys, &used);
                vo_reconstruct(v, frames, keys, k, r);
                for (int t = 0; t < frames; ++t) {
                    const double d = (double)v[t] - (double)r[t];
                    e2 += d * d;
                }
                for (int i = 0; i < k; ++i)
                    key_mask[(uint64_t)(keys[i] / 32) * series + (uint64_t)s] |= 1u << (keys[i] % 32);
                key_count[s] = (uint32_t)k;
                flags[s] = used ? 2 : 0;
            }
            if (recon)
                for (int t = 0; t < frames; ++t) recon[(uint64_t)t * frame_stride + (uint64_t)s] = r[t];
            if (err2) err2[s] = e2;
        }
        free(v);
        free(r);
        free(keys);
    }
}

/* ---- the encoder's coarse control fitting (:705-729) ------------------------------------------ */

/* std::clamp(v, lo, hi) */
static float clamp_r(float v, float lo, float hi) { return v < lo ? lo : (hi < v ? hi : v); }

/* sampleLeafBufferAtFractional (:2203-2237): trilinear over the leaf's reconstruction lt (voxel
 * (lz*8 + ly)*8 + lx, frames fastest), the position clamped to the leaf's extent. */
static float kf_sample_leaf(const float* lt, int frames, int t, int w, int h, int d, float fx, float fy, float fz)
{
    const float x = clamp_r(fx, 0.0f, (float)(w - 1 > 0 ? w - 1 : 0));
    const float y = clamp_r(fy, 0.0f, (float)(h - 1 > 0 ? h - 1 : 0));
    const float z = clamp_r(fz, 0.0f, (float)(d - 1 > 0 ? d - 1 : 0));
    const int x0 = (int)floorf(x), y0 = (int)floorf(y), z0 = (int)floorf(z);
    const int x1 = w - 1 < x0 + 1 ? w - 1 : x0 + 1, y1 = h - 1 < y0 + 1 ? h - 1 : y0 + 1,
              z1 = d - 1 < z0 + 1 ? d - 1 : z0 + 1;
    const float tx = x - (float)x0, ty = y - (float)y0, tz = z - (float)z0;
#define AT(lx, ly, lz) lt[(size_t)((((lz) * 8 + (ly)) * 8 + (lx))) * (size_t)frames + (size_t)t]
    const float c00 = AT(x0, y0, z0) * (1.0f - tx) + AT(x1, y0, z0) * tx;
    const float c01 = AT(x0, y0, z1) * (1.0f - tx) + AT(x1, y0, z1) * tx;
    const float c10 = AT(x0, y1, z0) * (1.0f - tx) + AT(x1, y1, z0) * tx;
    const float c11 = AT(x0, y1, z1) * (1.0f - tx) + AT(x1, y1, z1) * tx;
#undef AT
    const float c0 = c00 * (1.0f - ty) + c10 * ty;
    const float c1 = c01 * (1.0f - ty) + c11 * ty;
    return c0 * (1.0f - tz) + c1 * tz;
}

/* buildBinIndexFromKeys (:2288-2305): per time bin, the index before the first key at or after the
 * bin's first frame (0 for the first key), else the last key; stored in a byte. */
static void kf_bin_index(const int* keys, int k, int frames, int bins, uint8_t* out)
{
    for (int bin = 0; bin < bins; ++bin) {
        out[bin] = 0u;
        if (k == 0) continue;
        const int start = (int)(((int64_t)bin * (int64_t)frames) / (bins > 1 ? bins : 1));
        uint8_t local = (uint8_t)(k - 1);
        for (int i = 0; i < k; ++i)
            if (keys[i] >= start) {
                local = (uint8_t)(i > 0 ? i - 1 : 0);
                break;
            }
        out[bin] = local;
    }
}

/* controlCoords(4) (:189-198), then for each of the 4^3 controls in (gz, gy, gx) order: the sampled
 * series, its keys under the control profile, appendControlSequenceToStream (:2361-2399) with 8
 * time bins, and reconstructFromKeys into grid[ctrl * frames + t].  desc[c] = keyStart |
 * keyCount << 16 | reserved << 24; bins[c * 8 + b].  Returns the stream's key count (-1 beyond
 * key_cap); *required_max_local = requiredMaxBinLocalKeys. */
int vo_coarse_fit(const float* lt, int frames, int w, int h, int d, const vo_keyframe_profile* p, uint32_t* desc,
                  uint8_t* bins, uint16_t* key_frames, float* key_values, int key_cap, int* required_max_local,
                  float* grid)
{
    const float scale = 7.0f / (float)(4 - 1);
    float coords[4];
    for (int i = 0; i < 4; ++i) coords[i] = (float)i * scale;
    float* series = (float*)malloc((size_t)(frames > 0 ? frames : 1) * sizeof(float));
    int* keys = (int*)malloc((size_t)(frames > 0 ? frames : 1) * sizeof(int));
    int nk = 0, overflow = 0;
    uint8_t required = 1u;
    for (int gz = 0; gz < 4; ++gz)
        for (int gy = 0; gy < 4; ++gy)
            for (int gx = 0; gx < 4; ++gx) {
                const int ctrl = (gz * 4 + gy) * 4 + gx;
                for (int t = 0; t < frames; ++t)
                    series[t] = kf_sample_leaf(lt, frames, t, w, h, d, coords[gx], coords[gy], coords[gz]);
                const int k = vo_detect_keyframes(series, frames, p, keys, NULL);
                uint8_t* b = bins + ctrl * 8;
                kf_bin_index(keys, k, frames, 8, b);
                int local = 1;
                for (int bin = 0; bin < 8; ++bin) {
                    const int next = bin + 1 < 8 ? (int)b[bin + 1] : k;
                    const int span = next - (int)b[bin] > 1 ? next - (int)b[bin] : 1;
                    if (span > local) local = span;
                    if (span > (int)required) required = (uint8_t)span;
                }
                desc[ctrl] = (uint32_t)(uint16_t)nk | ((uint32_t)(k < 255 ? k : 255) << 16) |
                             ((uint32_t)(local < 255 ? local : 255) << 24);
                for (int i = 0; i < k; ++i) {
                    if (nk < key_cap) {
                        key_frames[nk] = (uint16_t)keys[i];
                        key_values[nk] = series[keys[i]];
                    } else {
                        overflow = 1;
                    }
                    ++nk;
                }
                vo_reconstruct(series, frames, keys, k, grid + (size_t)ctrl * (size_t)frames);
            }
    free(series);
    free(keys);
    *required_max_local = required;
    return overflow ? -1 : nk;
}

/* renderTemporalFloatToHalfBits over an array (vo_float_to_half, element by element). */
void vo_float_to_half_n(const float* v, uint64_t n, uint16_t* out)
{
    for (uint64_t i = 0; i < n; ++i) out[i] = vo_float_to_half(v[i]);
}

/* sampleControlGridValue (:2240-2286): trilinear over a fitted control grid grid[ctrl * frames + t]
 * of `res`^3 controls at controlCoords(res), the position clamped to the leaf's extent. */
static float kf_sample_grid(const float* grid, int res, int frames, int t, int w, int h, int d, float fx, float fy,
                            float fz)
{
    float coords[8];
    const float scale = res > 1 ? 7.0f / (float)(res - 1) : 0.0f;
    for (int i = 0; i < res && i < 8; ++i) coords[i] = res > 1 ? (float)i * scale : 0.0f;
    int i0[3], i1[3];
    float wt[3];
    const float pos[3] = {fx, fy, fz};
    const int ext[3] = {w, h, d};
    for (int a = 0; a < 3; ++a) {
        const float p = clamp_r(pos[a], 0.0f, (float)(ext[a] - 1 > 0 ? ext[a] - 1 : 0));
        int j1 = 1;
        while (j1 < res - 1 && coords[j1] < p) ++j1;
        const int j0 = j1 - 1 > 0 ? j1 - 1 : 0;
        const float c0 = coords[j0], c1 = coords[j1];
        i0[a] = j0;
        i1[a] = j1;
        wt[a] = c1 > c0 ? (p - c0) / (c1 - c0) : 0.0f;
    }
#define G(ix, iy, iz) grid[(size_t)(((iz) * res + (iy)) * res + (ix)) * (size_t)frames + (size_t)t]
    const float tx = wt[0], ty = wt[1], tz = wt[2];
    const float c00 = G(i0[0], i0[1], i0[2]) * (1.0f - tx) + G(i1[0], i0[1], i0[2]) * tx;
    const float c01 = G(i0[0], i0[1], i1[2]) * (1.0f - tx) + G(i1[0], i0[1], i1[2]) * tx;
    const float c10 = G(i0[0], i1[1], i0[2]) * (1.0f - tx) + G(i1[0], i1[1], i0[2]) * tx;
    const float c11 = G(i0[0], i1[1], i1[2]) * (1.0f - tx) + G(i1[0], i1[1], i1[2]) * tx;
#undef G
    const float c0 = c00 * (1.0f - ty) + c10 * ty;
    const float c1 = c01 * (1.0f - ty) + c11 * ty;
    return c0 * (1.0f - tz) + c1 * tz;
}

/* The FINE6 residual fitting (:815-850, the plain fine6 variant): for the 6^3 controls at
 * controlCoords(6), the series sampled from the reconstruction minus the coarse grid sampled at the
 * same position, keyed with the control profile and appended with 8 time bins; outputs as
 * vo_coarse_fit (desc and bins for 216 controls, grid [216][frames]). */
int vo_fine6_fit(const float* lt, int frames, int w, int h, int d, const vo_keyframe_profile* p,
                 const float* coarse_grid, uint32_t* desc, uint8_t* bins, uint16_t* key_frames, float* key_values,
                 int key_cap, int* required_max_local, float* grid)
{
    const float scale = 7.0f / (float)(6 - 1);
    float coords[6];
    for (int i = 0; i < 6; ++i) coords[i] = (float)i * scale;
    float* series = (float*)malloc((size_t)(frames > 0 ? frames : 1) * sizeof(float));
    int* keys = (int*)malloc((size_t)(frames > 0 ? frames : 1) * sizeof(int));
    int nk = 0, overflow = 0;
    uint8_t required = 1u;
    for (int gz = 0; gz < 6; ++gz)
        for (int gy = 0; gy < 6; ++gy)
            for (int gx = 0; gx < 6; ++gx) {
                const int ctrl = (gz * 6 + gy) * 6 + gx;
                for (int t = 0; t < frames; ++t) {
                    const float raw_like = kf_sample_leaf(lt, frames, t, w, h, d, coords[gx], coords[gy], coords[gz]);
                    const float coarse = kf_sample_grid(coarse_grid, 4, frames, t, w, h, d, coords[gx], coords[gy],
                                                        coords[gz]);
                    series[t] = raw_like - coarse;
                }
                const int k = vo_detect_keyframes(series, frames, p, keys, NULL);
                uint8_t* b = bins + ctrl * 8;
                kf_bin_index(keys, k, frames, 8, b);
                int local = 1;
                for (int bin = 0; bin < 8; ++bin) {
                    const int next = bin + 1 < 8 ? (int)b[bin + 1] : k;
                    const int span = next - (int)b[bin] > 1 ? next - (int)b[bin] : 1;
                    if (span > local) local = span;
                    if (span > (int)required) required = (uint8_t)span;
                }
                desc[ctrl] = (uint32_t)(uint16_t)nk | ((uint32_t)(k < 255 ? k : 255) << 16) |
                             ((uint32_t)(local < 255 ? local : 255) << 24);
                for (int i = 0; i < k; ++i) {
                    if (nk < key_cap) {
                        key_frames[nk] = (uint16_t)keys[i];
                        key_values[nk] = series[keys[i]];
                    } else {
                        overflow = 1;
                    }
                    ++nk;
                }
                if (grid) vo_reconstruct(series, frames, keys, k, grid + (size_t)ctrl * (size_t)frames);
            }
    free(series);
    free(keys);
    *required_max_local = required;
    return overflow ? -1 : nk;
}

/* The Mode2 shell stage (:930-1025): the shell voxels of a leaf (inside its extent) and, for each,
 * the residual of the reconstruction over the fitted coarse grid, keyed with the control profile
 * (plus, for a level set, addIsoSurfaceKeyFrames on the voxel's own series at 0 +- temporal_band),
 * reconstructed, and appended to a 4-bin stream with its reconstruction's values at the keys.
 * A voxel is a shell voxel when, at some frame, (level set) |value| <= surface_band, |coarse| <=
 * guard_band or their signs differ, or (density) value >= shell_cut.  Writes the 80-byte occupancy
 * section (8 x u64 voxel masks, 8 x u16 group prefixes), descriptors and 8-byte bin rows (first 4
 * bytes used) per active voxel; returns the stream's key count (-1 beyond key_cap). */
int vo_shell_fit(const float* lt, int frames, int w, int h, int d, const vo_keyframe_profile* p,
                 const float* coarse_grid, int levelset, float surface_band, float guard_band, float temporal_band,
                 float shell_cut, uint8_t* occupancy, uint32_t* desc, uint8_t* bins, uint16_t* key_frames,
                 float* key_values, int key_cap, int* active_count, int* required_max_local)
{
    float* series = (float*)malloc((size_t)(frames > 0 ? frames : 1) * sizeof(float));
    float* recon = (float*)malloc((size_t)(frames > 0 ? frames : 1) * sizeof(float));
    int* keys = (int*)malloc((size_t)(frames > 0 ? frames : 1) * sizeof(int));
    uint8_t* flag = (uint8_t*)malloc((size_t)(frames > 0 ? frames : 1));
    int nk = 0, overflow = 0, active = 0;
    uint8_t required = 1u;
    memset(occupancy, 0, 80);
    for (int group = 0; group < 8; ++group) {
        const uint16_t prefix = (uint16_t)active;
        memcpy(occupancy + 64 + 2 * group, &prefix, 2);
        uint64_t word = 0;
        for (int bit = 0; bit < 64; ++bit) {
            const int v = group * 64 + bit, lx = v % 8, ly = (v / 8) % 8, lz = v / 64;
            if (lx >= w || ly >= h || lz >= d) continue;
            const float* truth = lt + (size_t)v * (size_t)frames;
            int is_shell = 0;
            for (int t = 0; t < frames && !is_shell; ++t) {
                if (levelset) {
                    const float c = kf_sample_grid(coarse_grid, 4, frames, t, w, h, d, (float)lx, (float)ly, (float)lz);
                    is_shell = fabsf(truth[t]) <= surface_band || fabsf(c) <= guard_band ||
                               (truth[t] >= 0.0f) != (c >= 0.0f);
                } else {
                    is_shell = truth[t] >= shell_cut;
                }
            }
            if (!is_shell) continue;
            word |= 1ull << bit;
            for (int t = 0; t < frames; ++t)
                series[t] = truth[t] - kf_sample_grid(coarse_grid, 4, frames, t, w, h, d, (float)lx, (float)ly, (float)lz);
            int k = vo_detect_keyframes(series, frames, p, keys, NULL);
            if (levelset) {   /* addIsoSurfaceKeyFrames(truth, 0, temporal_band, keys), then sorted and unique */
                memset(flag, 0, (size_t)frames);
                for (int i = 0; i < k; ++i) flag[keys[i]] = 1;
                const float band = fmax_r(0.0f, temporal_band);
                for (int t = 0; t < frames; ++t) {
                    const float cur = truth[t] - 0.0f;
                    if (fabsf(cur) <= band)
                        for (int u = t - 1; u <= t + 1; ++u)
                            if (u >= 0 && u < frames) flag[u] = 1;
                    if (t > 0 && ((truth[t - 1] - 0.0f) >= 0.0f) != (cur >= 0.0f))
                        for (int u = t - 2; u <= t + 1; ++u)
                            if (u >= 0 && u < frames) flag[u] = 1;
                }
                k = 0;
                for (int t = 0; t < frames; ++t)
                    if (flag[t]) keys[k++] = t;
            }
            vo_reconstruct(series, frames, keys, k, recon);
            uint8_t* b = bins + (size_t)active * 8u;
            memset(b, 0, 8);
            kf_bin_index(keys, k, frames, 4, b);
            int local = 1;
            for (int bin = 0; bin < 4; ++bin) {
                const int next = bin + 1 < 4 ? (int)b[bin + 1] : k;
                const int span = next - (int)b[bin] > 1 ? next - (int)b[bin] : 1;
                if (span > local) local = span;
                if (span > (int)required) required = (uint8_t)span;
            }
            desc[active] = (uint32_t)(uint16_t)nk | ((uint32_t)(k < 255 ? k : 255) << 16) |
                           ((uint32_t)(local < 255 ? local : 255) << 24);
            for (int i = 0; i < k; ++i) {
                if (nk < key_cap) {
                    key_frames[nk] = (uint16_t)keys[i];
                    key_values[nk] = recon[keys[i]];
                } else {
                    overflow = 1;
                }
                ++nk;
            }
            ++active;
        }
        memcpy(occupancy + 8 * group, &word, 8);
    }
    free(series);
    free(recon);
    free(keys);
    free(flag);
    *active_count = active;
    *required_max_local = required;
    return overflow ? -1 : nk;
}
