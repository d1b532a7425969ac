// keyframes.cu -- the encoder's per-voxel keyframe pass on the GPU (vbt_detect_keyframes).
//
// For every voxel series of a raw frame-major volume, what the reference encoder's leaf loop does
// per voxel (src/render_temporal_kf_probe_main.cpp:619-659): the background test on the running
// max, detectDensityKeyFrames (:2080-2167: statistics, the constant test, dpRecurse's recursive
// split at the largest normalised error, cutoff and iso-surface protection), reconstructFromKeys
// (:2169-2201) and the squared error.  Keys, flags, reconstruction and error equal the reference's
// bit for bit.
//
// One thread owns one series.  A CTA stages its NV series (all frames) in shared memory as
// [frame][series], so lanes reading different frames of their own series never share a bank, and
// keeps the key set as a bitmask column beside it.  The recursion becomes a cursor walk over the
// key set (split the interval at the cursor until it holds, then step to the next key), flattened
// so that one loop iteration evaluates one frame of whatever interval each lane is in: lanes of a
// warp stay busy however different their splits are.
//
// Per evaluated frame the reference divides twice in double.  Here alpha = (t-a)/(b-a) comes from
// the correctly rounded reciprocal of b-a and one Markstein correction (exact for every integer
// pair this kernel meets; vbt_selftest_keyframe_division checks them all), and the normalised error
// is first bracketed by an approximation good to 2^-20 relative: only when it lies within 2^-15 of
// the running maximum (or of 1.0 for the split decision) is the exact double quotient formed.
#include <cuda_runtime.h>

#include <string>

#include "../../include/vbt_b200.h"

namespace vbtb {
int set_last_error(int status, const std::string& msg);
}

namespace {

constexpr uint32_t kKfMaxFrames = 1024;
constexpr double kHi = 1.0 + 1.0 / 32768.0;   // approximation margins (the approximation is good to 2^-20)
constexpr double kLo = 1.0 - 1.0 / 32768.0;

// std::max(a, b): a unless a < b.
__device__ __forceinline__ float fmax_r(float a, float b) { return a < b ? b : a; }
__device__ __forceinline__ double dmax_r(double a, double b) { return a < b ? b : a; }

// a / b for integers 0 <= a <= b <= 1024 held in doubles, given y = RN(1 / b): Markstein's
// correction step q = q0 + (a - q0 b) y, with the residual exact in an fma.
__device__ __forceinline__ double div_int_rn(double a, double b, double y)
{
    const double q0 = __dmul_rn(a, y);
    const double r = __fma_rn(-q0, b, a);
    return __fma_rn(r, y, q0);
}

// RN(1 / k) for k = 1 .. kKfMaxFrames (entry 0 unused), written by kf_rcp_init_kernel ahead of every
// pass on the pass's stream: one cached load where an interval or a key segment starts.
__device__ double g_kf_rcp[kKfMaxFrames + 1];

__global__ void kf_rcp_init_kernel()
{
    for (uint32_t k = 1u + threadIdx.x; k <= kKfMaxFrames; k += blockDim.x) g_kf_rcp[k] = __drcp_rn((double)k);
}

struct KfTotals {
    unsigned long long total_keys, protected_series, background_series;
    unsigned int max_keys, pad;
    double err2;
};

// cutoffState (:227-233).
__device__ __forceinline__ int cutoff_state(float v, float cutoff, float band)
{
    if (cutoff <= 0.0f) return 1;
    if (v < __fsub_rn(cutoff, band)) return 0;
    if (v > __fadd_rn(cutoff, band)) return 2;
    return 1;
}

template <int NV>
struct Column {
    const float* v;   // v[t * NV]
    uint32_t* m;      // m[w * NV]
    __device__ __forceinline__ float at(int t) const { return v[t * NV]; }
    __device__ __forceinline__ void set(int t) const { m[(t >> 5) * NV] |= 1u << (t & 31); }
    // The first key after frame a (the last frame is always a key, and a lies before it).
    __device__ __forceinline__ int next_key(int a, int words) const
    {
        int w = (a + 1) >> 5;
        uint32_t bits = m[w * NV] & (0xFFFFFFFFu << ((a + 1) & 31));
        while (bits == 0u && w + 1 < words) bits = m[++w * NV];
        return bits ? (w << 5) + __ffs(bits) - 1 : -1;
    }
};

struct SeriesStats {
    float stddev, ds;   // computeStats' stddev and max(1e-6, deltaScale)
};

// epsilonAt (:235-247), exactly.
__device__ __forceinline__ float eps_exact(float x, float prev, bool has_prev, const vbt_keyframe_profile& p,
                                           const SeriesStats& st, float floor_)
{
    float eps = __fadd_rn(p.eps_abs, __fmul_rn(p.eps_rel, fmax_r(fabsf(x), st.stddev)));
    if (p.gamma_delta > 0.0f && has_prev) {
        const float delta = __fdiv_rn(fabsf(__fsub_rn(x, prev)), st.ds);
        eps = __fdiv_rn(eps, __fadd_rn(1.0f, __fmul_rn(p.gamma_delta, delta)));
    }
    return fmax_r(eps, floor_);
}

struct SeriesOut {
    uint32_t count;
    uint8_t flag;
    double e2;
};

// The leaf loop's body for one series: key bits into col.m, the reconstruction into recon[t * fstride]
// (when not null); returns the key count, the flags and the squared error.
template <int NV>
__device__ __forceinline__ SeriesOut keyframe_series(const Column<NV>& col, float* top, int n, int words,
                                                  const vbt_keyframe_profile& p, float* recon,
                                                  unsigned long long fstride)
{
    for (int w = 0; w < words; ++w) col.m[w * NV] = 0u;

    // One pass: the running max of the leaf loop, and the sums of computeStats and of the constant test.
    float vmax = 0.0f;
    double sum = 0.0, sum2 = 0.0;
    for (int t = 0; t < n; ++t) {
        const float x = col.at(t);
        vmax = fmax_r(vmax, x);
        const double xd = (double)x;
        sum = __dadd_rn(sum, xd);
        sum2 = __dadd_rn(sum2, __dmul_rn(xd, xd));
    }

    uint32_t count;
    uint8_t flag = 0;
    double e2 = 0.0;
    const float floor_ = fmax_r(1e-6f, __fmul_rn(p.eps_abs, 0.1f));
    const double nd = (double)n;
    const double mean = __ddiv_rn(sum, nd);
    const double var_c = dmax_r(0.0, __dsub_rn(__ddiv_rn(sum2, nd), __dmul_rn(mean, mean)));
    const bool background = p.bg_threshold >= 0.0 && (double)vmax < p.bg_threshold;
    if (background || n == 1 || var_c < __dmul_rn((double)floor_, (double)floor_)) {
        // Background-zeroed (reconstruction 0, counted as one key), or a single key at frame 0
        // (one frame, or variance under the epsilon floor): the reconstruction is the first value.
        const float fill = background ? 0.0f : col.at(0);
        if (background) {
            e2 = sum2;      // the same sequence of squares the leaf loop sums
            flag = 1;
        } else {
            col.set(0);
            for (int t = 0; t < n; ++t) {
                const double d = __dsub_rn((double)col.at(t), (double)fill);
                e2 = __dadd_rn(e2, __dmul_rn(d, d));
            }
        }
        count = 1;
        if (recon)
            for (int t = 0; t < n; ++t) recon[(unsigned long long)t * fstride] = fill;
    } else {
        // computeStats (:200-225).
        SeriesStats st;
        {
            const float mean_f = __double2float_rn(mean);
            const double var_s =
                dmax_r(0.0, __dsub_rn(__ddiv_rn(sum2, nd), __dmul_rn((double)mean_f, (double)mean_f)));
            st.stddev = __double2float_rn(__dsqrt_rn(var_s));
            // deltas[min(m - 1, 9m / 10)] of the sorted |delta|s = the r-th largest, r = m - that index:
            // kept as an ascending list of the r largest seen.
            const int m = n - 1;
            const int r = m - min(m - 1, (m * 9) / 10);
            int cnt = 0;
            float prev = col.at(0);
            for (int t = 1; t < n; ++t) {
                const float x = col.at(t);
                const float d = fabsf(__fsub_rn(x, prev));
                prev = x;
                if (cnt < r) {
                    int k = cnt++;
                    while (k > 0 && top[(k - 1) * NV] > d) {
                        top[k * NV] = top[(k - 1) * NV];
                        --k;
                    }
                    top[k * NV] = d;
                } else if (d > top[0]) {
                    int k = 0;
                    while (k + 1 < r && top[(k + 1) * NV] < d) {
                        top[k * NV] = top[(k + 1) * NV];
                        ++k;
                    }
                    top[k * NV] = d;
                }
            }
            st.ds = fmax_r(1e-6f, fmax_r(1e-6f, top[0]));
        }
        const bool gamma_on = p.gamma_delta > 0.0f;
        const float inv_ds = __frcp_rn(st.ds), inv_floor = __frcp_rn(floor_);
        auto exact_err = [&](int t, double num) {
            const float e = eps_exact(col.at(t), t > 0 ? col.at(t - 1) : 0.0f, t > 0, p, st, floor_);
            return __ddiv_rn(num, (double)e);
        };

        // dpRecurse (:249-276) as a cursor walk over the key set.
        col.set(0);
        col.set(n - 1);
        uint32_t pushes = 2;
        int a = 0, b = n - 1;
        double v0 = (double)col.at(a), dv = __dsub_rn((double)col.at(b), v0);
        double den = (double)(b - a), y = __ldg(g_kf_rcp + (b - a));
        float xp = col.at(a);      // frame t - 1
        int t = a + 1, lead = -1;
        double lead_a = 0.0, lead_num = 0.0, lead_e = 0.0;
        bool lead_exact = true;    // lead_e holds the leader's exact error (0 for no leader)
        for (;;) {
            if (t < b) {
                const float x = col.at(t);
                const double alpha = div_int_rn((double)(t - a), den, y);
                const double pred = __dadd_rn(v0, __dmul_rn(alpha, dv));
                const double num = fabs(__dsub_rn((double)x, pred));
                if (num != 0.0) {
                    // 1 / epsilonAt = min((1 + gamma delta) / e0, 1 / floor), to 2^-21 relative
                    const float e0 = __fadd_rn(p.eps_abs, __fmul_rn(p.eps_rel, fmax_r(fabsf(x), st.stddev)));
                    float r = __frcp_rn(e0);
                    if (gamma_on) r *= fmaf(p.gamma_delta, fabsf(x - xp) * inv_ds, 1.0f);
                    const double e_a = num * (double)fminf(r, inv_floor);
                    if (e_a > lead_a * kHi) {
                        lead = t;
                        lead_a = e_a;
                        lead_num = num;
                        lead_exact = false;
                    } else if (!(e_a < lead_a * kLo)) {
                        if (!lead_exact) {
                            lead_e = exact_err(lead, lead_num);
                            lead_exact = true;
                        }
                        const double e = exact_err(t, num);
                        if (e > lead_e) {
                            lead = t;
                            lead_a = e_a;
                            lead_num = num;
                            lead_e = e;
                        }
                    }
                }
                xp = x;
                ++t;
                continue;
            }
            bool split = false;
            if (lead >= 0) {
                if (lead_a > kHi) split = true;
                else if (!(lead_a < kLo)) split = (lead_exact ? lead_e : exact_err(lead, lead_num)) > 1.0;
            }
            if (split) {
                col.set(lead);
                ++pushes;
                b = lead;
            } else {
                a = b;
                if (a >= n - 1) break;
                b = col.next_key(a, words);
                if (b < 0) break;   // unreachable: frame n - 1 is a key
            }
            xp = col.at(a);
            v0 = (double)xp;
            dv = __dsub_rn((double)col.at(b), v0);
            den = (double)(b - a);
            y = __ldg(g_kf_rcp + (b - a));
            t = a + 1;
            lead = -1;
            lead_a = 0.0;
            lead_e = 0.0;
            lead_exact = true;
        }

        // Cutoff protection (:2125-2146).
        bool used = false;
        if (p.cutoff_temporal_protect && p.render_cutoff > 0.0f && p.cutoff_band >= 0.0f) {
            int prev_state = 0;
            for (int u = 0; u < n; ++u) {
                const int cs = cutoff_state(col.at(u), p.render_cutoff, p.cutoff_band);
                if (cs == 1) {
                    if (u > 0) col.set(u - 1);
                    col.set(u);
                    if (u + 1 < n) col.set(u + 1);
                    pushes += 1u + (u > 0) + (u + 1 < n);
                    used = true;
                }
                if (u > 0 && prev_state != cs) {
                    col.set(u - 1);
                    col.set(u);
                    if (u + 1 < n) col.set(u + 1);
                    pushes += 2u + (u + 1 < n);
                    used = true;
                }
                prev_state = cs;
            }
        }
        count = 0;
        if (p.iso_surface_protect) {
            // addIsoSurfaceKeyFrames (:2051-2078); "added" compares the distinct keys after it with
            // the list length before it, duplicates included.
            const float band = fmax_r(0.0f, p.iso_band);
            float prev = 0.0f;
            for (int u = 0; u < n; ++u) {
                const float cur = __fsub_rn(col.at(u), p.iso_value);
                if (fabsf(cur) <= band) {
                    if (u > 0) col.set(u - 1);
                    col.set(u);
                    if (u + 1 < n) col.set(u + 1);
                }
                if (u > 0 && (prev >= 0.0f) != (cur >= 0.0f)) {
                    if (u > 1) col.set(u - 2);
                    col.set(u - 1);
                    col.set(u);
                    if (u + 1 < n) col.set(u + 1);
                }
                prev = cur;
            }
            for (int w = 0; w < words; ++w) count += __popc(col.m[w * NV]);
            used = used || count > pushes;
        } else {
            for (int w = 0; w < words; ++w) count += __popc(col.m[w * NV]);
        }
        flag = used ? 2 : 0;

        // reconstructFromKeys (:2169-2201): frame 0 is the first key and frame n - 1 the last, so
        // every later frame lies in (a, b] of two consecutive keys.
        int ka = 0, kb = col.next_key(0, words);
        float va = col.at(0), vb = col.at(kb);
        double kden = (double)kb, ky = __ldg(g_kf_rcp + kb);
        for (int u = 0; u < n; ++u) {
            const float x = col.at(u);
            float out;
            if (u == 0) {
                out = va;
            } else {
                if (u > kb) {
                    ka = kb;
                    kb = col.next_key(ka, words);
                    va = vb;
                    vb = col.at(kb);
                    kden = (double)(kb - ka);
                    ky = __ldg(g_kf_rcp + (kb - ka));
                }
                const double alpha = div_int_rn((double)(u - ka), kden, ky);
                out = __double2float_rn(__dadd_rn((double)va, __dmul_rn(alpha, (double)__fsub_rn(vb, va))));
            }
            const double d = __dsub_rn((double)x, (double)out);
            e2 = __dadd_rn(e2, __dmul_rn(d, d));
            if (recon) recon[(unsigned long long)u * fstride] = out;
        }
    }

    return SeriesOut{count, flag, e2};
}

template <int NV>
__global__ void __launch_bounds__(NV) keyframe_pass_kernel(const float* __restrict__ values, unsigned long long series,
                                                           int n, unsigned long long fstride,
                                                           unsigned long long sstride, vbt_keyframe_profile p,
                                                           int rmax, uint32_t* __restrict__ key_mask,
                                                           uint32_t* __restrict__ key_count, uint8_t* __restrict__ flags,
                                                           float* __restrict__ recon, double* __restrict__ err2_out,
                                                           KfTotals* __restrict__ totals)
{
    extern __shared__ __align__(16) float kf_smem[];
    const int words = (n + 31) >> 5;
    float* sv = kf_smem;                                               // [n][NV]
    uint32_t* sm = reinterpret_cast<uint32_t*>(sv + n * NV);           // [words][NV]
    float* stop = reinterpret_cast<float*>(sm + words * NV);           // [rmax][NV]
    const int j = threadIdx.x;
    const unsigned long long base = (unsigned long long)blockIdx.x * NV;

    if (sstride == 1ull) {              // frame-major: a warp reads 32 neighbouring series of one frame
        for (int idx = j; idx < n * NV; idx += NV) {
            const int t = idx / NV, c = idx - t * NV;
            const unsigned long long s = base + (unsigned long long)c;
            sv[idx] = s < series ? __ldcs(values + (unsigned long long)t * fstride + s) : 0.0f;
        }
    } else {                            // time fastest: a warp reads 32 neighbouring frames of one series
        for (int idx = j; idx < n * NV; idx += NV) {
            const int c = idx / n, t = idx - c * n;
            const unsigned long long s = base + (unsigned long long)c;
            sv[t * NV + c] = s < series ? __ldcs(values + (unsigned long long)t * fstride + s * sstride) : 0.0f;
        }
    }
    __syncthreads();

    const unsigned long long s = base + (unsigned long long)j;
    const bool valid = s < series;
    SeriesOut r{0u, 0, 0.0};
    if (valid) {
        const Column<NV> col{sv + j, sm + j};
        r = keyframe_series<NV>(col, stop + j, n, words, p, recon ? recon + s * sstride : nullptr, fstride);
        for (int w = 0; w < words; ++w) key_mask[(unsigned long long)w * series + s] = col.m[w * NV];
        key_count[s] = r.count;
        flags[s] = r.flag;
        if (err2_out) err2_out[s] = r.e2;
    }

    if (totals) {   // every lane of the warp is here (none returned early); idle lanes add zeros
        unsigned long long keys = r.count, prot = (r.flag >> 1) & 1u, bg = r.flag & 1u;
        unsigned int kmax = r.count;
        double e = r.e2;
        for (int o = 16; o > 0; o >>= 1) {
            keys += __shfl_xor_sync(0xFFFFFFFFu, keys, o);
            prot += __shfl_xor_sync(0xFFFFFFFFu, prot, o);
            bg += __shfl_xor_sync(0xFFFFFFFFu, bg, o);
            kmax = max(kmax, __shfl_xor_sync(0xFFFFFFFFu, kmax, o));
            e += __shfl_xor_sync(0xFFFFFFFFu, e, o);
        }
        if ((threadIdx.x & 31) == 0) {
            atomicAdd(&totals->total_keys, keys);
            atomicAdd(&totals->protected_series, prot);
            atomicAdd(&totals->background_series, bg);
            atomicMax(&totals->max_keys, kmax);
            atomicAdd(&totals->err2, e);
        }
    }
}

// Every a / b with 1 <= b <= b_max and 0 <= a <= b through div_int_rn against the IEEE quotient.
__global__ void keyframe_division_check_kernel(uint32_t b_max, unsigned long long* bad, unsigned long long* first)
{
    unsigned long long local = 0;
    for (uint32_t b = 1u + blockIdx.x; b <= b_max; b += gridDim.x) {
        const double bd = (double)b, y = __drcp_rn(bd);
        for (uint32_t a = threadIdx.x; a <= b; a += blockDim.x) {
            const double q = div_int_rn((double)a, bd, y);
            if (__double_as_longlong(q) != __double_as_longlong(__ddiv_rn((double)a, bd))) {
                ++local;
                atomicMin(first, ((unsigned long long)b << 16) | a);
            }
        }
    }
    if (local) atomicAdd(bad, local);
}

// ---- the encoder's coarse control fitting (src/render_temporal_kf_probe_main.cpp:705-729) ---------
// One CTA of 64 threads per leaf, one thread per coarse control c = (gz*4 + gy)*4 + gx: the control's
// series is sampled from the leaf's reconstruction at controlCoords(4)
// (sampleLeafBufferAtFractional, :2203-2237) into the same [frame][control] shared column the pass
// uses, keyed by keyframe_series under the control profile (no background test), and appended to
// the leaf's stream as appendControlSequenceToStream (:2361-2399) does: descriptor, bin row
// (buildBinIndexFromKeys, :2288-2305) and keyframes (frame, sampled value).

struct CoarseOut {
    uint32_t* desc;          // [leaf][C]
    uint8_t* bins;           // [leaf][C][8]
    uint16_t* key_frame;     // [leaf][C * frames]
    float* key_value;        // [leaf][C * frames]
    uint32_t* key_count;     // [leaf]
    uint8_t* required;       // [leaf] requiredMaxBinLocalKeys
    float* grid;             // optional [leaf][C][frames]
};

// std::clamp(v, lo, hi)
__device__ __forceinline__ float clamp_r(float v, float lo, float hi) { return v < lo ? lo : (hi < v ? hi : v); }

// One axis of sampleControlGridValue (:2240-2286) on a fitted 4^3 grid at controlCoords(4): the
// position clamped to the extent, the first coordinate at or above it (from the second on), the
// weight (p - c0) / (c1 - c0).
__device__ __forceinline__ void grid4_axis(float pos, int ext, int& j0, int& j1, float& w)
{
    const float scale = __fdiv_rn(7.0f, 3.0f);
    const float p = clamp_r(pos, 0.0f, (float)max(0, ext - 1));
    int k = 1;
    while (k < 3 && __fmul_rn((float)k, scale) < p) ++k;
    j1 = k;
    j0 = k - 1 > 0 ? k - 1 : 0;
    const float c0 = __fmul_rn((float)j0, scale), c1 = __fmul_rn((float)j1, scale);
    w = c1 > c0 ? __fdiv_rn(__fsub_rn(p, c0), __fsub_rn(c1, c0)) : 0.0f;
}

// The fitted 4^3 grid g[ctrl * n + t] sampled at frame t with the axes of grid4_axis, in the
// encoder's lerp order (x, then y, then z).
struct Grid4Sample {
    int x0, x1, y0, y1, z0, z1;
    float tx, ty, tz;
    __device__ __forceinline__ void init(float fx, float fy, float fz, int w, int h, int d)
    {
        grid4_axis(fx, w, x0, x1, tx);
        grid4_axis(fy, h, y0, y1, ty);
        grid4_axis(fz, d, z0, z1, tz);
    }
    __device__ __forceinline__ float at(const float* __restrict__ g, int n, int t) const
    {
        auto G = [&](int ix, int iy, int iz) { return __ldg(g + (unsigned)(((iz * 4 + iy) * 4 + ix) * n + t)); };
        const float ux = __fsub_rn(1.0f, tx), uy = __fsub_rn(1.0f, ty), uz = __fsub_rn(1.0f, tz);
        const float c00 = __fadd_rn(__fmul_rn(G(x0, y0, z0), ux), __fmul_rn(G(x1, y0, z0), tx));
        const float c01 = __fadd_rn(__fmul_rn(G(x0, y0, z1), ux), __fmul_rn(G(x1, y0, z1), tx));
        const float c10 = __fadd_rn(__fmul_rn(G(x0, y1, z0), ux), __fmul_rn(G(x1, y1, z0), tx));
        const float c11 = __fadd_rn(__fmul_rn(G(x0, y1, z1), ux), __fmul_rn(G(x1, y1, z1), tx));
        const float c0 = __fadd_rn(__fmul_rn(c00, uy), __fmul_rn(c10, ty));
        const float c1 = __fadd_rn(__fmul_rn(c01, uy), __fmul_rn(c11, ty));
        return __fadd_rn(__fmul_rn(c0, uz), __fmul_rn(c1, tz));
    }
};

// The control fitting of one leaf per CTA, one thread per control of an R^3 grid at
// controlCoords(R): R = 4 is the coarse fit (:705-729); R = 6 with RESID the FINE6 residual fit
// (:815-850), whose series is the sampled reconstruction minus the fitted coarse grid
// (cgrid[leaf][64][frames], from the coarse fit) sampled at the same position.
template <int R, bool RESID>
__global__ void __launch_bounds__(R * R * R) control_fit_kernel(const float* __restrict__ recon, uint32_t X,
                                                                uint32_t Y, uint32_t Z, int n,
                                                                unsigned long long fstride,
                                                                const uint32_t* __restrict__ leaves,
                                                                uint32_t n_leaves, vbt_keyframe_profile p, int rmax,
                                                                const float* __restrict__ cgrid, CoarseOut o)
{
    constexpr int NV = R * R * R;
    extern __shared__ __align__(16) float cf_smem[];
    __shared__ int s_count[NV], s_start[NV], s_span[NV * 8];
    const int words = (n + 31) >> 5;
    float* sv = cf_smem;                                               // [n][NV]
    uint32_t* sm = reinterpret_cast<uint32_t*>(sv + n * NV);           // [words][NV]
    float* stop = reinterpret_cast<float*>(sm + words * NV);           // [rmax][NV]
    const int c = threadIdx.x;
    const uint32_t li = blockIdx.x;
    if (li >= n_leaves) return;          // uniform per CTA
    const uint32_t leaf = leaves[li];
    const uint32_t lcx = (X + 7u) / 8u, lcy = (Y + 7u) / 8u, lcz = (Z + 7u) / 8u;
    if ((unsigned long long)leaf >= (unsigned long long)lcx * lcy * lcz) {   // uniform per CTA
        if (c == 0) o.key_count[li] = 0xFFFFFFFFu;
        return;
    }
    const uint32_t bx = leaf % lcx, by = (leaf / lcx) % lcy, bz = leaf / (lcx * lcy);
    const int w = (int)min(8u, X - 8u * bx), h = (int)min(8u, Y - 8u * by), d = (int)min(8u, Z - 8u * bz);
    const float scale = __fdiv_rn(7.0f, (float)(R - 1));
    const int gx = c % R, gy = (c / R) % R, gz = c / (R * R);
    const float px = __fmul_rn((float)gx, scale), py = __fmul_rn((float)gy, scale), pz = __fmul_rn((float)gz, scale);
    const float x = clamp_r(px, 0.0f, (float)max(0, w - 1));
    const float y = clamp_r(py, 0.0f, (float)max(0, h - 1));
    const float z = clamp_r(pz, 0.0f, (float)max(0, d - 1));
    const int x0 = (int)floorf(x), y0 = (int)floorf(y), z0 = (int)floorf(z);
    const int x1 = min(w - 1, x0 + 1), y1 = min(h - 1, y0 + 1), z1 = min(d - 1, z0 + 1);
    const float tx = __fsub_rn(x, (float)x0), ty = __fsub_rn(y, (float)y0), tz = __fsub_rn(z, (float)z0);
    const float ux = __fsub_rn(1.0f, tx), uy = __fsub_rn(1.0f, ty), uz = __fsub_rn(1.0f, tz);
    auto vox = [&](int lx, int ly, int lz) {
        return (unsigned long long)((8u * bz + (uint32_t)lz) * Y + 8u * by + (uint32_t)ly) * X + 8u * bx + (uint32_t)lx;
    };
    const unsigned long long v000 = vox(x0, y0, z0), v100 = vox(x1, y0, z0), v001 = vox(x0, y0, z1),
                             v101 = vox(x1, y0, z1), v010 = vox(x0, y1, z0), v110 = vox(x1, y1, z0),
                             v011 = vox(x0, y1, z1), v111 = vox(x1, y1, z1);
    Grid4Sample cs{};
    const float* cg = RESID ? cgrid + (unsigned long long)li * 64u * (unsigned)n : nullptr;
    if (RESID) cs.init(px, py, pz, w, h, d);
    for (int t = 0; t < n; ++t) {
        const float* f = recon + (unsigned long long)t * fstride;
        const float c00 = __fadd_rn(__fmul_rn(__ldg(f + v000), ux), __fmul_rn(__ldg(f + v100), tx));
        const float c01 = __fadd_rn(__fmul_rn(__ldg(f + v001), ux), __fmul_rn(__ldg(f + v101), tx));
        const float c10 = __fadd_rn(__fmul_rn(__ldg(f + v010), ux), __fmul_rn(__ldg(f + v110), tx));
        const float c11 = __fadd_rn(__fmul_rn(__ldg(f + v011), ux), __fmul_rn(__ldg(f + v111), tx));
        const float c0 = __fadd_rn(__fmul_rn(c00, uy), __fmul_rn(c10, ty));
        const float c1 = __fadd_rn(__fmul_rn(c01, uy), __fmul_rn(c11, ty));
        float v = __fadd_rn(__fmul_rn(c0, uz), __fmul_rn(c1, tz));
        if (RESID) v = __fsub_rn(v, cs.at(cg, n, t));
        sv[t * NV + c] = v;
    }
    const Column<NV> col{sv + c, sm + c};
    float* grid = o.grid ? o.grid + ((unsigned long long)li * NV + (unsigned)c) * (unsigned)n : nullptr;
    const SeriesOut r = keyframe_series<NV>(col, stop + c, n, words, p, grid, 1ull);
    const int count = (int)r.count;

    // buildBinIndexFromKeys: one merge of the sorted keys with the bins' first frames.
    uint8_t b8[8];
    {
        int b = 0, i = 0;
        for (int wd = 0; wd < words && b < 8; ++wd) {
            uint32_t bits = col.m[wd * NV];
            while (bits && b < 8) {
                const int key = (wd << 5) + __ffs(bits) - 1;
                bits &= bits - 1u;
                while (b < 8 && key >= (int)(((long long)b * n) / 8)) b8[b++] = (uint8_t)(i > 0 ? i - 1 : 0);
                ++i;
            }
        }
        for (; b < 8; ++b) b8[b] = (uint8_t)(count - 1);
    }
    int local = 1;
    for (int b = 0; b < 8; ++b) {
        const int next = b + 1 < 8 ? (int)b8[b + 1] : count;
        const int span = max(1, next - (int)b8[b]);
        s_span[c * 8 + b] = span;
        local = max(local, span);
    }
    s_count[c] = count;
    __syncthreads();
    if (c == 0) {            // keyStart: the keys of the controls before, in control order
        int run = 0, req = 1;
        for (int k = 0; k < NV; ++k) {
            s_start[k] = run;
            run += s_count[k];
            for (int b = 0; b < 8; ++b) req = (int)(uint8_t)max(req, s_span[k * 8 + b]);
        }
        o.key_count[li] = (uint32_t)run;
        o.required[li] = (uint8_t)req;
    }
    __syncthreads();
    const int start = s_start[c];
    o.desc[(unsigned long long)li * NV + (unsigned)c] =
        (uint32_t)(uint16_t)start | ((uint32_t)min(count, 255) << 16) | ((uint32_t)min(local, 255) << 24);
    uint8_t* brow = o.bins + ((unsigned long long)li * NV + (unsigned)c) * 8u;
    for (int b = 0; b < 8; ++b) brow[b] = b8[b];
    const unsigned long long kbase = (unsigned long long)li * NV * (unsigned)n + (unsigned)start;
    int i = 0;
    for (int wd = 0; wd < words; ++wd) {
        uint32_t bits = col.m[wd * NV];
        while (bits) {
            const int key = (wd << 5) + __ffs(bits) - 1;
            bits &= bits - 1u;
            o.key_frame[kbase + i] = (uint16_t)key;
            o.key_value[kbase + i] = col.at(key);
            ++i;
        }
    }
}

// ---- the Mode2 shell stage (:930-1025) ------------------------------------------------------
// One leaf per CTA, 128 threads, the 512 voxels in four rounds.  A voxel inside the leaf's extent
// is a shell voxel when at some frame (level set) |value| <= surface_band, |coarse| <= guard_band
// or their signs differ, or (density) value >= shell_cut -- value the pass's reconstruction,
// coarse the fitted coarse grid sampled at the voxel.  Its residual series (value - coarse) is
// keyed under the control profile, for a level set joined with addIsoSurfaceKeyFrames (:2051-2078)
// on the voxel's own series at 0 +- temporal_band, and appended to a 4-bin stream with its
// reconstructFromKeys values at the keys (:2169-2201).  Streams follow the voxel order; the
// occupancy section holds the 8 x u64 voxel masks and the 8 x u16 group prefixes.

struct ShellOut {
    uint8_t* occupancy;      // [leaf][80]
    uint32_t* desc;          // [leaf][512]
    uint8_t* bins;           // [leaf][512][8] (first 4 bytes used)
    uint16_t* key_frame;     // [leaf][512 * frames]
    float* key_value;        // [leaf][512 * frames]
    uint32_t* key_count;     // [leaf]
    uint32_t* active;        // [leaf]
    uint8_t* required;       // [leaf]
};

constexpr int kShellThreads = 128;

__global__ void __launch_bounds__(kShellThreads) shell_fit_kernel(
    const float* __restrict__ recon, uint32_t X, uint32_t Y, uint32_t Z, int n, unsigned long long fstride,
    const uint32_t* __restrict__ leaves, uint32_t n_leaves, vbt_keyframe_profile p, int rmax,
    const float* __restrict__ cgrid, int levelset, float surface_band, float guard_band, float temporal_band,
    float shell_cut, ShellOut o)
{
    constexpr int NT = kShellThreads;
    extern __shared__ __align__(16) float sh_smem[];
    __shared__ uint32_t s_mask[16];            // voxel bits, 32 per word
    __shared__ int s_wc[NT / 32], s_wk[NT / 32];
    __shared__ int s_run_active, s_run_keys, s_req;
    const int words = (n + 31) >> 5;
    float* sv = sh_smem;                                               // [n][NT]
    uint32_t* sm = reinterpret_cast<uint32_t*>(sv + n * NT);           // [words][NT]
    float* stop = reinterpret_cast<float*>(sm + words * NT);           // [rmax][NT]
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t li = blockIdx.x;
    if (li >= n_leaves) return;
    const uint32_t leaf = leaves[li];
    const uint32_t lcx = (X + 7u) / 8u, lcy = (Y + 7u) / 8u, lcz = (Z + 7u) / 8u;
    if ((unsigned long long)leaf >= (unsigned long long)lcx * lcy * lcz) {
        if (tid == 0) o.key_count[li] = 0xFFFFFFFFu;
        return;
    }
    const uint32_t bx = leaf % lcx, by = (leaf / lcx) % lcy, bz = leaf / (lcx * lcy);
    const int w = (int)min(8u, X - 8u * bx), h = (int)min(8u, Y - 8u * by), d = (int)min(8u, Z - 8u * bz);
    const float* cg = cgrid + (unsigned long long)li * 64u * (unsigned)n;
    if (tid == 0) {
        s_run_active = 0;
        s_run_keys = 0;
        s_req = 1;
    }
    if (tid < 16) s_mask[tid] = 0u;
    __syncthreads();
    const Column<NT> col{sv + tid, sm + tid};
    for (int round = 0; round < 512 / NT; ++round) {
        const int v = round * NT + tid;
        const int lx = v & 7, ly = (v >> 3) & 7, lz = v >> 6;
        const bool inside = lx < w && ly < h && lz < d;
        const unsigned long long vo =
            (unsigned long long)((8u * bz + (uint32_t)lz) * Y + 8u * by + (uint32_t)ly) * X + 8u * bx + (uint32_t)lx;
        Grid4Sample gs{};
        gs.init((float)lx, (float)ly, (float)lz, w, h, d);
        bool shell = false;
        if (inside) {
            for (int t = 0; t < n && !shell; ++t) {
                const float truth = __ldg(recon + (unsigned long long)t * fstride + vo);
                if (levelset) {
                    const float c = gs.at(cg, n, t);
                    shell = fabsf(truth) <= surface_band || fabsf(c) <= guard_band || (truth >= 0.0f) != (c >= 0.0f);
                } else {
                    shell = truth >= shell_cut;
                }
            }
        }
        int count = 0, local = 1;
        uint8_t b4[4] = {0, 0, 0, 0};
        if (shell) {
            for (int t = 0; t < n; ++t)
                sv[t * NT + tid] = __fsub_rn(__ldg(recon + (unsigned long long)t * fstride + vo), gs.at(cg, n, t));
            keyframe_series<NT>(col, stop + tid, n, words, p, nullptr, 1ull);
            if (levelset) {   // addIsoSurfaceKeyFrames(value, 0, temporal_band), sorted and unique
                const float band = fmax_r(0.0f, temporal_band);
                float prev = 0.0f;
                for (int t = 0; t < n; ++t) {
                    const float cur = __ldg(recon + (unsigned long long)t * fstride + vo);
                    if (fabsf(cur) <= band) {
                        if (t > 0) col.set(t - 1);
                        col.set(t);
                        if (t + 1 < n) col.set(t + 1);
                    }
                    if (t > 0 && (prev >= 0.0f) != (cur >= 0.0f)) {
                        if (t > 1) col.set(t - 2);
                        col.set(t - 1);
                        col.set(t);
                        if (t + 1 < n) col.set(t + 1);
                    }
                    prev = cur;
                }
            }
            for (int wd = 0; wd < words; ++wd) count += __popc(col.m[wd * NT]);
            // buildBinIndexFromKeys with 4 bins
            int b = 0, i = 0;
            for (int wd = 0; wd < words && b < 4; ++wd) {
                uint32_t bits = col.m[wd * NT];
                while (bits && b < 4) {
                    const int key = (wd << 5) + __ffs(bits) - 1;
                    bits &= bits - 1u;
                    while (b < 4 && key >= (int)(((long long)b * n) / 4)) b4[b++] = (uint8_t)(i > 0 ? i - 1 : 0);
                    ++i;
                }
            }
            for (; b < 4; ++b) b4[b] = (uint8_t)(count - 1);
            for (int bb = 0; bb < 4; ++bb) {
                const int next = bb + 1 < 4 ? (int)b4[bb + 1] : count;
                local = max(local, max(1, next - (int)b4[bb]));
            }
        }
        // voxel-order ranks of this round's shell voxels and key starts
        const unsigned bal = __ballot_sync(0xFFFFFFFFu, shell);
        int kincl = count;
        for (int off = 1; off < 32; off <<= 1) {
            const int y = __shfl_up_sync(0xFFFFFFFFu, kincl, off);
            if (lane >= off) kincl += y;
        }
        if (lane == 31) {
            s_wc[warp] = __popc(bal);
            s_wk[warp] = kincl;
        }
        if (lane == 0) s_mask[(round * NT + warp * 32) >> 5] = bal;
        __syncthreads();
        int abase = s_run_active, kbase = s_run_keys;
        for (int q = 0; q < warp; ++q) {
            abase += s_wc[q];
            kbase += s_wk[q];
        }
        if (shell) {
            const int a = abase + __popc(bal & ((1u << lane) - 1u));
            const int start = kbase + kincl - count;
            o.desc[(unsigned long long)li * 512u + (unsigned)a] =
                (uint32_t)(uint16_t)start | ((uint32_t)min(count, 255) << 16) | ((uint32_t)min(local, 255) << 24);
            uint8_t* brow = o.bins + ((unsigned long long)li * 512u + (unsigned)a) * 8u;
            for (int bb = 0; bb < 8; ++bb) brow[bb] = bb < 4 ? b4[bb] : 0u;
            // the reconstruction at each key: the first key's value, then per key
            // value(a) + 1 x (value(b) - value(a)) over the interval (a, b] that ends at it
            const unsigned long long kb = (unsigned long long)li * 512u * (unsigned)n + (unsigned)start;
            int i = 0, prev_key = -1;
            for (int wd = 0; wd < words; ++wd) {
                uint32_t bits = col.m[wd * NT];
                while (bits) {
                    const int key = (wd << 5) + __ffs(bits) - 1;
                    bits &= bits - 1u;
                    float val = col.at(key);
                    if (prev_key >= 0) {
                        const float va = col.at(prev_key);
                        val = __double2float_rn(__dadd_rn((double)va, (double)__fsub_rn(val, va)));
                    }
                    o.key_frame[kb + i] = (uint16_t)key;
                    o.key_value[kb + i] = val;
                    prev_key = key;
                    ++i;
                }
            }
            atomicMax(&s_req, local);
        }
        __syncthreads();
        if (tid == 0) {
            for (int q = 0; q < NT / 32; ++q) {
                s_run_active += s_wc[q];
                s_run_keys += s_wk[q];
            }
        }
        __syncthreads();
    }
    // occupancy: 8 x u64 masks, then 8 x u16 prefixes (shell voxels before the group)
    if (tid < 8) {
        uint32_t pre = 0;
        for (int g = 0; g < tid; ++g) pre += __popc(s_mask[2 * g]) + __popc(s_mask[2 * g + 1]);
        uint8_t* occ = o.occupancy + (unsigned long long)li * 80u;
        const uint32_t lo = s_mask[2 * tid], hi = s_mask[2 * tid + 1];
        for (int k = 0; k < 4; ++k) {
            occ[8 * tid + k] = (uint8_t)(lo >> (8 * k));
            occ[8 * tid + 4 + k] = (uint8_t)(hi >> (8 * k));
        }
        occ[64 + 2 * tid] = (uint8_t)pre;
        occ[64 + 2 * tid + 1] = (uint8_t)(pre >> 8);
    }
    if (tid == 0) {
        o.key_count[li] = (uint32_t)s_run_keys;
        o.active[li] = (uint32_t)s_run_active;
        o.required[li] = (uint8_t)min(s_req, 255);
    }
}

// ---- the density route (:1105-1245, routeRenderTemporalLeaf :27-66) --------------------------
// Per listed leaf, the encoder's sampling lattice (every 8th frame, the leaf's voxel (0, 0, 0) --
// control 0 of either fitted grid): the raw value against the coarse prediction and against coarse
// + FINE6, in double as the encoder accumulates them; FINE6 (mode 3) when the coarse fit is too
// rough, the points are visible and the fine fit gains enough, else GRID4 (mode 1).
__global__ void route_kernel(const float* __restrict__ raw, uint32_t X, uint32_t Y, uint32_t Z, int n,
                             unsigned long long fstride, const uint32_t* __restrict__ leaves, uint32_t n_leaves,
                             const float* __restrict__ cgrid, const float* __restrict__ fgrid, double peak, double lo,
                             double hi, uint8_t* __restrict__ mode)
{
    const uint32_t li = blockIdx.x * blockDim.x + threadIdx.x;
    if (li >= n_leaves) return;
    const uint32_t leaf = leaves[li];
    const uint32_t lcx = (X + 7u) / 8u, lcy = (Y + 7u) / 8u, lcz = (Z + 7u) / 8u;
    if ((unsigned long long)leaf >= (unsigned long long)lcx * lcy * lcz) {
        mode[li] = 0;
        return;
    }
    const uint32_t bx = leaf % lcx, by = (leaf / lcx) % lcy, bz = leaf / (lcx * lcy);
    const unsigned long long vo = (unsigned long long)(8u * bz * Y + 8u * by) * X + 8u * bx;
    const float* cg = cgrid + (unsigned long long)li * 64u * (unsigned)n;
    const float* fg = fgrid + (unsigned long long)li * 216u * (unsigned)n;
    int cnt = 0, vis = 0, bnd = 0;
    double ce2 = 0.0, fe2 = 0.0, cpk = 0.0;
    for (int t = 0; t < n; t += 8) {
        const double truth = (double)__ldg(raw + (unsigned long long)t * fstride + vo);
        const float cp = __ldg(cg + t), fp = __ldg(fg + t);
        ++cnt;
        vis += truth >= lo;
        bnd += lo <= truth && truth <= hi;
        const double cd = __dsub_rn(truth, (double)cp), fd = __dsub_rn(truth, (double)__fadd_rn(cp, fp));
        ce2 = __dadd_rn(ce2, __dmul_rn(cd, cd));
        fe2 = __dadd_rn(fe2, __dmul_rn(fd, fd));
        cpk = dmax_r(cpk, __ddiv_rn(fabs(cd), peak));
    }
    const double c = (double)(cnt > 1 ? cnt : 1);
    const double crm = __ddiv_rn(__dsqrt_rn(__ddiv_rn(ce2, c)), peak);
    const double frm = __ddiv_rn(__dsqrt_rn(__ddiv_rn(fe2, c)), peak);
    const bool rough = crm > (double)0.008f || cpk > (double)0.03f;
    const bool sensitive = __ddiv_rn((double)vis, c) >= (double)0.005f || __ddiv_rn((double)bnd, c) >= (double)0.005f;
    const double gain = __ddiv_rn(__dsub_rn(crm, frm), dmax_r(crm, 1e-12));
    mode[li] = (rough && sensitive && gain >= (double)0.05f) ? 3 : 1;
}

template <int NV>
size_t kf_smem_bytes(int n, int rmax)
{
    return (size_t)NV * 4u * ((size_t)n + (size_t)((n + 31) / 32) + (size_t)rmax);
}

}  // namespace

static_assert(sizeof(KfTotals) == sizeof(vbt_keyframe_totals), "vbt_keyframe_totals layout");

extern "C" int vbt_detect_keyframes(const float* d_values, uint64_t series, uint32_t frames, uint64_t frame_stride,
                                    uint64_t series_stride,
                                    const vbt_keyframe_profile* profile, uint32_t* d_key_mask, uint32_t* d_key_count,
                                    uint8_t* d_flags, float* d_recon, double* d_err2, vbt_keyframe_totals* d_totals,
                                    void* stream)
{
    using vbtb::set_last_error;
    if (!profile) return set_last_error(VBT_STATUS_INVALID_ARGUMENT, "null profile");
    if (frames == 0) return set_last_error(VBT_STATUS_INVALID_ARGUMENT, "frames must be at least 1");
    if (frames > kKfMaxFrames) return set_last_error(VBT_STATUS_LIMIT, "frames above 1024");
    const bool frame_major = series_stride == 1u && frame_stride >= series;
    const bool time_fastest = frame_stride == 1u && series_stride >= frames;
    if (!frame_major && !time_fastest)
        return set_last_error(VBT_STATUS_INVALID_ARGUMENT,
                              "layout must be frame-major (series_stride 1, frame_stride >= series) or time-fastest "
                              "(frame_stride 1, series_stride >= frames)");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (d_totals) {
        const cudaError_t e = cudaMemsetAsync(d_totals, 0, sizeof(vbt_keyframe_totals), s);
        if (e != cudaSuccess) return set_last_error(VBT_STATUS_CUDA, std::string("cudaMemsetAsync: ") + cudaGetErrorString(e));
    }
    if (series == 0) return VBT_STATUS_OK;
    if ((series + 63u) / 32u > 0x7FFFFFFFull) return set_last_error(VBT_STATUS_LIMIT, "series above 2^36");
    if (!d_values || !d_key_mask || !d_key_count || !d_flags)
        return set_last_error(VBT_STATUS_INVALID_ARGUMENT, "null argument");
    const int n = (int)frames;
    const int m = n - 1;
    const int rmax = n >= 2 ? m - (m - 1 < (m * 9) / 10 ? m - 1 : (m * 9) / 10) : 1;
    int dev = 0, smem_max = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    KfTotals* totals = reinterpret_cast<KfTotals*>(d_totals);
    const unsigned long long fs = frame_stride, ss = frame_major ? 1ull : series_stride;
    kf_rcp_init_kernel<<<1, 1024, 0, s>>>();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_last_error(VBT_STATUS_CUDA, std::string("kf_rcp_init_kernel: ") + cudaGetErrorString(e));
    if (kf_smem_bytes<64>(n, rmax) <= (size_t)smem_max) {
        const size_t smem = kf_smem_bytes<64>(n, rmax);
        e = cudaFuncSetAttribute(keyframe_pass_kernel<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e == cudaSuccess) {
            const unsigned long long grid = (series + 63) / 64;
            keyframe_pass_kernel<64><<<(unsigned)grid, 64, smem, s>>>(d_values, series, n, fs, ss, *profile, rmax, d_key_mask,
                                                                      d_key_count, d_flags, d_recon, d_err2, totals);
            e = cudaGetLastError();
        }
    } else {
        const size_t smem = kf_smem_bytes<32>(n, rmax);
        e = cudaFuncSetAttribute(keyframe_pass_kernel<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e == cudaSuccess) {
            const unsigned long long grid = (series + 31) / 32;
            keyframe_pass_kernel<32><<<(unsigned)grid, 32, smem, s>>>(d_values, series, n, fs, ss, *profile, rmax, d_key_mask,
                                                                      d_key_count, d_flags, d_recon, d_err2, totals);
            e = cudaGetLastError();
        }
    }
    return e == cudaSuccess ? VBT_STATUS_OK
                            : set_last_error(VBT_STATUS_CUDA, std::string("keyframe_pass_kernel: ") + cudaGetErrorString(e));
}

extern "C" int vbt_selftest_keyframe_division(uint32_t b_max, uint64_t* result, int device)
{
    using vbtb::set_last_error;
    if (!result) return set_last_error(VBT_STATUS_INVALID_ARGUMENT, "null argument");
    if (b_max < 1u || b_max > 65535u) return set_last_error(VBT_STATUS_INVALID_ARGUMENT, "b_max must lie in [1, 65535]");
    int dev_count = 0;
    if (cudaGetDeviceCount(&dev_count) != cudaSuccess || dev_count == 0)
        return set_last_error(VBT_STATUS_CUDA, "no CUDA device");
    if (device < 0 || device >= dev_count) return set_last_error(VBT_STATUS_INVALID_ARGUMENT, "device out of range");
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(device);
    unsigned long long* d = nullptr;
    cudaError_t e = cudaMalloc(&d, 2 * sizeof(unsigned long long));
    unsigned long long h[2] = {0ull, ~0ull};
    if (e == cudaSuccess) e = cudaMemcpy(d, h, sizeof(h), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        int sms = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        keyframe_division_check_kernel<<<8 * (sms > 0 ? sms : 1), 256>>>(b_max, d, d + 1);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(h, d, sizeof(h), cudaMemcpyDeviceToHost);
    if (d) cudaFree(d);
    cudaSetDevice(prev);
    if (e != cudaSuccess) return set_last_error(VBT_STATUS_CUDA, std::string("keyframe division check: ") + cudaGetErrorString(e));
    result[0] = h[0];
    result[1] = h[1];
    return VBT_STATUS_OK;
}

extern "C" int vbt_coarse_fit(const float* d_recon, uint32_t width, uint32_t height, uint32_t depth, uint32_t frames,
                              uint64_t frame_stride, const uint32_t* d_leaves, uint32_t leaf_count,
                              const vbt_keyframe_profile* control_profile, uint32_t* d_desc, uint8_t* d_bins,
                              uint16_t* d_key_frames, float* d_key_values, uint32_t* d_key_count,
                              uint8_t* d_required_max_local, float* d_grid, void* stream)
{
    using vbtb::set_last_error;
    if (!control_profile) return set_last_error(VBT_STATUS_INVALID_ARGUMENT, "null profile");
    if (frames == 0 || width == 0 || height == 0 || depth == 0)
        return set_last_error(VBT_STATUS_INVALID_ARGUMENT, "empty volume");
    if (frames > kKfMaxFrames) return set_last_error(VBT_STATUS_LIMIT, "frames above 1024");
    const unsigned long long voxels = (unsigned long long)width * height * depth;
    if (frame_stride < voxels) return set_last_error(VBT_STATUS_INVALID_ARGUMENT, "frame_stride smaller than the volume");
    if (leaf_count == 0) return VBT_STATUS_OK;
    if (!d_recon || !d_leaves || !d_desc || !d_bins || !d_key_frames || !d_key_values || !d_key_count ||
        !d_required_max_local)
        return set_last_error(VBT_STATUS_INVALID_ARGUMENT, "null argument");
    const int n = (int)frames;
    const int m = n - 1;
    const int rmax = n >= 2 ? m - (m - 1 < (m * 9) / 10 ? m - 1 : (m * 9) / 10) : 1;
    int dev = 0, smem_max = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    const size_t smem = kf_smem_bytes<64>(n, rmax);
    const size_t static_smem = (64 + 64 + 512) * sizeof(int);
    if (smem + static_smem > (size_t)smem_max) return set_last_error(VBT_STATUS_LIMIT, "too many frames for one leaf's CTA");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    kf_rcp_init_kernel<<<1, 1024, 0, s>>>();
    cudaError_t e = cudaFuncSetAttribute(control_fit_kernel<4, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e == cudaSuccess) {
        vbt_keyframe_profile prof = *control_profile;
        prof.bg_threshold = -1.0;          // the control fitting has no background test
        const CoarseOut o{d_desc, d_bins, d_key_frames, d_key_values, d_key_count, d_required_max_local, d_grid};
        control_fit_kernel<4, false><<<leaf_count, 64, smem, s>>>(d_recon, width, height, depth, n, frame_stride,
                                                                  d_leaves, leaf_count, prof, rmax, nullptr, o);
        e = cudaGetLastError();
    }
    return e == cudaSuccess ? VBT_STATUS_OK
                            : set_last_error(VBT_STATUS_CUDA, std::string("control_fit_kernel<4>: ") + cudaGetErrorString(e));
}

extern "C" int vbt_fine6_fit(const float* d_recon, uint32_t width, uint32_t height, uint32_t depth, uint32_t frames,
                             uint64_t frame_stride, const uint32_t* d_leaves, uint32_t leaf_count,
                             const vbt_keyframe_profile* control_profile, const float* d_coarse_grid, uint32_t* d_desc,
                             uint8_t* d_bins, uint16_t* d_key_frames, float* d_key_values, uint32_t* d_key_count,
                             uint8_t* d_required_max_local, float* d_grid, void* stream)
{
    using vbtb::set_last_error;
    if (!control_profile) return set_last_error(VBT_STATUS_INVALID_ARGUMENT, "null profile");
    if (frames == 0 || width == 0 || height == 0 || depth == 0)
        return set_last_error(VBT_STATUS_INVALID_ARGUMENT, "empty volume");
    if (frames > kKfMaxFrames) return set_last_error(VBT_STATUS_LIMIT, "frames above 1024");
    const unsigned long long voxels = (unsigned long long)width * height * depth;
    if (frame_stride < voxels) return set_last_error(VBT_STATUS_INVALID_ARGUMENT, "frame_stride smaller than the volume");
    if (leaf_count == 0) return VBT_STATUS_OK;
    if (!d_recon || !d_leaves || !d_coarse_grid || !d_desc || !d_bins || !d_key_frames || !d_key_values ||
        !d_key_count || !d_required_max_local)
        return set_last_error(VBT_STATUS_INVALID_ARGUMENT, "null argument");
    const int n = (int)frames;
    const int m = n - 1;
    const int rmax = n >= 2 ? m - (m - 1 < (m * 9) / 10 ? m - 1 : (m * 9) / 10) : 1;
    int dev = 0, smem_max = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    const size_t smem = kf_smem_bytes<216>(n, rmax);
    const size_t static_smem = (216 + 216 + 216 * 8) * sizeof(int);
    if (smem + static_smem > (size_t)smem_max) return set_last_error(VBT_STATUS_LIMIT, "too many frames for one leaf's CTA");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    kf_rcp_init_kernel<<<1, 1024, 0, s>>>();
    cudaError_t e = cudaFuncSetAttribute(control_fit_kernel<6, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e == cudaSuccess) {
        vbt_keyframe_profile prof = *control_profile;
        prof.bg_threshold = -1.0;
        const CoarseOut o{d_desc, d_bins, d_key_frames, d_key_values, d_key_count, d_required_max_local, d_grid};
        control_fit_kernel<6, true><<<leaf_count, 216, smem, s>>>(d_recon, width, height, depth, n, frame_stride,
                                                                  d_leaves, leaf_count, prof, rmax, d_coarse_grid, o);
        e = cudaGetLastError();
    }
    return e == cudaSuccess ? VBT_STATUS_OK
                            : set_last_error(VBT_STATUS_CUDA, std::string("control_fit_kernel<6>: ") + cudaGetErrorString(e));
}

extern "C" int vbt_shell_fit(const float* d_recon, uint32_t width, uint32_t height, uint32_t depth, uint32_t frames,
                             uint64_t frame_stride, const uint32_t* d_leaves, uint32_t leaf_count,
                             const vbt_keyframe_profile* control_profile, const float* d_coarse_grid, int levelset,
                             float surface_band, float guard_band, float temporal_band, float shell_cut,
                             uint8_t* d_occupancy, uint32_t* d_desc, uint8_t* d_bins, uint16_t* d_key_frames,
                             float* d_key_values, uint32_t* d_key_count, uint32_t* d_active,
                             uint8_t* d_required_max_local, void* stream)
{
    using vbtb::set_last_error;
    if (!control_profile) return set_last_error(VBT_STATUS_INVALID_ARGUMENT, "null profile");
    if (frames == 0 || width == 0 || height == 0 || depth == 0)
        return set_last_error(VBT_STATUS_INVALID_ARGUMENT, "empty volume");
    if (frames > kKfMaxFrames) return set_last_error(VBT_STATUS_LIMIT, "frames above 1024");
    const unsigned long long voxels = (unsigned long long)width * height * depth;
    if (frame_stride < voxels) return set_last_error(VBT_STATUS_INVALID_ARGUMENT, "frame_stride smaller than the volume");
    if (leaf_count == 0) return VBT_STATUS_OK;
    if (!d_recon || !d_leaves || !d_coarse_grid || !d_occupancy || !d_desc || !d_bins || !d_key_frames ||
        !d_key_values || !d_key_count || !d_active || !d_required_max_local)
        return set_last_error(VBT_STATUS_INVALID_ARGUMENT, "null argument");
    const int n = (int)frames;
    const int m = n - 1;
    const int rmax = n >= 2 ? m - (m - 1 < (m * 9) / 10 ? m - 1 : (m * 9) / 10) : 1;
    int dev = 0, smem_max = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    const size_t smem = kf_smem_bytes<kShellThreads>(n, rmax);
    if (smem + 1024 > (size_t)smem_max) return set_last_error(VBT_STATUS_LIMIT, "too many frames for one leaf's CTA");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    kf_rcp_init_kernel<<<1, 1024, 0, s>>>();
    cudaError_t e = cudaFuncSetAttribute(shell_fit_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) {
        vbt_keyframe_profile prof = *control_profile;
        prof.bg_threshold = -1.0;
        const ShellOut o{d_occupancy, d_desc, d_bins, d_key_frames, d_key_values, d_key_count, d_active,
                         d_required_max_local};
        shell_fit_kernel<<<leaf_count, kShellThreads, smem, s>>>(d_recon, width, height, depth, n, frame_stride,
                                                                  d_leaves, leaf_count, prof, rmax, d_coarse_grid,
                                                                  levelset, surface_band, guard_band, temporal_band,
                                                                  shell_cut, o);
        e = cudaGetLastError();
    }
    return e == cudaSuccess ? VBT_STATUS_OK
                            : set_last_error(VBT_STATUS_CUDA, std::string("shell_fit_kernel: ") + cudaGetErrorString(e));
}

extern "C" int vbt_route_density(const float* d_raw, uint32_t width, uint32_t height, uint32_t depth, uint32_t frames,
                                 uint64_t frame_stride, const uint32_t* d_leaves, uint32_t leaf_count,
                                 const float* d_coarse_grid, const float* d_fine_grid, double peak, double visible_lo,
                                 double visible_hi, uint8_t* d_mode, void* stream)
{
    using vbtb::set_last_error;
    if (frames == 0 || width == 0 || height == 0 || depth == 0)
        return set_last_error(VBT_STATUS_INVALID_ARGUMENT, "empty volume");
    if (leaf_count == 0) return VBT_STATUS_OK;
    if (!d_raw || !d_leaves || !d_coarse_grid || !d_fine_grid || !d_mode)
        return set_last_error(VBT_STATUS_INVALID_ARGUMENT, "null argument");
    if (!(peak > 0.0)) return set_last_error(VBT_STATUS_INVALID_ARGUMENT, "peak must be positive");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    route_kernel<<<(leaf_count + 127) / 128, 128, 0, s>>>(d_raw, width, height, depth, (int)frames, frame_stride,
                                                          d_leaves, leaf_count, d_coarse_grid, d_fine_grid, peak,
                                                          visible_lo, visible_hi, d_mode);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? VBT_STATUS_OK
                            : set_last_error(VBT_STATUS_CUDA, std::string("route_kernel: ") + cudaGetErrorString(e));
}
