// rt_kernel_leaf.cuh -- the render-temporal decode kernel: one CTA per leaf, all frames of the
// launch, leaf bytes staged in shared memory by a TMA bulk copy.  Included by kernels.cu (it uses
// that file's axis table g_axis and helpers).
//
// Per leaf, frames are processed in batches that fit the control buffer.  For each batch:
//  1. controls: every (control, frame range) unit decodes its values into ctrl[frame][control].
//     A leaf with few controls splits each control's frames over several threads, so all 256
//     threads work.  Timeline batches (frame steps of 0 or 1) on leaves with strictly increasing
//     key frames use the streaming cursor; anything else uses the reference's bracket search.
//  2. voxels: each warp reconstructs whole frames with the separable trilinear and stores them.
#pragma once

namespace vbtb {

constexpr int kLeafThreads = 256;   // the render window kernel (render_window.cuh)
constexpr int kLeafWarps = kLeafThreads / 32;
constexpr int kDecWarps = 9;         // the decode kernel: 288 threads, one per FINE6 control
constexpr int kDecThreads = 32 * kDecWarps;
constexpr int kLeafCtrlBudget = 3072;   // floats: frames x controls of one batch
constexpr uint32_t leaf_fixed_bytes(int nw)
{
    return 16 + 6 * kMaxLaunchFrames + 576 + nw * 196 * 8 + nw * 112 * 16 + kLeafCtrlBudget * 4 + 256 * 4 + 768;
}
constexpr uint32_t kLeafFixed = leaf_fixed_bytes(kLeafWarps);
constexpr uint32_t kDecFixed = leaf_fixed_bytes(kDecWarps);
constexpr uint32_t kStagePad = 16;   // readable bytes past the largest staged window
static_assert(kDecFixed == kLeafFixedBytes, "host stage sizing must match the kernel's shared-memory layout");

struct LeafSmem {
    uint64_t* bar;
    int* fr;
    uint8_t *b8, *b4;
    AxisWeight (*w)[3][8];
    float2* x2;      // [warp][196]
    float4* y4;      // [warp][112]
    float* ctrl;     // [kLeafCtrlBudget]
    float* rcp;      // [256] RN(1/i)
    float4* w16;     // [grid][axis][8] {t, 1 - t, i0, i1}: the axis weights as 16-byte rows
    uint8_t* stage;  // leaf window (16-byte aligned), kStagePad bytes of padding after it
};

// Shared-memory layout for NW warps (x-lerp and y-lerp rows per warp).
template <int NW = kLeafWarps>
__device__ __forceinline__ LeafSmem leaf_layout(uint8_t* dyn)
{
    LeafSmem s;
    s.bar = reinterpret_cast<uint64_t*>(dyn);
    s.fr = reinterpret_cast<int*>(dyn + 16);
    s.b8 = dyn + 16 + 4 * kMaxLaunchFrames;
    s.b4 = s.b8 + kMaxLaunchFrames;
    s.w = reinterpret_cast<AxisWeight(*)[3][8]>(dyn + 16 + 6 * kMaxLaunchFrames);
    s.x2 = reinterpret_cast<float2*>(dyn + 16 + 6 * kMaxLaunchFrames + 576);
    s.y4 = reinterpret_cast<float4*>(reinterpret_cast<uint8_t*>(s.x2) + NW * 196 * 8);
    s.ctrl = reinterpret_cast<float*>(reinterpret_cast<uint8_t*>(s.y4) + NW * 112 * 16);
    s.rcp = s.ctrl + kLeafCtrlBudget;
    s.w16 = reinterpret_cast<float4*>(s.rcp + 256);
    s.stage = reinterpret_cast<uint8_t*>(s.w16 + 48);
    return s;
}

struct LeafGeom {
    uint32_t li, bx, by, bz;
    int w, h, d;
};

}  // namespace vbtb
#include "rt_leaf_fast.cuh"
namespace vbtb {

template <bool DENSE>
__device__ __forceinline__ void store_quad(const DeviceAsset& a, const LeafGeom& G, float* __restrict__ out,
                                           uint64_t frame_stride, int fi, int lane, int i, float4 v)
{
    const int lz = 2 * i + (lane >> 4), ly = (lane >> 1) & 7, lx0 = 4 * (lane & 1);
    if (DENSE) {
        if (ly < G.h && lz < G.d) {
            float* dst = out + (uint64_t)fi * frame_stride +
                         ((uint64_t)(G.bz * 8 + lz) * a.g.height + (G.by * 8 + ly)) * a.g.width + G.bx * 8 + lx0;
            if (lx0 + 4 <= G.w && (((uintptr_t)dst) & 15u) == 0u) {
                *reinterpret_cast<float4*>(dst) = v;
            } else {
                const float vv[4] = {v.x, v.y, v.z, v.w};
                for (int k = 0; k < 4 && lx0 + k < G.w; ++k) dst[k] = vv[k];
            }
        }
    } else {
        reinterpret_cast<float4*>(out + (uint64_t)fi * frame_stride + (uint64_t)G.li * 512u)[lane + 32 * i] = v;
    }
}

// Where leaf_decode puts a finished voxel quad: the current-frame cache or dense frames.
template <bool DENSE>
struct FrameSink {
    const DeviceAsset& a;
    const LeafGeom& G;
    float* __restrict__ out;
    uint64_t frame_stride;
    __device__ __forceinline__ void operator()(int fi, int lane, int i, float4 v) const
    {
        store_quad<DENSE>(a, G, out, frame_stride, fi, lane, i, v);
    }
};

// The same stores from values held by the sink itself (no references to the launch's asset or the
// leaf's geometry), for the specialised path.
template <bool DENSE>
struct QuadSink {
    float* __restrict__ out;
    uint64_t frame_stride;
    uint32_t li, width, height, bx, by, bz;
    int w, h, d;
    __device__ __forceinline__ void operator()(int fi, int lane, int i, float4 v) const
    {
        const int lz = 2 * i + (lane >> 4), ly = (lane >> 1) & 7, lx0 = 4 * (lane & 1);
        if (DENSE) {
            if (ly < h && lz < d) {
                float* dst = out + (uint64_t)fi * frame_stride +
                             ((uint64_t)(bz * 8 + lz) * height + (by * 8 + ly)) * width + bx * 8 + lx0;
                if (lx0 + 4 <= w && (((uintptr_t)dst) & 15u) == 0u) {
                    *reinterpret_cast<float4*>(dst) = v;
                } else {
                    const float vv[4] = {v.x, v.y, v.z, v.w};
                    for (int k = 0; k < 4 && lx0 + k < w; ++k) dst[k] = vv[k];
                }
            }
        } else {
            reinterpret_cast<float4*>(out + (uint64_t)fi * frame_stride + (uint64_t)li * 512u)[lane + 32 * i] = v;
        }
    }
};

// Decode one validated, non-EMPTY leaf for all frames of the launch with word reader `m` and NW
// warps; each finished quad of 4 voxels goes to `sink(frame index, lane, quad, values)`.  Frame
// lists that step by 0 or 1 stream each control's keys; other non-decreasing lists (`monotone`)
// walk a cursor; anything else, or keys that do not strictly increase, uses the reference's search.
template <class M, class Sink, int NW = kLeafWarps>
__device__ __forceinline__ void leaf_decode(const DeviceAsset& a, const M& m, const LeafSmem& s, const LeafEntry& e,
                                            int nframes, bool steps01, bool monotone, const LeafGeom& G,
                                            const Sink& sink)
{
    constexpr int NT = 32 * NW;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint64_t base = 4ull * e.word_off;
    const int cres = (int)((e.header >> 6) & 7u), fres = (int)((e.header >> 9) & 7u);
    const bool fine = (e.info & kFlagFine) != 0u, shell = (e.info & kFlagShell) != 0u;
    const bool occ = (e.info & kFlagOccClamp) != 0u;
    const StreamRef cs{base + 8u, (uint32_t)(cres * cres * cres), 8u, e.kf & 0xFFFFu, (e.header >> 2) & 3u};
    const StreamRef fs{base + 8u + e.coarse_bytes, (uint32_t)(fres * fres * fres), 8u, e.kf >> 16,
                       (e.header >> 4) & 3u};
    const StreamRef ss{base + e.shell_off, entry_shell_active(e), 4u, e.kf >> 16, (e.header >> 4) & 3u};
    const int Cc = (int)cs.controls;
    const int Cf = fine ? (int)fs.controls : (shell ? (int)ss.controls : 0);
    const int Ctot = Cc + Cf;
    // frames per batch: as many as the control buffer holds, rounded down to a multiple of the
    // warp count when that still leaves a full round (each warp reconstructs whole frames)
    int nb_max = min(nframes, kLeafCtrlBudget / max(Ctot, 1));
    if (nb_max < nframes && nb_max > NW) nb_max -= nb_max % NW;
    const bool stream = steps01 && (e.info & kFlagSorted) != 0u;
    const bool cursor = !stream && monotone && (e.info & kFlagSorted) != 0u;
    const bool plain = !occ && G.w == 8 && G.h == 8 && G.d == 8;
    const int ly = (lane >> 1) & 7, lx0 = 4 * (lane & 1);
    uint64_t mask[4] = {0, 0, 0, 0};
    uint32_t pref[4] = {0, 0, 0, 0};
    if (occ) {
        const uint64_t ob = base + 8u + e.coarse_bytes;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const uint32_t g = (uint32_t)(2 * i + (lane >> 4));
            mask[i] = ((uint64_t)m((uint32_t)((ob + 8u * g + 4u) >> 2)) << 32) | m((uint32_t)((ob + 8u * g) >> 2));
            pref[i] = (m((uint32_t)((ob + 64u + 2u * g) >> 2)) >> ((g & 1u) * 16u)) & 0xFFFFu;
        }
    }
    float2* x2 = s.x2 + warp * 196;
    float4* y4 = s.y4 + warp * 112;
    for (int fb0 = 0; fb0 < nframes; fb0 += nb_max) {
        const int nb = min(nb_max, nframes - fb0);
        // 1. controls, as (control, frame range) units.  With at most one control per thread, each
        //    control's frames are split over tpc threads so that all threads work; with more, each
        //    thread owns one whole control and the remaining controls are cut into short frame
        //    ranges spread over all threads (each thread starts at most one extra range).
        auto run_unit = [&](int c, int j0, int j1) {
            const StreamRef st = c < Cc ? cs : (fine ? fs : ss);
            const uint32_t ci = (uint32_t)(c < Cc ? c : c - Cc);
            float* dst = s.ctrl + j0 * Ctot + c;
            if (stream) {
                const uint32_t bin0 = st.bins == 8u ? s.b8[fb0 + j0] : s.b4[fb0 + j0];
                m_control_stream(m, st, ci, s.fr + fb0 + j0, bin0, j1 - j0, dst, Ctot, s.rcp);
            } else {
                const FrameBatch fb{s.fr + fb0 + j0, s.b8 + fb0 + j0, s.b4 + fb0 + j0, j1 - j0};
                if (cursor) m_control_cursor(m, st, ci, fb, dst, Ctot);
                else m_control_search(m, st, ci, fb, dst, Ctot);
            }
        };
        const int c0 = Ctot > NT ? NT : 0;   // controls [0, c0) are owned whole
        if (c0) run_unit(tid, 0, nb);
        const int rest = Ctot - c0;
        const int tpc = min(8, max(1, NT / rest));
        const int part_len = (nb + tpc - 1) / tpc;
        for (int unit = tid; unit < rest * tpc; unit += NT) {
            const int c = c0 + unit / tpc, q = unit % tpc;
            const int j0 = q * part_len, j1 = min(nb, j0 + part_len);
            if (j0 < j1) run_unit(c, j0, j1);
        }
        __syncthreads();
        // 2. voxels
        for (int j = warp; j < nb; j += NW) {
            const float* g = s.ctrl + j * Ctot;
            float4 q[4];
            if (cres >= 2) trilinear_quads_ptr(s.w[0], x2, y4, g, cres, lane, q);
            else constant_quads(g, cres, q);
            if (fine) {
                float4 qf[4];
                if (fres >= 2) trilinear_quads_ptr(s.w[1], x2, y4, g + Cc, fres, lane, qf);
                else constant_quads(g + Cc, fres, qf);
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const float2 lo2 = add2_rn(make_float2(q[i].x, q[i].y), make_float2(qf[i].x, qf[i].y));
                    const float2 hi2 = add2_rn(make_float2(q[i].z, q[i].w), make_float2(qf[i].z, qf[i].w));
                    q[i] = make_float4(lo2.x, lo2.y, hi2.x, hi2.y);
                }
            }
            const int fi = fb0 + j;
            if (plain) {
#pragma unroll
                for (int i = 0; i < 4; ++i) sink(fi, lane, i, q[i]);
                continue;
            }
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int lz = 2 * i + (lane >> 4);
                float v[4] = {q[i].x, q[i].y, q[i].z, q[i].w};
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const uint32_t bit = (uint32_t)(ly * 8 + lx0 + k);
                    const bool in_occ = occ && ((mask[i] >> bit) & 1ull);
                    if (shell && in_occ) {
                        const uint32_t di = (pref[i] + __popcll(mask[i] & ((1ull << bit) - 1ull))) & 0xFFFFu;
                        v[k] = __fadd_rn(v[k], g[Cc + di]);
                    }
                    if (occ && !in_occ && v[k] < 0.0f) v[k] = 0.0f;
                    if (lx0 + k >= G.w || ly >= G.h || lz >= G.d) v[k] = 0.0f;
                }
                sink(fi, lane, i, make_float4(v[0], v[1], v[2], v[3]));
            }
        }
        __syncthreads();
    }
}

// Next leaf index of this launch from its work counter ([epoch:32 | next index:32]).  The slot
// still carries an older launch's epoch until the first CTA of this launch installs its own
// (taking index 0); from then on a grab is one atomicAdd.  Every failed compare-and-swap means
// another CTA changed the slot, so the loop ends; the bound only guards against a corrupt slot.
__device__ __forceinline__ uint32_t grab_leaf(unsigned long long* slot, uint32_t epoch, bool& timed_out)
{
    unsigned long long v = atomicAdd(slot, 1ull);
    if ((uint32_t)(v >> 32) == epoch) return (uint32_t)v;
    unsigned long long expect = v + 1ull;
    const unsigned long long mine = ((unsigned long long)epoch << 32) | 1ull;
    for (int it = 0; it < (1 << 20); ++it) {
        const unsigned long long seen = atomicCAS(slot, expect, mine);
        if (seen == expect) return 0u;
        if ((uint32_t)(seen >> 32) == epoch) {
            v = atomicAdd(slot, 1ull);
            return (uint32_t)v;
        }
        expect = seen;
    }
    timed_out = true;
    return 0xFFFFFFFFu;
}

// Dense frames, EMPTY leaves: zero their segments of the eight lines of y-band `by` in z-plane zz,
// in every frame of the launch, the whole CTA.  The band's inactive leaves are a 64-bit mask per 64
// leaves along x (a ballot over the page table, the same for every line and frame); the warps take
// (line, frame) pairs and the lanes store consecutive 16-byte chunks (a chunk never straddles two
// leaves).  Inactive leaves with a walker status record it once (the leaf's first plane).  vec:
// rows 16-byte aligned (X % 4 == 0, 16-byte aligned output and frame stride); otherwise one float
// per store.
template <int NW>
__device__ __forceinline__ void zero_band(const DeviceAsset& a, float* __restrict__ out, uint64_t frame_stride,
                                          int nframes, uint32_t zz, uint32_t by, bool vec)
{
    const uint32_t X = a.g.width, Y = a.g.height;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t lrow = ((zz >> 3) * a.g.lcy + by) * a.g.lcx;
    const uint32_t lines = min(8u, Y - 8u * by);
    for (uint32_t b0 = 0; b0 < a.g.lcx; b0 += 64u) {
        const uint32_t bx0 = b0 + (uint32_t)lane, bx1 = bx0 + 32u;
        const bool e0 = bx0 < a.g.lcx && __ldg(a.compact + lrow + bx0) == kNoRank;
        const bool e1 = bx1 < a.g.lcx && __ldg(a.compact + lrow + bx1) == kNoRank;
        if (warp == 0 && (zz & 7u) == 0u) {
            if (e0) {
                const uint32_t st = entry_status(a.entries[lrow + bx0]);
                if (st != kOk) record_error(a.err, lrow + bx0, st);
            }
            if (e1) {
                const uint32_t st = entry_status(a.entries[lrow + bx1]);
                if (st != kOk) record_error(a.err, lrow + bx1, st);
            }
        }
        const uint64_t mask = (uint64_t)__ballot_sync(0xFFFFFFFFu, e0) | ((uint64_t)__ballot_sync(0xFFFFFFFFu, e1) << 32);
        if (mask == 0ull) continue;
        const uint32_t x_end = min(X, 8u * (b0 + 64u));
        for (uint32_t pr = (uint32_t)warp; pr < lines * (uint32_t)nframes; pr += NW) {
            const uint32_t fi = pr / lines, y = 8u * by + (pr - fi * lines);
            float* row = out + (uint64_t)fi * frame_stride + ((uint64_t)zz * Y + y) * X;
            if (vec) {
                for (uint32_t x = 8u * b0 + 4u * (uint32_t)lane; x < x_end; x += 128u)
                    if ((mask >> ((x >> 3) - b0)) & 1ull) *reinterpret_cast<float4*>(row + x) = make_float4(0.f, 0.f, 0.f, 0.f);
            } else {
                for (uint32_t x = 8u * b0 + (uint32_t)lane; x < x_end; x += 32u)
                    if ((mask >> ((x >> 3) - b0)) & 1ull) row[x] = 0.0f;
            }
        }
    }
}

// GLOBAL_FALLBACK: leaves whose window exceeds the stage are decoded from global memory (only
// instantiated for assets that have such leaves; it costs registers).
// Leaves are handed out dynamically (grab_leaf), one at a time per CTA, so that CTAs that drew
// cheap leaves (few controls, few keys) take more of them.
// The general decode as a call of its own, so that its registers do not crowd the fast path's
// (the kernel's shared-memory layout is recomputed from the dynamic shared-memory base).
template <class M, bool DENSE>
__device__ __noinline__ void leaf_decode_general(const DeviceAsset& a, M m, LeafEntry e, int nframes, bool steps01,
                                                 bool monotone, LeafGeom G, float* __restrict__ out,
                                                 uint64_t frame_stride)
{
    extern __shared__ __align__(128) uint8_t dyn[];
    const LeafSmem s = leaf_layout<kDecWarps>(dyn);
    leaf_decode<M, FrameSink<DENSE>, kDecWarps>(a, m, s, e, nframes, steps01, monotone, G,
                                                FrameSink<DENSE>{a, G, out, frame_stride});
}

// The specialised decode (rt_leaf_fast.cuh) as a call of its own too: each path gets the whole
// register budget of the 288-thread launch.  The leaf's bytes are read from the shared-memory
// stage, or (GLOBAL_KEYS: a leaf larger than the stage) straight from the payload through L1 --
// the same byte offsets from the 16-byte-aligned window start a0; the payload's 16-byte tail
// padding keeps the second word of the last key read inside the allocation.
template <bool FINE, bool DENSE, bool GLOBAL_KEYS>
__device__ __noinline__ void leaf_decode_fast_call(const DeviceAsset& a, LeafEntry e, uint32_t lb, uint64_t a0,
                                                   int nframes, LeafGeom G, float* __restrict__ out,
                                                   uint64_t frame_stride)
{
    extern __shared__ __align__(128) uint8_t dyn[];
    const LeafSmem s = leaf_layout<kDecWarps>(dyn);
    const QuadSink<DENSE> sink{out, frame_stride, G.li, a.g.width, a.g.height, G.bx, G.by, G.bz, G.w, G.h, G.d};
    const uint8_t* st = GLOBAL_KEYS ? reinterpret_cast<const uint8_t*>(a.payload) + a0 : s.stage;
    leaf_decode_fast<FINE, kDecWarps>(st, lb, s, e, nframes, G, sink);
}

// GRID4 / FINE6 leaves of the common shape take leaf_decode_fast (rt_leaf_fast.cuh), staged or
// (GLOBAL_FALLBACK) from global memory; every other leaf the general leaf_decode.
template <bool DENSE, bool GLOBAL_FALLBACK>
__global__ void __launch_bounds__(kDecThreads, 2) decode_leaf_kernel(const __grid_constant__ DeviceAsset a,
                                                                     FrameList fl, float* __restrict__ out,
                                                                     uint64_t frame_stride, unsigned long long* work,
                                                                     uint32_t epoch)
{
    extern __shared__ __align__(128) uint8_t dyn[];
    const LeafSmem s = leaf_layout<kDecWarps>(dyn);
    uint32_t* const s_next = reinterpret_cast<uint32_t*>(dyn + 8);   // beside the 8-byte barrier
    const int tid = threadIdx.x;
    const int total = (int)a.g.frames;
    // work items: the active leaves by rank and, for dense frames of a volume with inactive leaves,
    // one item per (z-plane, y-band of leaves) that zeroes the inactive leaves' segments of that
    // band in every frame.  The two kinds are interleaved in proportion (item i is leaf
    // floor(i A / N) when that value steps at i, else zero band i - floor(i A / N)), so
    // bandwidth-bound zeroing and latency-bound decoding share the GPU throughout the launch.
    const uint32_t n_leaves = *(volatile const uint32_t*)a.counters;
    const uint32_t n_zero = DENSE && n_leaves < a.g.leaf_count ? a.g.depth * a.g.lcy : 0u;
    const uint64_t n_items = (uint64_t)n_leaves + n_zero;
    const bool vec = (a.g.width & 3u) == 0u && (reinterpret_cast<uintptr_t>(out) & 15u) == 0u &&
                     (frame_stride & 3u) == 0u;

    if (tid == 0) {
        mbar_init(s.bar, 1);
        mbar_init_fence();
        bool to = false;
        const uint32_t first = grab_leaf(work, epoch, to);
        if (to) record_error(a.err, 0u, kErrWaitTimeout);
        *s_next = first;
    }
    if (tid < 256) s.rcp[tid] = __frcp_rn((float)tid);
    if (tid < fl.n) {
        const int fr = clamp_frame(fl.f[tid], total);
        s.fr[tid] = fr;
        s.b8[tid] = (uint8_t)time_bin(fr, 8u, total);
        s.b4[tid] = (uint8_t)time_bin(fr, 4u, total);
    }
    __syncthreads();
    const bool steps01 =
        __syncthreads_and(tid == 0 || tid >= fl.n || (unsigned)(s.fr[tid] - s.fr[tid - 1]) <= 1u) != 0;
    const bool monotone = __syncthreads_and(tid == 0 || tid >= fl.n || s.fr[tid] >= s.fr[tid - 1]) != 0;
    const uint8_t* pay_bytes = reinterpret_cast<const uint8_t*>(a.payload);
    uint32_t phase = 0;
    uint32_t li = *s_next;
    while (li < n_items) {
        // every thread has read li, and the previous leaf's shared-memory reads are complete
        __syncthreads();
        uint32_t rank = li;
        if (DENSE && n_zero) {
            const uint32_t d = (uint32_t)((uint64_t)li * n_leaves / n_items);
            const uint32_t d1 = (uint32_t)((uint64_t)(li + 1u) * n_leaves / n_items);
            if (d1 == d) {   // a zero band
                if (tid == 0) {
                    bool to = false;
                    *s_next = grab_leaf(work, epoch, to);
                    if (to) record_error(a.err, 0u, kErrWaitTimeout);
                }
                const uint32_t zi = li - d;
                zero_band<kDecWarps>(a, out, frame_stride, fl.n, zi / a.g.lcy, zi % a.g.lcy, vec);
                __syncthreads();   // the next index is visible
                li = *s_next;
                continue;
            }
            rank = d;
        }
        const uint32_t leaf = __ldg(a.active_list + rank);
        const LeafEntry e = a.entries[leaf];
        LeafGeom G;
        G.li = rank;
        leaf_extent(a.g, leaf, G.bx, G.by, G.bz, G.w, G.h, G.d);
        const uint32_t st = entry_status(e);
        const uint64_t b0 = 4ull * e.word_off;
        const uint64_t b1 = 4ull * (uint64_t)__ldg(a.offsets + leaf + 1);
        const uint64_t a0 = b0 & ~15ull, a1 = (b1 + 15u) & ~15ull;
        const bool skip = st != kOk || (e.header & 3u) == kModeEmpty;
        const bool staged = !skip && a1 - a0 <= a.g.stage_bytes;
        if (tid == 0) {
            if (staged) mbar_expect_and_copy(s.bar, s.stage, pay_bytes + a0, (uint32_t)(a1 - a0));
            bool to = false;
            const uint32_t nx = grab_leaf(work, epoch, to);
            if (to) record_error(a.err, leaf, kErrWaitTimeout);
            *s_next = nx;
        }
        if (skip) {
            if (st != kOk && tid == 0) record_error(a.err, leaf, st);
            for (int idx = tid; idx < fl.n * 128; idx += kDecThreads)
                store_quad<DENSE>(a, G, out, frame_stride, idx >> 7, (idx & 127) & 31, (idx & 127) >> 5,
                                  make_float4(0.f, 0.f, 0.f, 0.f));
        } else if (!GLOBAL_FALLBACK && !staged) {   // the launcher never lets this happen
            if (tid == 0) record_error(a.err, leaf, kErrDecodeOob);
        } else {
            if (tid < 48) {
                const int ws = tid / 24, axis = (tid % 24) >> 3, p = tid & 7;
                const int R = ws == 0 ? (int)((e.header >> 6) & 7u) : (int)((e.header >> 9) & 7u);
                const int ext = axis == 0 ? G.w : (axis == 1 ? G.h : G.d);
                const AxisWeight aw = g_axis[axis_index(R, ext, p)];
                s.w[ws][axis][p] = aw;
                s.w16[tid] = make_float4(aw.t, aw.omt, __int_as_float((int)aw.i0), __int_as_float((int)aw.i1));
            }
            const bool ok = !staged || mbar_wait(s.bar, phase);
            if (__syncthreads_or(!ok)) {   // any thread gave up: the whole CTA stops, together
                if (tid == 0) record_error(a.err, leaf, kErrWaitTimeout);
                if (staged) mbar_wait(s.bar, phase);   // a second bounded wait for the copy in flight
                return;
            }
            if (staged) phase ^= 1u;
            bool fine = false;
            if (fast_leaf_shape(e, steps01, fine) && (staged || GLOBAL_FALLBACK)) {
                const uint32_t lb = (uint32_t)(b0 - a0);
                if (staged) {
                    if (fine) leaf_decode_fast_call<true, DENSE, false>(a, e, lb, a0, fl.n, G, out, frame_stride);
                    else leaf_decode_fast_call<false, DENSE, false>(a, e, lb, a0, fl.n, G, out, frame_stride);
                } else if constexpr (GLOBAL_FALLBACK) {
                    if (fine) leaf_decode_fast_call<true, DENSE, true>(a, e, lb, a0, fl.n, G, out, frame_stride);
                    else leaf_decode_fast_call<false, DENSE, true>(a, e, lb, a0, fl.n, G, out, frame_stride);
                }
            } else if (staged) {
                const SharedWords m{reinterpret_cast<const uint32_t*>(s.stage), (uint32_t)(a0 >> 2)};
                leaf_decode_general<SharedWords, DENSE>(a, m, e, fl.n, steps01, monotone, G, out, frame_stride);
            } else if (GLOBAL_FALLBACK) {
                const GlobalWords m{a.payload};
                leaf_decode_general<GlobalWords, DENSE>(a, m, e, fl.n, steps01, monotone, G, out, frame_stride);
            }
        }
        __syncthreads();   // the next index is visible
        li = *s_next;
    }
}

template <bool DENSE, bool GF>
static int leaf_grid(uint32_t smem_bytes)
{
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, decode_leaf_kernel<DENSE, GF>, kDecThreads, smem_bytes);
    return sms * (per > 0 ? per : 1);
}

template <bool DENSE, bool GF>
static void launch_leaf_variant(const DeviceAsset& a, uint32_t seq, const FrameList& fl, float* out, uint64_t stride,
                                int grid, cudaStream_t s)
{
    const uint32_t smem = kDecFixed + a.g.stage_bytes + kStagePad;
    cudaFuncSetAttribute(decode_leaf_kernel<DENSE, GF>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    const int g = grid > 0 ? grid : leaf_grid<DENSE, GF>(smem);
    unsigned long long* slot = a.work + seq % kWorkSlots;
    // Inside a stream capture the epoch is frozen into the graph: every replay starts from a
    // cleared slot instead (a graph is never replayed concurrently with itself).
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cs) == cudaSuccess && cs == cudaStreamCaptureStatusActive)
        cudaMemsetAsync(slot, 0, sizeof(unsigned long long), s);
    decode_leaf_kernel<DENSE, GF><<<g, kDecThreads, smem, s>>>(a, fl, out, stride, slot, seq + 1u);
}

static void launch_rt_leaf(const DeviceAsset& a, uint32_t seq, const FrameList& fl, float* out, uint64_t stride,
                           int grid, bool dense, cudaStream_t s)
{
    const bool gf = a.g.max_window > a.g.stage_bytes;
    if (dense) {
        if (gf) launch_leaf_variant<true, true>(a, seq, fl, out, stride, grid, s);
        else launch_leaf_variant<true, false>(a, seq, fl, out, stride, grid, s);
    } else {
        if (gf) launch_leaf_variant<false, true>(a, seq, fl, out, stride, grid, s);
        else launch_leaf_variant<false, false>(a, seq, fl, out, stride, grid, s);
    }
}

}  // namespace vbtb
