// render_window.cuh -- (d) window decode of render-temporal leaves as a hat-basis contraction on
// the tensor cores, and its FP64 error oracle.  Included by kernels.cu after sci_window.cuh (it
// uses that file's tcgen05 helpers and rt_kernel_leaf.cuh's leaf decode).
//
// A render-temporal control is piecewise linear in t between its key frames and constant outside
// them (decodeFromSequence, src/render_temporal_decode.cpp:79-131, on strictly increasing keys).
// The trilinear reconstruction is linear in the controls, so between two consecutive frames of
// the union U of every control's key frames inside the window (plus the window's first and last
// frame) every voxel is linear in t.  For one leaf and a window of n <= 16 frames:
//     V(512 x n) = Coef(512 x K) . H(K x n),
// Coef = the voxels at the K knots of U, decoded exactly (the leaf kernel's control and voxel
// phases on K frames instead of n), H = the hat functions of U at the window's frames (a frame on
// a knot has a unit row).  Coef and H are each split into three BF16 terms; the six products
// whose terms sum to at most 2^-24 of the value run as tcgen05.mma kind::f16 (M = 128 voxels,
// N = 16 frames, K = 16 knots) accumulated in FP32 in tensor memory: 4 M tiles x 6 = 24 MMAs per
// leaf-window.  A knot frame's value is the sum of its three exact terms: bit-identical to the
// per-frame decode.  Leaves whose keys do not strictly increase, and Mode2 leaves (the clamp to
// zero outside the occupancy is not linear), take every frame as a knot; a window whose every
// frame is a knot is decoded exactly, without the contraction.
// A launch covers up to 64 frames as consecutive 16-frame windows: each leaf is staged once and
// its knots are found for all windows in one pass over its keys.
#pragma once

namespace vbtb {

constexpr int kRwWin = 16;                      // frames per window (the MMA's N)
constexpr int kRwMaxN = 64;                     // frames per launch
constexpr uint32_t kRwA = 4u * 3u * 4096u;      // 4 M tiles x 3 terms x (128 voxel rows x 16 knots)
constexpr uint32_t kRwB = 3u * 512u;            // 3 terms x (16 frame rows x 16 knots)
constexpr uint32_t kRwMisc = 128u;              // MMA barrier, TMEM address, knot mask, knot offsets
constexpr uint32_t kRwHead = kRwA + kRwB + kRwMisc;   // the leaf-kernel layout follows
// The FP32 voxels at the knots ([knot][voxel], 32 KiB) live in the first half of the A region
// until the split into A's BF16 terms overwrites them.
static_assert(16u * 512u * 4u <= kRwA, "the knot values fit inside the A operand region");
constexpr uint32_t kRwTmemCols = 64u;           // 4 M tiles x 16 FP32 columns
static_assert(kRwHead % 128u == 0u, "the leaf-kernel layout after the window head stays aligned");

struct CoefSink {
    float* coef;
    __device__ __forceinline__ void operator()(int k, int lane, int i, float4 v) const
    {
        reinterpret_cast<float4*>(coef + k * 512)[lane + 32 * i] = v;
    }
};

__device__ __forceinline__ void win_split3(float x, uint16_t& b0, uint16_t& b1, uint16_t& b2)
{
    b0 = win_bf16_bits(x);
    const float r1 = __fsub_rn(x, win_bf16_val(b0));
    b1 = win_bf16_bits(r1);
    b2 = win_bf16_bits(__fsub_rn(r1, win_bf16_val(b1)));
}

// One leaf, every window of the launch.  Returns false when a bounded wait gave up (the CTA then
// stops).
template <class M>
__device__ __forceinline__ bool render_window_leaf(const DeviceAsset& a, const M& m, const LeafSmem& s,
                                                   const LeafEntry& e, const LeafGeom& G, int t0, int n,
                                                   uint8_t* sA, uint8_t* sB, unsigned long long* s_mask,
                                                   int* s_knot, uint64_t* bar_mma, uint32_t taddr, uint32_t& ph_mma,
                                                   float* __restrict__ out, uint64_t frame_stride, uint32_t leaf)
{
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int total = (int)a.g.frames;
    float* const sCoef = reinterpret_cast<float*>(sA);
    // 1. knots: every control's key frames strictly inside the launch's frames (each window's
    //    first and last frame are set already)
    const bool interp = (e.info & kFlagSorted) != 0u && (e.info & (kFlagOccClamp | kFlagShell)) == 0u;
    if (interp) {
        const uint64_t base = 4ull * e.word_off;
        const int cres = (int)((e.header >> 6) & 7u), fres = (int)((e.header >> 9) & 7u);
        const bool fine = (e.info & kFlagFine) != 0u;
        const StreamRef cs{base + 8u, (uint32_t)(cres * cres * cres), 8u, e.kf & 0xFFFFu, (e.header >> 2) & 3u};
        const StreamRef fs{base + 8u + e.coarse_bytes, (uint32_t)(fres * fres * fres), 8u, e.kf >> 16,
                           (e.header >> 4) & 3u};
        const int Cc = (int)cs.controls, Ctot = Cc + (fine ? (int)fs.controls : 0);
        for (int c = tid; c < Ctot; c += kLeafThreads) {
            const StreamRef& st = c < Cc ? cs : fs;
            const uint32_t ci = (uint32_t)(c < Cc ? c : c - Cc);
            const uint32_t desc = m((uint32_t)((st.base + 4ull * ci) >> 2));
            const uint32_t kc = (desc >> 16) & 0xFFu, ks = desc & 0xFFFFu;
            if (kc == 0u || ks + kc > st.kf) continue;
            const uint64_t kb = stream_key_base(st);
            uint32_t lo = 0, hi = kc;   // first key with frame > t0
            while (lo < hi) {
                const uint32_t mid = (lo + hi) >> 1;
                if (m_key_frame(m, kb, st.codec, ks + mid) > t0) hi = mid;
                else lo = mid + 1u;
            }
            unsigned long long bits = 0ull;
            for (uint32_t k = lo; k < kc; ++k) {
                const int f = m_key_frame(m, kb, st.codec, ks + k);
                if (f >= t0 + n - 1) break;
                bits |= 1ull << (f - t0);
            }
            if (bits) atomicOr(s_mask, bits);
        }
    } else if (tid == 0) {
        *s_mask = n == 64 ? ~0ull : ((1ull << n) - 1ull);
    }
    __syncthreads();
    const unsigned long long mask = *s_mask;
    for (int w0 = 0; w0 < n; w0 += kRwWin) {
        const int nw = min(kRwWin, n - w0);
        const uint32_t sub = (uint32_t)(mask >> w0) & ((1u << nw) - 1u);
        const int K = __popc(sub);
        if (tid < nw && ((sub >> tid) & 1u)) {
            const int k = __popc(sub & ((1u << tid) - 1u));
            const int fr = t0 + w0 + tid;
            s.fr[k] = fr;
            s.b8[k] = (uint8_t)time_bin(fr, 8u, total);
            s.b4[k] = (uint8_t)time_bin(fr, 4u, total);
            s_knot[k] = tid;
        }
        __syncthreads();
        // A window whose every frame is a knot has nothing to interpolate: its frames are decoded
        // exactly, straight into the output.
        if (K == nw) {
            leaf_decode(a, m, s, e, nw, true, true, G,
                        FrameSink<false>{a, G, out + (uint64_t)w0 * frame_stride, frame_stride});
            continue;
        }
        // 2. exact voxels at the knots
        leaf_decode(a, m, s, e, K, false, true, G, CoefSink{sCoef});
        // 3. A = Coef split into three BF16 terms (knot columns >= K are 0), through registers
        //    since A overwrites the knot values; B = H split likewise
        uint32_t w[4][3][4];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const int it = tid + r * kLeafThreads;
            const uint32_t v = (uint32_t)it & 511u, g = (uint32_t)it >> 9;
            if ((int)(8u * g) >= K) {   // a knot group past K: zeros (B's rows there are 0 too)
#pragma unroll
                for (int p = 0; p < 3; ++p) w[r][p][0] = w[r][p][1] = w[r][p][2] = w[r][p][3] = 0u;
                continue;
            }
#pragma unroll
            for (int kk = 0; kk < 8; kk += 2) {
                const int k = (int)(8u * g) + kk;
                const float x0 = k < K ? sCoef[k * 512 + (int)v] : 0.0f;
                const float x1 = k + 1 < K ? sCoef[(k + 1) * 512 + (int)v] : 0.0f;
                uint16_t a0[3], a1[3];
                win_split3(x0, a0[0], a0[1], a0[2]);
                win_split3(x1, a1[0], a1[1], a1[2]);
#pragma unroll
                for (int p = 0; p < 3; ++p) w[r][p][kk >> 1] = (uint32_t)a0[p] | ((uint32_t)a1[p] << 16);
            }
        }
        __syncthreads();
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const int it = tid + r * kLeafThreads;
            const uint32_t v = (uint32_t)it & 511u, g = (uint32_t)it >> 9;
            const uint32_t mt = v >> 7, row = v & 127u;
#pragma unroll
            for (int p = 0; p < 3; ++p)
                *reinterpret_cast<uint4*>(sA + (mt * 3u + (uint32_t)p) * 4096u + win_off(row, 8u * g)) =
                    make_uint4(w[r][p][0], w[r][p][1], w[r][p][2], w[r][p][3]);
        }
        {
            const int j = tid >> 4, k = tid & 15;   // 256 threads = 16 frames x 16 knots
            float h = 0.0f;
            if (j < nw && k < K) {
                const int u = s_knot[k];
                if (u == j) h = 1.0f;
                else if (u < j && k + 1 < K && s_knot[k + 1] > j)
                    h = __fdiv_rn((float)(s_knot[k + 1] - j), (float)(s_knot[k + 1] - u));
                else if (u > j && k > 0 && s_knot[k - 1] < j)
                    h = __fdiv_rn((float)(j - s_knot[k - 1]), (float)(u - s_knot[k - 1]));
            }
            uint16_t t[3];
            win_split3(h, t[0], t[1], t[2]);
#pragma unroll
            for (int p = 0; p < 3; ++p)
                *reinterpret_cast<uint16_t*>(sB + (uint32_t)p * 512u + win_off((uint32_t)j, (uint32_t)k)) = t[p];
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        win_tc_fence_before();
        __syncthreads();
        win_tc_fence_after();
        // 4. one thread issues the 24 MMAs (term pairs p + q <= 2) and commits them
        if (tid == 0) {
            const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((16u >> 3) << 17) | ((128u >> 4) << 24);
            for (uint32_t mt = 0; mt < 4u; ++mt) {
                uint32_t acc = 0u;
                for (uint32_t p = 0; p < 3u; ++p)
                    for (uint32_t q = 0; p + q < 3u; ++q) {
                        win_mma(taddr + mt * 16u, win_desc(win_smem_u32(sA + (mt * 3u + p) * 4096u)),
                                win_desc(win_smem_u32(sB + q * 512u)), idesc, acc);
                        acc = 1u;
                    }
            }
            win_commit(bar_mma);
        }
        const bool ok = mbar_wait(bar_mma, ph_mma);
        if (__syncthreads_or(!ok)) {
            if (tid == 0) record_error(a.err, leaf, kErrWaitTimeout);
            mbar_wait(bar_mma, ph_mma);
            return false;
        }
        ph_mma ^= 1u;
        win_tc_fence_after();
        // 5. epilogue: warp w reads voxel rows 32 (w % 4) .. +31 of M tiles 2 (w / 4) and
        //    2 (w / 4) + 1
        const uint32_t quarter = (uint32_t)(warp & 3), half = (uint32_t)(warp >> 2);
#pragma unroll
        for (uint32_t mm = 0; mm < 2u; ++mm) {
            const uint32_t mt = half * 2u + mm;
            float d[16];
            win_ld16(taddr + ((quarter * 32u) << 16) + mt * 16u, d);
            const uint32_t v = mt * 128u + quarter * 32u + (uint32_t)lane;
            float* o = out + (uint64_t)w0 * frame_stride + (uint64_t)G.li * 512u + v;
#pragma unroll
            for (int j = 0; j < kRwWin; ++j)
                if (j < nw) o[(uint64_t)j * frame_stride] = d[j];
        }
        win_tc_fence_before();
        __syncthreads();   // D, A, B and the knot buffers are free for the next window or leaf
        win_tc_fence_after();
    }
    return true;
}

// Persistent CTAs over the active leaves, 256 threads, as many per SM as shared memory allows;
// leaves are handed out one at a time by the launch's work counter (grab_leaf), so that CTAs that
// drew cheap leaves (few knots) take more of them.  out[f * frame_stride + rank * 512 + voxel] for f < n, the current-frame cache
// layout of frames t0 .. t0 + n - 1.
template <bool GLOBAL_FALLBACK>
__global__ void __launch_bounds__(kLeafThreads, 2) render_window_kernel(DeviceAsset a, int t0, int n,
                                                                        float* __restrict__ out, uint64_t frame_stride,
                                                                        unsigned long long* work, uint32_t epoch)
{
    extern __shared__ __align__(1024) uint8_t rdyn[];
    uint8_t* sA = rdyn;
    uint8_t* sB = rdyn + kRwA;
    uint8_t* misc = rdyn + kRwA + kRwB;
    uint64_t* bar_mma = reinterpret_cast<uint64_t*>(misc);
    unsigned long long* s_mask = reinterpret_cast<unsigned long long*>(misc + 8);
    uint32_t* s_taddr = reinterpret_cast<uint32_t*>(misc + 16);
    int* s_knot = reinterpret_cast<int*>(misc + 32);   // a window's knot offsets, ascending
    uint32_t* s_next = reinterpret_cast<uint32_t*>(misc + 96);   // the next rank from the work counter
    const LeafSmem s = leaf_layout(rdyn + kRwHead);
    const int tid = threadIdx.x, warp = tid >> 5;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(win_smem_u32(s_taddr)),
                     "r"(kRwTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        mbar_init(s.bar, 1);
        mbar_init(bar_mma, 1);
        mbar_init_fence();
        bool to = false;
        const uint32_t first = grab_leaf(work, epoch, to);
        if (to) record_error(a.err, 0u, kErrWaitTimeout);
        *s_next = first;
    }
    s.rcp[tid] = __frcp_rn((float)tid);
    win_tc_fence_before();
    __syncthreads();
    win_tc_fence_after();
    const uint32_t taddr = *s_taddr;
    const uint32_t n_leaves = *(volatile const uint32_t*)a.counters;
    const uint8_t* pay_bytes = reinterpret_cast<const uint8_t*>(a.payload);
    uint32_t ph_tma = 0, ph_mma = 0;

    uint32_t rank = *s_next;
    while (rank < n_leaves) {
        __syncthreads();   // every thread has read the rank
        if (tid == 0) {
            bool to = false;
            const uint32_t nx = grab_leaf(work, epoch, to);
            if (to) record_error(a.err, 0u, kErrWaitTimeout);
            *s_next = nx;
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
        if (skip || (!GLOBAL_FALLBACK && !staged)) {   // uniform over the CTA
            if (tid == 0) record_error(a.err, leaf, st != kOk ? st : kErrDecodeOob);
            for (int i = tid; i < n * 512; i += kLeafThreads)
                out[(uint64_t)(i >> 9) * frame_stride + (uint64_t)rank * 512u + (i & 511)] = 0.0f;
            __syncthreads();   // the next rank is visible
            rank = *s_next;
            continue;
        }
        if (tid == 0) {
            if (staged) mbar_expect_and_copy(s.bar, s.stage, pay_bytes + a0, (uint32_t)(a1 - a0));
            unsigned long long ends = 0ull;
            for (int w0 = 0; w0 < n; w0 += kRwWin) ends |= (1ull << w0) | (1ull << min(n - 1, w0 + kRwWin - 1));
            *s_mask = ends;
        }
        if (tid < 48) {
            const int ws = tid / 24, axis = (tid % 24) >> 3, p = tid & 7;
            const int R = ws == 0 ? (int)((e.header >> 6) & 7u) : (int)((e.header >> 9) & 7u);
            const int ext = axis == 0 ? G.w : (axis == 1 ? G.h : G.d);
            s.w[ws][axis][p] = g_axis[axis_index(R, ext, p)];
        }
        const bool ok = !staged || mbar_wait(s.bar, ph_tma);
        if (__syncthreads_or(!ok)) {
            if (tid == 0) record_error(a.err, leaf, kErrWaitTimeout);
            if (staged) mbar_wait(s.bar, ph_tma);
            break;
        }
        if (staged) ph_tma ^= 1u;
        bool done;
        if (staged) {
            const SharedWords m{reinterpret_cast<const uint32_t*>(s.stage), (uint32_t)(a0 >> 2)};
            done = render_window_leaf(a, m, s, e, G, t0, n, sA, sB, s_mask, s_knot, bar_mma, taddr, ph_mma, out,
                                      frame_stride, leaf);
        } else {
            const GlobalWords m{a.payload};
            done = render_window_leaf(a, m, s, e, G, t0, n, sA, sB, s_mask, s_knot, bar_mma, taddr, ph_mma, out,
                                      frame_stride, leaf);
        }
        if (!done) break;
        __syncthreads();   // the next rank is visible
        rank = *s_next;
    }
    win_tc_fence_before();
    __syncthreads();
    win_tc_fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(kRwTmemCols) : "memory");
}

// Exact-arithmetic trilinear of one control grid (resolution R) at voxel (lx, ly, lz): the
// reference's nested lerps with its FP32 weights t and 1 - t, expanded without rounding.
__device__ __forceinline__ double trilinear_f64(const AxisWeight (*w)[8], const double* g, int R, int lx, int ly,
                                                int lz)
{
    if (R < 2) return R == 1 ? g[0] : 0.0;
    const AxisWeight ax = w[0][lx], ay = w[1][ly], az = w[2][lz];
    double v = 0.0;
    for (int cz = 0; cz < 2; ++cz)
        for (int cy = 0; cy < 2; ++cy)
            for (int cx = 0; cx < 2; ++cx) {
                const int ci = ((cz ? az.i1 : az.i0) * R + (cy ? ay.i1 : ay.i0)) * R + (cx ? ax.i1 : ax.i0);
                v += (double)(cx ? ax.t : ax.omt) * (double)(cy ? ay.t : ay.omt) * (double)(cz ? az.t : az.omt) * g[ci];
            }
    return v;
}

// FP64 error oracle of any render-temporal cache of frames [t0, t0 + n) (cache layout, active
// ranks of the current page table): per voxel and frame the reference composition
// (render_smoke_vbt_bench_main.cpp:277-387) evaluated in double without intermediate rounding --
// controls from the bracket the reference's search selects, interpolated exactly; the trilinear
// with the reference's FP32 weights; fine grid or Mode2 shell residual; Mode2's clamp of negatives
// outside the occupancy -- reduced as sci_window_oracle_kernel reduces.
__global__ void __launch_bounds__(256) render_window_oracle_kernel(DeviceAsset a, int t0, int n,
                                                                   const float* __restrict__ vals,
                                                                   uint64_t frame_stride, unsigned long long* stats)
{
    __shared__ double s_ctrl[343 + 512];
    __shared__ AxisWeight s_w[2][3][8];
    __shared__ double s_max[8], s_sum[8];
    __shared__ unsigned long long s_lo[8], s_hi[8];
    const int tid = threadIdx.x;
    const int total = (int)a.g.frames;
    double my_max = 0.0, my_sum = 0.0;
    unsigned long long my_lo = ~0ull, my_hi = 0ull;
    const GlobalWords m{a.payload};
    const uint32_t n_leaves = *(volatile const uint32_t*)a.counters;
    for (uint32_t rank = blockIdx.x; rank < n_leaves; rank += gridDim.x) {
        const uint32_t leaf = __ldg(a.active_list + rank);
        const LeafEntry e = a.entries[leaf];
        int ew, eh, ed;
        uint32_t gx, gy, gz;
        leaf_extent(a.g, leaf, gx, gy, gz, ew, eh, ed);
        const float* row0 = vals + (uint64_t)rank * 512u;
        if (entry_status(e) != kOk || (e.header & 3u) == kModeEmpty) {   // the cache holds 0
            for (int i = tid; i < n * 512; i += 256)
                my_max = fmax(my_max, fabs((double)row0[(uint64_t)(i >> 9) * frame_stride + (i & 511)]));
            continue;
        }
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
        if (tid < 48) {
            const int ws = tid / 24, axis = (tid % 24) >> 3, p = tid & 7;
            const int R = ws == 0 ? cres : fres;
            const int ext = axis == 0 ? ew : (axis == 1 ? eh : ed);
            s_w[ws][axis][p] = g_axis[axis_index(R, ext, p)];
        }
        for (int f = 0; f < n; ++f) {
            const int t = t0 + f;
            for (int c = tid; c < Cc + Cf; c += 256) {
                const StreamRef& st = c < Cc ? cs : (fine ? fs : ss);
                const uint32_t ci = (uint32_t)(c < Cc ? c : c - Cc);
                s_ctrl[c] = m_control_value_f64(m, st, ci, t, time_bin(t, st.bins, total));
            }
            __syncthreads();
            for (int v = tid; v < 512; v += 256) {
                const int lx = v & 7, ly = (v >> 3) & 7, lz = v >> 6;
                double ref = 0.0;
                if (lx < ew && ly < eh && lz < ed) {
                    ref = trilinear_f64(s_w[0], s_ctrl, cres, lx, ly, lz);
                    if (fine) ref += trilinear_f64(s_w[1], s_ctrl + Cc, fres, lx, ly, lz);
                    if (occ) {
                        const uint64_t ob = base + 8u + e.coarse_bytes;
                        const uint32_t g = (uint32_t)v >> 6, bit = (uint32_t)v & 63u;
                        const uint64_t mk = ((uint64_t)m((uint32_t)((ob + 8u * g + 4u) >> 2)) << 32) |
                                            m((uint32_t)((ob + 8u * g) >> 2));
                        const uint32_t pref = (m((uint32_t)((ob + 64u + 2u * g) >> 2)) >> ((g & 1u) * 16u)) & 0xFFFFu;
                        const bool in_occ = ((mk >> bit) & 1ull) != 0ull;
                        if (shell && in_occ) {
                            const uint32_t di = (pref + (uint32_t)__popcll(mk & ((1ull << bit) - 1ull))) & 0xFFFFu;
                            ref += s_ctrl[Cc + (int)di];
                        }
                        if (!in_occ && ref < 0.0) ref = 0.0;
                    }
                }
                const double got = (double)row0[(uint64_t)f * frame_stride + v];
                const double err = fabs(got - ref);
                my_max = fmax(my_max, err);
                my_sum += err * err;
                const unsigned long long o = win_ordered(ref);
                my_lo = o < my_lo ? o : my_lo;
                my_hi = o > my_hi ? o : my_hi;
            }
            __syncthreads();
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        my_max = fmax(my_max, __shfl_down_sync(0xFFFFFFFFu, my_max, o));
        my_sum += __shfl_down_sync(0xFFFFFFFFu, my_sum, o);
        const unsigned long long lo2 = __shfl_down_sync(0xFFFFFFFFu, my_lo, o);
        const unsigned long long hi2 = __shfl_down_sync(0xFFFFFFFFu, my_hi, o);
        my_lo = lo2 < my_lo ? lo2 : my_lo;
        my_hi = hi2 > my_hi ? hi2 : my_hi;
    }
    const int warp = tid >> 5, lane = tid & 31;
    if (lane == 0) {
        s_max[warp] = my_max;
        s_sum[warp] = my_sum;
        s_lo[warp] = my_lo;
        s_hi[warp] = my_hi;
    }
    __syncthreads();
    if (tid == 0) {
        double mx = 0.0, sm = 0.0;
        unsigned long long lo = ~0ull, hi = 0ull;
        for (int w = 0; w < 8; ++w) {
            mx = fmax(mx, s_max[w]);
            sm += s_sum[w];
            lo = s_lo[w] < lo ? s_lo[w] : lo;
            hi = s_hi[w] > hi ? s_hi[w] : hi;
        }
        atomicMax(stats + 0, (unsigned long long)__double_as_longlong(mx));
        atomicAdd(reinterpret_cast<double*>(stats + 1), sm);
        atomicMin(stats + 2, lo);
        atomicMax(stats + 3, hi);
    }
}

void launch_render_window(const DeviceAsset& asset, uint32_t seq, int t0, int n, float* out, uint64_t frame_stride,
                          cudaStream_t s)
{
    // Two CTAs per SM when the leaf stage allows; leaves whose window exceeds that stage are read
    // from global memory (the GLOBAL_FALLBACK instantiation).
    DeviceAsset a = asset;
    constexpr uint32_t cap2 = ((233472u / 2u - 1024u - kRwHead - kLeafFixed - kStagePad) / 1024u) * 1024u;
    if (a.g.stage_bytes > cap2) a.g.stage_bytes = cap2;
    const uint32_t smem = kRwHead + kLeafFixed + a.g.stage_bytes + kStagePad;
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    auto go = [&](auto kernel) {
        cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        // CTAs per SM from the shared memory per SM and per block (registers allow two: the
        // kernel's launch bounds)
        int per_sm = 0, reserved = 0;
        cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
        cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev);
        const int fit = (int)((uint32_t)per_sm / (smem + (uint32_t)reserved));
        const int per = fit >= 2 ? 2 : 1;
        unsigned long long* slot = a.work + seq % kWorkSlots;
        // inside a stream capture every replay starts from a cleared slot (see launch_leaf_variant)
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        if (cudaStreamIsCapturing(s, &cs) == cudaSuccess && cs == cudaStreamCaptureStatusActive)
            cudaMemsetAsync(slot, 0, sizeof(unsigned long long), s);
        kernel<<<sms * per, kLeafThreads, smem, s>>>(a, t0, n, out, frame_stride, slot, seq + 1u);
    };
    if (a.g.max_window > a.g.stage_bytes) go(render_window_kernel<true>);
    else go(render_window_kernel<false>);
}

void launch_render_window_oracle(const DeviceAsset& a, int t0, int n, const float* vals, uint64_t frame_stride,
                                 unsigned long long* stats, cudaStream_t s)
{
    cudaMemsetAsync(stats, 0, 4 * sizeof(unsigned long long), s);
    cudaMemsetAsync(stats + 2, 0xFF, sizeof(unsigned long long), s);
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    render_window_oracle_kernel<<<4 * sms, 256, 0, s>>>(a, t0, n, vals, frame_stride, stats);
}

}  // namespace vbtb
