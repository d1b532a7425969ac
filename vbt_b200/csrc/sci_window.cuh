// sci_window.cuh -- (d) multi-frame window decode of scientific leaves on the tensor cores, and
// its FP64 error oracle.  Included by kernels.cu (it uses that file's scientific helpers).
//
// For one leaf and a window of n <= 64 frames starting at t0, the voxels are
//     V(512 x n) = S(512 x 64) . C(64 x n) + residual,
// C = the 64 coarse controls at the window's frames (DC b0(t) + sum_k q_k b_k(t), the DCT-II
// contraction of render/src/scientific_decode.cpp:82-97) and S = the trilinear weights of
// sampleCoarseAt (:99-123).  Those weights are products of three axis weights that are multiples
// of 1/7, so S' = 343 S is an integer matrix with entries <= 343.  Every entry but 343 (the eight
// voxels that sit on a control point, weight 1) is exact in one BF16; the A operand holds S' with
// 343 entered as 342, and the missing 1 x C term of those eight voxels is added on the CUDA cores.
// C is computed in FP64 (exact products, one rounding per term), rounded once to FP32 and split
// into three BF16 terms c = c_hi + c_mid + c_lo
// (residual below 2^-26 |c|).  The contraction is 3 tcgen05.mma products per 16-wide K step
// (S'.c_hi + S'.c_mid + S'.c_lo), accumulated in FP32 in tensor memory: 4 M tiles (128 voxels)
// x 4 K steps x 3 terms = 48 MMAs of 128 x N x 16 per leaf-window, N = n rounded up to 16.
// The epilogue reads D from tensor memory, adds the corner terms, scales by 1/343, adds the
// sparse-event or DenseGrid residual (CUDA cores, as the per-frame path) and writes the cache
// layout.
//
// Shared-memory operand layout (canonical K-major, no swizzle): per K step, core matrices of
// 8 rows x 16 bytes; the two 8-element K halves 128 bytes apart (leading byte offset), 8-row
// groups 256 bytes apart (stride byte offset).
#pragma once

namespace vbtb {

constexpr int kWinThreads = 256;
constexpr int kWinMaxN = 64;
constexpr uint32_t kWinTmemCols = 256;                  // 4 M tiles x 64 columns of FP32
constexpr uint32_t kWinA = 4u * 4u * 4096u;             // 4 M tiles x 4 K steps x (128 rows x 32 B)
constexpr uint32_t kWinB = 4u * 3u * (kWinMaxN * 32u);  // 4 K steps x 3 terms x (64 rows x 32 B)
constexpr uint32_t kWinCorner = 8u * kWinMaxN * 4u;     // corner controls x frames, FP32
constexpr uint32_t kWinQ = 64u * 64u * 4u;              // 64 controls x keep (<= 64) coefficients
constexpr int kWinBasisK = 4;                            // basis terms held in FP64 per frame
constexpr int kWinBdStride = kWinBasisK + 1;             // doubles per frame row (8 rows: 8 bank pairs)
constexpr uint32_t kWinBd = kWinMaxN * kWinBdStride * 8u;   // b_k(t0 + f), k < 4, FP64
constexpr uint32_t kWinSmem = kWinA + kWinB + kWinCorner + kWinQ + kWinBd + 256u;   // + barrier, TMEM address, sparse header

__device__ __forceinline__ uint32_t win_smem_u32(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor: start >> 4 [0,14), LBO >> 4 [16,30), SBO >> 4 [32,46),
// version 1 [46,48), no swizzle [61,64).
__device__ __forceinline__ uint64_t win_desc(uint32_t saddr)
{
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(128u >> 4) << 16) | ((uint64_t)(256u >> 4) << 32) |
           (1ull << 46);
}

// Byte offset of (row, k) inside one K step of a K-major operand tile.
__device__ __forceinline__ uint32_t win_off(uint32_t row, uint32_t k)
{
    return (row >> 3) * 256u + (k >> 3) * 128u + (row & 7u) * 16u + (k & 7u) * 2u;
}

// 7 x the trilinear weight of control coordinate c (0..3) for voxel coordinate x (0..7): the
// sample position is 3x/7 control spacings (scientific_decode.cpp:99-123, f = x/7*3 clamped to
// cell 0..2).
__device__ __forceinline__ uint32_t win_w7(uint32_t x, uint32_t c)
{
    const uint32_t f7 = 3u * x;
    const uint32_t i0 = min(2u, f7 / 7u);
    const uint32_t t7 = f7 - 7u * i0;
    return c == i0 ? 7u - t7 : (c == i0 + 1u ? t7 : 0u);
}

// Index 0..7 of a corner control ((cx, cy, cz) in {0, 3}^3), or -1.
__device__ __forceinline__ int win_corner_of_control(uint32_t ci)
{
    const uint32_t cx = ci & 3u, cy = (ci >> 2) & 3u, cz = ci >> 4;
    if ((cx != 0u && cx != 3u) || (cy != 0u && cy != 3u) || (cz != 0u && cz != 3u)) return -1;
    return (int)((cx ? 1u : 0u) | (cy ? 2u : 0u) | (cz ? 4u : 0u));
}
// Index 0..7 of a voxel on a control point ((lx, ly, lz) in {0, 7}^3), or -1.
__device__ __forceinline__ int win_corner_of_voxel(uint32_t v)
{
    const uint32_t lx = v & 7u, ly = (v >> 3) & 7u, lz = v >> 6;
    if ((lx != 0u && lx != 7u) || (ly != 0u && ly != 7u) || (lz != 0u && lz != 7u)) return -1;
    return (int)((lx ? 1u : 0u) | (ly ? 2u : 0u) | (lz ? 4u : 0u));
}

__device__ __forceinline__ uint16_t win_bf16_bits(float x)
{
    const __nv_bfloat16 b = __float2bfloat16_rn(x);
    return *reinterpret_cast<const uint16_t*>(&b);
}
__device__ __forceinline__ float win_bf16_val(uint16_t bits)
{
    return __uint_as_float((uint32_t)bits << 16);
}

__device__ __forceinline__ void win_tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void win_tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// D[tmem] (+)= A[desc] x B[desc], kind::f16 (BF16 inputs, FP32 accumulate).
__device__ __forceinline__ void win_mma(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc, uint32_t acc)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
        "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(acc)
        : "memory");
}

__device__ __forceinline__ void win_commit(uint64_t* bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(win_smem_u32(bar))
                 : "memory");
}

// 16 consecutive FP32 columns of this thread's tensor-memory lane.
__device__ __forceinline__ void win_ld16(uint32_t taddr, float (&v)[16])
{
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// L2 prefetch of a scientific leaf's payload, one 128-byte line per thread: the coefficient block
// with the sparse section's header, mask, bins and the keys of its events (or 512 bytes past the
// block for other modes), and the events' 4-bit codes.  Only lines that start inside the payload.
__device__ __forceinline__ void win_prefetch_leaf(const DeviceAsset& a, const LeafEntry& e, int tid)
{
    const uint32_t hdr = e.header, mode = hdr & 3u;
    const uint32_t keep = ((hdr >> 2) & 0x3Fu) + 1u, count = (hdr >> 16) & 0x0FFFu;
    const uint64_t base = 4ull * e.word_off, sb = base + 4u + 64u * (keep + 1u);
    const uint64_t end = mode == 1u ? sb + 100u + 2u * count : sb + 512u;
    const uint32_t tier = (hdr >> 8) & 3u;
    const uint32_t cap = tier == 0u ? 64u : tier == 1u ? 256u : tier == 2u ? 768u : 1024u;
    const uint64_t rb = sb + 100u + 2u * cap;
    const uint64_t lim = 4ull * a.g.payload_words;
    const uint64_t l0 = base & ~127ull, n0 = (end - l0 + 127u) / 128u;
    uint64_t at = ~0ull;
    if ((uint64_t)tid < n0) at = l0 + 128u * (uint64_t)tid;
    else if (mode == 1u && count && (uint64_t)tid >= 128u && (uint64_t)tid < 128u + (count / 2u + 128u) / 128u + 1u)
        at = (rb & ~127ull) + 128u * (uint64_t)(tid - 128);
    if (at < lim)
        asm volatile("prefetch.global.L2 [%0];" ::"l"(reinterpret_cast<const uint8_t*>(a.payload) + at));
}

// One CTA per leaf at a time (grid-stride), 256 threads, 2 CTAs per SM (shared memory and the
// 256 tensor-memory columns each).  out[f * frame_stride + leaf * 512 + voxel] for f < n.
__global__ void __launch_bounds__(kWinThreads, 2) sci_window_kernel(DeviceAsset a, int t0, int n,
                                                                    float* __restrict__ out, uint64_t frame_stride)
{
    extern __shared__ __align__(1024) uint8_t wdyn[];
    uint8_t* sA = wdyn;
    uint8_t* sB = wdyn + kWinA;
    float* sCorner = reinterpret_cast<float*>(wdyn + kWinA + kWinB);
    float* sQ = reinterpret_cast<float*>(wdyn + kWinA + kWinB + kWinCorner);
    double* sBd = reinterpret_cast<double*>(wdyn + kWinA + kWinB + kWinCorner + kWinQ);
    uint64_t* bar = reinterpret_cast<uint64_t*>(wdyn + kWinA + kWinB + kWinCorner + kWinQ + kWinBd);
    uint32_t* s_taddr = reinterpret_cast<uint32_t*>(bar + 1);
    SparseLeaf* s_sparse = reinterpret_cast<SparseLeaf*>(bar + 2);                 // 40 bytes
    uint32_t* s_mask = reinterpret_cast<uint32_t*>(reinterpret_cast<uint8_t*>(bar) + 64);   // 16 words
    uint32_t* s_bin = reinterpret_cast<uint32_t*>(reinterpret_cast<uint8_t*>(bar) + 128);   // 16 bin starts
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int N = (n + 15) & ~15;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(win_smem_u32(s_taddr)),
                     "r"(kWinTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        mbar_init(bar, 1);
        mbar_init_fence();
    }
    // A = S' (343 entered as 342), one exact BF16 per entry; the 32 axis weights 7 w(x, c) come
    // from a table in shared memory (in the Q region, not yet in use)
    uint32_t* s_w7 = reinterpret_cast<uint32_t*>(sQ);
    if (tid < 32) s_w7[tid] = win_w7((uint32_t)tid >> 2, (uint32_t)tid & 3u);
    // the window's first basis values in FP64 (the same for every leaf)
    for (int i = tid; i < kWinMaxN * kWinBasisK; i += kWinThreads) {
        const int f = i / kWinBasisK, k = i % kWinBasisK;
        sBd[f * kWinBdStride + k] = f < n ? (double)__ldg(a.basis + (uint64_t)(t0 + f) * 64u + k) : 0.0;
    }
    __syncthreads();
    // two adjacent controls per 32-bit store; a warp's 32 stores cover 8 rows x 4 words of one
    // 8-row core group: 32 distinct banks
    for (uint32_t P = tid; P < 512u * 32u; P += kWinThreads) {
        const uint32_t v = (P & 7u) | (((P >> 5) & 63u) << 3);
        const uint32_t ci = 2u * (((P >> 3) & 3u) | ((P >> 11) << 2));
        const uint32_t yz = s_w7[(((v >> 3) & 7u) << 2) | ((ci >> 2) & 3u)] * s_w7[((v >> 6) << 2) | (ci >> 4)];
        uint32_t w0 = s_w7[((v & 7u) << 2) | (ci & 3u)] * yz, w1 = s_w7[((v & 7u) << 2) | ((ci & 3u) | 1u)] * yz;
        if (w0 == 343u) w0 = 342u;
        if (w1 == 343u) w1 = 342u;
        const uint32_t m = v >> 7, sk = ci >> 4;
        *reinterpret_cast<uint32_t*>(sA + (m * 4u + sk) * 4096u + win_off(v & 127u, ci & 15u)) =
            (uint32_t)win_bf16_bits((float)w0) | ((uint32_t)win_bf16_bits((float)w1) << 16);
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    win_tc_fence_before();
    __syncthreads();
    win_tc_fence_after();
    const uint32_t taddr = *s_taddr;
    const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
    uint32_t phase = 0;

    // leaf table entries are read two leaves ahead; the next leaf's payload is prefetched into
    // L2 while this one decodes (its coefficient block and, for SparseEvents, the event keys and
    // codes), so the leaf's first reads are L2 hits
    const uint32_t L = a.g.leaf_count, G = gridDim.x;
    LeafEntry e_n1 = blockIdx.x < L ? a.entries[blockIdx.x] : LeafEntry{};
    LeafEntry e_n2 = blockIdx.x + G < L ? a.entries[blockIdx.x + G] : LeafEntry{};
    for (uint32_t leaf = blockIdx.x; leaf < L; leaf += G) {
        const LeafEntry e = e_n1;
        e_n1 = e_n2;
        if (leaf + 2u * G < L) e_n2 = a.entries[leaf + 2u * G];
        if (leaf + G < L && entry_status(e_n1) == kOk) win_prefetch_leaf(a, e_n1, tid);
        const uint32_t st = entry_status(e);
        const uint32_t hdr = e.header, mode = hdr & 3u;
        const int keep = (int)((hdr >> 2) & 0x3Fu) + 1;
        if (st != kOk) {   // uniform over the CTA
            if (tid == 0) record_error(a.err, leaf, st);
            for (int i = tid; i < n * 512; i += kWinThreads)
                out[(uint64_t)(i >> 9) * frame_stride + (uint64_t)leaf * 512u + (i & 511)] = 0.0f;
            continue;
        }
        const uint64_t base = 4ull * e.word_off;
        // 1. coefficients q[ci][k]: DC (fp16) for k = 0, int8 x acScale[k-1] otherwise
        SciReader rd{a.payload, a.g.payload_words, false};
        // the coarse block inside the payload: 32-bit windows instead of checked byte reads
        const bool block_in = base + 4u + (uint64_t)(64 * (keep + 1)) + 4u <= 4ull * a.g.payload_words;
        for (int i = tid; i < 64 * keep; i += kWinThreads) {
            const int ci = i / keep, k = i % keep;
            const uint64_t cb = base + 4u + (uint64_t)ci * (keep + 1);
            if (block_in) {
                const uint32_t w = pay_u32(a.payload, k == 0 ? cb : cb + 2u + (k - 1));
                sQ[i] = k == 0 ? half_bits_to_float(w & 0xFFFFu)
                               : __fmul_rn((float)(int8_t)(w & 0xFFu), __ldg(a.scales + k - 1));
            } else {
                sQ[i] = k == 0 ? half_bits_to_float(rd.u16(cb))
                               : __fmul_rn((float)(int8_t)rd.byte(cb + 2u + (k - 1)), __ldg(a.scales + k - 1));
            }
        }
        // the sparse section's header and occupancy mask, once per leaf
        if (mode == 1u && tid < 16) {
            const SparseLeaf sp = sparse_leaf(rd, base, hdr, keep);
            const bool any = sp.count && sp.es > 0.0f;
            s_mask[tid] = any ? sparse_mask_word(rd, sp, (uint32_t)tid) : 0u;
            s_bin[tid] = any ? rd.u16(sp.bb + 2u * (uint32_t)tid) : 0u;
            if (tid == 0) *s_sparse = sp;
        }
        if (rd.oob) record_error(a.err, leaf, kErrDecodeOob);
        __syncthreads();
        // Events are scattered onto their (frame, voxel) on leaves whose keys strictly increase
        // within every bin (kFlagSorted, set at load) and whose event scale is finite; otherwise
        // each voxel with events searches per frame, as the reference does.
        const bool scatter = mode == 1u && (e.info & kFlagSorted) != 0u && s_sparse->count &&
                             s_sparse->es > 0.0f && s_sparse->es <= 3.40282347e38f;
        // 2. C[f][ci] = sum_k q[ci][k] b_k(t0 + f) in FP64 (exact products, one rounding per
        //    term) rounded once to FP32, split into three BF16 terms, B tiles and corners.  Thread
        //    owns controls ci0 = 8 warp + 2 (lane / 8) and ci0 + 1 (coefficients in registers) and
        //    frames lane % 8 + 8 j; its three 32-bit stores per frame hit 32 distinct banks per warp.
        {
            const int ci0 = 8 * warp + 2 * (lane >> 3);
            double qa[kWinBasisK], qb[kWinBasisK];
#pragma unroll
            for (int k = 0; k < kWinBasisK; ++k) {
                qa[k] = k < keep ? (double)sQ[ci0 * keep + k] : 0.0;
                qb[k] = k < keep ? (double)sQ[(ci0 + 1) * keep + k] : 0.0;
            }
            const uint32_t sk = (uint32_t)ci0 >> 4, kk = (uint32_t)ci0 & 15u;
            const int cora = win_corner_of_control((uint32_t)ci0), corb = win_corner_of_control((uint32_t)ci0 + 1u);
            for (int f = lane & 7; f < N; f += 8) {
                float ca = 0.0f, cb = 0.0f;
                if (f < n) {
                    const double* bd = sBd + f * kWinBdStride;
                    double xa = 0.0, xb = 0.0;
#pragma unroll
                    for (int k = 0; k < kWinBasisK; ++k)
                        if (k < keep) {
                            const double b = bd[k];
                            xa = __fma_rn(qa[k], b, xa);
                            xb = __fma_rn(qb[k], b, xb);
                        }
                    if (keep > kWinBasisK) {
                        const float* brow = a.basis + (uint64_t)(t0 + f) * 64u;
                        for (int k = kWinBasisK; k < keep; ++k) {
                            const double b = (double)__ldg(brow + k);
                            xa = __fma_rn((double)sQ[ci0 * keep + k], b, xa);
                            xb = __fma_rn((double)sQ[(ci0 + 1) * keep + k], b, xb);
                        }
                    }
                    ca = __double2float_rn(xa);
                    cb = __double2float_rn(xb);
                }
                const uint16_t a0 = win_bf16_bits(ca), b0 = win_bf16_bits(cb);
                const float ra = __fsub_rn(ca, win_bf16_val(a0)), rb = __fsub_rn(cb, win_bf16_val(b0));
                const uint16_t a1 = win_bf16_bits(ra), b1 = win_bf16_bits(rb);
                const uint16_t a2 = win_bf16_bits(__fsub_rn(ra, win_bf16_val(a1)));
                const uint16_t b2 = win_bf16_bits(__fsub_rn(rb, win_bf16_val(b1)));
                uint8_t* dst = sB + sk * 3u * (uint32_t)(N * 32) + win_off((uint32_t)f, kk);
                *reinterpret_cast<uint32_t*>(dst) = (uint32_t)a0 | ((uint32_t)b0 << 16);
                *reinterpret_cast<uint32_t*>(dst + (uint32_t)(N * 32)) = (uint32_t)a1 | ((uint32_t)b1 << 16);
                *reinterpret_cast<uint32_t*>(dst + 2u * (uint32_t)(N * 32)) = (uint32_t)a2 | ((uint32_t)b2 << 16);
                if (cora >= 0) sCorner[cora * kWinMaxN + f] = ca;
                if (corb >= 0) sCorner[corb * kWinMaxN + f] = cb;
            }
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        win_tc_fence_before();
        __syncthreads();
        win_tc_fence_after();
        // 3. one thread issues the 48 MMAs and commits them to the barrier
        if (tid == 0) {
            for (uint32_t m = 0; m < 4u; ++m)
                for (uint32_t s = 0; s < 4u; ++s) {
                    const uint64_t ad = win_desc(win_smem_u32(sA + (m * 4u + s) * 4096u));
                    for (uint32_t p = 0; p < 3u; ++p) {
                        const uint64_t bd = win_desc(win_smem_u32(sB + (s * 3u + p) * (uint32_t)(N * 32)));
                        win_mma(taddr + m * (uint32_t)N, ad, bd, idesc, (s | p) != 0u ? 1u : 0u);
                    }
                }
            win_commit(bar);
        }
        // DenseGrid leaves, while the products run: the residual grids in place of the coarse
        // coefficients (no longer read) -- the per-frame BFP grid of every frame of the window,
        // or the temporal-basis grids (render/src/scientific_decode.cpp:125-233), decoded as the
        // per-frame path decodes them (sci_decode_controls)
        const int dres = mode == 2u ? 3 : 4, dper = dres * dres * dres;
        const int dbits = (int)((hdr >> 8) & 0xFu);
        const uint32_t dsub = (hdr >> 12) & 7u;
        const int dtkeep = (int)((hdr >> 15) & 0xFu) + 1;
        if (mode >= 2u) {
            const uint64_t scales = base + 4u + (uint64_t)(64 * (keep + 1));
            if (dsub == 1u) {
                const int bbytes = (dper * dbits + 7) / 8;
                const uint64_t data = scales + (uint64_t)(dtkeep * 2);
                if (dbits > 0)
                    for (int i = tid; i < dtkeep * dper; i += kWinThreads) {
                        const int k = i / dper, ci = i % dper;
                        const float sc = half_bits_to_float(rd.u16(scales + (uint64_t)(k * 2)));
                        sQ[i] = bfp_sample(rd, data + (uint64_t)(k * bbytes), dres, dbits, sc, ci);
                    }
            } else {
                const int fbytes = (dper * dbits + 7) / 8;
                for (int i = tid; i < n * dper; i += kWinThreads) {
                    const int f = i / dper, ci = i % dper;
                    const uint32_t t = (uint32_t)(t0 + f);
                    const uint64_t data = scales + (uint64_t)a.g.frames * 2u + (uint64_t)t * fbytes;
                    const float sc = half_bits_to_float(rd.u16(scales + t * 2u));
                    sQ[i] = bfp_sample(rd, data, dres, dbits, sc, ci);
                }
            }
        }
        // SparseEvents leaves with scattered events, while the products run: the 4-bit residual
        // code q of every event that a window frame's search would find, as nibble f & 7 of word
        // (f >> 3) * 512 + voxel of a table in place of the coefficients (all zeros elsewhere).
        // An event key (lt << 9 | voxel) of bin b belongs to the frames b * fpb + lt for b < 15
        // (lt < fpb), and for the last bin to every frame 15 * fpb + lt + 128 j (the search key
        // keeps 7 bits of the local time).  The bin ranges follow one another (kFlagSorted), so the
        // events of the window's bins are one run and each event finds its bin among 16 starts.
        uint32_t* s_ev = reinterpret_cast<uint32_t*>(sQ);
        if (scatter) {
            for (int i = tid; i < (int)(kWinQ / 16u); i += kWinThreads)
                reinterpret_cast<uint4*>(s_ev)[i] = make_uint4(0u, 0u, 0u, 0u);
            __syncthreads();
            const SparseLeaf sp = *s_sparse;
            const uint64_t cb = sp.bb + 32u, rb = cb + sp.cap * 2u;
            const uint32_t t1 = (uint32_t)(t0 + n);
            const uint32_t b_lo = min(15u, (uint32_t)t0 / sp.fpb), b_hi = min(15u, (t1 - 1u) / sp.fpb);
            const uint32_t e_lo = s_bin[b_lo], e_hi = b_hi < 15u ? s_bin[b_hi + 1u] : (sp.count & 0xFFFFu);
            for (uint32_t ev = e_lo + (uint32_t)tid; ev < e_hi; ev += kWinThreads) {
                uint32_t b = b_lo;
                while (b < b_hi && s_bin[b + 1u] <= ev) ++b;
                const uint32_t key = sp.inside ? (pay_u32(a.payload, cb + 2u * ev) & 0xFFFFu) : rd.u16(cb + 2u * ev);
                const uint32_t lt = key >> 9, li = key & 511u;
                if (b < 15u && lt >= sp.fpb) continue;
                const uint32_t byte = sp.inside ? (pay_u32(a.payload, rb + (ev >> 1)) & 0xFFu) : rd.byte(rb + (ev >> 1));
                const uint32_t nib = (ev & 1u) == 0u ? (byte & 0xFu) : ((byte >> 4) & 0xFu);
                const uint32_t tend = b < 15u ? min((b + 1u) * sp.fpb, a.g.frames) : a.g.frames;
                for (uint32_t t = b * sp.fpb + lt; t < tend && t < t1; t += 128u)
                    if (t >= (uint32_t)t0) {
                        const uint32_t f = t - (uint32_t)t0;
                        atomicOr(s_ev + (f >> 3) * 512u + li, nib << ((f & 7u) * 4u));
                    }
            }
        }
        // 4. wait for the products (bounded): one thread polls the barrier while the others sleep
        //    in the CTA barrier (no issue slots spent spinning); a timeout stops the whole CTA
        //    after a second wait
        bool ok = true;
        if (tid == 0) ok = mbar_wait(bar, phase);
        if (__syncthreads_or(!ok)) {
            if (tid == 0) {
                record_error(a.err, leaf, kErrWaitTimeout);
                mbar_wait(bar, phase);
            }
            break;
        }
        phase ^= 1u;
        win_tc_fence_after();
        // 5. epilogue: warp w reads lanes 32 (w % 4) .. +31 (voxel rows), half of the columns;
        //    voxels outside a boundary leaf's extent are 0, as in the per-frame cache
        uint32_t gx, gy, gz;
        int ew, eh, ed;
        leaf_extent(a.g, leaf, gx, gy, gz, ew, eh, ed);
        const uint32_t quarter = (uint32_t)(warp & 3), half = (uint32_t)(warp >> 2);
        const uint32_t row = quarter * 32u + (uint32_t)lane;
        const int cols_per_half = N / 2;
        const bool full_leaf = ew == 8 && eh == 8 && ed == 8;
        for (uint32_t m = 0; m < 4u; ++m) {
            const uint32_t v = m * 128u + row;
            const int corner = win_corner_of_voxel(v);
            const bool inside = (int)(v & 7u) < ew && (int)((v >> 3) & 7u) < eh && (int)(v >> 6) < ed;
            const bool events = mode == 1u && !scatter && ((s_mask[v >> 5] >> (v & 31u)) & 1u) != 0u;
            // the branch is taken by whole warps: tcgen05.ld is a warp-wide instruction that every
            // lane must issue together (a warp with any searched voxel takes the general case,
            // whose operations for the others are the same as here)
            if (mode <= 1u && !__any_sync(0xFFFFFFFFu, events)) {
                // no residual at this voxel (CoarseOnly, or none here), or the scattered events of
                // the table: D (+ the corner term) / 343 (+ q * es), the same operations as the
                // general case (an absent event is q = 0, which adds +0 as the search's 0 does)
                const bool wcorner = __any_sync(0xFFFFFFFFu, corner >= 0);
                const float es = scatter ? s_sparse->es : 0.0f;
                for (int c0 = (int)half * cols_per_half; c0 < (int)(half + 1) * cols_per_half; c0 += 16) {
                    float d[16];
                    win_ld16(taddr + ((quarter * 32u) << 16) + m * (uint32_t)N + (uint32_t)c0, d);
                    uint32_t q0 = 0u, q1 = 0u;
                    if (scatter) {
                        q0 = s_ev[(uint32_t)(c0 >> 3) * 512u + v];
                        q1 = s_ev[(uint32_t)((c0 >> 3) + 1) * 512u + v];
                    }
                    float* o = out + (uint64_t)c0 * frame_stride + (uint64_t)leaf * 512u + v;
                    // the common chunk -- 16 frames inside the window, a full leaf, no corner voxel
                    // in the warp -- without the per-output tests (same operations)
                    if (!wcorner && full_leaf && c0 + 16 <= n) {
                        if (scatter) {
                            // q as a float without a conversion: the code's bits (sign bit
                            // flipped) in the mantissa of 1.5 * 2^23, minus 1.5 * 2^23 + 8 (exact)
                            const uint32_t x0 = q0 ^ 0x88888888u, x1 = q1 ^ 0x88888888u;
#pragma unroll
                            for (int j = 0; j < 16; ++j) {
                                const uint32_t u = ((j < 8 ? x0 : x1) >> (4 * (j & 7))) & 0xFu;
                                const float qf = __fsub_rn(__uint_as_float(0x4B400000u | u), 12582920.0f);
                                *o = __fadd_rn(__fmul_rn(d[j], 1.0f / 343.0f), __fmul_rn(qf, es));
                                o += frame_stride;
                            }
                        } else if (mode == 1u) {
#pragma unroll
                            for (int j = 0; j < 16; ++j) {
                                *o = __fadd_rn(__fmul_rn(d[j], 1.0f / 343.0f), 0.0f);
                                o += frame_stride;
                            }
                        } else {
#pragma unroll
                            for (int j = 0; j < 16; ++j) {
                                *o = __fmul_rn(d[j], 1.0f / 343.0f);
                                o += frame_stride;
                            }
                        }
                        continue;
                    }
#pragma unroll
                    for (int j = 0; j < 16; ++j) {
                        if (c0 + j < n) {
                            float val = d[j];
                            if (corner >= 0) val = __fadd_rn(val, sCorner[corner * kWinMaxN + c0 + j]);
                            val = __fmul_rn(val, 1.0f / 343.0f);
                            if (mode == 1u) {
                                const int q = ((int)((j < 8 ? q0 : q1) << (28 - 4 * (j & 7)))) >> 28;
                                val = __fadd_rn(val, scatter ? __fmul_rn((float)q, es) : 0.0f);
                            }
                            o[(uint64_t)j * frame_stride] = inside ? val : 0.0f;
                        }
                    }
                }
                continue;
            }
            const int dsel = mode == 2u ? 1 : 2;
            const AxisWeight dx = c_sci_axis[dsel][v & 7u], dy = c_sci_axis[dsel][(v >> 3) & 7u],
                             dz = c_sci_axis[dsel][v >> 6];
            for (int c0 = (int)half * cols_per_half; c0 < (int)(half + 1) * cols_per_half; c0 += 16) {
                float d[16];
                win_ld16(taddr + ((quarter * 32u) << 16) + m * (uint32_t)N + (uint32_t)c0, d);
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const int f = c0 + j;
                    if (f < n) {
                        float val = d[j];
                        if (corner >= 0) val = __fadd_rn(val, sCorner[corner * kWinMaxN + f]);
                        val = __fmul_rn(val, 1.0f / 343.0f);
                        if (mode == 1u) {
                            val = __fadd_rn(val, events ? sparse_at(rd, *s_sparse, v, (uint32_t)(t0 + f)) : 0.0f);
                        } else if (mode >= 2u) {
                            float r = 0.0f;
                            if (dsub == 1u) {
                                if (dbits > 0) {
                                    const float* brow = a.basis + (uint64_t)(t0 + f) * 64u;
                                    for (int k = 0; k < dtkeep; ++k)
                                        r = __fadd_rn(r, __fmul_rn(tri_small(sQ + k * dper, dres, dx, dy, dz),
                                                                   __ldg(brow + k)));
                                }
                            } else {
                                r = tri_small(sQ + f * dper, dres, dx, dy, dz);
                            }
                            val = __fadd_rn(val, r);
                        }
                        out[(uint64_t)f * frame_stride + (uint64_t)leaf * 512u + v] = inside ? val : 0.0f;
                    }
                }
            }
        }
        if (rd.oob) record_error(a.err, leaf, kErrDecodeOob);
        win_tc_fence_before();
        __syncthreads();   // D and the B tiles are free for the next leaf
        win_tc_fence_after();
    }
    win_tc_fence_before();
    __syncthreads();
    win_tc_fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(kWinTmemCols) : "memory");
}

// FP64 error oracle of a window (any scientific output of frames [t0, t0 + n) in the cache
// layout; voxels outside a boundary leaf's extent must be 0): per voxel and frame the reference
// model evaluated in double -- the coarse controls
// as sum_k q_k b_k(t) over the same FP32 coefficients and basis values, the trilinear weights as
// the reference's FP32 t and 1 - t, both without rounding, plus the FP32 sparse residual -- and
// the reduction stats[0] = max |value - oracle| (as ordered bits), stats[1] = sum of squares,
// stats[2] / stats[3] = oracle min / max (as ordered bits), in double.
__device__ __forceinline__ unsigned long long win_ordered(double x)
{
    const unsigned long long b = __double_as_longlong(x);
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}

// The DenseGrid residual of voxel (lx, ly, lz) at frame t in double without intermediate rounding:
// the decoded BFP samples and the reference's FP32 axis weights, the per-frame grid or the sum of
// the temporal-basis grids times the basis values (render/src/scientific_decode.cpp:125-233).
__device__ double dense_residual_f64(const DeviceAsset& a, SciReader& rd, uint64_t base, uint32_t hdr, int keep,
                                     uint32_t lx, uint32_t ly, uint32_t lz, uint32_t t)
{
    const uint32_t mode = hdr & 3u;
    const int res = mode == 2u ? 3 : 4, per = res * res * res;
    const int bits = (int)((hdr >> 8) & 0xFu);
    const uint32_t sub = (hdr >> 12) & 7u;
    const int tkeep = (int)((hdr >> 15) & 0xFu) + 1;
    const int sel = mode == 2u ? 1 : 2;
    const AxisWeight ax = c_sci_axis[sel][lx], ay = c_sci_axis[sel][ly], az = c_sci_axis[sel][lz];
    const uint64_t scales = base + 4u + (uint64_t)(64 * (keep + 1));
    auto tri = [&](uint64_t data, float sc) {
        double r = 0.0;
        for (int cz = 0; cz < 2; ++cz)
            for (int cy = 0; cy < 2; ++cy)
                for (int cx = 0; cx < 2; ++cx) {
                    const int ci = ((cz ? az.i1 : az.i0) * res + (cy ? ay.i1 : ay.i0)) * res + (cx ? ax.i1 : ax.i0);
                    const double w = (double)(cx ? ax.t : ax.omt) * (double)(cy ? ay.t : ay.omt) *
                                     (double)(cz ? az.t : az.omt);
                    r += w * (double)bfp_sample(rd, data, res, bits, sc, ci);
                }
        return r;
    };
    if (sub == 1u) {
        if (bits <= 0) return 0.0;
        const int bbytes = (per * bits + 7) / 8;
        const uint64_t data = scales + (uint64_t)(tkeep * 2);
        const float* brow = a.basis + (uint64_t)t * 64u;
        double r = 0.0;
        for (int k = 0; k < tkeep; ++k)
            r += tri(data + (uint64_t)(k * bbytes), half_bits_to_float(rd.u16(scales + (uint64_t)(k * 2)))) *
                 (double)__ldg(brow + k);
        return r;
    }
    const int fbytes = (per * bits + 7) / 8;
    return tri(scales + (uint64_t)a.g.frames * 2u + (uint64_t)t * fbytes, half_bits_to_float(rd.u16(scales + t * 2u)));
}

__global__ void __launch_bounds__(256) sci_window_oracle_kernel(DeviceAsset a, int t0, int n,
                                                                const float* __restrict__ vals, uint64_t frame_stride,
                                                                unsigned long long* stats)
{
    __shared__ double s_max[8], s_sum[8];
    __shared__ unsigned long long s_lo[8], s_hi[8];
    double my_max = 0.0, my_sum = 0.0;
    unsigned long long my_lo = ~0ull, my_hi = 0ull;
    const uint64_t items = (uint64_t)a.g.leaf_count * 512u;
    for (uint64_t it = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; it < items;
         it += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t leaf = (uint32_t)(it >> 9), v = (uint32_t)(it & 511u);
        const LeafEntry e = a.entries[leaf];
        const uint32_t hdr = e.header, mode = hdr & 3u;
        if (entry_status(e) != kOk) continue;
        const int keep = (int)((hdr >> 2) & 0x3Fu) + 1;
        const uint64_t base = 4ull * e.word_off;
        SciReader rd{a.payload, a.g.payload_words, false};
        const uint32_t lx = v & 7u, ly = (v >> 3) & 7u, lz = v >> 6;
        uint32_t gx, gy, gz;
        int ew, eh, ed;
        leaf_extent(a.g, leaf, gx, gy, gz, ew, eh, ed);
        if ((int)lx >= ew || (int)ly >= eh || (int)lz >= ed) {   // outside the volume: the cache holds 0
            for (int f = 0; f < n; ++f)
                my_max = fmax(my_max, fabs((double)vals[(uint64_t)f * frame_stride + (uint64_t)leaf * 512u + v]));
            continue;
        }
        const AxisWeight ax = c_sci_axis[0][lx], ay = c_sci_axis[0][ly], az = c_sci_axis[0][lz];
        for (int f = 0; f < n; ++f) {
            const uint32_t t = (uint32_t)(t0 + f);
            const float* brow = a.basis + (uint64_t)t * 64u;
            double ref = 0.0;
            for (int cz = 0; cz < 2; ++cz)
                for (int cy = 0; cy < 2; ++cy)
                    for (int cx = 0; cx < 2; ++cx) {
                        const int ci = ((cz ? az.i1 : az.i0) * 4 + (cy ? ay.i1 : ay.i0)) * 4 + (cx ? ax.i1 : ax.i0);
                        const double w = (double)(cx ? ax.t : ax.omt) * (double)(cy ? ay.t : ay.omt) *
                                         (double)(cz ? az.t : az.omt);
                        const uint64_t cb = base + 4u + (uint64_t)ci * (keep + 1);
                        double c = (double)half_bits_to_float(rd.u16(cb)) * (double)__ldg(brow);
                        for (int k = 1; k < keep; ++k) {
                            const float q = __fmul_rn((float)(int8_t)rd.byte(cb + 2u + (k - 1)), __ldg(a.scales + k - 1));
                            c += (double)q * (double)__ldg(brow + k);
                        }
                        ref += w * c;
                    }
            if (mode == 1u) ref += (double)sci_sparse(rd, base, hdr, keep, v, t);
            else if (mode >= 2u) ref += dense_residual_f64(a, rd, base, hdr, keep, lx, ly, lz, t);
            const double got = (double)vals[(uint64_t)f * frame_stride + (uint64_t)leaf * 512u + v];
            const double err = fabs(got - ref);
            my_max = fmax(my_max, err);
            my_sum += err * err;
            const unsigned long long o = win_ordered(ref);
            my_lo = o < my_lo ? o : my_lo;
            my_hi = o > my_hi ? o : my_hi;
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
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
        s_max[warp] = my_max;
        s_sum[warp] = my_sum;
        s_lo[warp] = my_lo;
        s_hi[warp] = my_hi;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double mx = 0.0, sm = 0.0;
        unsigned long long lo = ~0ull, hi = 0ull;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
            mx = fmax(mx, s_max[w]);
            sm += s_sum[w];
            lo = s_lo[w] < lo ? s_lo[w] : lo;
            hi = s_hi[w] > hi ? s_hi[w] : hi;
        }
        atomicMax(stats + 0, (unsigned long long)__double_as_longlong(mx));   // non-negative: bits order
        atomicAdd(reinterpret_cast<double*>(stats + 1), sm);
        atomicMin(stats + 2, lo);
        atomicMax(stats + 3, hi);
    }
}

void launch_sci_window(const DeviceAsset& a, int t0, int n, float* out, uint64_t frame_stride, cudaStream_t s)
{
    cudaFuncSetAttribute(sci_window_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kWinSmem);
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int grid = (int)(a.g.leaf_count < (uint32_t)(2 * sms) ? a.g.leaf_count : (uint32_t)(2 * sms));
    sci_window_kernel<<<grid, kWinThreads, kWinSmem, s>>>(a, t0, n, out, frame_stride);
}

void launch_sci_window_oracle(const DeviceAsset& a, int t0, int n, const float* vals, uint64_t frame_stride,
                              unsigned long long* stats, cudaStream_t s)
{
    cudaMemsetAsync(stats, 0, 4 * sizeof(unsigned long long), s);       // max, sum (0.0), -, max
    cudaMemsetAsync(stats + 2, 0xFF, sizeof(unsigned long long), s);   // min starts at the top
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    sci_window_oracle_kernel<<<4 * sms, 256, 0, s>>>(a, t0, n, vals, frame_stride, stats);
}

}  // namespace vbtb
