// rt_staged.cuh -- render-temporal leaf decode from a shared-memory copy of the leaf (or, for
// leaves larger than the stage, straight from the payload through the same word reader).
//
// The leaf's bytes are brought into shared memory by one TMA bulk copy (cp.async.bulk,
// completion on an mbarrier), so the per-control keyframe walks -- chains of dependent 3-byte
// reads -- run at shared-memory latency instead of L2 latency.  The copied window is the leaf
// rounded out to 16-byte boundaries (the payload allocation is 16-byte aligned and padded by 16
// bytes, so the window never leaves it).
//
// Controls: leaves whose key frames strictly increase (checked once per asset) are walked by a
// cursor that reads each key once -- for such keys the reference's hinted bracket search returns
// the first key's value before it, the last key's value after it, the key's value on an exact hit
// and v0 + a (v1 - v0) with a = (t - f0) / (f1 - f0) for the adjacent pair around t, so a cursor
// k = "first key with frame > t" that only moves forward yields the same bits; other leaves, and
// frame lists that go backwards, use the reference's search (src/render_temporal_decode.cpp:79-131).
//
// Voxels: the reference's trilinear (render/src/render_smoke_vbt_bench_main.cpp:236-267) lerps
// along x first, then y, then z:  c00 = lerp_x(g[z0][y0][x0], g[z0][y0][x1]), c0 = lerp_y(c00,
// c10), v = lerp_z(c0, c1).  The x-lerp depends only on (lx, control row y, control row z), and
// the y-lerp only on (lx, ly, control row z), so they are computed once per leaf and frame
// (R*R*8 and R*64 lerps) and shared by every voxel that uses them: the same operations on the
// same operands in the same order, hence the same bits, with 4-6x fewer lerps than per voxel.
#pragma once
#include <cuda_fp16.h>

#include "rt_search.cuh"

namespace vbtb {

// Two lerps side by side, each a*(1-t) + b*t rounded after every operation.  Scalar _rn
// operations on purpose: a packed FP32x2 multiply followed by a packed add is contracted into a
// packed FMA by this toolkit's assembler even when both carry .rn (measured on sm_100a: every
// packed multiply and every packed add alone rounds like the scalar one, the pair does not),
// which would break bit-equality with the reference's separately rounded float arithmetic.
__device__ __forceinline__ float2 add2_rn(float2 a, float2 b)
{
    return make_float2(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y));
}

__device__ __forceinline__ float2 lerp2(float2 a, float2 b, float2 t, float2 omt)
{
    return make_float2(__fadd_rn(__fmul_rn(a.x, omt.x), __fmul_rn(b.x, t.x)),
                       __fadd_rn(__fmul_rn(a.y, omt.y), __fmul_rn(b.y, t.y)));
}

// binary16 -> binary32 with the hardware conversion; NaNs keep their payload bits exactly as
// src/render_temporal_decode.cpp:167-199 maps them.
__device__ __forceinline__ float half_to_float_exact(uint32_t h)
{
    const float f = __half2float(__ushort_as_half((unsigned short)h));
    const bool nan = (h & 0x7C00u) == 0x7C00u && (h & 0x3FFu) != 0u;
    return nan ? __uint_as_float(((h & 0x8000u) << 16) | 0x7F800000u | ((h & 0x3FFu) << 13)) : f;
}

__device__ __forceinline__ uint32_t row_byte(uint32_t r0, uint32_t r1, uint32_t b)
{
    return ((b < 4u ? r0 : r1) >> ((b & 3u) * 8u)) & 0xFFu;
}


// Word readers: global (read-only path) or a shared-memory window that starts at word `w0`.
struct GlobalWords {
    const uint32_t* __restrict__ pw;
    __device__ __forceinline__ uint32_t operator()(uint32_t i) const { return __ldg(pw + i); }
};
struct SharedWords {
    const uint32_t* s;
    uint32_t w0;
    __device__ __forceinline__ uint32_t operator()(uint32_t i) const { return s[i - w0]; }
};

template <class M>
__device__ __forceinline__ uint32_t m_key24(const M& m, uint64_t b)
{
    const uint32_t w = (uint32_t)(b >> 2);
    const uint32_t sh = (uint32_t)(b & 3u) * 8u;
    const uint32_t lo = m(w);
    if (sh <= 8u) return (lo >> sh) & 0xFFFFFFu;
    return __funnelshift_r(lo, m(w + 1u), sh) & 0xFFFFFFu;
}

template <class M>
__device__ __forceinline__ int m_key_frame(const M& m, uint64_t kb, uint32_t codec, uint32_t i)
{
    if (codec == 1u) return (int)(m((uint32_t)((kb + 8ull * i) >> 2)) & 0xFFFFu);
    const uint64_t b = kb + 3ull * i;
    return (int)((m((uint32_t)(b >> 2)) >> ((uint32_t)(b & 3u) * 8u)) & 0xFFu);
}

template <class M>
__device__ __forceinline__ void m_key_read(const M& m, uint64_t kb, uint32_t codec, uint32_t i, int& frame,
                                           float& value)
{
    if (codec == 1u) {
        const uint32_t w = (uint32_t)((kb + 8ull * i) >> 2);
        frame = (int)(m(w) & 0xFFFFu);
        value = __uint_as_float(m(w + 1u));
    } else {
        const uint32_t k = m_key24(m, kb + 3ull * i);
        frame = (int)(k & 0xFFu);
        value = half_to_float_exact(k >> 8);
    }
}

struct FrameBatch {
    const int* fr;          // clamped frames
    const uint8_t* b8;      // time bins for 8-bin streams
    const uint8_t* b4;      // time bins for 4-bin streams
    int nb;
};

// Cursor walk (strictly increasing key frames, non-decreasing frames); see the
// head of this file for why it equals the reference's search.
template <class M>
__device__ __forceinline__ void m_control_cursor(const M& m, const StreamRef& s, uint32_t c, const FrameBatch& fb,
                                                 float* dst, int stride)
{
    const uint32_t desc = m((uint32_t)((s.base + 4ull * c) >> 2));
    const uint32_t kc = (desc >> 16) & 0xFFu;
    if (kc == 0u || (desc & 0xFFFFu) + kc > s.kf) {   // see decode_control (rt_search.cuh)
        for (int j = 0; j < fb.nb; ++j) dst[j * stride] = 0.0f;
        return;
    }
    const uint32_t ks = desc & 0xFFFFu;
    const uint64_t kb = stream_key_base(s);
    const int t0 = fb.fr[0];
    const uint32_t bin = s.bins == 8u ? fb.b8[0] : fb.b4[0];
    const uint64_t row = s.base + 4ull * s.controls + (uint64_t)c * s.bins;
    const uint32_t hb = (m((uint32_t)((row + (bin & ~3u)) >> 2)) >> ((bin & 3u) * 8u)) & 0xFFu;
    uint32_t k = hb < kc - 1u ? hb : kc - 1u;
    if (m_key_frame(m, kb, s.codec, ks + k) > t0) {
        uint32_t lo = 0, hi = k;
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (m_key_frame(m, kb, s.codec, ks + mid) > t0) hi = mid;
            else lo = mid + 1u;
        }
        k = lo;
    } else {
        ++k;
        while (k < kc && m_key_frame(m, kb, s.codec, ks + k) <= t0) ++k;
    }
    int fp = 0, fn = 0;
    float vp = 0.0f, vn = 0.0f;
    if (k > 0u) m_key_read(m, kb, s.codec, ks + k - 1u, fp, vp);
    if (k < kc) m_key_read(m, kb, s.codec, ks + k, fn, vn);
    for (int j = 0; j < fb.nb; ++j) {
        const int t = fb.fr[j];
        while (k < kc && fn <= t) {
            fp = fn;
            vp = vn;
            ++k;
            if (k < kc) m_key_read(m, kb, s.codec, ks + k, fn, vn);
        }
        float out;
        if (k == 0u) out = vn;
        else if (k == kc || fp == t) out = vp;
        else {
            const float alpha = __fdiv_rn((float)(t - fp), (float)(fn - fp));
            out = __fadd_rn(vp, __fmul_rn(alpha, __fsub_rn(vn, vp)));
        }
        dst[j * stride] = out;
    }
}

// Correctly rounded a / b for integers 0 < a < b < 2^16 given y = RN(1/b), without a division:
// q0 = RN(a y) is within one ulp of a / b, the remainder a - b q0 is exact in one fused
// multiply-add, and RN(q0 + r y) is the correctly rounded quotient (P. Markstein, "Computation of
// elementary functions on the IBM RISC System/6000 processor", IBM J. Res. Dev. 34(1), 1990).
// vbt_selftest_key_division checks it against IEEE division for every such pair.
__device__ __forceinline__ float div_small_rn(float a, float b, float y)
{
    const float q0 = __fmul_rn(a, y);
    const float r = __fmaf_rn(-q0, b, a);
    return __fmaf_rn(r, y, q0);
}

// Key read with no data-dependent branch: a 3-byte key is always taken from two words (the
// shared-memory stage and the payload both carry 16 bytes of padding past any key).
template <class M>
__device__ __forceinline__ void m_key_read_nb(const M& m, uint64_t kb, uint32_t codec, uint32_t i, int& frame,
                                              float& value)
{
    if (codec == 1u) {
        const uint32_t w = (uint32_t)((kb + 8ull * i) >> 2);
        frame = (int)(m(w) & 0xFFFFu);
        value = __uint_as_float(m(w + 1u));
    } else {
        const uint64_t b = kb + 3ull * i;
        const uint32_t w = (uint32_t)(b >> 2);
        const uint32_t k = __funnelshift_r(m(w), m(w + 1u), (uint32_t)(b & 3u) * 8u) & 0xFFFFFFu;
        frame = (int)(k & 0xFFu);
        value = half_to_float_exact(k >> 8);
    }
}

// Streaming cursor over frames t0, t1, ... with t(j+1) - t(j) in {0, 1} (a clamped timeline
// window), for a control whose key frames strictly increase.  The cursor k (first key with
// frame > t) then advances at most once per frame, so the key after next is prefetched one
// advance ahead and no frame waits on a load.  Per key interval the span b = f1 - f0, its
// reciprocal RN(1/b) (`rcp`, a table of RN(1/i) for i < 256) and the difference v1 - v0 are
// formed once; per frame the value is v0 + RN(RN((t - f0) / b) * (v1 - v0)), the quotient by
// div_small_rn, the first key's value before it, the last key's after it and the key's value on
// an exact hit -- the bits of the reference's search (see the head of
// this file), with selects instead of branches.
template <class M>
__device__ __forceinline__ void m_control_stream(const M& m, const StreamRef& s, uint32_t c, const int* fr,
                                                 uint32_t bin0, int n, float* dst, int stride,
                                                 const float* __restrict__ rcp)
{
    const uint32_t desc = m((uint32_t)((s.base + 4ull * c) >> 2));
    const uint32_t kc = (desc >> 16) & 0xFFu;
    if (kc == 0u || (desc & 0xFFFFu) + kc > s.kf) {   // see decode_control (rt_search.cuh)
        for (int j = 0; j < n; ++j) dst[j * stride] = 0.0f;
        return;
    }
    const uint32_t ks = desc & 0xFFFFu;
    const uint64_t kb = stream_key_base(s);
    const int t0 = fr[0];
    const uint64_t row = s.base + 4ull * s.controls + (uint64_t)c * s.bins;
    const uint32_t hb = (m((uint32_t)((row + (bin0 & ~3u)) >> 2)) >> ((bin0 & 3u) * 8u)) & 0xFFu;
    uint32_t k = hb < kc - 1u ? hb : kc - 1u;
    if (m_key_frame(m, kb, s.codec, ks + k) > t0) {
        uint32_t lo = 0, hi = k;
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (m_key_frame(m, kb, s.codec, ks + mid) > t0) hi = mid;
            else lo = mid + 1u;
        }
        k = lo;
    } else {
        ++k;
        while (k < kc && m_key_frame(m, kb, s.codec, ks + k) <= t0) ++k;
    }
    int fp = 0, fn = 0, fnn = 0;
    float vp = 0.0f, vn = 0.0f, vnn = 0.0f;
    if (k > 0u) m_key_read_nb(m, kb, s.codec, ks + k - 1u, fp, vp);
    if (k < kc) m_key_read_nb(m, kb, s.codec, ks + k, fn, vn);
    if (k + 1u < kc) m_key_read_nb(m, kb, s.codec, ks + k + 1u, fnn, vnn);
    // the interval [fp, fn); outside 0 < k < kc its values are never selected
    float bf, y, d;
    auto interval = [&]() {
        const uint32_t b = (uint32_t)(fn - fp);
        bf = (float)(int)b;
        y = b < 256u ? rcp[b] : __frcp_rn(bf);
        d = __fsub_rn(vn, vp);
    };
    interval();
    for (int j = 0; j < n; ++j) {
        const int t = fr[j];
        if (k < kc && fn <= t) {
            fp = fn;
            vp = vn;
            fn = fnn;
            vn = vnn;
            ++k;
            if (k + 1u < kc) m_key_read_nb(m, kb, s.codec, ks + k + 1u, fnn, vnn);
            interval();
        }
        const int ai = t - fp;
        const float lerp = __fadd_rn(vp, __fmul_rn(div_small_rn((float)ai, bf, y), d));
        dst[j * stride] = k == 0u ? vn : ((k == kc || ai == 0) ? vp : lerp);
    }
}

// The reference's hinted bracket search for one frame (src/render_temporal_decode.cpp:79-131) on a
// control with keys [ks, ks + kc), kc > 0: kind 1 = the value v0, kind 2 = the value v1,
// kind 3 = v0 + (frame - f0) / (f1 - f0) * (v1 - v0).  r0 / r1 hold the control's bin hint bytes.
struct Bracket {
    int kind, f0, f1;
    float v0, v1;
};

template <class M>
__device__ __forceinline__ Bracket m_search_bracket(const M& m, uint64_t kb, uint32_t codec, uint32_t ks, uint32_t kc,
                                                    uint32_t bins, uint32_t r0, uint32_t r1, int frame, uint32_t bin)
{
    const uint32_t last = kc - 1u;
    const uint32_t hb = row_byte(r0, r1, bin);
    uint32_t lo = hb < last ? hb : last;
    Bracket b{1, 0, 0, 0.0f, 0.0f};
    m_key_read(m, kb, codec, ks + lo, b.f0, b.v0);
    if (b.f0 > frame) {
        lo = 0u;
        m_key_read(m, kb, codec, ks, b.f0, b.v0);
    }
    if (b.f0 >= frame || lo == last) return b;
    uint32_t hi = last;
    if (bin + 1u < bins) {
        const uint32_t h = row_byte(r0, r1, bin + 1u) + 1u;
        hi = h < last ? h : last;
    }
    if (hi < lo + 1u) hi = lo + 1u;
    m_key_read(m, kb, codec, ks + hi, b.f1, b.v1);
    if (b.f1 < frame) {
        hi = last;
        m_key_read(m, kb, codec, ks + hi, b.f1, b.v1);
    }
    if (b.f1 <= frame) {
        b.kind = 2;
        return b;
    }
    bool moved_lo = false, moved_hi = false;
    while (hi > lo + 1u) {
        const uint32_t mid = lo + (hi - lo) / 2u;
        const int fm = m_key_frame(m, kb, codec, ks + mid);
        if (fm < frame) {
            lo = mid;
            b.f0 = fm;
            moved_lo = true;
        } else {
            hi = mid;
            b.f1 = fm;
            moved_hi = true;
        }
    }
    if (moved_hi) m_key_read(m, kb, codec, ks + hi, b.f1, b.v1);
    if (b.f1 == frame) {
        b.kind = 2;
        return b;
    }
    if (moved_lo) m_key_read(m, kb, codec, ks + lo, b.f0, b.v0);
    b.kind = 3;
    return b;
}

// The reference's search for every frame of a batch, rounded as the reference rounds.
template <class M>
__device__ __forceinline__ void m_control_search(const M& m, const StreamRef& s, uint32_t c, const FrameBatch& fb,
                                                 float* dst, int stride)
{
    const uint32_t desc = m((uint32_t)((s.base + 4ull * c) >> 2));
    const uint64_t row = s.base + 4ull * s.controls + (uint64_t)c * s.bins;
    const uint32_t r0 = m((uint32_t)(row >> 2));
    const uint32_t r1 = s.bins == 8u ? m((uint32_t)(row >> 2) + 1u) : 0u;
    const uint32_t kc = (desc >> 16) & 0xFFu;
    if (kc == 0u || (desc & 0xFFFFu) + kc > s.kf) {
        for (int j = 0; j < fb.nb; ++j) dst[j * stride] = 0.0f;
        return;
    }
    const uint32_t ks = desc & 0xFFFFu;
    const uint64_t kb = stream_key_base(s);
    const uint8_t* bins_of_frame = s.bins == 8u ? fb.b8 : fb.b4;
    for (int j = 0; j < fb.nb; ++j) {
        const int frame = fb.fr[j];
        const Bracket b = m_search_bracket(m, kb, s.codec, ks, kc, s.bins, r0, r1, frame, bins_of_frame[j]);
        float out;
        if (b.kind == 1) out = b.v0;
        else if (b.kind == 2) out = b.v1;
        else {
            const float alpha = __fdiv_rn((float)(frame - b.f0), (float)(b.f1 - b.f0));
            out = __fadd_rn(b.v0, __fmul_rn(alpha, __fsub_rn(b.v1, b.v0)));
        }
        dst[j * stride] = out;
    }
}

// The same control value in double without intermediate rounding (the FP64 error oracle): the
// bracket the reference's search selects, interpolated exactly.
template <class M>
__device__ __forceinline__ double m_control_value_f64(const M& m, const StreamRef& s, uint32_t c, int frame,
                                                      uint32_t bin)
{
    const uint32_t desc = m((uint32_t)((s.base + 4ull * c) >> 2));
    const uint64_t row = s.base + 4ull * s.controls + (uint64_t)c * s.bins;
    const uint32_t r0 = m((uint32_t)(row >> 2));
    const uint32_t r1 = s.bins == 8u ? m((uint32_t)(row >> 2) + 1u) : 0u;
    const uint32_t kc = (desc >> 16) & 0xFFu;
    if (kc == 0u || (desc & 0xFFFFu) + kc > s.kf) return 0.0;
    const Bracket b = m_search_bracket(m, stream_key_base(s), s.codec, desc & 0xFFFFu, kc, s.bins, r0, r1, frame, bin);
    if (b.kind == 1) return (double)b.v0;
    if (b.kind == 2) return (double)b.v1;
    return (double)b.v0 + (double)(frame - b.f0) / (double)(b.f1 - b.f0) * ((double)b.v1 - (double)b.v0);
}

// Separable trilinear of one control grid (resolution R >= 2) for one frame.  On return each
// lane holds its 4 voxel quads: quad i covers voxels 4*(lane + 32 i) .. +3, i.e. lz = 2i +
// (lane >> 4), ly = (lane >> 1) & 7, lx = 4*(lane & 1) .. +3.
// w[axis][p] are the axis weights of this grid; x2 (R*R*4 float2) and y4 (R*16 float4) are the
// warp's scratch rows in shared memory.
__device__ __forceinline__ void trilinear_quads_ptr(const AxisWeight (*w)[8], float2* x2, float4* y4,
                                                    const float* __restrict__ g, int R, int lane, float4 q[4])
{
    // x-lerps: X[z*R + y][pair] for lx pair (2p, 2p+1)
    const int nx = R * R * 4;
    for (int it = lane; it < nx; it += 32) {
        const int row = it >> 2, p = it & 3;
        const AxisWeight wa = w[0][2 * p], wb = w[0][2 * p + 1];
        const float* gr = g + row * R;
        const float2 A = make_float2(gr[wa.i0], gr[wb.i0]);
        const float2 B = make_float2(gr[wa.i1], gr[wb.i1]);
        x2[it] = lerp2(A, B, make_float2(wa.t, wb.t), make_float2(wa.omt, wb.omt));
    }
    __syncwarp();
    // y-lerps: Y[z][ly][quad] for lx quad (4k .. 4k+3), two float2 lerps each
    const int ny = R * 16;
    for (int it = lane; it < ny; it += 32) {
        const int z = it >> 4, ly = (it >> 1) & 7, k = it & 1;
        const AxisWeight wy = w[1][ly];
        const float2* xa = x2 + (z * R + wy.i0) * 4 + 2 * k;
        const float2* xb = x2 + (z * R + wy.i1) * 4 + 2 * k;
        const float2 t = make_float2(wy.t, wy.t), omt = make_float2(wy.omt, wy.omt);
        const float2 lo2 = lerp2(xa[0], xb[0], t, omt);
        const float2 hi2 = lerp2(xa[1], xb[1], t, omt);
        y4[it] = make_float4(lo2.x, lo2.y, hi2.x, hi2.y);
    }
    __syncwarp();
    // z-lerps: the lane's four voxel quads
    const int ly = (lane >> 1) & 7, k = lane & 1;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int lz = 2 * i + (lane >> 4);
        const AxisWeight wz = w[2][lz];
        const float4 A = y4[(wz.i0 * 8 + ly) * 2 + k];
        const float4 B = y4[(wz.i1 * 8 + ly) * 2 + k];
        const float2 t = make_float2(wz.t, wz.t), omt = make_float2(wz.omt, wz.omt);
        const float2 lo2 = lerp2(make_float2(A.x, A.y), make_float2(B.x, B.y), t, omt);
        const float2 hi2 = lerp2(make_float2(A.z, A.w), make_float2(B.z, B.w), t, omt);
        q[i] = make_float4(lo2.x, lo2.y, hi2.x, hi2.y);
    }
    __syncwarp();
}

// Grid sample for resolutions 0 and 1 (no interpolation: 0, or the single control).
__device__ __forceinline__ void constant_quads(const float* __restrict__ g, int R, float4 q[4])
{
    const float v = R == 1 ? g[0] : 0.0f;
#pragma unroll
    for (int i = 0; i < 4; ++i) q[i] = make_float4(v, v, v, v);
}

// ---- TMA bulk copy global -> shared with mbarrier completion (sm_90+ PTX, no multicast) ----

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_init_fence()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Issue one bulk copy of `bytes` (multiple of 16; both addresses 16-byte aligned) and arm the
// barrier with the byte count.  The proxy fence orders this CTA's earlier generic-proxy reads of
// the destination before the async-proxy writes.
__device__ __forceinline__ void mbar_expect_and_copy(uint64_t* bar, void* dst, const void* src, uint32_t bytes)
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

// Bounded wait for phase `parity` of the mbarrier: returns false if it did not complete within
// the iteration limit (the caller records a timeout status instead of hanging).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity)
{
    for (uint32_t it = 0; it < (1u << 22); ++it) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(smem_addr(bar)), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

}  // namespace vbtb
