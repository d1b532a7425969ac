// rt_decode_v2.cuh -- render-temporal leaf decode, one warp per (leaf, frame chunk).
//
// Controls: every control of the leaf is decoded for a batch of frames at once.  Leaves whose key
// frames are strictly increasing (checked once per asset) use a forward cursor that reads each
// key once; other leaves, and frame lists that go backwards, use the reference's bracket search
// with the descriptor and bin-hint row hoisted out of the frame loop.  Both give the reference's
// bits (rt_decode.cuh).
//
// Voxels: the reference's trilinear (render/src/render_smoke_vbt_bench_main.cpp:236-267) lerps
// along x first, then y, then z:  c00 = lerp_x(g[z0][y0][x0], g[z0][y0][x1]), c0 = lerp_y(c00,
// c10), v = lerp_z(c0, c1).  The x-lerp depends only on (lx, control row y, control row z), and
// the y-lerp only on (lx, ly, control row z), so they are computed once per leaf and frame
// (R*R*8 and R*64 lerps) and shared by every voxel that uses them: the same operations on the
// same operands in the same order, hence the same bits, with 4-6x fewer lerps than per voxel.
#pragma once
#include "rt_decode.cuh"

namespace vbtb {

constexpr int kV2Warps = 4;             // warps per CTA
constexpr int kV2CtrlBudget = 1536;     // floats of control values per warp (frames x controls)
constexpr int kV2MaxBatch = 16;         // frames per control batch
constexpr int kV2ChunkFrames = 16;      // frames per work item

struct __align__(16) V2WarpSmem {
    float ctrl[kV2CtrlBudget];
    float2 x2[7 * 7 * 4];               // x-lerps: [z*R + y][lx pair]
    float4 y4[7 * 8 * 2];               // y-lerps: [z][ly][lx quad]
    AxisWeight w[2][3][8];              // axis weights of the coarse [0] and fine [1] grids
    int fr[kV2MaxBatch];                // clamped frames of the batch
    uint8_t b8[kV2MaxBatch], b4[kV2MaxBatch];
};

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

__device__ __forceinline__ void key_read_v2(const uint32_t* __restrict__ pw, uint64_t kb, uint32_t codec, uint32_t i,
                                            int& frame, float& value)
{
    if (codec == 1u) {
        const uint32_t w = (uint32_t)((kb + 8ull * i) >> 2);
        frame = (int)(ldw(pw, w) & 0xFFFFu);
        value = __uint_as_float(ldw(pw, w + 1u));
    } else {
        const uint32_t k = ld_key24(pw, kb + 3ull * i);
        frame = (int)(k & 0xFFu);
        value = half_to_float_exact(k >> 8);
    }
}

__device__ __forceinline__ uint32_t row_byte(uint32_t r0, uint32_t r1, uint32_t b)
{
    return ((b < 4u ? r0 : r1) >> ((b & 3u) * 8u)) & 0xFFu;
}

// Decode control c of stream s for the batch's frames into dst[j * stride].
__device__ __forceinline__ void decode_control_batch(const uint32_t* __restrict__ pw, const StreamRef& s, uint32_t c,
                                                     const V2WarpSmem& sm, int nb, float* dst, int stride)
{
    const uint32_t desc = ldw(pw, (uint32_t)((s.base + 4ull * c) >> 2));
    const uint64_t row = s.base + 4ull * s.controls + (uint64_t)c * s.bins;
    const uint32_t r0 = ldw(pw, (uint32_t)(row >> 2));
    const uint32_t r1 = s.bins == 8u ? ldw(pw, (uint32_t)(row >> 2) + 1u) : 0u;
    const uint32_t kc = (desc >> 16) & 0xFFu;
    if (kc == 0u || (desc & 0xFFFFu) + kc > s.kf) {   // see decode_control (rt_decode.cuh)
        for (int j = 0; j < nb; ++j) dst[j * stride] = 0.0f;
        return;
    }
    const uint32_t ks = desc & 0xFFFFu, last = kc - 1u;
    const uint64_t kb = stream_key_base(s);
    const uint8_t* bins_of_frame = s.bins == 8u ? sm.b8 : sm.b4;
    for (int j = 0; j < nb; ++j) {
        const int frame = sm.fr[j];
        const uint32_t bin = bins_of_frame[j];
        const uint32_t hb = row_byte(r0, r1, bin);
        uint32_t lo = hb < last ? hb : last;
        int f0, f1;
        float v0, v1, out;
        key_read_v2(pw, kb, s.codec, ks + lo, f0, v0);
        if (f0 > frame) {
            lo = 0u;
            key_read_v2(pw, kb, s.codec, ks, f0, v0);
        }
        if (f0 >= frame || lo == last) {
            out = v0;
        } else {
            uint32_t hi = last;
            if (bin + 1u < s.bins) {
                const uint32_t h = row_byte(r0, r1, bin + 1u) + 1u;
                hi = h < last ? h : last;
            }
            if (hi < lo + 1u) hi = lo + 1u;
            key_read_v2(pw, kb, s.codec, ks + hi, f1, v1);
            if (f1 < frame) {
                hi = last;
                key_read_v2(pw, kb, s.codec, ks + hi, f1, v1);
            }
            if (f1 <= frame) {
                out = v1;
            } else {
                bool moved_lo = false, moved_hi = false;
                while (hi > lo + 1u) {
                    const uint32_t mid = lo + (hi - lo) / 2u;
                    const int fm = key_frame(pw, kb, s.codec, ks + mid);
                    if (fm < frame) {
                        lo = mid;
                        f0 = fm;
                        moved_lo = true;
                    } else {
                        hi = mid;
                        f1 = fm;
                        moved_hi = true;
                    }
                }
                if (moved_hi) key_read_v2(pw, kb, s.codec, ks + hi, f1, v1);
                if (f1 == frame) {
                    out = v1;
                } else {
                    if (moved_lo) key_read_v2(pw, kb, s.codec, ks + lo, f0, v0);
                    const float alpha = __fdiv_rn((float)(frame - f0), (float)(f1 - f0));
                    out = __fadd_rn(v0, __fmul_rn(alpha, __fsub_rn(v1, v0)));
                }
            }
        }
        dst[j * stride] = out;
    }
}

// Cursor decode of control c for a batch of non-decreasing frames, valid when the control's key
// frames are strictly increasing (checked once per asset, kFlagSorted).  For such keys the
// reference's hinted bracket search returns: the first key's value before it, the last key's
// value after it, the key's value on an exact hit, else v0 + a*(v1 - v0) with a = (t-f0)/(f1-f0)
// for the adjacent pair around t -- so a cursor k = "first key with frame > t" that only moves
// forward, reading each key once, yields the same bits.
__device__ __forceinline__ void decode_control_cursor(const uint32_t* __restrict__ pw, const StreamRef& s, uint32_t c,
                                                      const V2WarpSmem& sm, int nb, float* dst, int stride)
{
    const uint32_t desc = ldw(pw, (uint32_t)((s.base + 4ull * c) >> 2));
    const uint32_t kc = (desc >> 16) & 0xFFu;
    if (kc == 0u || (desc & 0xFFFFu) + kc > s.kf) {   // see decode_control (rt_decode.cuh)
        for (int j = 0; j < nb; ++j) dst[j * stride] = 0.0f;
        return;
    }
    const uint32_t ks = desc & 0xFFFFu;
    const uint64_t kb = stream_key_base(s);
    // initial cursor for the first frame: start from the bin hint (a predecessor candidate)
    const int t0 = sm.fr[0];
    const uint32_t bin = s.bins == 8u ? sm.b8[0] : sm.b4[0];
    const uint64_t row = s.base + 4ull * s.controls + (uint64_t)c * s.bins;
    const uint32_t hb = (ldw(pw, (uint32_t)((row + (bin & ~3u)) >> 2)) >> ((bin & 3u) * 8u)) & 0xFFu;
    uint32_t k = hb < kc - 1u ? hb : kc - 1u;
    int fk;
    float vk;
    key_read_v2(pw, kb, s.codec, ks + k, fk, vk);
    if (fk > t0) {   // hint overshoots: binary search for the first key > t0 in [0, k]
        uint32_t lo = 0, hi = k;
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (key_frame(pw, kb, s.codec, ks + mid) > t0) hi = mid;
            else lo = mid + 1u;
        }
        k = lo;
    } else {          // step forward from the hint
        ++k;
        while (k < kc && key_frame(pw, kb, s.codec, ks + k) <= t0) ++k;
    }
    // prev = key k-1, next = key k (when they exist)
    int fp = 0, fn = 0;
    float vp = 0.0f, vn = 0.0f;
    if (k > 0u) key_read_v2(pw, kb, s.codec, ks + k - 1u, fp, vp);
    if (k < kc) key_read_v2(pw, kb, s.codec, ks + k, fn, vn);
    for (int j = 0; j < nb; ++j) {
        const int t = sm.fr[j];
        while (k < kc && fn <= t) {
            fp = fn;
            vp = vn;
            ++k;
            if (k < kc) key_read_v2(pw, kb, s.codec, ks + k, fn, vn);
        }
        float out;
        if (k == 0u) out = vn;               // before the first key
        else if (k == kc || fp == t) out = vp;   // after the last key, or an exact hit
        else {
            const float alpha = __fdiv_rn((float)(t - fp), (float)(fn - fp));
            out = __fadd_rn(vp, __fmul_rn(alpha, __fsub_rn(vn, vp)));
        }
        dst[j * stride] = out;
    }
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

__device__ __forceinline__ void trilinear_quads(V2WarpSmem& sm, int ws, const float* __restrict__ g, int R, int lane,
                                                float4 q[4])
{
    trilinear_quads_ptr(sm.w[ws], sm.x2, sm.y4, g, R, lane, q);
}

__device__ __forceinline__ void load_axis_weights(V2WarpSmem& sm, int ws, int R, int w, int h, int d, int lane)
{
    if (lane < 24) {
        const int axis = lane >> 3, p = lane & 7;
        const int ext = axis == 0 ? w : (axis == 1 ? h : d);
        sm.w[ws][axis][p] = g_axis[axis_index(R, ext, p)];
    }
}

// Grid sample for resolutions 0 and 1 (no interpolation: 0, or the single control).
__device__ __forceinline__ void constant_quads(const float* __restrict__ g, int R, float4 q[4])
{
    const float v = R == 1 ? g[0] : 0.0f;
#pragma unroll
    for (int i = 0; i < 4; ++i) q[i] = make_float4(v, v, v, v);
}

}  // namespace vbtb
