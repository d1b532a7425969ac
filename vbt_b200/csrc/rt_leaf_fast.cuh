// rt_leaf_fast.cuh -- the render decode kernel's specialised path for the two leaf shapes that make
// up nearly every render-temporal asset: GRID4 (a 4^3 coarse grid) and FINE6 (4^3 coarse + 6^3
// fine), FP16 key frames that strictly increase, over a timeline (frames stepping by 0 or 1).
// Included by rt_kernel_leaf.cuh; the general leaf_decode there covers every other leaf.
//
// Same arithmetic as the general path, operation for operation (so the same bits):
//  - controls: the streaming cursor of rt_staged.cuh (m_control_stream), but each cursor is set
//    up once per launch and then carried in registers across the frame batches.  A unit is one
//    control and one contiguous part of the launch's frames: GRID4 splits each of its 64 controls
//    into 4 parts (256 units), FINE6 keeps its 280 controls whole (one unit per thread of the
//    288).  A batch takes the next frames of every part, as many as the control buffer holds.
//    Key reads are byte offsets into the staged leaf (32-bit arithmetic), and the FP16 value is
//    the hardware conversion, exact for every value but NaN -- such leaves (kFlagHalfPlain
//    unset) take the general path, which keeps the reference's NaN payloads.  Key spans are
//    below 256 frames (u8 frames), so RN(1/span) always comes from the table.
//  - voxels: the separable trilinear with the grid resolution a compile-time constant, each axis
//    weight one 128-bit shared load.
#pragma once

namespace vbtb {

// A cursor over one control's keys: k = first key with frame > t (0..kc), [fp, fn) the key
// interval around t with values vp, vn, the key after it prefetched (fnn, vnn), and per interval
// bf = span, y = RN(1/span), d = vn - vp.
struct KeyCursor {
    uint32_t kb;   // stage byte offset of the control's first key
    int k, kc;
    int fp, fn, fnn;
    float vp, vn, vnn;
    float bf, y, d;
};

// Key i of an FP16 stream at stage byte offset `off`: frame byte and binary16 value (hardware
// conversion; the leaf holds no NaN key).  The stage is padded, so the second word always exists.
__device__ __forceinline__ void fast_key(const uint8_t* __restrict__ st, uint32_t off, int& frame, float& value)
{
    const uint32_t* w = reinterpret_cast<const uint32_t*>(st + (off & ~3u));
    const uint32_t k = __funnelshift_r(w[0], w[1], (off & 3u) * 8u);
    frame = (int)(k & 0xFFu);
    value = __half2float(__ushort_as_half((unsigned short)(k >> 8)));
}

__device__ __forceinline__ void fast_interval(KeyCursor& cu, const float* __restrict__ rcp)
{
    const int b = cu.fn - cu.fp;
    cu.bf = (float)b;
    cu.y = rcp[b & 255];   // outside 0 < k < kc the interval is never selected
    cu.d = __fsub_rn(cu.vn, cu.vp);
}

// Set the cursor of control ci of the 8-bin stream at stage offset sbase (C controls, kf keys in
// its pool) for first frame t0 in time bin bin0: the start of m_control_stream.
__device__ __forceinline__ void fast_cursor_init(const uint8_t* __restrict__ st, uint32_t sbase, uint32_t C,
                                                 uint32_t ci, uint32_t kf, int t0, uint32_t bin0,
                                                 const float* __restrict__ rcp, KeyCursor& cu)
{
    cu.k = 0;
    cu.kc = 0;
    cu.fp = cu.fn = cu.fnn = 0;
    cu.vp = cu.vn = cu.vnn = 0.0f;
    cu.bf = cu.y = 1.0f;
    cu.d = 0.0f;
    cu.kb = 0u;
    const uint32_t desc = *reinterpret_cast<const uint32_t*>(st + sbase + 4u * ci);
    const uint32_t kc = (desc >> 16) & 0xFFu, ks = desc & 0xFFFFu;
    if (kc == 0u || ks + kc > kf) return;   // decodes to 0 (see decode_control, rt_search.cuh)
    cu.kc = (int)kc;
    cu.kb = sbase + 12u * C + 3u * ks;      // descriptors (4 C) + 8-bin rows (8 C, 4-aligned)
    const uint32_t hb = st[sbase + 4u * C + 8u * ci + bin0];
    uint32_t k = hb < kc - 1u ? hb : kc - 1u;
    if ((int)st[cu.kb + 3u * k] > t0) {
        uint32_t lo = 0, hi = k;
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if ((int)st[cu.kb + 3u * mid] > t0) hi = mid;
            else lo = mid + 1u;
        }
        k = lo;
    } else {
        ++k;
        while (k < kc && (int)st[cu.kb + 3u * k] <= t0) ++k;
    }
    cu.k = (int)k;
    if (k > 0u) fast_key(st, cu.kb + 3u * (k - 1u), cu.fp, cu.vp);
    if (k < kc) fast_key(st, cu.kb + 3u * k, cu.fn, cu.vn);
    if (k + 1u < kc) fast_key(st, cu.kb + 3u * (k + 1u), cu.fnn, cu.vnn);
    fast_interval(cu, rcp);
}

// The control's value at frame t (t >= the previous call's t, by at most one frame).
__device__ __forceinline__ float fast_cursor_step(KeyCursor& cu, const uint8_t* __restrict__ st, int t,
                                                  const float* __restrict__ rcp)
{
    if (cu.k < cu.kc && cu.fn <= t) {
        cu.fp = cu.fn;
        cu.vp = cu.vn;
        cu.fn = cu.fnn;
        cu.vn = cu.vnn;
        ++cu.k;
        if (cu.k + 1 < cu.kc) fast_key(st, cu.kb + 3u * (uint32_t)(cu.k + 1), cu.fnn, cu.vnn);
        fast_interval(cu, rcp);
    }
    const int ai = t - cu.fp;
    const float lerp = __fadd_rn(cu.vp, __fmul_rn(div_small_rn((float)ai, cu.bf, cu.y), cu.d));
    return cu.k == 0 ? cu.vn : ((cu.k == cu.kc || ai == 0) ? cu.vp : lerp);
}

// The axis weights of a leaf as 16-byte rows {t, 1 - t, i0, i1} (the kernel's shared table w16,
// [grid][axis][position], written beside the AxisWeight table at the start of every leaf): one
// 128-bit shared load per weight, read right where it is used, so no weight stays in a register
// across the frame loop.
__device__ __forceinline__ void axis_row(const float4* __restrict__ w16, int axis, int pos, float& t, float& omt,
                                         int& i0, int& i1)
{
    const float4 r = w16[axis * 8 + pos];
    t = r.x;
    omt = r.y;
    i0 = __float_as_int(r.z);
    i1 = __float_as_int(r.w);
}

// The x- and y-phases of trilinear_quads_ptr (rt_staged.cuh) for a compile-time even resolution R:
// the same lerps on the same operands in the same order, item loops unrolled.  x-lerps go to x2
// ([control row z*R + y][lx pair]), y-lerps to y4 ([control row z][ly][lx quad]).
template <int R>
__device__ __forceinline__ void trilinear_xy(const float4* __restrict__ w16, float2* x2, float4* y4,
                                             const float* __restrict__ g, int lane)
{
    static_assert(R % 2 == 0 && R >= 2 && R <= 6, "even resolutions up to 6");
    constexpr int NX = R * R * 4;
    {
        const int p = lane & 3;
        float ta, oa, tb, ob;
        int a0, a1, b0, b1;
        axis_row(w16, 0, 2 * p, ta, oa, a0, a1);
        axis_row(w16, 0, 2 * p + 1, tb, ob, b0, b1);
#pragma unroll
        for (int m = 0; m < (NX + 31) / 32; ++m) {
            const int row = (lane >> 2) + 8 * m;
            if (NX % 32 == 0 || row < R * R) {
                const float* gr = g + row * R;
                const float2 A = make_float2(gr[a0], gr[b0]);
                const float2 B = make_float2(gr[a1], gr[b1]);
                x2[lane + 32 * m] = lerp2(A, B, make_float2(ta, tb), make_float2(oa, ob));
            }
        }
    }
    __syncwarp();
    const int k = lane & 1;
    float t, o;
    int i0, i1;
    axis_row(w16, 1, (lane >> 1) & 7, t, o, i0, i1);
    const float2 ty = make_float2(t, t), oy = make_float2(o, o);
#pragma unroll
    for (int m = 0; m < R / 2; ++m) {   // R * 16 y items
        const int z = (lane >> 4) + 2 * m;
        const float4 a = *reinterpret_cast<const float4*>(x2 + (z * R + i0) * 4 + 2 * k);
        const float4 b = *reinterpret_cast<const float4*>(x2 + (z * R + i1) * 4 + 2 * k);
        const float2 lo2 = lerp2(make_float2(a.x, a.y), make_float2(b.x, b.y), ty, oy);
        const float2 hi2 = lerp2(make_float2(a.z, a.w), make_float2(b.z, b.w), ty, oy);
        y4[lane + 32 * m] = make_float4(lo2.x, lo2.y, hi2.x, hi2.y);
    }
    __syncwarp();
}

// The z-phase of trilinear_quads_ptr for the lane's quad i (voxels 4 (lane + 32 i) .. + 3).
__device__ __forceinline__ float4 trilinear_z(const float4* __restrict__ w16, const float4* y4, int lane, int i)
{
    const int k = lane & 1, ly = (lane >> 1) & 7;
    float tz, oz;
    int i0, i1;
    axis_row(w16, 2, 2 * i + (lane >> 4), tz, oz, i0, i1);
    const float4 A = y4[(i0 * 8 + ly) * 2 + k];
    const float4 B = y4[(i1 * 8 + ly) * 2 + k];
    const float2 t = make_float2(tz, tz), omt = make_float2(oz, oz);
    const float2 lo2 = lerp2(make_float2(A.x, A.y), make_float2(B.x, B.y), t, omt);
    const float2 hi2 = lerp2(make_float2(A.z, A.w), make_float2(B.z, B.w), t, omt);
    return make_float4(lo2.x, lo2.y, hi2.x, hi2.y);
}

// Can leaf_decode_fast take this leaf?  (Staged, timeline frames, strictly increasing FP16 keys
// without NaN, coarse resolution 4, no Mode2 shell, and fine resolution 6 when there is a fine
// stream.)
__device__ __forceinline__ bool fast_leaf_shape(const LeafEntry& e, bool steps01, bool& fine)
{
    const uint32_t need = kFlagSorted | kFlagHalfPlain;
    if (!steps01 || (e.info & need) != need || (e.info & (kFlagOccClamp | kFlagShell)) != 0u) return false;
    if (((e.header >> 6) & 7u) != 4u || ((e.header >> 2) & 3u) == 1u) return false;
    fine = (e.info & kFlagFine) != 0u;
    return !fine || (((e.header >> 9) & 7u) == 6u && ((e.header >> 4) & 3u) != 1u);
}

// Decode one staged leaf of the fast shape for all nframes frames of the launch (NW warps; the
// leaf's bytes start at stage offset lb).  Quads go to sink(frame index, lane, quad, values).
// Per lane and slot the voxel phase holds one quad at a time.
template <bool FINE, int NW, class Sink>
__device__ __forceinline__ void leaf_decode_fast(const uint8_t* __restrict__ st, uint32_t lb, const LeafSmem& s,
                                                 const LeafEntry& e, int nframes, const LeafGeom& G,
                                                 const Sink& sink)
{
    constexpr int CC = 64, CT = FINE ? 64 + 216 : 64;
    constexpr int P = FINE ? 1 : 4;   // parts per control
    static_assert(CT * P <= 32 * NW, "one unit per thread");
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int Lp = (nframes + P - 1) / P;   // frames per part
    int m = kLeafCtrlBudget / (CT * P);     // frames per part per batch
    if (m > Lp) m = Lp;
    if (P == 1 && m > NW) m -= m % NW;      // whole voxel rounds
    // this thread's unit
    const bool unit = tid < CT * P;
    const int c = FINE ? tid : (tid & 63);
    const int p = FINE ? 0 : (tid >> 6);
    const bool is_fine = FINE && c >= CC;
    const uint32_t C = is_fine ? 216u : 64u;
    const uint32_t ci = (uint32_t)(is_fine ? c - CC : c);
    const int f_lo = p * Lp, f_hi = min(nframes, f_lo + Lp);
    KeyCursor cu;
    if (unit && f_lo < f_hi) {
        const uint32_t sbase = lb + 8u + (is_fine ? e.coarse_bytes : 0u);
        const uint32_t kf = is_fine ? (e.kf >> 16) : (e.kf & 0xFFFFu);
        fast_cursor_init(st, sbase, C, ci, kf, s.fr[f_lo], s.b8[f_lo], s.rcp, cu);
    }
    const bool plain = G.w == 8 && G.h == 8 && G.d == 8;
    float2* x2 = s.x2 + warp * 196;
    float4* y4 = s.y4 + warp * 112;
    for (int b0 = 0; b0 < Lp; b0 += m) {
        const int mb = min(m, Lp - b0);
        // 1. controls: slot p * mb + j holds frame f_lo + b0 + j
        if (unit) {
            float* dst = s.ctrl + (p * mb) * CT + c;
            for (int j = 0; j < mb; ++j) {
                const int fi = f_lo + b0 + j;
                if (fi >= f_hi) break;
                dst[j * CT] = fast_cursor_step(cu, st, s.fr[fi], s.rcp);
            }
        }
        __syncthreads();
        // 2. voxels, one slot (frame) per warp
        for (int slot = warp; slot < P * mb; slot += NW) {
            const int pp = P == 1 ? 0 : slot / mb, j = slot - pp * mb;
            const int fi = pp * Lp + b0 + j;
            if (fi >= min(nframes, (pp + 1) * Lp)) continue;
            const float* g = s.ctrl + slot * CT;
            // FINE6: the fine grid's x/y tables first (y4 region), then the coarse grid's into the
            // x2 region ([x2: 64 float2][y: 64 float4]); each quad is then coarse + fine, rounded
            // once (the reference's sum; addition is commutative) and stored at once
            float4* yc = FINE ? reinterpret_cast<float4*>(x2 + 64) : y4;
            if (FINE) trilinear_xy<6>(s.w16 + 24, x2, y4, g + CC, lane);
            trilinear_xy<4>(s.w16, x2, yc, g, lane);
            const int ly = (lane >> 1) & 7, lx0 = 4 * (lane & 1);
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                float4 v = trilinear_z(s.w16, yc, lane, i);
                if (FINE) {
                    const float4 f = trilinear_z(s.w16 + 24, y4, lane, i);
                    v = make_float4(__fadd_rn(v.x, f.x), __fadd_rn(v.y, f.y), __fadd_rn(v.z, f.z), __fadd_rn(v.w, f.w));
                }
                if (!plain) {
                    const int lz = 2 * i + (lane >> 4);
                    const bool row_in = ly < G.h && lz < G.d;
                    if (!row_in || lx0 >= G.w) v.x = 0.0f;
                    if (!row_in || lx0 + 1 >= G.w) v.y = 0.0f;
                    if (!row_in || lx0 + 2 >= G.w) v.z = 0.0f;
                    if (!row_in || lx0 + 3 >= G.w) v.w = 0.0f;
                }
                sink(fi, lane, i, v);
            }
            __syncwarp();   // the tables are read before the next slot overwrites them
        }
        __syncthreads();
    }
}

}  // namespace vbtb
