// rt_search.cuh -- device-side decode of render-temporal control streams from the payload
// (the reference search, one control at one frame).
//
// A control stream is [desc u32 x C][bins u8 x C*B, pad 4][keyframes, pad 4].  Decoding one
// control at one frame follows src/render_temporal_decode.cpp:79-131 (decodeFromSequence):
// clamp the frame, take the bin hint as the predecessor key, fall back to key 0 when the hint
// overshoots, take the next bin's hint + 1 as the upper bracket (fallback: the last key), binary
// search inside the bracket, then lerp v0 + a*(v1 - v0).  Every float operation uses the _rn
// intrinsics so nvcc cannot contract a multiply and an add into an FMA: the result is bit-equal
// to the reference CPU decoder, which rounds after every operation.
//
// All reads go through the payload as aligned 32-bit words (the leaf block is 4-byte aligned);
// byte fields are extracted with funnel shifts.  Bounds were validated once by the payload walker
// (kernel a), so no read here can leave the leaf: keyframe indices stay in [keyStart,
// keyStart + keyCount) and keyStart + keyCount <= keyframe count was checked for every control.
#pragma once
#include "vbt_format.cuh"

namespace vbtb {

__device__ __forceinline__ uint32_t ldw(const uint32_t* __restrict__ words, uint32_t word_index)
{
    return __ldg(words + word_index);
}

// Byte at absolute byte offset `b` of the payload.
__device__ __forceinline__ uint32_t ld_byte(const uint32_t* __restrict__ pw, uint64_t b)
{
    return (ldw(pw, (uint32_t)(b >> 2)) >> ((uint32_t)(b & 3u) * 8u)) & 0xFFu;
}

// Three bytes (b, b+1, b+2) as the low 24 bits: frame byte and fp16 value of an FP16 keyframe.
__device__ __forceinline__ uint32_t ld_key24(const uint32_t* __restrict__ pw, uint64_t b)
{
    const uint32_t w = (uint32_t)(b >> 2);
    const uint32_t sh = (uint32_t)(b & 3u) * 8u;
    const uint32_t lo = ldw(pw, w);
    if (sh <= 8u) return (lo >> sh) & 0xFFFFFFu;
    const uint32_t hi = ldw(pw, w + 1u);
    return __funnelshift_r(lo, hi, sh) & 0xFFFFFFu;
}

struct StreamRef {
    uint64_t base;    // absolute payload byte offset of the stream (4-byte aligned)
    uint32_t controls;
    uint32_t bins;    // 8 (coarse / fine) or 4 (Mode2 shell)
    uint32_t kf;      // keyframe count of the stream
    uint32_t codec;   // 1 = FP32 keyframes, otherwise FP16
};

__device__ __forceinline__ uint64_t stream_key_base(const StreamRef& s)
{
    return s.base + (uint64_t)s.controls * 4u + align4(s.controls * s.bins);
}

// Frame index of key i (absolute index inside the stream's keyframe pool).
__device__ __forceinline__ int key_frame(const uint32_t* __restrict__ pw, uint64_t kb, uint32_t codec, uint32_t i)
{
    if (codec == 1u) return (int)(ldw(pw, (uint32_t)((kb + 8ull * i) >> 2)) & 0xFFFFu);
    return (int)ld_byte(pw, kb + 3ull * i);
}

// Value of key i.
__device__ __forceinline__ float key_value(const uint32_t* __restrict__ pw, uint64_t kb, uint32_t codec, uint32_t i)
{
    if (codec == 1u) return __uint_as_float(ldw(pw, (uint32_t)((kb + 8ull * i + 4u) >> 2)));
    return half_bits_to_float(ld_key24(pw, kb + 3ull * i) >> 8);
}

// Frame and value of key i in one read.
__device__ __forceinline__ void key_read(const uint32_t* __restrict__ pw, uint64_t kb, uint32_t codec, uint32_t i,
                                         int& frame, float& value)
{
    if (codec == 1u) {
        const uint32_t w = (uint32_t)((kb + 8ull * i) >> 2);
        frame = (int)(ldw(pw, w) & 0xFFFFu);
        value = __uint_as_float(ldw(pw, w + 1u));
    } else {
        const uint32_t k = ld_key24(pw, kb + 3ull * i);
        frame = (int)(k & 0xFFu);
        value = half_bits_to_float(k >> 8);
    }
}

// Time bin for a clamped frame: min(bins-1, frame*bins / max(1, total)).
__device__ __forceinline__ uint32_t time_bin(int frame, uint32_t bins, int total)
{
    if (bins == 0u) return 0u;
    const uint32_t q = (uint32_t)(((long long)frame * bins) / (total > 1 ? total : 1));
    return q < bins - 1u ? q : bins - 1u;
}

__device__ __forceinline__ int clamp_frame(int frame_index, int total)
{
    const int tmax = total - 1 > 0 ? total - 1 : 0;
    return frame_index < 0 ? 0 : (frame_index > tmax ? tmax : frame_index);
}

// Decode control c of stream s at clamped frame `frame` (bin = time_bin(frame, s.bins, total)).
__device__ __forceinline__ float decode_control(const uint32_t* __restrict__ pw, const StreamRef& s, uint32_t c,
                                                int frame, uint32_t bin)
{
    const uint32_t desc = ldw(pw, (uint32_t)((s.base + 4ull * c) >> 2));
    const uint32_t kc = (desc >> 16) & 0xFFu;
    // bin row: bins bytes at base + 4C + c*bins (4-byte aligned for bins = 4 or 8)
    const uint64_t row = s.base + 4ull * s.controls + (uint64_t)c * s.bins;
    const uint32_t w0 = ldw(pw, (uint32_t)((row + (bin & ~3u)) >> 2));
    // keyCount 0 decodes to 0; a key range past the pool only occurs for Mode2 shell controls of
    // voxels outside a boundary leaf's extent, which are never sampled (the walker validated all
    // others), so it is not read either.
    if (kc == 0u || (desc & 0xFFFFu) + kc > s.kf) return 0.0f;
    const uint32_t ks = desc & 0xFFFFu;
    const uint32_t last = kc - 1u;
    const uint64_t kb = stream_key_base(s) ;
    const uint32_t hb = (w0 >> ((bin & 3u) * 8u)) & 0xFFu;
    uint32_t lo = hb < last ? hb : last;
    int f0;
    float v0;
    key_read(pw, kb, s.codec, ks + lo, f0, v0);
    if (f0 > frame) {
        lo = 0u;
        key_read(pw, kb, s.codec, ks, f0, v0);
    }
    if (f0 >= frame || lo == last) return v0;
    uint32_t hi = last;
    if (bin + 1u < s.bins) {
        const uint32_t nb = bin + 1u;
        const uint32_t wn = (nb & ~3u) == (bin & ~3u) ? w0 : ldw(pw, (uint32_t)((row + (nb & ~3u)) >> 2));
        const uint32_t h = ((wn >> ((nb & 3u) * 8u)) & 0xFFu) + 1u;
        hi = h < last ? h : last;
    }
    if (hi < lo + 1u) hi = lo + 1u;
    int f1;
    float v1;
    key_read(pw, kb, s.codec, ks + hi, f1, v1);
    if (f1 < frame) {
        hi = last;
        key_read(pw, kb, s.codec, ks + hi, f1, v1);
    }
    if (f1 <= frame) return v1;
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
    if (moved_hi) v1 = key_value(pw, kb, s.codec, ks + hi);
    if (f1 == frame) return v1;
    if (moved_lo) v0 = key_value(pw, kb, s.codec, ks + lo);
    const float alpha = __fdiv_rn((float)(frame - f0), (float)(f1 - f0));
    return __fadd_rn(v0, __fmul_rn(alpha, __fsub_rn(v1, v0)));
}

// a*(1-t) + b*t with the reference's rounding (two products, one sum; 1-t precomputed exactly).
__device__ __forceinline__ float lerp_ref(float a, float b, float t, float omt)
{
    return __fadd_rn(__fmul_rn(a, omt), __fmul_rn(b, t));
}

}  // namespace vbtb
