// scalar.cu -- checked decode of arbitrary control streams (the scalar C++ API's device path).
//
// Unlike the asset kernels, the stream here was never walked, so every check of
// decodeRenderTemporalControlValue (src/render_temporal_decode.cpp:304-356) and of
// readPackedKeyframe (:33-66) runs per call, in the reference's order, and the first failing
// check is reported as a status instead of a thrown exception.  Any bin count (1..255) and both
// aligned and unaligned stream layouts are accepted, so bytes are read one at a time.
#include <cuda_runtime.h>

#include "vbt_format.cuh"

namespace vbtb {

struct CheckedStream {
    const uint8_t* p;
    uint32_t bytes, codec, cc, bins, kf, align;
    int total;
};

__device__ __forceinline__ uint32_t b8(const CheckedStream& s, uint64_t o) { return __ldg(s.p + o); }

__device__ int checked_decode(const CheckedStream& s, uint32_t ci, int frame_index, float& out)
{
    out = 0.0f;
    if (ci >= s.cc) return kErrControlIndex;
    const uint32_t stride = key_stride(s.codec);
    const uint32_t descb = s.cc * 4u;
    uint32_t binb = s.cc * s.bins, keyb = s.kf * stride;
    if (s.align) {
        binb = align4(binb);
        keyb = align4(keyb);
    }
    if (descb + binb + keyb > s.bytes) return kErrStreamOob;
    if ((uint64_t)ci * 4u + 4u > s.bytes) return kErrDecodeOob;
    const uint32_t ks = b8(s, 4ull * ci) | (b8(s, 4ull * ci + 1) << 8);
    const uint32_t kc = b8(s, 4ull * ci + 2);
    if (kc == 0u) return kOk;
    if (ks + kc > s.kf) return kErrKeyRangeOob;
    // The check above is the reference's, in 32-bit arithmetic: a keyframe count near 2^32 / stride
    // wraps it and the reference then reads keys past the stream.  Here no key is read unless the
    // stream's true extent, in 64 bits, fits.
    const uint64_t keyb_wide = s.align ? (((uint64_t)s.kf * stride + 3u) & ~3ull) : (uint64_t)s.kf * stride;
    if ((uint64_t)descb + binb + keyb_wide > s.bytes) return kErrStreamOob;
    const uint64_t kb = descb + binb;
    const uint64_t lb = descb + (uint64_t)ci * s.bins;
    auto kframe = [&](uint32_t i) -> int {
        const uint64_t o = kb + (uint64_t)i * stride;
        return s.codec == 1u ? (int)(b8(s, o) | (b8(s, o + 1) << 8)) : (int)b8(s, o);
    };
    auto kvalue = [&](uint32_t i, float& v) -> int {
        if (i >= s.kf) return kErrKeyIndex;
        const uint64_t o = kb + (uint64_t)i * stride;
        const uint64_t limit = (uint64_t)s.kf * stride;
        if (s.codec == 1u) {
            if ((uint64_t)i * stride + 8u > limit) return kErrDecodeOob;
            const uint32_t w = b8(s, o + 4) | (b8(s, o + 5) << 8) | (b8(s, o + 6) << 16) | (b8(s, o + 7) << 24);
            v = __uint_as_float(w);
        } else {
            if ((uint64_t)i * stride + 3u > limit) return kErrDecodeOob;
            v = half_bits_to_float(b8(s, o + 1) | (b8(s, o + 2) << 8));
        }
        return kOk;
    };
    const int tmax = s.total - 1 > 0 ? s.total - 1 : 0;
    const int frame = frame_index < 0 ? 0 : (frame_index > tmax ? tmax : frame_index);
    const uint32_t last = kc - 1u;
    uint32_t bin = 0;
    if (s.bins != 0u) {
        const uint32_t q = (uint32_t)(((long long)frame * s.bins) / (s.total > 1 ? s.total : 1));
        bin = q < s.bins - 1u ? q : s.bins - 1u;
    }
    uint32_t lo = 0;
    if (s.bins != 0u) {
        const uint32_t h = b8(s, lb + bin);
        lo = h < last ? h : last;
    }
    int f0 = kframe(ks + lo);
    if (f0 > frame) {
        lo = 0u;
        f0 = kframe(ks);
    }
    if (f0 >= frame || lo == last) return kvalue(ks + lo, out);
    uint32_t hi = last;
    if (bin + 1u < s.bins) {
        const uint32_t h = b8(s, lb + bin + 1u) + 1u;
        hi = h < last ? h : last;
    }
    if (hi < lo + 1u) hi = lo + 1u;
    int f1 = kframe(ks + hi);
    if (f1 < frame) {
        hi = last;
        f1 = kframe(ks + hi);
    }
    if (f1 <= frame) return kvalue(ks + hi, out);
    while (hi > lo + 1u) {
        const uint32_t mid = lo + (hi - lo) / 2u;
        const int fm = kframe(ks + mid);
        if (fm < frame) {
            lo = mid;
            f0 = fm;
        } else {
            hi = mid;
            f1 = fm;
        }
    }
    float v1, v0;
    int st = kvalue(ks + hi, v1);
    if (st) return st;
    if (f1 == frame) {
        out = v1;
        return kOk;
    }
    st = kvalue(ks + lo, v0);
    if (st) return st;
    const float alpha = __fdiv_rn((float)(frame - f0), (float)(f1 - f0));
    out = __fadd_rn(v0, __fmul_rn(alpha, __fsub_rn(v1, v0)));
    return kOk;
}

__global__ void __launch_bounds__(128) checked_decode_kernel(CheckedStream s, const uint32_t* __restrict__ ci,
                                                             const int32_t* __restrict__ fr, uint64_t n,
                                                             float* __restrict__ out, int32_t* __restrict__ status)
{
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float v;
    const int st = checked_decode(s, ci[i], fr[i], v);
    out[i] = v;
    if (status) status[i] = st;
}

void launch_checked_decode(const uint8_t* stream, uint32_t bytes, uint32_t codec, uint32_t cc, uint32_t bins,
                           uint32_t kf, int align, int total, const uint32_t* ci, const int32_t* fr, uint64_t n,
                           float* out, int32_t* status, cudaStream_t st)
{
    if (n == 0) return;
    CheckedStream s{stream, bytes, codec, cc, bins, kf, (uint32_t)(align != 0), total};
    checked_decode_kernel<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(s, ci, fr, n, out, status);
}

}  // namespace vbtb
