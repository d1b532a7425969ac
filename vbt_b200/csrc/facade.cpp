// facade.cpp -- the reference's C++ decoder API (namespace vbt / vbt::render) over the C-ABI.
//
// Format functions (header/prefix packing, stream layout, leaf parsing/building, stream
// packing, half conversion, the VBTPACK4 reader) are host code with the reference's semantics
// and error messages (src/render_temporal_payload.cpp, src/render_temporal_decode.cpp:133-302,
// render/src/vbt_file.cpp).  Every value decode runs on the GPU through include/vbt_b200.h:
// control values through vbt_decode_control_values, frames and point queries through a device
// copy of the VbtFile kept resident between calls.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

#include "vbt/dct_codec.h"
#include "vbt/query_patterns.h"
#include "vbt/render_temporal_decode.h"
#include "vbt/render_temporal_payload.h"
#include "vbt/scientific_decode.h"
#include "vbt/vbt_file.h"
#include "vbt_b200.h"

namespace vbt {

namespace {

uint32_t align4(uint32_t b) { return (b + 3u) & ~3u; }

uint16_t controls_for_resolution(uint32_t r) { return r == 0u ? uint16_t(0) : static_cast<uint16_t>(r * r * r); }

RenderTemporalStreamLayout stream_layout(uint32_t start, uint32_t controls, uint32_t bins, uint32_t keyframes,
                                         RenderTemporalSequenceCodec codec, bool align)
{
    RenderTemporalStreamLayout s;
    s.descriptorOffset = start;
    s.descriptorBytes = controls * kRenderTemporalControlDescriptorBytes;
    s.binIndexOffset = s.descriptorOffset + s.descriptorBytes;
    s.binIndexBytes = align ? align4(controls * bins) : controls * bins;
    s.keyframeOffset = s.binIndexOffset + s.binIndexBytes;
    const uint32_t kb = keyframes * renderTemporalKeyframeBytes(codec);
    s.keyframeBytes = align ? align4(kb) : kb;
    s.totalBytes = s.descriptorBytes + s.binIndexBytes + s.keyframeBytes;
    return s;
}

[[noreturn]] void throw_status(int status)
{
    throw std::runtime_error(vbt_status_string(status));
}

void cuda_check(cudaError_t e, const char* what)
{
    if (e != cudaSuccess) throw std::runtime_error(std::string("no usable CUDA device (") + what + "): " + cudaGetErrorString(e));
}

// Per-thread device staging for the scalar decode calls: a non-blocking stream of the thread's
// own (threads that decode at the same time do not queue behind one another on the legacy default
// stream), the last stream bytes uploaded, and one pinned host block and one device block for the
// (control, frame) pairs in and the (value, status) pairs out, so that a call is one copy in, one
// launch, one copy out and one stream synchronisation.
struct Staging {
    cudaStream_t stream = nullptr;
    uint8_t* d_stream = nullptr;
    size_t stream_cap = 0;
    std::vector<uint8_t> last;   // host copy of the bytes currently in d_stream
    void* d_io = nullptr;
    void* h_io = nullptr;        // pinned
    size_t io_cap = 0;
    ~Staging()
    {
        if (stream) cudaStreamDestroy(stream);
        if (d_stream) cudaFree(d_stream);
        if (d_io) cudaFree(d_io);
        if (h_io) cudaFreeHost(h_io);
    }
};
thread_local Staging g_stage;

// Decode n (control, frame) pairs of one stream on the GPU; statuses per pair.
void gpu_decode(const uint8_t* stream, uint32_t bytes, RenderTemporalSequenceCodec codec, uint32_t cc, uint32_t bins,
                uint32_t kf, bool align, int total, const uint32_t* ci, const int32_t* fr, size_t n, float* out,
                int32_t* status)
{
    Staging& s = g_stage;
    if (!s.stream) cuda_check(cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking), "cudaStreamCreate");
    if (bytes > s.stream_cap) {
        if (s.d_stream) cudaFree(s.d_stream);
        s.d_stream = nullptr;
        s.stream_cap = 0;
        s.last.clear();
        cuda_check(cudaMalloc(&s.d_stream, bytes), "cudaMalloc");
        s.stream_cap = bytes;
    }
    if (bytes && (s.last.size() != bytes || std::memcmp(s.last.data(), stream, bytes) != 0)) {
        cuda_check(cudaMemcpyAsync(s.d_stream, stream, bytes, cudaMemcpyHostToDevice, s.stream), "cudaMemcpyAsync");
        s.last.assign(stream, stream + bytes);
    }
    const size_t io = n * 16;
    if (io > s.io_cap) {
        if (s.d_io) cudaFree(s.d_io);
        if (s.h_io) cudaFreeHost(s.h_io);
        s.d_io = s.h_io = nullptr;
        s.io_cap = 0;
        cuda_check(cudaMalloc(&s.d_io, io), "cudaMalloc");
        cuda_check(cudaHostAlloc(&s.h_io, io, cudaHostAllocDefault), "cudaHostAlloc");
        s.io_cap = io;
    }
    // [control indices][frames] in, [values][statuses] out, adjacent in both blocks
    auto* h = static_cast<uint8_t*>(s.h_io);
    std::memcpy(h, ci, 4 * n);
    std::memcpy(h + 4 * n, fr, 4 * n);
    auto* d = static_cast<uint8_t*>(s.d_io);
    cuda_check(cudaMemcpyAsync(d, h, 8 * n, cudaMemcpyHostToDevice, s.stream), "cudaMemcpyAsync");
    const int st = vbt_decode_control_values(s.d_stream, bytes, static_cast<uint32_t>(codec), cc, bins, kf, align ? 1 : 0,
                                             total, reinterpret_cast<const uint32_t*>(d),
                                             reinterpret_cast<const int32_t*>(d + 4 * n), n,
                                             reinterpret_cast<float*>(d + 8 * n), reinterpret_cast<int32_t*>(d + 12 * n),
                                             s.stream);
    if (st) throw std::runtime_error(vbt_last_error());
    cuda_check(cudaMemcpyAsync(h + 8 * n, d + 8 * n, 8 * n, cudaMemcpyDeviceToHost, s.stream), "cudaMemcpyAsync");
    cuda_check(cudaStreamSynchronize(s.stream), "cudaStreamSynchronize");
    std::memcpy(out, h + 8 * n, 4 * n);
    std::memcpy(status, h + 12 * n, 4 * n);
}

// The reference's pre-decode checks of decodeRenderTemporalControlValue
// (src/render_temporal_decode.cpp:316-340), in its order, run on the host bytes: control index,
// stream extent (32-bit, as the reference computes it), descriptor in bounds, key range.  Returns
// the bytes the device needs, or 0 when the control has no keys (its value is 0 and no launch is
// needed).  Where the reference's 32-bit extent wraps (a keyframe count near 2^32 / stride) it
// would read keys past the stream; here that case is refused with its extent message before any
// key is read, and the descriptor-only cases keep the reference's results.
uint32_t checked_extent(const uint8_t* base, uint16_t controlCount, uint8_t timeBinCount, uint32_t keyframeCount,
                        uint32_t streamBytes, bool align, RenderTemporalSequenceCodec codec, uint32_t controlIndex)
{
    if (controlIndex >= controlCount) throw_status(VBT_STATUS_CONTROL_INDEX);
    const uint32_t desc = static_cast<uint32_t>(controlCount) * kRenderTemporalControlDescriptorBytes;
    uint32_t bins = static_cast<uint32_t>(controlCount) * timeBinCount;
    uint32_t keys = keyframeCount * renderTemporalKeyframeBytes(codec);
    if (align) {
        bins = align4(bins);
        keys = align4(keys);
    }
    const uint32_t total = desc + bins + keys;
    if (total > streamBytes) throw_status(VBT_STATUS_STREAM_OOB);
    if (static_cast<uint64_t>(controlIndex) * 4u + 4u > streamBytes) throw_status(VBT_STATUS_DECODE_OOB);
    const uint8_t* d = base + static_cast<size_t>(controlIndex) * 4u;
    const uint32_t keyStart = d[0] | (static_cast<uint32_t>(d[1]) << 8), keyCount = d[2];
    if (keyCount == 0u) return 0u;
    if (keyStart + keyCount > keyframeCount) throw_status(VBT_STATUS_KEY_RANGE_OOB);
    const uint64_t keys_wide = static_cast<uint64_t>(keyframeCount) * renderTemporalKeyframeBytes(codec);
    const uint64_t wide = static_cast<uint64_t>(desc) + bins + (align ? ((keys_wide + 3u) & ~3ull) : keys_wide);
    if (wide > streamBytes) throw_status(VBT_STATUS_STREAM_OOB);
    return total;
}

}  // namespace

const char* toString(TemporalFirstPackedMode mode)
{
    switch (mode) {
    case TemporalFirstPackedMode::EMPTY: return "Empty";
    case TemporalFirstPackedMode::TEMPORAL_GRID4: return "TemporalGrid4";
    case TemporalFirstPackedMode::TEMPORAL_FINE_COMPACT: return "TemporalFineCompact";
    case TemporalFirstPackedMode::TEMPORAL_FINE6: return "TemporalFine6";
    }
    return "Unknown";
}

// ----------------------------------------------------------------- render_temporal_payload.h

uint32_t renderTemporalKeyframeBytes(RenderTemporalSequenceCodec codec)
{
    return codec == RenderTemporalSequenceCodec::DP_KEYFRAME_FP32 ? 8u : 3u;
}

uint32_t packRenderTemporalHeader(const RenderTemporalPackedHeaderFields& f)
{
    uint32_t p = static_cast<uint32_t>(f.mode) & 3u;
    p |= (static_cast<uint32_t>(f.coarseCodec) & 3u) << 2;
    p |= (static_cast<uint32_t>(f.fineCodec) & 3u) << 4;
    p |= (std::min<uint32_t>(f.coarseResolution, 7u) & 7u) << 6;
    p |= (std::min<uint32_t>(f.fineResolution, 7u) & 7u) << 9;
    return p;
}

RenderTemporalPackedHeaderFields unpackRenderTemporalHeader(uint32_t p)
{
    RenderTemporalPackedHeaderFields f;
    f.mode = static_cast<TemporalFirstPackedMode>(p & 3u);
    f.coarseCodec = static_cast<RenderTemporalSequenceCodec>((p >> 2) & 3u);
    f.fineCodec = static_cast<RenderTemporalSequenceCodec>((p >> 4) & 3u);
    f.coarseResolution = static_cast<uint8_t>((p >> 6) & 7u);
    f.fineResolution = static_cast<uint8_t>((p >> 9) & 7u);
    return f;
}

RenderTemporalPackedLeafPrefix makeRenderTemporalLeafPrefix(TemporalFirstPackedMode, uint32_t coarseKf, uint32_t fineKf)
{
    if (coarseKf > 0xFFFFu || fineKf > 0xFFFFu)
        throw std::runtime_error("render temporal prefix keyframe count exceeds uint16");
    RenderTemporalPackedLeafPrefix p;
    p.coarseKeyframeCount = static_cast<uint16_t>(coarseKf);
    p.fineKeyframeCount = static_cast<uint16_t>(fineKf);
    return p;
}

bool validateRenderTemporalLeafPrefix(const RenderTemporalPackedLeafPrefix& prefix,
                                      const RenderTemporalPackedHeaderFields& header,
                                      const TemporalFirstEncoderOptions& options)
{
    if (options.timeBinCount != kRenderTemporalPackedTimeBinCount) return false;
    if (controls_for_resolution(header.coarseResolution) == 0 && prefix.coarseKeyframeCount != 0) return false;
    const bool fineMode = header.mode == TemporalFirstPackedMode::TEMPORAL_FINE6 ||
                          header.mode == TemporalFirstPackedMode::TEMPORAL_FINE_COMPACT;
    if (fineMode && controls_for_resolution(header.fineResolution) == 0 && prefix.fineKeyframeCount != 0) return false;
    return true;
}

RenderTemporalPackedLeafLayout computeRenderTemporalLeafLayout(const RenderTemporalPackedHeaderFields& header,
                                                              const RenderTemporalPackedLeafPrefix& prefix, bool align)
{
    RenderTemporalPackedLeafLayout out;
    out.coarseOffset = out.prefixOffset + out.prefixBytes;
    out.coarse = stream_layout(out.coarseOffset, controls_for_resolution(header.coarseResolution),
                               kRenderTemporalPackedTimeBinCount, prefix.coarseKeyframeCount, header.coarseCodec, align);
    out.fineOffset = out.coarseOffset + out.coarse.totalBytes;
    if (header.mode == TemporalFirstPackedMode::TEMPORAL_FINE6) {
        out.fine = stream_layout(out.fineOffset, controls_for_resolution(header.fineResolution),
                                 kRenderTemporalPackedTimeBinCount, prefix.fineKeyframeCount, header.fineCodec, align);
        out.totalBytes = out.fineOffset + out.fine.totalBytes;
    } else if (header.mode == TemporalFirstPackedMode::TEMPORAL_FINE_COMPACT) {
        // occupancy (80 bytes) + the residual keyframe bytes; the residual descriptors and bins
        // depend on the occupancy popcount and are sized by parseRenderTemporalPackedLeaf
        out.fine = RenderTemporalStreamLayout{};
        out.fine.descriptorOffset = out.fineOffset;
        out.fine.descriptorBytes = 80u;
        out.fine.binIndexOffset = out.fineOffset + 80u;
        out.fine.keyframeOffset = out.fineOffset + 80u;
        const uint32_t kb = prefix.fineKeyframeCount * renderTemporalKeyframeBytes(header.fineCodec);
        out.fine.keyframeBytes = align ? align4(kb) : kb;
        out.fine.totalBytes = 80u + out.fine.keyframeBytes;
        out.totalBytes = out.fineOffset + out.fine.totalBytes;
    } else {
        out.totalBytes = out.coarseOffset + out.coarse.totalBytes;
    }
    if (header.mode == TemporalFirstPackedMode::EMPTY) {
        out.coarseOffset = 0;
        out.fineOffset = 0;
        out.coarse = {};
        out.fine = {};
        out.totalBytes = out.headerBytes;
    }
    return out;
}

std::vector<uint8_t> buildRenderTemporalPackedLeafBytes(const RenderTemporalPackedHeaderFields& header,
                                                        const RenderTemporalPackedLeafPrefix& prefix,
                                                        const std::vector<uint8_t>& coarse,
                                                        const std::vector<uint8_t>& fine, bool align)
{
    const auto layout = computeRenderTemporalLeafLayout(header, prefix, align);
    const uint32_t packed = packRenderTemporalHeader(header);
    if (header.mode == TemporalFirstPackedMode::EMPTY) {
        std::vector<uint8_t> out(4, 0u);
        std::memcpy(out.data(), &packed, 4);
        return out;
    }
    if (coarse.size() != layout.coarse.totalBytes)
        throw std::runtime_error("render temporal coarse stream bytes do not match computed layout");
    if (header.mode == TemporalFirstPackedMode::TEMPORAL_FINE6 && fine.size() != layout.fine.totalBytes)
        throw std::runtime_error("render temporal fine stream bytes do not match computed layout");
    std::vector<uint8_t> out(layout.totalBytes, 0u);
    if (!fine.empty() && fine.size() > out.size() - std::min<size_t>(out.size(), layout.fineOffset))
        throw std::runtime_error("render temporal fine stream bytes do not fit the computed layout");
    std::memcpy(out.data(), &packed, 4);
    std::memcpy(out.data() + layout.prefixOffset, &prefix, sizeof(prefix));
    std::memcpy(out.data() + layout.coarseOffset, coarse.data(), coarse.size());
    if (!fine.empty()) std::memcpy(out.data() + layout.fineOffset, fine.data(), fine.size());
    return out;
}

std::vector<uint8_t> buildRenderTemporalPackedLeafBytes(const RenderTemporalPackedHeaderFields& header,
                                                        const RenderTemporalPackedLeafPrefix& prefix,
                                                        const std::vector<uint8_t>& coarse,
                                                        const std::vector<uint8_t>& occupancy,
                                                        const std::vector<uint8_t>& residual, bool align)
{
    std::vector<uint8_t> out(8, 0u);
    const uint32_t packed = packRenderTemporalHeader(header);
    std::memcpy(out.data(), &packed, 4);
    std::memcpy(out.data() + 4, &prefix, 4);
    auto append = [&](const std::vector<uint8_t>& part) {
        if (part.empty()) return;
        out.insert(out.end(), part.begin(), part.end());
        if (align)
            while (out.size() % 4 != 0) out.push_back(0);
    };
    append(coarse);
    append(occupancy);
    append(residual);
    return out;
}

std::vector<uint8_t> packRenderTemporalShellOccupancySection(const RenderTemporalShellOccupancySection& section)
{
    std::vector<uint8_t> out(80, 0u);
    std::memcpy(out.data(), section.shellMask.data(), 64);
    std::memcpy(out.data() + 64, section.groupPrefix.data(), 16);
    return out;
}

RenderTemporalShellOccupancySection unpackRenderTemporalShellOccupancySection(const uint8_t* data, std::uint64_t size)
{
    RenderTemporalShellOccupancySection s{};
    if (data == nullptr || size < 80) return s;
    std::memcpy(s.shellMask.data(), data, 64);
    std::memcpy(s.groupPrefix.data(), data + 64, 16);
    return s;
}

std::uint16_t renderTemporalShellActiveVoxelCount(const RenderTemporalShellOccupancySection& section)
{
    uint32_t n = 0;
    for (uint64_t w : section.shellMask) n += static_cast<uint32_t>(__builtin_popcountll(w));
    return static_cast<uint16_t>(n);
}

RenderTemporalPackedLeafView parseRenderTemporalPackedLeaf(const uint8_t* leaf, size_t bytes, bool align)
{
    if (leaf == nullptr || bytes < 4) throw std::runtime_error("render temporal leaf bytes too small");
    RenderTemporalPackedLeafView v;
    uint32_t packed;
    std::memcpy(&packed, leaf, 4);
    v.header = unpackRenderTemporalHeader(packed);
    if (v.header.mode == TemporalFirstPackedMode::EMPTY) {
        v.layout = computeRenderTemporalLeafLayout(v.header, v.prefix, align);
        return v;
    }
    if (bytes < 8) throw std::runtime_error("render temporal leaf prefix missing");
    std::memcpy(&v.prefix, leaf + 4, 4);
    v.layout = computeRenderTemporalLeafLayout(v.header, v.prefix, align);
    if (v.layout.totalBytes > bytes) throw std::runtime_error("render temporal leaf shorter than computed layout");
    if (v.header.mode == TemporalFirstPackedMode::TEMPORAL_FINE_COMPACT) {
        const size_t occOff = v.layout.fine.descriptorOffset, occBytes = v.layout.fine.descriptorBytes;
        if (occBytes != 80u || occOff > bytes || occBytes > bytes - occOff)
            throw std::runtime_error("render temporal shell occupancy is out of bounds");
        const auto occ = unpackRenderTemporalShellOccupancySection(leaf + occOff, occBytes);
        uint16_t expect = 0;
        for (size_t g = 0; g < 8; ++g) {
            if (occ.groupPrefix[g] != expect) throw std::runtime_error("render temporal shell group prefix is inconsistent");
            expect = static_cast<uint16_t>(expect + __builtin_popcountll(occ.shellMask[g]));
        }
        if (expect == 0u) throw std::runtime_error("render temporal shell mode contains no active voxels");
        size_t resOff = occOff + occBytes;
        if (align) resOff = (resOff + 3u) & ~size_t{3u};
        size_t binBytes = size_t(expect) * kRenderTemporalShellPackedTimeBinCount;
        size_t keyBytes = size_t(v.prefix.fineKeyframeCount) * renderTemporalKeyframeBytes(v.header.fineCodec);
        if (align) {
            binBytes = (binBytes + 3u) & ~size_t{3u};
            keyBytes = (keyBytes + 3u) & ~size_t{3u};
        }
        const size_t resBytes = size_t(expect) * kRenderTemporalControlDescriptorBytes + binBytes + keyBytes;
        if (resOff > bytes || resBytes > bytes - resOff)
            throw std::runtime_error("render temporal shell residual stream is out of bounds");
        if (resOff + resBytes != bytes) throw std::runtime_error("render temporal shell leaf contains trailing bytes");
        v.shellActiveVoxelCount = expect;
        v.shellResidualOffset = static_cast<uint32_t>(resOff);
        v.shellResidualBytes = static_cast<uint32_t>(resBytes);
    }
    return v;
}

// ----------------------------------------------------------------- render_temporal_decode.h

// IEEE binary32 -> binary16, round half up on the 13 dropped mantissa bits, overflow to
// infinity, underflow to signed zero (the conversion of src/render_temporal_decode.cpp:133-165).
uint16_t renderTemporalFloatToHalfBits(float value)
{
    uint32_t bits;
    std::memcpy(&bits, &value, 4);
    const uint32_t sign = (bits >> 16) & 0x8000u;
    int32_t exp = static_cast<int32_t>((bits >> 23) & 0xFFu) - 112;
    uint32_t man = bits & 0x7FFFFFu;
    if (exp <= 0) {
        if (exp < -10) return static_cast<uint16_t>(sign);
        man |= 0x800000u;
        const uint32_t shifted = man >> static_cast<uint32_t>(1 - exp);
        return static_cast<uint16_t>(sign | ((shifted + 0x1000u) >> 13));
    }
    if (exp >= 31) return static_cast<uint16_t>(sign | 0x7C00u);
    const uint32_t rounded = (man + 0x1000u) >> 13;
    if (rounded == 0x400u) {
        ++exp;
        if (exp >= 31) return static_cast<uint16_t>(sign | 0x7C00u);
        return static_cast<uint16_t>(sign | (static_cast<uint32_t>(exp) << 10));
    }
    return static_cast<uint16_t>(sign | (static_cast<uint32_t>(exp) << 10) | (rounded & 0x3FFu));
}

// Exact binary16 -> binary32 (subnormals normalised, NaN payloads kept).
float renderTemporalHalfBitsToFloat(uint16_t h)
{
    const uint32_t sign = static_cast<uint32_t>(h & 0x8000u) << 16;
    uint32_t e = (h >> 10) & 0x1Fu, m = h & 0x3FFu, bits;
    if (e == 0) {
        if (m == 0) {
            bits = sign;
        } else {
            int shift = 0;
            while ((m & 0x400u) == 0) {
                m <<= 1;
                ++shift;
            }
            bits = sign | (static_cast<uint32_t>(113 - shift) << 23) | ((m & 0x3FFu) << 13);
        }
    } else if (e == 31) {
        bits = sign | 0x7F800000u | (m << 13);
    } else {
        bits = sign | ((e + 112u) << 23) | (m << 13);
    }
    float f;
    std::memcpy(&f, &bits, 4);
    return f;
}

bool validateRenderTemporalControlStreamData(const RenderTemporalControlStreamData& s)
{
    if (s.controlCount == 0 || s.timeBinCount == 0 || s.maxBinLocalKeys == 0) return false;
    if (s.descriptors.size() != s.controlCount) return false;
    if (s.binIndex.size() != size_t(s.controlCount) * s.timeBinCount) return false;
    for (const auto& d : s.descriptors) {
        if (size_t(d.keyStart) + d.keyCount > s.keyframes.size()) return false;
        if (d.keyCount > s.timeBinCount * s.maxBinLocalKeys) return false;
        if (d.reserved != 0u && d.reserved > s.maxBinLocalKeys) return false;
    }
    return true;
}

std::vector<uint8_t> packRenderTemporalControlStream(const RenderTemporalControlStreamData& s, bool align)
{
    if (!validateRenderTemporalControlStreamData(s)) throw std::runtime_error("invalid render temporal control stream");
    const uint32_t stride = renderTemporalKeyframeBytes(s.codec);
    const uint32_t descBytes = static_cast<uint32_t>(s.descriptors.size() * 4);
    uint32_t binBytes = static_cast<uint32_t>(s.binIndex.size());
    uint32_t keyBytes = static_cast<uint32_t>(s.keyframes.size()) * stride;
    if (align) {
        binBytes = align4(binBytes);
        keyBytes = align4(keyBytes);
    }
    std::vector<uint8_t> out(size_t(descBytes) + binBytes + keyBytes, 0u);
    std::memcpy(out.data(), s.descriptors.data(), descBytes);
    std::memcpy(out.data() + descBytes, s.binIndex.data(), s.binIndex.size());
    uint8_t* keys = out.data() + descBytes + binBytes;
    for (size_t i = 0; i < s.keyframes.size(); ++i) {
        const auto& k = s.keyframes[i];
        uint8_t* p = keys + i * stride;
        if (s.codec == RenderTemporalSequenceCodec::DP_KEYFRAME_FP32) {
            std::memcpy(p, &k.frame, 2);
            std::memcpy(p + 4, &k.value, 4);
        } else {
            if (k.frame > 255u) throw std::runtime_error("render temporal fp16 keyframe frame exceeds uint8 range");
            const uint16_t hv = renderTemporalFloatToHalfBits(k.value);
            p[0] = static_cast<uint8_t>(k.frame);
            p[1] = static_cast<uint8_t>(hv & 0xFFu);
            p[2] = static_cast<uint8_t>(hv >> 8);
        }
    }
    return out;
}

RenderTemporalControlStreamData unpackRenderTemporalControlStream(const uint8_t* base, RenderTemporalSequenceCodec codec,
                                                                 uint16_t cc, uint8_t bins, uint8_t maxLocal,
                                                                 uint32_t kf, uint32_t streamBytes, bool align)
{
    RenderTemporalControlStreamData out;
    out.codec = codec;
    out.controlCount = cc;
    out.timeBinCount = bins;
    out.maxBinLocalKeys = maxLocal;
    out.descriptors.resize(cc);
    out.binIndex.resize(size_t(cc) * bins);
    out.keyframes.resize(kf);
    const uint32_t stride = renderTemporalKeyframeBytes(codec);
    const uint32_t descBytes = static_cast<uint32_t>(cc) * 4u;
    uint32_t binBytes = static_cast<uint32_t>(cc) * bins, keyBytes = kf * stride;
    if (align) {
        binBytes = align4(binBytes);
        keyBytes = align4(keyBytes);
    }
    if (descBytes + binBytes + keyBytes > streamBytes) throw std::runtime_error("render temporal stream bytes too small");
    std::memcpy(out.descriptors.data(), base, descBytes);
    std::memcpy(out.binIndex.data(), base + descBytes, out.binIndex.size());
    const uint8_t* keys = base + descBytes + binBytes;
    for (uint32_t i = 0; i < kf; ++i) {
        const uint8_t* p = keys + size_t(i) * stride;
        if (codec == RenderTemporalSequenceCodec::DP_KEYFRAME_FP32) {
            std::memcpy(&out.keyframes[i].frame, p, 2);
            std::memcpy(&out.keyframes[i].value, p + 4, 4);
        } else {
            out.keyframes[i].frame = p[0];
            out.keyframes[i].value = renderTemporalHalfBitsToFloat(static_cast<uint16_t>(p[1] | (p[2] << 8)));
        }
    }
    return out;
}

std::vector<float> decodeRenderTemporalControlValues(const uint8_t* base, RenderTemporalSequenceCodec codec,
                                                     uint16_t cc, uint8_t bins, uint32_t kf, uint32_t streamBytes,
                                                     bool align, int totalFrames, const std::vector<uint16_t>& ci,
                                                     const std::vector<int>& frames)
{
    if (ci.size() != frames.size()) throw std::invalid_argument("controlIndex and frameIndex sizes differ");
    if (ci.empty()) return {};
    uint32_t extent = 0;
    for (uint16_t c : ci) extent = std::max(extent, checked_extent(base, cc, bins, kf, streamBytes, align, codec, c));
    if (extent == 0u) return std::vector<float>(ci.size(), 0.0f);   // no control has keys
    std::vector<uint32_t> c32(ci.begin(), ci.end());
    std::vector<int32_t> f32(frames.begin(), frames.end());
    std::vector<float> out(ci.size());
    std::vector<int32_t> st(ci.size());
    gpu_decode(base, extent, codec, cc, bins, kf, align, totalFrames, c32.data(), f32.data(), ci.size(), out.data(),
               st.data());
    for (int32_t s : st)
        if (s) throw_status(s);
    return out;
}

float decodeRenderTemporalControlValue(const uint8_t* base, RenderTemporalSequenceCodec codec, uint16_t cc, uint8_t bins,
                                       uint8_t /*maxBinLocalKeys: unused by the decode, as in the reference*/,
                                       uint32_t kf, uint32_t streamBytes, bool align, int totalFrames,
                                       uint16_t controlIndex, int frameIndex)
{
    const uint32_t extent = checked_extent(base, cc, bins, kf, streamBytes, align, codec, controlIndex);
    if (extent == 0u) return 0.0f;   // a control without keys decodes to 0
    const uint32_t c = controlIndex;
    const int32_t f = frameIndex;
    float out = 0.0f;
    int32_t st = 0;
    gpu_decode(base, extent, codec, cc, bins, kf, align, totalFrames, &c, &f, 1, &out, &st);
    if (st) throw_status(st);
    return out;
}

float decodeRenderTemporalLeafControlValue(const uint8_t* leafBase, const RenderTemporalPackedHeaderFields& header,
                                           const RenderTemporalPackedLeafPrefix& prefix,
                                           const RenderTemporalPackedLeafLayout& layout, bool useFine, bool align,
                                           int totalFrames, uint16_t controlIndex, int frameIndex)
{
    if (useFine)
        return decodeRenderTemporalControlValue(leafBase + layout.fineOffset, header.fineCodec,
                                                controls_for_resolution(header.fineResolution),
                                                kRenderTemporalPackedTimeBinCount, 0u, prefix.fineKeyframeCount,
                                                layout.fine.totalBytes, align, totalFrames, controlIndex, frameIndex);
    return decodeRenderTemporalControlValue(leafBase + layout.coarseOffset, header.coarseCodec,
                                            static_cast<uint16_t>(header.coarseResolution * header.coarseResolution *
                                                                  header.coarseResolution),
                                            kRenderTemporalPackedTimeBinCount, 0u, prefix.coarseKeyframeCount,
                                            layout.coarse.totalBytes, align, totalFrames, controlIndex, frameIndex);
}

float decodeRenderTemporalLeafShellVoxelValue(const uint8_t* leafBase, const RenderTemporalPackedLeafView& v, bool align,
                                              int totalFrames, std::uint16_t voxel, int frameIndex)
{
    if (leafBase == nullptr || voxel >= 512) return 0.0f;
    if (v.header.mode != TemporalFirstPackedMode::TEMPORAL_FINE_COMPACT) return 0.0f;
    const auto occ = unpackRenderTemporalShellOccupancySection(leafBase + v.layout.fine.descriptorOffset,
                                                               v.layout.fine.descriptorBytes);
    const uint32_t g = voxel >> 6, bit = voxel & 63u;
    const uint64_t mask = occ.shellMask[g];
    if ((mask & (1ull << bit)) == 0ull) return 0.0f;
    const uint16_t di =
        static_cast<uint16_t>(occ.groupPrefix[g] + __builtin_popcountll(mask & ((1ull << bit) - 1ull)));
    if (v.shellActiveVoxelCount == 0 || v.prefix.fineKeyframeCount == 0) return 0.0f;
    return decodeRenderTemporalControlValue(leafBase + v.shellResidualOffset, v.header.fineCodec,
                                            v.shellActiveVoxelCount, kRenderTemporalShellPackedTimeBinCount, 0u,
                                            v.prefix.fineKeyframeCount, v.shellResidualBytes, align, totalFrames, di,
                                            frameIndex);
}

// ----------------------------------------------------------------- dct_codec.h (encoder side)

namespace {
constexpr double kPi = 3.14159265358979323846;
double basis(int n, int k, int i)
{
    const double invN = 1.0 / static_cast<double>(n);
    const double alpha = k == 0 ? std::sqrt(invN) : std::sqrt(2.0 * invN);
    return alpha * std::cos((kPi / static_cast<double>(n)) * (static_cast<double>(i) + 0.5) * static_cast<double>(k));
}
}  // namespace

std::vector<float> dctEncodeKeep(const std::vector<float>& series, int keepCount)
{
    const int n = static_cast<int>(series.size());
    const int keep = std::max(1, std::min(keepCount, n));
    std::vector<float> c(static_cast<size_t>(keep), 0.0f);
    const double invN = 1.0 / static_cast<double>(n);
    for (int k = 0; k < keep; ++k) {
        const double alpha = k == 0 ? std::sqrt(invN) : std::sqrt(2.0 * invN);
        double sum = 0.0;
        for (int i = 0; i < n; ++i)
            sum += static_cast<double>(series[i]) *
                   std::cos((kPi / static_cast<double>(n)) * (static_cast<double>(i) + 0.5) * static_cast<double>(k));
        c[static_cast<size_t>(k)] = static_cast<float>(alpha * sum);
    }
    return c;
}

std::vector<float> dctEncodeKeepWeighted(const std::vector<float>& series, const std::vector<float>& weights,
                                         int keepCount)
{
    const int n = static_cast<int>(series.size());
    const int keep = std::max(1, std::min(keepCount, n));
    if (weights.empty()) return dctEncodeKeep(series, keep);
    // weighted least squares: (B^T W B) c = B^T W s, solved by Gauss-Jordan with partial pivoting
    std::vector<double> A(size_t(keep) * keep, 0.0), b(size_t(keep), 0.0);
    for (int i = 0; i < n; ++i) {
        const double w = std::max(1e-6, static_cast<double>(weights[size_t(i)]));
        for (int r = 0; r < keep; ++r) {
            const double br = basis(n, r, i);
            b[size_t(r)] += w * br * static_cast<double>(series[size_t(i)]);
            for (int c = 0; c < keep; ++c) A[size_t(r) * keep + c] += w * br * basis(n, c, i);
        }
    }
    for (int i = 0; i < keep; ++i) {
        int piv = i;
        for (int r = i + 1; r < keep; ++r)
            if (std::abs(A[size_t(r) * keep + i]) > std::abs(A[size_t(piv) * keep + i])) piv = r;
        if (std::abs(A[size_t(piv) * keep + i]) < 1e-12) return dctEncodeKeep(series, keep);
        if (piv != i) {
            for (int c = i; c < keep; ++c) std::swap(A[size_t(i) * keep + c], A[size_t(piv) * keep + c]);
            std::swap(b[size_t(i)], b[size_t(piv)]);
        }
        const double diag = A[size_t(i) * keep + i];
        for (int c = i; c < keep; ++c) A[size_t(i) * keep + c] /= diag;
        b[size_t(i)] /= diag;
        for (int r = 0; r < keep; ++r) {
            if (r == i) continue;
            const double f = A[size_t(r) * keep + i];
            if (std::abs(f) < 1e-18) continue;
            for (int c = i; c < keep; ++c) A[size_t(r) * keep + c] -= f * A[size_t(i) * keep + c];
            b[size_t(r)] -= f * b[size_t(i)];
        }
    }
    std::vector<float> out(static_cast<size_t>(keep), 0.0f);
    for (int i = 0; i < keep; ++i) out[size_t(i)] = static_cast<float>(b[size_t(i)]);
    return out;
}

// Same operand order as the reference (coefficient x alpha, then x cosine) so that the double
// sums, and therefore the float results, are identical.
float dctDecodeAt(const std::vector<float>& coeffs, int totalLength, int index)
{
    const double invN = 1.0 / static_cast<double>(totalLength);
    double v = 0.0;
    for (size_t k = 0; k < coeffs.size(); ++k) {
        const double alpha = k == 0 ? std::sqrt(invN) : std::sqrt(2.0 * invN);
        v += static_cast<double>(coeffs[k]) * alpha *
             std::cos((kPi / static_cast<double>(totalLength)) * (static_cast<double>(index) + 0.5) *
                      static_cast<double>(k));
    }
    return static_cast<float>(v);
}

}  // namespace vbt

// ===================================================================== vbt::render

namespace vbt::render {

namespace {

uint32_t rd32(const uint8_t* p)
{
    uint32_t v;
    std::memcpy(&v, p, 4);
    return v;
}

std::vector<uint8_t> image_of(const VbtFile& f)
{
    std::vector<uint8_t> img(52 + 4 * (f.coarseAcScales.size() + f.offsetsWords.size() + f.payloadWords.size()));
    std::memcpy(img.data(), f.header.magic, 8);
    const uint32_t h[11] = {f.header.version, f.header.width, f.header.height, f.header.depth, f.header.frames,
                            f.header.leafSize, f.header.coarseResolution, f.header.maxCoarseKeep, f.header.leafCount,
                            f.header.profileType, f.header.coarseAcScaleCount};
    std::memcpy(img.data() + 8, h, 44);
    uint8_t* p = img.data() + 52;
    std::memcpy(p, f.coarseAcScales.data(), 4 * f.coarseAcScales.size());
    p += 4 * f.coarseAcScales.size();
    std::memcpy(p, f.offsetsWords.data(), 4 * f.offsetsWords.size());
    p += 4 * f.offsetsWords.size();
    std::memcpy(p, f.payloadWords.data(), 4 * f.payloadWords.size());
    return img;
}

// Device copies of VbtFile objects for the GPU-backed calls.  The reference's decoders read the
// VbtFile's vectors on every call, so a copy made earlier must never decode bytes the caller has
// since changed: each call compares, against the image it last uploaded, exactly the bytes it is
// about to decode -- the header, the AC scales and, per leaf it reads, that leaf's two offsets and
// its payload words -- and uploads the file again when any of them differ.  A different file that
// reuses a freed VbtFile's address is caught the same way.  Copies are kept for the most recently
// used files only (kMaxCopies, and at most kMaxCopyBytes of device memory in all), so files that
// are destroyed without releaseDeviceCopy hold no device memory beyond those bounds.
constexpr size_t kMaxCopies = 8;
constexpr uint64_t kMaxCopyBytes = 2ull << 30;

struct DeviceCopy {
    std::mutex mu;               // one call at a time on a copy (a call may upload it again)
    vbt_asset* asset = nullptr;
    std::vector<uint8_t> image;  // the bytes last uploaded
    uint64_t device_bytes = 0;
    uint64_t tick = 0;
    ~DeviceCopy()
    {
        if (asset) vbt_asset_destroy(asset);
    }
};
std::mutex g_cache_mu;
std::map<const VbtFile*, std::shared_ptr<DeviceCopy>> g_cache;
uint64_t g_tick = 0;

// The copy of `f` (created empty when absent), most recently used; older copies beyond the
// bounds are dropped from the cache (a call still using one keeps it alive until it returns).
std::shared_ptr<DeviceCopy> cache_entry(const VbtFile& f)
{
    std::vector<std::shared_ptr<DeviceCopy>> dropped;   // destroyed after the lock is released
    std::lock_guard<std::mutex> lock(g_cache_mu);
    auto& slot = g_cache[&f];
    if (!slot) slot = std::make_shared<DeviceCopy>();
    slot->tick = ++g_tick;
    std::shared_ptr<DeviceCopy> mine = slot;
    for (;;) {
        uint64_t bytes = 0;
        auto oldest = g_cache.end();
        for (auto it = g_cache.begin(); it != g_cache.end(); ++it) {
            bytes += it->second->device_bytes;
            if (it->second != mine && (oldest == g_cache.end() || it->second->tick < oldest->second->tick)) oldest = it;
        }
        if (oldest == g_cache.end() || (g_cache.size() <= kMaxCopies && bytes <= kMaxCopyBytes)) break;
        dropped.push_back(std::move(oldest->second));
        g_cache.erase(oldest);
    }
    return mine;
}

bool same_words(const uint8_t* a, const void* b, size_t words) { return std::memcmp(a, b, 4 * words) == 0; }

// Make c->asset decode `f`: compare the header, the scales and the payload of the leaves in
// `leaves` (every leaf when `all`) with the uploaded image, and upload `f` again when they differ.
// Called with c->mu held.
vbt_asset* synced(DeviceCopy& c, const VbtFile& f, const std::vector<uint32_t>& leaves, bool all)
{
    const size_t ns = f.coarseAcScales.size(), no = f.offsetsWords.size(), np = f.payloadWords.size();
    const size_t bytes = 52 + 4 * (ns + no + np);
    bool fresh = c.asset != nullptr && c.image.size() == bytes;
    if (fresh) {
        uint8_t head[52];
        std::memcpy(head, f.header.magic, 8);
        const uint32_t w[11] = {f.header.version, f.header.width, f.header.height, f.header.depth, f.header.frames,
                                f.header.leafSize, f.header.coarseResolution, f.header.maxCoarseKeep,
                                f.header.leafCount, f.header.profileType, f.header.coarseAcScaleCount};
        std::memcpy(head + 8, w, 44);
        const uint8_t* img = c.image.data();
        const uint8_t* off = img + 52 + 4 * ns;
        const uint8_t* pay = off + 4 * no;
        fresh = std::memcmp(img, head, 52) == 0 && same_words(img + 52, f.coarseAcScales.data(), ns);
        if (fresh && all) {
            fresh = same_words(off, f.offsetsWords.data(), no) && same_words(pay, f.payloadWords.data(), np);
        } else if (fresh) {
            fresh = no > 0 && same_words(off + 4 * (no - 1), &f.offsetsWords[no - 1], 1);
            for (size_t i = 0; fresh && i < leaves.size(); ++i) {
                const uint32_t l = leaves[i];
                if (l + 1u >= no) continue;   // the decode reads no such leaf
                fresh = same_words(off + 4ull * l, &f.offsetsWords[l], 2);
                const uint32_t w0 = f.offsetsWords[l], w1 = f.offsetsWords[l + 1];
                if (fresh && w0 < w1 && w1 <= np) fresh = same_words(pay + 4ull * w0, &f.payloadWords[w0], w1 - w0);
            }
        }
    }
    if (fresh) return c.asset;
    std::vector<uint8_t> img = image_of(f);
    if (c.asset && c.image.size() == img.size() && std::memcmp(c.image.data(), img.data(), 52) == 0) {
        // same header and sizes: into the resident buffers
        int st = vbt_asset_upload(c.asset, img.data(), img.size(), nullptr);
        if (st == VBT_STATUS_OK && cudaDeviceSynchronize() != cudaSuccess) st = VBT_STATUS_CUDA;
        if (st) throw std::runtime_error(vbt_last_error());
    } else {
        if (c.asset) vbt_asset_destroy(c.asset);
        c.asset = nullptr;
        c.device_bytes = 0;
        vbt_asset* a = nullptr;
        if (vbt_asset_create(img.data(), img.size(), 0, &a)) throw std::runtime_error(vbt_last_error());
        c.asset = a;
        vbt_asset_info info{};
        if (vbt_asset_get_info(a, &info) == VBT_STATUS_OK) c.device_bytes = info.device_bytes;
    }
    c.image = std::move(img);
    return c.asset;
}

}  // namespace

bool loadVbtFile(const std::filesystem::path& path, VbtFile& outFile, std::string& error)
{
    error.clear();
    std::error_code ec;
    const uintmax_t size = std::filesystem::file_size(path, ec);
    if (ec) {
        error = "Failed to query file size: " + path.string();
        return false;
    }
    FILE* fp = std::fopen(path.string().c_str(), "rb");
    if (!fp) {
        error = "Failed to open file: " + path.string();
        return false;
    }
    std::vector<uint8_t> img(static_cast<size_t>(size));
    const size_t got = img.empty() ? 0 : std::fread(img.data(), 1, img.size(), fp);
    std::fclose(fp);
    if (got != img.size()) {
        error = "Failed to read VBTPACK header.";
        return false;
    }
    vbt_header h{};
    if (vbt_validate_file_image(img.data(), img.size(), &h) != VBT_STATUS_OK) {
        error = vbt_last_error();
        return false;
    }
    VbtFile loaded;
    std::memcpy(loaded.header.magic, img.data(), 8);
    loaded.header.version = h.version;
    loaded.header.width = h.width;
    loaded.header.height = h.height;
    loaded.header.depth = h.depth;
    loaded.header.frames = h.frames;
    loaded.header.leafSize = h.leaf_size;
    loaded.header.coarseResolution = h.coarse_resolution;
    loaded.header.maxCoarseKeep = h.max_coarse_keep;
    loaded.header.leafCount = h.leaf_count;
    loaded.header.profileType = h.profile_type;
    loaded.header.coarseAcScaleCount = h.coarse_ac_scale_count;
    const uint8_t* p = img.data() + 52;
    loaded.coarseAcScales.resize(h.coarse_ac_scale_count);
    std::memcpy(loaded.coarseAcScales.data(), p, 4ull * h.coarse_ac_scale_count);
    p += 4ull * h.coarse_ac_scale_count;
    loaded.offsetsWords.resize(size_t(h.leaf_count) + 1u);
    std::memcpy(loaded.offsetsWords.data(), p, 4 * loaded.offsetsWords.size());
    p += 4 * loaded.offsetsWords.size();
    loaded.payloadWords.resize(loaded.offsetsWords.back());
    std::memcpy(loaded.payloadWords.data(), p, 4 * loaded.payloadWords.size());
    outFile = std::move(loaded);
    return true;
}

uint32_t readPackedHeaderWord(const VbtFile& file, uint32_t leafIndex)
{
    if (leafIndex >= file.header.leafCount) return 0u;
    const uint32_t w = file.offsetsWords[leafIndex];
    if (w >= file.payloadWords.size()) return 0u;
    return file.payloadWords[w];
}

ScientificHeaderV2 decodeScientificHeaderV2(uint32_t p)
{
    ScientificHeaderV2 d{};
    d.mode = static_cast<ScientificMode>(p & 3u);
    switch (d.mode) {
    case ScientificMode::CoarseOnly:
        d.coarseKeepMinus1 = (p >> 2) & 0x3Fu;
        d.coarseQuantClass = (p >> 8) & 0x7u;
        break;
    case ScientificMode::SparseEvents:
        d.coarseKeepMinus1 = (p >> 2) & 0x3Fu;
        d.tierId = (p >> 8) & 0x3u;
        d.framesPerBinMinus1 = (p >> 10) & 0xFu;
        d.eventQuantCode = (p >> 14) & 0x3u;
        d.packedEventCount = (p >> 16) & 0x0FFFu;
        d.sparseSubtype = (p >> 28) & 0xFu;
        break;
    case ScientificMode::DenseGrid3:
    case ScientificMode::DenseGrid4:
        d.coarseKeepMinus1 = (p >> 2) & 0x3Fu;
        d.denseQuantBits = (p >> 8) & 0xFu;
        d.denseSubtype = (p >> 12) & 0x7u;
        d.denseTemporalKeepMinus1 = (p >> 15) & 0xFu;
        break;
    }
    return d;
}

uint32_t leafIndexForVoxel(const VbtFileHeader& h, uint32_t x, uint32_t y, uint32_t z)
{
    if (h.width == 0u || h.height == 0u || h.depth == 0u || h.leafSize == 0u) return 0u;
    const uint32_t s = h.leafSize;
    const uint32_t lx = (h.width + s - 1u) / s, ly = (h.height + s - 1u) / s, lz = (h.depth + s - 1u) / s;
    const uint32_t bx = std::min(lx - 1u, x / s), by = std::min(ly - 1u, y / s), bz = std::min(lz - 1u, z / s);
    return (bz * ly + by) * lx + bx;
}

bool parseQueryPattern(const std::string& text, QueryPattern& out)
{
    if (text == "random") out = QueryPattern::RandomFull;
    else if (text == "same-t") out = QueryPattern::SameT;
    else if (text == "same-xyz") out = QueryPattern::SameXYZ;
    else if (text == "coherent") out = QueryPattern::CoherentTiles;
    else return false;
    return true;
}

// Draw order of render/src/query_patterns.cpp:29-86 (four fixed draws, then per query), so a
// seed gives the reference's queries.
std::vector<Query4D> generateQueries(const VbtFileHeader& h, QueryPattern pattern, uint32_t count, uint32_t seed)
{
    std::mt19937 rng(seed);
    std::uniform_int_distribution<uint32_t> dx(0, std::max(1u, h.width) - 1u), dy(0, std::max(1u, h.height) - 1u),
        dz(0, std::max(1u, h.depth) - 1u), dt(0, std::max(1u, h.frames) - 1u);
    std::vector<Query4D> q(count);
    const uint32_t fx = dx(rng), fy = dy(rng), fz = dz(rng), ft = dt(rng);
    for (uint32_t i = 0; i < count; ++i) {
        Query4D r{};
        switch (pattern) {
        case QueryPattern::RandomFull:
            r.x = dx(rng);
            r.y = dy(rng);
            r.z = dz(rng);
            r.t = dt(rng);
            break;
        case QueryPattern::SameT:
            r.x = dx(rng);
            r.y = dy(rng);
            r.z = dz(rng);
            r.t = ft;
            break;
        case QueryPattern::SameXYZ:
            r.x = fx;
            r.y = fy;
            r.z = fz;
            r.t = dt(rng);
            break;
        case QueryPattern::CoherentTiles: {
            const uint32_t bx = (dx(rng) / 8u) * 8u, by = (dy(rng) / 8u) * 8u, bz = (dz(rng) / 8u) * 8u;
            r.x = std::min(h.width - 1u, bx + (i % 8u));
            r.y = std::min(h.height - 1u, by + ((i / 8u) % 8u));
            r.z = std::min(h.depth - 1u, bz + ((i / 64u) % 8u));
            r.t = ft;
            break;
        }
        }
        q[i] = r;
    }
    return q;
}

void fillLeafIndices(const VbtFileHeader& h, std::vector<Query4D>& queries)
{
    for (auto& q : queries) q.leafIndex = leafIndexForVoxel(h, q.x, q.y, q.z);
}

void sortQueriesByLeaf(std::vector<Query4D>& queries)
{
    std::stable_sort(queries.begin(), queries.end(), [](const Query4D& a, const Query4D& b) {
        if (a.leafIndex != b.leafIndex) return a.leafIndex < b.leafIndex;
        if (a.t != b.t) return a.t < b.t;
        if (a.z != b.z) return a.z < b.z;
        if (a.y != b.y) return a.y < b.y;
        return a.x < b.x;
    });
}

std::vector<float> decodeValuesGpu(const VbtFile& file, const std::vector<Query4D>& queries)
{
    std::vector<uint32_t> q(queries.size() * 4);
    std::vector<uint32_t> leaves;
    leaves.reserve(queries.size());
    const VbtFileHeader& h = file.header;
    for (size_t i = 0; i < queries.size(); ++i) {
        q[4 * i] = queries[i].x;
        q[4 * i + 1] = queries[i].y;
        q[4 * i + 2] = queries[i].z;
        q[4 * i + 3] = queries[i].t;
        if (queries[i].x < h.width && queries[i].y < h.height && queries[i].z < h.depth)
            leaves.push_back(leafIndexForVoxel(h, queries[i].x, queries[i].y, queries[i].z));
    }
    std::sort(leaves.begin(), leaves.end());
    leaves.erase(std::unique(leaves.begin(), leaves.end()), leaves.end());
    const bool all = leaves.size() * 4 >= h.leafCount;   // most leaves: compare the file in one pass
    std::vector<float> out(queries.size());
    const std::shared_ptr<DeviceCopy> c = cache_entry(file);
    std::lock_guard<std::mutex> lock(c->mu);
    vbt_asset* a = synced(*c, file, leaves, all);
    const int st = vbt_query_points_host(a, q.data(), queries.size(), out.data(), nullptr);
    if (st) throw std::runtime_error(vbt_last_error());
    return out;
}

namespace {
// A dense frame of `file` through its device copy (every leaf is read).
std::vector<float> frames_of(const VbtFile& file, int frameIndex)
{
    std::vector<float> out(size_t(file.header.width) * file.header.height * file.header.depth);
    const std::shared_ptr<DeviceCopy> c = cache_entry(file);
    std::lock_guard<std::mutex> lock(c->mu);
    vbt_asset* a = synced(*c, file, {}, true);
    const int st = vbt_decode_frames_host(a, &frameIndex, 1, out.data(), nullptr);
    if (st) throw std::runtime_error(vbt_last_error());
    return out;
}
}  // namespace

float decodeScientificValueAtCpu(const VbtFile& file, const Query4D& query)
{
    if (query.leafIndex != leafIndexForVoxel(file.header, query.x, query.y, query.z))
        throw std::invalid_argument("Query4D.leafIndex differs from leafIndexForVoxel(x, y, z)");
    if (query.t >= file.header.frames) throw std::out_of_range("query frame outside the asset's frames");
    return decodeValuesGpu(file, {query})[0];
}

std::vector<float> reconstructScientificFrameCpu(const VbtFile& file, uint32_t frameIndex)
{
    if (frameIndex >= file.header.frames) throw std::out_of_range("frame outside the asset's frames");
    return frames_of(file, static_cast<int>(frameIndex));
}

std::vector<float> decodeRenderTemporalFrame(const VbtFile& file, int frameIndex)
{
    return frames_of(file, frameIndex);
}

void releaseDeviceCopy(const VbtFile& file)
{
    std::shared_ptr<DeviceCopy> dropped;   // destroyed after the lock, once no call uses it
    std::lock_guard<std::mutex> lock(g_cache_mu);
    auto it = g_cache.find(&file);
    if (it != g_cache.end()) {
        dropped = std::move(it->second);
        g_cache.erase(it);
    }
}

size_t deviceCopyCount()
{
    std::lock_guard<std::mutex> lock(g_cache_mu);
    return g_cache.size();
}

}  // namespace vbt::render
