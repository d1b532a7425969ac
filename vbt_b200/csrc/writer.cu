// writer.cu -- a VBTPACK4 writer on the GPU.
//
// vbt_pack_payload: packed leaf blocks, each padded with zero bytes to a whole number of words,
// concatenated into the payload pool, and the word offset table -- what
// writeRenderTemporalProbeFile (src/render_temporal_kf_probe_main.cpp:2561-2585) builds on the host
// before it writes the 52-byte header, the offsets and the payload.
//
// vbt_pack_leaves: the leaves themselves, from their control streams, straight into that payload:
// packRenderTemporalControlStream (src/render_temporal_decode.cpp:201-264) for every stream and
// buildRenderTemporalPackedLeafBytes (src/render_temporal_payload.cpp:199-232 for EMPTY, GRID4 and
// FINE6, :348-386 for the Mode2 shell layout) with 4-byte alignment, the only form the encoder
// writes (render_temporal_kf_probe_main.cpp:1276-1419).
#include <cuda_runtime.h>

#include <string>

#include "../../include/vbt_b200.h"

namespace vbtb {
int set_last_error(int status, const std::string& msg);
}

namespace {

constexpr int kScanThreads = 1024;

// Exclusive scan of the padded word counts into offsets[0..n], in one CTA: each thread sums a
// contiguous run of leaves, the CTA scans the run totals, each thread writes its run.  offsets[n]
// is the payload size in words; *overflow is set when it does not fit 32 bits.
__global__ void __launch_bounds__(kScanThreads) payload_offsets_kernel(const unsigned long long* __restrict__ block_off,
                                                                       uint32_t n, uint32_t* __restrict__ offsets,
                                                                       unsigned long long* total)
{
    __shared__ unsigned long long s_part[kScanThreads];
    const uint32_t tid = threadIdx.x;
    const uint32_t per = (n + kScanThreads - 1) / kScanThreads;
    const uint32_t b = tid * per, e = min(n, b + per);
    unsigned long long sum = 0;
    for (uint32_t i = b; i < e; ++i) sum += (block_off[i + 1] - block_off[i] + 3ull) >> 2;
    s_part[tid] = sum;
    __syncthreads();
    for (uint32_t off = 1; off < kScanThreads; off <<= 1) {   // inclusive Hillis-Steele scan
        const unsigned long long v = tid >= off ? s_part[tid - off] : 0ull;
        __syncthreads();
        s_part[tid] += v;
        __syncthreads();
    }
    unsigned long long run = s_part[tid] - sum;
    for (uint32_t i = b; i < e; ++i) {
        offsets[i] = (uint32_t)run;
        run += (block_off[i + 1] - block_off[i] + 3ull) >> 2;
    }
    if (tid == kScanThreads - 1) {
        offsets[n] = (uint32_t)s_part[tid];
        *total = s_part[tid];
    }
}

// One warp per leaf: word w of the leaf's padded block is bytes 4w .. 4w+3 of the block, zero past
// its end.
__global__ void __launch_bounds__(256) payload_copy_kernel(const uint8_t* __restrict__ blocks,
                                                           const unsigned long long* __restrict__ block_off, uint32_t n,
                                                           const uint32_t* __restrict__ offsets,
                                                           uint32_t* __restrict__ payload)
{
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    for (uint32_t leaf = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); leaf < n; leaf += warps) {
        const unsigned long long b0 = block_off[leaf], len = block_off[leaf + 1] - b0;
        const uint8_t* src = blocks + b0;
        uint32_t* dst = payload + offsets[leaf];
        const unsigned long long words = (len + 3ull) >> 2;
        const bool aligned = ((reinterpret_cast<uintptr_t>(src) & 3u) == 0u);
        for (unsigned long long w = lane; w < words; w += 32u) {
            uint32_t v;
            if (aligned && 4ull * w + 4ull <= len) {
                v = reinterpret_cast<const uint32_t*>(src)[w];
            } else {
                v = 0u;
                for (uint32_t k = 0; k < 4u; ++k)
                    if (4ull * w + k < len) v |= (uint32_t)src[4ull * w + k] << (8u * k);
            }
            dst[w] = v;
        }
    }
}

// ---- leaves from control streams ----------------------------------------------------------------

struct LeafStreams {   // vbt_leaf_streams
    uint32_t header;
    uint16_t coarse_kf, fine_kf;
    uint32_t coarse_control, coarse_key, fine_control, fine_key, occupancy;
    uint8_t coarse_max_local, fine_max_local, pad0, pad1;
};

struct PackInputs {
    const LeafStreams* leaves;
    const uint32_t* desc;        // one RenderTemporalControlDescriptor word per control row
    const uint8_t* bins;         // 8 bytes per control row (4-bin streams use the first 4)
    const uint16_t* key_frame;
    const float* key_value;
    const uint8_t* occupancy;    // 80-byte Mode2 sections
    unsigned long long control_rows, key_rows, occupancy_rows;
};

__device__ __forceinline__ uint32_t align4(uint32_t b) { return (b + 3u) & ~3u; }

// One control stream of a leaf: its controls, time bins, keyframes and codec (1 = FP32 keys of
// 8 bytes, otherwise FP16 keys of 3 bytes, keyframeBytesForCodec), and the rows it reads.
struct StreamPlan {
    uint32_t controls, bins, keys, codec, first_control, first_key, max_local;
    __device__ uint32_t key_stride() const { return codec == 1u ? 8u : 3u; }
    __device__ uint32_t desc_bytes() const { return controls * 4u; }
    __device__ uint32_t bin_bytes() const { return align4(controls * bins); }
    __device__ uint32_t key_bytes() const { return align4(keys * key_stride()); }
    __device__ uint32_t bytes() const { return desc_bytes() + bin_bytes() + key_bytes(); }
};

struct LeafPlan {
    uint32_t mode, total;    // total bytes (a multiple of 4)
    StreamPlan coarse, fine; // fine: FINE6's stream or the Mode2 shell residual stream
    bool has_fine, has_occupancy, bad_occupancy;
};

__device__ LeafPlan plan_leaf(const PackInputs& in, const LeafStreams& l)
{
    LeafPlan p{};
    p.mode = l.header & 3u;
    if (p.mode == 0u) {          // EMPTY: the header word alone
        p.total = 4u;
        return p;
    }
    const uint32_t cres = (l.header >> 6) & 7u, fres = (l.header >> 9) & 7u;
    p.coarse = StreamPlan{cres * cres * cres, 8u, l.coarse_kf, (l.header >> 2) & 3u, l.coarse_control,
                          l.coarse_key, l.coarse_max_local};
    p.total = 8u + p.coarse.bytes();
    if (p.mode == 3u) {          // FINE6
        p.fine = StreamPlan{fres * fres * fres, 8u, l.fine_kf, (l.header >> 4) & 3u, l.fine_control, l.fine_key,
                            l.fine_max_local};
        p.has_fine = true;
        p.total += p.fine.bytes();
    } else if (p.mode == 2u) {   // Mode2: occupancy, then the residual stream over the active voxels
        uint32_t active = 0;
        p.bad_occupancy = in.occupancy == nullptr || l.occupancy >= in.occupancy_rows;
        if (!p.bad_occupancy) {
            const uint32_t* occ = reinterpret_cast<const uint32_t*>(in.occupancy + (size_t)l.occupancy * 80u);
            for (int w = 0; w < 16; ++w) active += __popc(occ[w]);   // the 8 x 64-bit voxel mask
        }
        p.fine = StreamPlan{active, 4u, l.fine_kf, (l.header >> 4) & 3u, l.fine_control, l.fine_key,
                            l.fine_max_local};
        p.has_fine = p.has_occupancy = true;
        p.total += 80u + p.fine.bytes();
    }
    return p;
}

// validateRenderTemporalControlStreamData (src/render_temporal_decode.cpp:201-222) and the FP16
// frame range of packRenderTemporalControlStream (:254-256), over the lanes of a warp: 0, 1
// ("invalid render temporal control stream"), 2 ("render temporal fp16 keyframe frame exceeds
// uint8 range") or 3 (rows beyond the caller's arrays).
__device__ uint32_t check_stream(const PackInputs& in, const StreamPlan& st, uint32_t lane)
{
    if ((unsigned long long)st.first_control + st.controls > in.control_rows ||
        (unsigned long long)st.first_key + st.keys > in.key_rows)
        return 3u;
    bool bad = st.controls == 0u || st.max_local == 0u;
    for (uint32_t c = lane; c < st.controls && !bad; c += 32u) {
        const uint32_t d = in.desc[st.first_control + c];
        const uint32_t start = d & 0xFFFFu, count = (d >> 16) & 0xFFu, reserved = d >> 24;
        bad = start + count > st.keys || count > st.bins * st.max_local || (reserved != 0u && reserved > st.max_local);
    }
    if (__any_sync(0xFFFFFFFFu, bad)) return 1u;
    bool range = false;
    if (st.codec != 1u)
        for (uint32_t k = lane; k < st.keys && !range; k += 32u) range = in.key_frame[st.first_key + k] > 255u;
    return __any_sync(0xFFFFFFFFu, range) ? 2u : 0u;
}

// renderTemporalFloatToHalfBits (src/render_temporal_decode.cpp:135-165): truncating exponent
// rebias with the mantissa rounded half up, overflow to infinity, small values to signed zero.
__device__ __forceinline__ uint32_t float_to_half_bits(float value)
{
    const uint32_t bits = __float_as_uint(value);
    const uint32_t sign = (bits >> 16) & 0x8000u;
    int exponent = (int)((bits >> 23) & 0xFFu) - 127 + 15;
    uint32_t mantissa = bits & 0x7FFFFFu;
    if (exponent <= 0) {
        if (exponent < -10) return sign;
        mantissa |= 0x800000u;
        return sign | (((mantissa >> (uint32_t)(1 - exponent)) + 0x1000u) >> 13);
    }
    if (exponent >= 31) return sign | 0x7C00u;
    const uint32_t rounded = (mantissa + 0x1000u) >> 13;
    if (rounded == 0x400u) {
        ++exponent;
        return exponent >= 31 ? (sign | 0x7C00u) : (sign | ((uint32_t)exponent << 10));
    }
    return sign | ((uint32_t)exponent << 10) | (rounded & 0x3FFu);
}

// Writes a stream at out[0 ..): descriptors, bin index and keyframes, each section padded to words.
// Bin rows are 8 bytes apart and 4-byte aligned: an 8-bin section is a straight copy of its rows, a
// 4-bin section the first word of each.  FP32 keys are two words each (frame and zero half, value);
// FP16 keys go four at a time into three words (3 bytes each: frame, half low, half high).
__device__ void write_stream(const PackInputs& in, const StreamPlan& st, uint32_t* out, uint32_t lane)
{
    for (uint32_t c = lane; c < st.controls; c += 32u) out[c] = in.desc[st.first_control + c];
    out += st.controls;
    const uint32_t* rows = reinterpret_cast<const uint32_t*>(in.bins + (size_t)st.first_control * 8u);
    if (st.bins == 8u) {
        for (uint32_t w = lane; w < 2u * st.controls; w += 32u) out[w] = rows[w];
    } else {                     // 4 bins
        for (uint32_t c = lane; c < st.controls; c += 32u) out[c] = rows[2u * c];
    }
    out += st.bin_bytes() / 4u;
    const uint16_t* fr = in.key_frame + st.first_key;
    const float* val = in.key_value + st.first_key;
    if (st.codec == 1u) {        // RenderTemporalPackedKeyframeFp32: u16 frame, u16 0, f32 value
        for (uint32_t k = lane; k < st.keys; k += 32u) {
            out[2u * k] = fr[k];
            out[2u * k + 1u] = __float_as_uint(val[k]);
        }
        return;
    }
    const uint32_t words = st.key_bytes() / 4u;
    for (uint32_t g = lane; 3u * g < words; g += 32u) {
        uint32_t b[12];
        for (uint32_t j = 0; j < 4u; ++j) {
            const uint32_t k = 4u * g + j;
            const bool on = k < st.keys;
            const uint32_t h = on ? float_to_half_bits(val[k]) : 0u;
            b[3u * j] = on ? (fr[k] & 0xFFu) : 0u;
            b[3u * j + 1u] = h & 0xFFu;
            b[3u * j + 2u] = h >> 8;
        }
        for (uint32_t q = 0; q < 3u && 3u * g + q < words; ++q)
            out[3u * g + q] = b[4u * q] | (b[4u * q + 1u] << 8) | (b[4u * q + 2u] << 16) | (b[4u * q + 3u] << 24);
    }
}

// Pass 1, one warp per leaf: the leaf's size in words into words[leaf], and the lowest failing
// leaf (leaf << 2 | reason) into *err.
__global__ void __launch_bounds__(256) leaf_sizes_kernel(PackInputs in, uint32_t n, uint32_t* __restrict__ words,
                                                        unsigned long long* err)
{
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    for (uint32_t leaf = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); leaf < n; leaf += warps) {
        const LeafStreams l = in.leaves[leaf];
        const LeafPlan p = plan_leaf(in, l);
        uint32_t reason = p.bad_occupancy ? 3u : 0u;
        if (p.mode != 0u && !reason) {
            reason = check_stream(in, p.coarse, lane);
            if (!reason && p.has_fine) reason = check_stream(in, p.fine, lane);
        }
        if (lane == 0) {
            words[leaf] = p.total / 4u;
            if (reason) atomicMin(err, ((unsigned long long)leaf << 2) | reason);
        }
    }
}

// In-place exclusive scan of words[0..n) by one CTA (each thread a contiguous run); words[n] and
// *total receive the sum.
__global__ void __launch_bounds__(kScanThreads) words_scan_kernel(uint32_t* __restrict__ words, uint32_t n,
                                                                  unsigned long long* total)
{
    __shared__ unsigned long long s_part[kScanThreads];
    const uint32_t tid = threadIdx.x;
    const uint32_t per = (n + kScanThreads - 1) / kScanThreads;
    const uint32_t b = tid * per, e = min(n, b + per);
    unsigned long long sum = 0;
    for (uint32_t i = b; i < e; ++i) sum += words[i];
    s_part[tid] = sum;
    __syncthreads();
    for (uint32_t off = 1; off < kScanThreads; off <<= 1) {
        const unsigned long long v = tid >= off ? s_part[tid - off] : 0ull;
        __syncthreads();
        s_part[tid] += v;
        __syncthreads();
    }
    unsigned long long run = s_part[tid] - sum;
    for (uint32_t i = b; i < e; ++i) {
        const uint32_t w = words[i];
        words[i] = (uint32_t)run;
        run += w;
    }
    if (tid == kScanThreads - 1) {
        words[n] = (uint32_t)s_part[tid];
        *total = s_part[tid];
    }
}

// Pass 2, one warp per leaf: every word of the leaf, header and prefix included.
__global__ void __launch_bounds__(256) leaf_write_kernel(PackInputs in, uint32_t n, const uint32_t* __restrict__ offsets,
                                                        uint32_t* __restrict__ payload)
{
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    for (uint32_t leaf = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); leaf < n; leaf += warps) {
        const LeafStreams l = in.leaves[leaf];
        const LeafPlan p = plan_leaf(in, l);
        uint32_t* out = payload + offsets[leaf];
        if (lane == 0) out[0] = l.header;
        if (p.mode == 0u) continue;
        if (lane == 0) out[1] = (uint32_t)l.coarse_kf | ((uint32_t)l.fine_kf << 16);
        out += 2;
        write_stream(in, p.coarse, out, lane);
        out += p.coarse.bytes() / 4u;
        if (p.has_occupancy) {
            const uint32_t* occ = reinterpret_cast<const uint32_t*>(in.occupancy + (size_t)l.occupancy * 80u);
            if (lane < 20u) out[lane] = occ[lane];
            out += 20;
        }
        if (p.has_fine) write_stream(in, p.fine, out, lane);
    }
}

}  // namespace

extern "C" int vbt_pack_payload(const uint8_t* d_blocks, const uint64_t* d_block_offsets, uint32_t leaf_count,
                                uint32_t* d_offsets, uint32_t* d_payload, uint64_t payload_capacity_words,
                                uint64_t* total_words, void* stream)
{
    using vbtb::set_last_error;
    if (!d_block_offsets || !d_offsets || !total_words || (leaf_count && !d_blocks))
        return set_last_error(VBT_STATUS_INVALID_ARGUMENT, "null argument");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    unsigned long long* d_total = nullptr;
    cudaError_t e = cudaMallocAsync(reinterpret_cast<void**>(&d_total), sizeof(unsigned long long), s);
    if (e != cudaSuccess) return set_last_error(VBT_STATUS_CUDA, std::string("cudaMallocAsync: ") + cudaGetErrorString(e));
    payload_offsets_kernel<<<1, kScanThreads, 0, s>>>(reinterpret_cast<const unsigned long long*>(d_block_offsets),
                                                      leaf_count, d_offsets, d_total);
    unsigned long long total = 0;
    e = cudaMemcpyAsync(&total, d_total, sizeof(total), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFreeAsync(d_total, s);
    if (e != cudaSuccess) return set_last_error(VBT_STATUS_CUDA, std::string("payload offsets: ") + cudaGetErrorString(e));
    *total_words = total;
    if (total > 0xFFFFFFFFull) return set_last_error(VBT_STATUS_LIMIT, "payload exceeds 2^32 words (the format's offsets are 32-bit)");
    if (total > payload_capacity_words) return set_last_error(VBT_STATUS_LIMIT, "payload buffer smaller than the packed payload");
    if (total == 0) return VBT_STATUS_OK;
    if (!d_payload) return set_last_error(VBT_STATUS_INVALID_ARGUMENT, "null payload buffer");
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const uint32_t need = (leaf_count + 7u) / 8u;
    const uint32_t grid = need < 8u * (uint32_t)sms ? (need ? need : 1u) : 8u * (uint32_t)sms;
    payload_copy_kernel<<<grid, 256, 0, s>>>(d_blocks, reinterpret_cast<const unsigned long long*>(d_block_offsets),
                                             leaf_count, d_offsets, d_payload);
    e = cudaGetLastError();
    return e == cudaSuccess ? VBT_STATUS_OK
                            : set_last_error(VBT_STATUS_CUDA, std::string("payload_copy_kernel: ") + cudaGetErrorString(e));
}

extern "C" int vbt_pack_leaves(const vbt_leaf_streams* d_leaves, uint32_t leaf_count, const uint32_t* d_descriptors,
                               const uint8_t* d_bins, uint64_t control_rows, const uint16_t* d_key_frames,
                               const float* d_key_values, uint64_t key_rows, const uint8_t* d_occupancy,
                               uint64_t occupancy_rows, uint32_t* d_offsets, uint32_t* d_payload,
                               uint64_t payload_capacity_words, uint64_t* total_words, void* stream)
{
    using vbtb::set_last_error;
    static_assert(sizeof(LeafStreams) == sizeof(vbt_leaf_streams), "vbt_leaf_streams layout");
    if (!d_offsets || !total_words || (leaf_count && !d_leaves))
        return set_last_error(VBT_STATUS_INVALID_ARGUMENT, "null argument");
    if ((control_rows && (!d_descriptors || !d_bins)) || (key_rows && (!d_key_frames || !d_key_values)))
        return set_last_error(VBT_STATUS_INVALID_ARGUMENT, "null stream array");
    if (((reinterpret_cast<uintptr_t>(d_occupancy) | reinterpret_cast<uintptr_t>(d_bins)) & 3u) != 0u)
        return set_last_error(VBT_STATUS_INVALID_ARGUMENT, "bin rows and occupancy sections must be 4-byte aligned");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    unsigned long long* d_tmp = nullptr;   // [0] total words, [1] lowest failing leaf << 2 | reason
    cudaError_t e = cudaMallocAsync(reinterpret_cast<void**>(&d_tmp), 2 * sizeof(unsigned long long), s);
    if (e != cudaSuccess) return set_last_error(VBT_STATUS_CUDA, std::string("cudaMallocAsync: ") + cudaGetErrorString(e));
    e = cudaMemsetAsync(d_tmp + 1, 0xFF, sizeof(unsigned long long), s);
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const uint32_t need = (leaf_count + 7u) / 8u;
    const uint32_t grid = need < 8u * (uint32_t)sms ? (need ? need : 1u) : 8u * (uint32_t)sms;
    const PackInputs in{reinterpret_cast<const LeafStreams*>(d_leaves), d_descriptors, d_bins, d_key_frames,
                        d_key_values, d_occupancy, control_rows, key_rows, d_occupancy ? occupancy_rows : 0ull};
    if (e == cudaSuccess) {
        leaf_sizes_kernel<<<grid, 256, 0, s>>>(in, leaf_count, d_offsets, d_tmp + 1);
        words_scan_kernel<<<1, kScanThreads, 0, s>>>(d_offsets, leaf_count, d_tmp);
        e = cudaGetLastError();
    }
    unsigned long long h[2] = {0ull, ~0ull};
    if (e == cudaSuccess) e = cudaMemcpyAsync(h, d_tmp, sizeof(h), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFreeAsync(d_tmp, s);
    if (e != cudaSuccess) return set_last_error(VBT_STATUS_CUDA, std::string("leaf sizes: ") + cudaGetErrorString(e));
    *total_words = h[0];
    if (h[1] != ~0ull) {
        const unsigned long long leaf = h[1] >> 2;
        return set_last_error(VBT_STATUS_INVALID_ARGUMENT,
                              std::string((h[1] & 3u) == 1u   ? "invalid render temporal control stream"
                                          : (h[1] & 3u) == 2u ? "render temporal fp16 keyframe frame exceeds uint8 range"
                                                              : "stream rows outside the given arrays") +
                                  " (leaf " + std::to_string(leaf) + ")");
    }
    if (h[0] > 0xFFFFFFFFull) return set_last_error(VBT_STATUS_LIMIT, "payload exceeds 2^32 words (the format's offsets are 32-bit)");
    if (h[0] > payload_capacity_words) return set_last_error(VBT_STATUS_LIMIT, "payload buffer smaller than the packed payload");
    if (h[0] == 0) return VBT_STATUS_OK;
    if (!d_payload) return set_last_error(VBT_STATUS_INVALID_ARGUMENT, "null payload buffer");
    leaf_write_kernel<<<grid, 256, 0, s>>>(in, leaf_count, d_offsets, d_payload);
    e = cudaGetLastError();
    return e == cudaSuccess ? VBT_STATUS_OK
                            : set_last_error(VBT_STATUS_CUDA, std::string("leaf_write_kernel: ") + cudaGetErrorString(e));
}
