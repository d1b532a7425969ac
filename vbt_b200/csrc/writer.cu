// writer.cu -- the payload half of a VBTPACK4 writer on the GPU (vbt_pack_payload): packed leaf
// blocks, each padded with zero bytes to a whole number of words, concatenated into the payload
// pool, and the word offset table -- what writeRenderTemporalProbeFile
// (src/render_temporal_kf_probe_main.cpp:2561-2585) builds on the host before it writes the
// 52-byte header, the offsets and the payload.
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
