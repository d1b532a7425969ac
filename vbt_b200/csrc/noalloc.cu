// noalloc.cu -- the active-leaf page table built without allocating any device memory.
//
// Some callers cannot let a library allocate: a renderer or plugin host that sub-allocates all
// device memory from its own pool and hands libraries finished buffers, or a per-frame loop that
// must not call cudaMalloc because it synchronises the device and stalls the frame.  For them,
// vbt_build_page_table_noalloc takes the offsets and payload already in device memory plus the
// output buffers, and keeps its only scratch -- the per-tile descriptors of the cross-CTA prefix
// scan -- in a fixed array of this file that every GPU loading the library holds until exit.
//
// Scratch: kNoAllocMaxTiles descriptors of 8 bytes (512 KiB), one per 256 leaves, so at most
// kNoAllocMaxTiles * 256 leaves per call.  The array is shared by all calls in the process and
// keeps the last call's contents; each call clears the part it uses first.  Calls whose kernels
// overlap on the GPU (on different streams) race on the array.
#include <cuda/atomic>
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/vbt_b200.h"

namespace vbtb {
int set_last_error(int status, const std::string& msg);   // capi.cu: the message of vbt_last_error()
}

namespace {

constexpr uint32_t kTile = 256;
constexpr uint32_t kNoAllocMaxTiles = 65536;
constexpr uint64_t kNoAllocMaxLeaves = (uint64_t)kNoAllocMaxTiles * kTile;

static __device__ __align__(256) unsigned long long g_noalloc_scratch[kNoAllocMaxTiles];

// Same leaf predicate as the asset walker: a render-temporal leaf is active when its offsets stay
// inside the payload and its header's route tag is not EMPTY; every scientific leaf is active.
__global__ void __launch_bounds__(kTile) page_table_noalloc_kernel(const uint32_t* __restrict__ offsets,
                                                                   const uint32_t* __restrict__ payload,
                                                                   uint64_t payload_words, uint32_t leaf_count,
                                                                   uint32_t profile, unsigned long long* tiles,
                                                                   uint32_t* compact, uint32_t* active_list,
                                                                   uint32_t* active_count)
{
    __shared__ uint32_t s_warp[kTile / 32];
    __shared__ uint32_t s_base;
    const uint32_t tile = blockIdx.x;
    const uint32_t leaf = tile * kTile + threadIdx.x;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    bool flag = false;
    if (leaf < leaf_count) {
        if (profile == 2u) {
            flag = true;
        } else {
            const uint32_t wb = __ldg(offsets + leaf), we = __ldg(offsets + leaf + 1);
            flag = we > wb && we <= payload_words && (__ldg(payload + wb) & 3u) != 0u;
        }
    }
    const unsigned bal = __ballot_sync(0xFFFFFFFFu, flag);
    const uint32_t in_warp = __popc(bal & ((1u << lane) - 1u));
    if (lane == 0) s_warp[warp] = __popc(bal);
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t run = 0;
        for (int w = 0; w < (int)(kTile / 32); ++w) {
            const uint32_t c = s_warp[w];
            s_warp[w] = run;
            run += c;
        }
        // descriptor: flag[33:32] (1 = aggregate, 2 = inclusive prefix) | count; zeroed by the host
        cuda::atomic_ref<unsigned long long, cuda::thread_scope_device> self(tiles[tile]);
        uint32_t excl = 0;
        if (tile == 0) {
            self.store((2ull << 32) | run, cuda::memory_order_release);
        } else {
            self.store((1ull << 32) | run, cuda::memory_order_release);
            int j = (int)tile - 1;
            uint32_t spins = 0;
            bool timed_out = false;
            while (j >= 0) {
                cuda::atomic_ref<unsigned long long, cuda::thread_scope_device> st(tiles[j]);
                const unsigned long long v = st.load(cuda::memory_order_acquire);
                const unsigned long long f = (v >> 32) & 3ull;
                if (f == 0ull) {
                    if (++spins > (1u << 22)) {   // bounded wait: report through the count, never hang
                        timed_out = true;
                        break;
                    }
                    __nanosleep(64);
                    continue;
                }
                excl += (uint32_t)(v & 0xFFFFFFFFull);
                if (f == 2ull) break;
                --j;
            }
            self.store((2ull << 32) | (excl + run), cuda::memory_order_release);
            if (timed_out) atomicExch(active_count, 0xFFFFFFFFu);
        }
        s_base = excl;
        if ((tile + 1) * kTile >= leaf_count) atomicCAS(active_count, 0u, excl + run);
    }
    __syncthreads();
    if (leaf < leaf_count) {
        const uint32_t rank = s_base + s_warp[warp] + in_warp;
        compact[leaf] = flag ? rank : 0xFFFFFFFFu;
        if (flag) active_list[rank] = leaf;
    }
}

// Device address of the scratch array, looked up once per device with that device current.  The
// address belongs to the device's primary context, the one the CUDA runtime uses; a process that
// destroys that context (cudaDeviceReset) must not call the entry point again on that device,
// because the cached address would then name memory that is no longer mapped.
std::mutex g_setup_mu;
unsigned long long* g_scratch_ptr[64] = {};

int scratch_for_current_device(unsigned long long** out)
{
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= 64)
        return vbtb::set_last_error(VBT_STATUS_CUDA, std::string("no usable CUDA device: ") + cudaGetErrorString(e));
    std::lock_guard<std::mutex> lock(g_setup_mu);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return vbtb::set_last_error(VBT_STATUS_CUDA, std::string("cudaGetSymbolAddress(page-table scratch): ") +
                                                             cudaGetErrorString(e));
        g_scratch_ptr[dev] = static_cast<unsigned long long*>(p);
    }
    *out = g_scratch_ptr[dev];
    return VBT_STATUS_OK;
}

}  // namespace

extern "C" {

int vbt_build_page_table_noalloc(const uint32_t* d_offsets, const uint32_t* d_payload, uint64_t payload_words,
                                 uint32_t leaf_count, uint32_t profile_type, uint32_t* d_compact,
                                 uint32_t* d_active_list, uint32_t* d_active_count, void* stream)
{
    if (leaf_count == 0 || !d_offsets || !d_compact || !d_active_list || !d_active_count ||
        (profile_type != 2u && !d_payload))
        return vbtb::set_last_error(VBT_STATUS_INVALID_ARGUMENT, "null buffer or zero leaf count");
    if (profile_type > 2u)
        return vbtb::set_last_error(VBT_STATUS_INVALID_ARGUMENT, "Invalid VBTPACK4 profile type.");
    if ((uint64_t)leaf_count > kNoAllocMaxLeaves)
        return vbtb::set_last_error(VBT_STATUS_LIMIT, "leaf_count " + std::to_string(leaf_count) +
                                                          " exceeds the allocation-free page table's limit of " +
                                                          std::to_string(kNoAllocMaxLeaves) + " leaves");
    unsigned long long* scratch = nullptr;
    int st = scratch_for_current_device(&scratch);
    if (st) return st;
    const uint32_t tiles = (leaf_count + kTile - 1) / kTile;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemsetAsync(scratch, 0, sizeof(unsigned long long) * tiles, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_active_count, 0, sizeof(uint32_t), s);
    if (e != cudaSuccess) return vbtb::set_last_error(VBT_STATUS_CUDA, std::string("cudaMemsetAsync: ") + cudaGetErrorString(e));
    page_table_noalloc_kernel<<<tiles, kTile, 0, s>>>(d_offsets, d_payload, payload_words, leaf_count, profile_type,
                                                      scratch, d_compact, d_active_list, d_active_count);
    e = cudaGetLastError();
    if (e != cudaSuccess)
        return vbtb::set_last_error(VBT_STATUS_CUDA, std::string("page_table_noalloc_kernel: ") + cudaGetErrorString(e));
    return VBT_STATUS_OK;
}

}  // extern "C"
