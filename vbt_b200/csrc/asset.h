// asset.h -- the resident asset behind the opaque vbt_asset handle (shared by the C-ABI and the
// serving loop).
#pragma once

#include <atomic>
#include <cstdint>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/vbt_b200.h"
#include "kernels.cuh"

struct vbt_asset {
    int device = 0;
    vbt_header hdr{};
    vbtb::DeviceAsset dev{};
    uint32_t epoch = 0;
    std::atomic<uint32_t> launch_seq{0};   // decode launches: selects and tags a work-counter slot
    bool sparse = false;   // render-temporal image given at creation with most leaves EMPTY (point-query shape)
    uint64_t device_bytes = 0;
    std::vector<void*> allocations;
    // staging for the host-buffer calls (grow-only)
    void* stage_in = nullptr;
    size_t stage_in_bytes = 0;
    void* stage_out = nullptr;
    size_t stage_out_bytes = 0;
    std::mutex mu;
    unsigned long long* d_stats = nullptr;   // 4 words for the window error oracle's reduction
    // cache-timeline configuration (vbt_autotune_cache / vbt_set_tuning) and its captured graphs,
    // keyed by (first frame, frame count, output, frame stride)
    vbt_tuning tuning{0u, 48u, 0, 0.0f, 0.0f};
    std::mutex graph_mu;
    std::map<std::tuple<int, int, uintptr_t, uint64_t>, cudaGraphExec_t> graphs;
};

namespace vbtb {
// Destroys the asset's captured timeline graphs (tune.cu).
void release_timeline_graphs(vbt_asset* a);
}
