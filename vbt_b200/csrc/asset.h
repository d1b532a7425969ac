// asset.h -- the resident asset behind the opaque vbt_asset handle (shared by the C-ABI and the
// serving loop).
#pragma once

#include <atomic>
#include <cstdint>
#include <mutex>
#include <vector>

#include "../../include/vbt_b200.h"
#include "kernels.cuh"

struct vbt_asset {
    int device = 0;
    vbt_header hdr{};
    vbtb::DeviceAsset dev{};
    uint32_t epoch = 0;
    std::atomic<uint32_t> launch_seq{0};   // decode launches: selects and tags a work-counter slot
    uint64_t device_bytes = 0;
    std::vector<void*> allocations;
    // staging for the host-buffer calls (grow-only)
    void* stage_in = nullptr;
    size_t stage_in_bytes = 0;
    void* stage_out = nullptr;
    size_t stage_out_bytes = 0;
    std::mutex mu;
};
