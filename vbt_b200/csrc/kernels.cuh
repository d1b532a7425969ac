// kernels.cuh -- launch-argument structs and launchers shared between the kernel and C-ABI units.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

#include "vbt_format.cuh"

namespace vbtb {

struct AssetGeom {
    uint32_t width, height, depth, frames;
    uint32_t lcx, lcy, lcz, leaf_count;
    uint32_t profile;       // 2 = scientific, otherwise render-temporal
    uint32_t scale_count;
    uint64_t payload_words;
    uint32_t stage_bytes;   // shared-memory leaf stage of the render decode kernel (0 = none)
    uint32_t max_window;    // largest 16-byte-aligned window of a non-EMPTY leaf
    uint32_t sparse;        // 1: render-temporal with most leaves EMPTY (the point-query shape)
};

struct DeviceAsset {
    AssetGeom g;
    const uint32_t* offsets;     // leaf_count + 1 words
    const uint32_t* payload;     // payload words
    const float* scales;         // coarse AC scales (scientific)
    const float* basis;          // scientific DCT basis table [frames][64]
    LeafEntry* entries;          // leaf table (kernel a)
    uint32_t* compact;           // page table: leaf -> rank or kNoRank
    uint32_t* active_list;       // rank -> leaf
    uint32_t* counters;          // [0] active count, [1] walk error flags
    unsigned long long* err;     // first failing (leaf << 8 | status), ~0 when none
    unsigned long long* tile_state;  // look-back tile descriptors
    uint8_t* key_sorted;         // per leaf: bit 0 its decoded controls' key frames strictly increase,
                                 // bit 1 none of their FP16 key values is a NaN
    unsigned long long* work;    // kWorkSlots leaf-work counters [epoch:32 | next index:32]
};

// Decode launches of one asset take their leaves from a work counter; launch number n uses slot
// n % kWorkSlots tagged with epoch n + 1, so up to kWorkSlots launches of one asset may run at
// the same time.
constexpr uint32_t kWorkSlots = 64;

// Frames of one decode launch (the frame list travels as a kernel parameter).
constexpr int kMaxLaunchFrames = 128;

// Fixed shared memory of the render decode kernel besides its leaf stage (rt_kernel_leaf.cuh:
// barrier, frame tables, axis weights, 9 warps x (x-lerp + y-lerp rows), 3072-float controls,
// reciprocal table, axis weights as 16-byte rows).
constexpr uint32_t kLeafFixedBytes =
    16 + 6 * kMaxLaunchFrames + 576 + 9 * 196 * 8 + 9 * 112 * 16 + 3072 * 4 + 256 * 4 + 768;

constexpr int kWalkThreads = 256;
constexpr int kWalkTile = 256;   // leaves per walker CTA (one scan element per thread)

// Decode work is done one leaf per warp; kDecodeWarps warps per CTA.
constexpr int kDecodeWarps = 8;
constexpr int kCtrlSlots = 343 + 512;   // coarse (<= 7^3) + fine (<= 7^3) or shell (<= 512) values
// per-warp shared slots: max(render controls, scientific 64 controls + 16 basis grids of 4^3)
constexpr int kWarpSlots = 64 + 16 * 64 > kCtrlSlots ? 64 + 16 * 64 : kCtrlSlots;

// One slice or frame request of a mixed serving step (serve_mixed_kernel, serve_mixed.cuh): the
// kind, the asset (an index into the step's DeviceAsset array), its running tile offset and its
// device buffers.
constexpr uint32_t kMixedSlice = 1, kMixedFrames = 2;
constexpr uint32_t kMaxMixedReqs = 256;
struct MixedReq {
    uint32_t kind, asset;
    uint32_t n;       // frames: frames
    uint32_t a0;      // slice: z
    int32_t t0, t1;   // slice: frames [t0, t1)
    uint64_t first;   // tiles of the step before this request's
    uint64_t in;      // frames: device address of its int32 frame list
    uint64_t out;     // device address of its result
};
// Tiles of one request of a mixed step (host and device agree on this count).
uint64_t mixed_request_tiles(const MixedReq& r, const AssetGeom& g);
// A mixed step as a CUDA graph (work-counter reset, then the persistent kernel), built on first
// use and relaunched with the next step's parameters.
struct MixedStepGraph {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaGraphNode_t kernel = nullptr;
};
// Launch one mixed step: reqs[k] (device) with running tile offsets summing to n_tiles; errs[k]
// receive each request's first failing (leaf << 8 | status).  counter: an 8-byte device word of
// the caller's (reset by the step).  With a graph, the step replays it (its parameters updated).
int launch_serve_mixed(const DeviceAsset* assets, const MixedReq* reqs, uint32_t k, uint64_t n_tiles,
                       unsigned long long* counter, unsigned long long* errs, MixedStepGraph* graph, cudaStream_t s);
void release_mixed_graph(MixedStepGraph& g);

void launch_walk(const DeviceAsset& a, uint32_t epoch, cudaStream_t s);
// page table only, from the leaf table the walker built (same predicate, same ranks)
void launch_page_table(const DeviceAsset& a, uint32_t epoch, cudaStream_t s);
// Per-asset key-order analysis (after a walk): sets key_sorted[] and the kFlagSorted /
// kFlagHalfPlain bits of the leaf table.  Runs at load and after every re-upload; later walks copy
// the bits from key_sorted.
void launch_key_order(const DeviceAsset& a, cudaStream_t s);
// Decode `nframes` frames (frames[] on the host, <= kMaxLaunchFrames) of every active leaf into the cache:
// out[f * cache_frame_stride + rank * 512 + voxel].
void launch_decode_cache(const DeviceAsset& a, uint32_t seq, const int* frames, int nframes, float* out,
                         uint64_t cache_frame_stride, int grid, cudaStream_t s);
// Dense frames: out[f * X*Y*Z + (z*Y + y)*X + x]; every leaf (EMPTY ones write zeros).
void launch_decode_dense(const DeviceAsset& a, uint32_t seq, const int* frames, int nframes, float* out, int grid,
                         cudaStream_t s);
// Leaf-per-warp cache decode (same output as launch_decode_cache); grid 0 = one wave.
void launch_decode_cache_warp(const DeviceAsset& a, const int* frames, int nframes, float* out, uint64_t stride,
                              int grid, cudaStream_t s);
int decode_warp_grid();
// (d) scientific window decode on the tensor cores, frames [t0, t0 + n), n <= 64, cache layout.
void launch_sci_window(const DeviceAsset& a, int t0, int n, float* out, uint64_t frame_stride, cudaStream_t s);
// FP64 oracle of a scientific window: stats[0] max |err| (double bits), stats[1] sum err^2
// (double), stats[2] / stats[3] oracle min / max (order-preserving bits).
void launch_control_cache(const DeviceAsset& a, const int* frames, int nframes, float* out, uint64_t stride,
                          cudaStream_t s);
void launch_render_window(const DeviceAsset& a, uint32_t seq, int t0, int n, float* out, uint64_t frame_stride,
                          cudaStream_t s);
void launch_render_window_oracle(const DeviceAsset& a, int t0, int n, const float* vals, uint64_t frame_stride,
                                 unsigned long long* stats, cudaStream_t s);
void launch_key_division_check(uint32_t b_max, unsigned long long* d_out, cudaStream_t s);
void launch_sci_window_oracle(const DeviceAsset& a, int t0, int n, const float* vals, uint64_t frame_stride,
                              unsigned long long* stats, cudaStream_t s);
// Plain path: one CTA per leaf of the whole leaf grid, one frame per launch (the reference
// Studio dispatch shape, VBTStudio/frontend/src/volume_renderer.cpp:704-735).
void launch_decode_cache_plain(const DeviceAsset& a, int frame, float* out, cudaStream_t s);
// Point queries: q[4*i..] = (x, y, z, t); out[i].
// sparse: most leaves are EMPTY (the compacting kernel), else one thread per query
void launch_query_points(const DeviceAsset& a, const uint32_t* q, uint64_t n, float* out, bool sparse, cudaStream_t s);
// Point queries of k requests over several assets in one launch (a device array of DeviceAsset).
// seg: starts[0..k] (first query of each request, starts[k] = n), asset[k], then 8-byte aligned
// outs[k] (result arrays, as 64-bit addresses); decode errors of request r are recorded in errs[r].
void launch_query_points_batch(const DeviceAsset* assets, const uint32_t* seg, uint32_t k, const uint4* q, uint64_t n,
                               unsigned long long* errs, int sparse, cudaStream_t s);   // sparse: 0 none, 1 some, 2 all
// Z-slice over a frame range: out[(t - t0) * X*Y + y*X + x] for t in [t0, t1).
void launch_query_slice(const DeviceAsset& a, uint32_t z, int t0, int t1, float* out, cudaStream_t s);

void upload_axis_tables();

}  // namespace vbtb
