// serve_mixed.cuh -- one persistent launch over the slice and frame requests a serving step
// admitted, of any resident assets, mixed.  Included by kernels.cu (it uses that file's decode
// helpers).  (The step's point requests go to the multi-asset point kernel beside it: a point is a
// chain of dependent loads that wants every thread an SM can hold in flight, while a leaf tile
// needs this kernel's 128 registers per thread.)
//
// The requests form a table (MixedReq, in device memory) with a running count of tiles.  A tile is
// one warp's piece of work:
//   slice   one (leaf of the z layer, frame): the leaf's controls at the frame, then its rows of
//           the layer -- the body of query_slice_kernel;
//   frames  one (leaf, frame) of a dense frame: controls, then all 64 rows of the leaf (zeros for
//           an EMPTY leaf) -- the body of the warp-per-leaf decode_kernel<DENSE>.
// Warps take tiles kTileGrab at a time from a work counter (zeroed before the launch), so the
// tiles of large and small requests spread over the GPU as they come.  Each request has its own
// result array and error word; the values are those of the per-request kernels, bit for bit.
#pragma once

namespace vbtb {

constexpr uint32_t kTileGrab = 4;

// Tiles of one request (the host's count: same arithmetic).
__host__ __device__ __forceinline__ uint64_t mixed_tiles(const MixedReq& r, const AssetGeom& g)
{
    return r.kind == kMixedSlice ? (uint64_t)g.lcx * g.lcy * (uint64_t)(r.t1 - r.t0) : (uint64_t)g.leaf_count * r.n;
}

// Slice tile: rows of leaf `li` of the z layer at frame t into the request's [t - t0][y][x] output.
__device__ __forceinline__ void mixed_slice_tile(const DeviceAsset& a, const MixedReq& r, uint32_t li, int t,
                                                 float* __restrict__ s_ctrl, unsigned long long* err, int lane)
{
    const uint32_t bz = min(a.g.lcz - 1u, r.a0 >> 3);
    const int lz = (int)(r.a0 - bz * 8u);
    const uint32_t leaf = bz * a.g.lcx * a.g.lcy + li;
    const LeafEntry e = a.entries[leaf];
    uint32_t bx, by, bzz;
    int w, h, d;
    leaf_extent(a.g, leaf, bx, by, bzz, w, h, d);
    const uint32_t st = entry_status(e);
    const bool sci = a.g.profile == 2u;
    const bool empty = !sci && (e.header & 3u) == kModeEmpty;
    bool oob = false;
    const bool in_range = lz < d && (!sci || (uint32_t)t < a.g.frames);
    if (st != kOk && lane == 0) record_error(err, leaf, st);
    if (in_range && !empty && st == kOk) {
        if (sci) sci_decode_controls(a, e, (uint32_t)t, s_ctrl, lane, oob);
        else rt_decode_controls(a, e, clamp_frame(t, (int)a.g.frames), s_ctrl, lane);
    }
    __syncwarp();
    if (lane < 8 && lane < h) {
        float v[8];
        if (!in_range || empty || st != kOk) {
            for (int i = 0; i < 8; ++i) v[i] = 0.0f;
        } else if (sci) {
            sci_row(a, e, s_ctrl, (uint32_t)t, w, h, d, lane, lz, v, oob);
        } else {
            rt_row(a, e, s_ctrl, w, h, d, lane, lz, v);
        }
        float* out = reinterpret_cast<float*>(r.out);
        float* dst = out + (uint64_t)(t - r.t0) * a.g.width * a.g.height + (uint64_t)(by * 8 + lane) * a.g.width + bx * 8;
        for (int i = 0; i < w; ++i) dst[i] = v[i];
    }
    if (__any_sync(0xFFFFFFFFu, oob) && lane == 0) record_error(err, leaf, kErrDecodeOob);
    __syncwarp();
}

// Frame tile: all voxels of `leaf` at frame index `fr` (as given) into the dense frame `frame_out`.
__device__ __forceinline__ void mixed_frame_tile(const DeviceAsset& a, uint32_t leaf, int fr, float* __restrict__ fb,
                                                 float* __restrict__ s_ctrl, unsigned long long* err, int lane)
{
    const LeafEntry e = a.entries[leaf];
    uint32_t bx, by, bz;
    int w, h, d;
    leaf_extent(a.g, leaf, bx, by, bz, w, h, d);
    const bool sci = a.g.profile == 2u;
    const bool empty = !sci && (e.header & 3u) == kModeEmpty;
    const uint32_t st = entry_status(e);
    if (st != kOk && lane == 0) record_error(err, leaf, st);
    const bool scatter = sci && st == kOk && (e.header & 3u) == 1u && (e.info & kFlagSorted) != 0u;
    bool oob = false;
    if (!empty && st == kOk) {
        if (sci) sci_decode_controls(a, e, (uint32_t)fr, s_ctrl, lane, oob);
        else rt_decode_controls(a, e, clamp_frame(fr, (int)a.g.frames), s_ctrl, lane);
    }
    __syncwarp();
    for (int rr = lane; rr < 64; rr += 32) {
        const int ly = rr & 7, lz = rr >> 3;
        float v[8];
        if (empty || st != kOk) {
#pragma unroll
            for (int i = 0; i < 8; ++i) v[i] = 0.0f;
        } else if (sci) {
            sci_row(a, e, s_ctrl, (uint32_t)fr, w, h, d, ly, lz, v, oob, scatter);
        } else {
            rt_row(a, e, s_ctrl, w, h, d, ly, lz, v);
        }
        if (ly < h && lz < d) {
            float* dst = fb + ((uint64_t)(bz * 8 + lz) * a.g.height + (by * 8 + ly)) * a.g.width + bx * 8;
            if (w == 8 && (((uintptr_t)dst) & 15u) == 0u) {
                reinterpret_cast<float4*>(dst)[0] = make_float4(v[0], v[1], v[2], v[3]);
                reinterpret_cast<float4*>(dst)[1] = make_float4(v[4], v[5], v[6], v[7]);
            } else {
                for (int i = 0; i < w; ++i) dst[i] = v[i];
            }
        }
    }
    if (scatter && (uint32_t)fr < a.g.frames) {
        __syncwarp();   // the rows written by the other lanes are visible
        sci_scatter_frame(a, e, (uint32_t)fr, w, h, d, lane,
                          [&](uint32_t li) {
                              return fb + ((uint64_t)(bz * 8 + (li >> 6)) * a.g.height + (by * 8 + ((li >> 3) & 7u))) *
                                              a.g.width +
                                          bx * 8 + (li & 7u);
                          },
                          oob);
    }
    if (__any_sync(0xFFFFFFFFu, oob) && lane == 0) record_error(err, leaf, kErrDecodeOob);
    __syncwarp();
}

constexpr int kMixedWarps = 8;

__global__ void __launch_bounds__(kMixedWarps * 32) serve_mixed_kernel(const DeviceAsset* __restrict__ assets,
                                                                       const MixedReq* __restrict__ reqs, uint32_t k,
                                                                       uint64_t n_tiles, unsigned long long* counter,
                                                                       unsigned long long* errs)
{
    __shared__ __align__(16) float s_ctrl_all[kMixedWarps][kWarpSlots];
    __shared__ uint64_t s_first[kMaxMixedReqs + 1];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (uint32_t i = (uint32_t)tid; i < k; i += blockDim.x) s_first[i] = reqs[i].first;
    if (tid == 0) s_first[k] = n_tiles;
    __syncthreads();
    float* s_ctrl = s_ctrl_all[warp];
    for (;;) {
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(counter, (unsigned long long)kTileGrab);
        base = __shfl_sync(0xFFFFFFFFu, base, 0);
        if (base >= n_tiles) break;   // the counter only grows: every later grab is past the end too
        for (uint32_t j = 0; j < kTileGrab; ++j) {
            const uint64_t tile = base + j;
            if (tile >= n_tiles) break;
            int lo = 0, hi = (int)k - 1;
            while (lo < hi) {   // the last request whose first tile is at or before this one
                const int mid = (lo + hi + 1) >> 1;
                if (s_first[mid] <= tile) lo = mid;
                else hi = mid - 1;
            }
            const MixedReq rq = reqs[lo];
            const DeviceAsset& a = assets[rq.asset];
            const uint64_t u = tile - rq.first;
            unsigned long long* err = errs + lo;
            if (rq.kind == kMixedSlice) {
                const uint32_t layer = a.g.lcx * a.g.lcy;
                mixed_slice_tile(a, rq, (uint32_t)(u % layer), rq.t0 + (int)(u / layer), s_ctrl, err, lane);
            } else {
                const uint32_t L = a.g.leaf_count;
                const uint64_t fi = u / L;
                const int fr = reinterpret_cast<const int*>(rq.in)[fi];
                float* fb = reinterpret_cast<float*>(rq.out) + fi * ((uint64_t)a.g.width * a.g.height * a.g.depth);
                mixed_frame_tile(a, (uint32_t)(u % L), fr, fb, s_ctrl, err, lane);
            }
        }
    }
}

static int mixed_grid(uint64_t n_tiles)
{
    static int full = 0;
    if (!full) {
        int dev = 0, sms = 0, per = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, serve_mixed_kernel, kMixedWarps * 32, 0);
        full = sms * (per > 0 ? per : 1);
    }
    const uint64_t want = (n_tiles + (uint64_t)kTileGrab * kMixedWarps - 1) / ((uint64_t)kTileGrab * kMixedWarps);
    return (int)(want < (uint64_t)full ? (want > 0 ? want : 1) : (uint64_t)full);
}

}  // namespace vbtb
