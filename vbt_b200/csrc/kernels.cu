// kernels.cu -- the hand-written sm_100a kernels of the decode path.
//
//  (a) walk_kernel          payload walker: validates every leaf once per upload, writes the
//                           32-byte leaf table, and builds the active-leaf page table by
//                           warp-ballot/popc compaction with a single-pass decoupled look-back.
//      page_table_kernel    the per-frame page table from the leaf table's active flags.
//  (b) decode_*_kernel      warp-per-leaf decode into the current-frame voxel cache (512 FP32
//                           per active leaf) or into dense frames, several frames per launch.
//  (c) query_*_kernel       batched (x, y, z, t) point queries and z-slice queries.
//
// Render-temporal arithmetic is bit-exact with the reference CPU decoder (every float op is an
// explicitly rounded _rn intrinsic; see rt_search.cuh).  Scientific coarse controls are summed in
// compensated float-float arithmetic (error-free products and two-sums) to track the reference's
// double accumulation (render/src/scientific_decode.cpp:82-97) without FP64 on the device.
#include <cuda/atomic>

#include <mutex>

#include "kernels.cuh"
#include "rt_search.cuh"

namespace vbtb {

// Axis weight table (see AxisWeight), filled once per process by upload_axis_tables().
__constant__ AxisWeight c_axis[kAxisRes * kAxisExt * kAxisPos];
__device__ AxisWeight g_axis[kAxisRes * kAxisExt * kAxisPos];
// Scientific trilinear axes: [0] coarse 4^3 grid (f = x/7*3, clamp 0..2), [1] dense 3^3, [2] dense 4^3.
__constant__ AxisWeight c_sci_axis[3][8];
}  // namespace vbtb

#include <cuda_fp16.h>

#include "rt_staged.cuh"

namespace vbtb {

// ---------------------------------------------------------------------------------------------
// host: axis tables, computed with the same float expressions as the reference
// (render/src/render_smoke_vbt_bench_main.cpp:201-234; render/src/scientific_decode.cpp:99-123,
// :137-149).  Host float arithmetic is IEEE binary32 with round-to-nearest and no contraction
// (this translation unit's host code is compiled with -ffp-contract=off).
void upload_axis_tables()
{
    static AxisWeight tab[kAxisRes * kAxisExt * kAxisPos];
    for (int res = 0; res < kAxisRes; ++res)
        for (int ext = 0; ext < kAxisExt; ++ext)
            for (int pos = 0; pos < kAxisPos; ++pos) {
                AxisWeight w{0, 0, 0, 0, 0.0f, 1.0f};
                if (res >= 2) {
                    const float scale = 7.0f / (float)(res - 1);
                    const float maxp = (float)(ext - 1 > 0 ? ext - 1 : 0);
                    float p = (float)pos;
                    p = p < 0.0f ? 0.0f : (p > maxp ? maxp : p);
                    int i1 = 1;
                    while (i1 < res - 1 && (float)i1 * scale < p) ++i1;
                    const int i0 = i1 - 1 > 0 ? i1 - 1 : 0;
                    const float c0 = (float)i0 * scale, c1 = (float)i1 * scale;
                    const volatile float num = p - c0;
                    const volatile float den = c1 - c0;
                    const float t = (c1 > c0) ? (num / den) : 0.0f;
                    w.i0 = (uint8_t)i0;
                    w.i1 = (uint8_t)i1;
                    w.t = t;
                    w.omt = 1.0f - t;
                }
                tab[axis_index(res, ext, pos)] = w;
            }
    cudaMemcpyToSymbol(c_axis, tab, sizeof(tab));
    cudaMemcpyToSymbol(g_axis, tab, sizeof(tab));
    AxisWeight sci[3][8];
    const int grids[3] = {4, 3, 4};
    for (int g = 0; g < 3; ++g)
        for (int p = 0; p < 8; ++p) {
            const int res = grids[g];
            const volatile float q = (float)p / 7.0f;
            const float f = q * (float)(res - 1);
            int i0 = (int)floorf(f);
            i0 = i0 < 0 ? 0 : (i0 > res - 2 ? res - 2 : i0);
            const float t = f - (float)i0;
            sci[g][p] = AxisWeight{(uint8_t)i0, (uint8_t)(i0 + 1), 0, 0, t, 1.0f - t};
        }
    cudaMemcpyToSymbol(c_sci_axis, sci, sizeof(sci));
}

// ---------------------------------------------------------------------------------------------
// shared helpers

__device__ __forceinline__ void record_error(unsigned long long* err, uint32_t leaf, uint32_t status)
{
    atomicMin(err, ((unsigned long long)leaf << 8) | status);
}

__device__ __forceinline__ void leaf_extent(const AssetGeom& g, uint32_t leaf, uint32_t& bx, uint32_t& by,
                                            uint32_t& bz, int& w, int& h, int& d)
{
    bx = leaf % g.lcx;
    by = (leaf / g.lcx) % g.lcy;
    bz = leaf / (g.lcx * g.lcy);
    const int ex = (int)g.width - (int)bx * 8, ey = (int)g.height - (int)by * 8, ez = (int)g.depth - (int)bz * 8;
    w = ex < 8 ? ex : 8;
    h = ey < 8 ? ey : 8;
    d = ez < 8 ? ez : 8;
}

// ---------------------------------------------------------------------------------------------
// (a) payload walker + page table

// Validate one render-temporal leaf with the whole warp (src/render_temporal_payload.cpp:234-311
// for the layout and Mode2 occupancy checks; src/render_temporal_decode.cpp:316-339 for the
// stream-size and keyframe-range checks the decoder would make on every control it decodes).
__device__ LeafEntry walk_rt_leaf(const DeviceAsset& a, uint32_t leaf, int lane)
{
    const uint32_t* __restrict__ pw = a.payload;
    LeafEntry e{};
    const uint32_t wb = __ldg(a.offsets + leaf), we = __ldg(a.offsets + leaf + 1);
    e.word_off = wb;
    if (we <= wb || we > a.g.payload_words) {   // offsets are re-checked here for re-uploaded images
        e.info = kErrDecodeOob << 16;
        return e;
    }
    const uint64_t bytes = 4ull * (we - wb);
    e.header = ldw(pw, wb);
    const uint32_t mode = e.header & 3u;
    if (mode == kModeEmpty) return e;
    uint32_t status = kOk, flags = kFlagActive;
    if (bytes < 8u) {
        e.info = flags | (kErrPrefixMissing << 16);
        return e;
    }
    const uint32_t ccodec = (e.header >> 2) & 3u, fcodec = (e.header >> 4) & 3u;
    const uint32_t cres = (e.header >> 6) & 7u, fres = (e.header >> 9) & 7u;
    e.kf = ldw(pw, wb + 1);
    const uint32_t ckf = e.kf & 0xFFFFu, fkf = e.kf >> 16;
    const uint32_t cc = cres * cres * cres, fc = fres * fres * fres;
    e.coarse_bytes = stream_bytes(cc, 8u, ckf, ccodec);
    const uint32_t fine_off = 8u + e.coarse_bytes;
    uint32_t total = fine_off;
    if (mode == kModeFine6) {
        e.fine_bytes = stream_bytes(fc, 8u, fkf, fcodec);
        total = fine_off + e.fine_bytes;
    } else if (mode == kModeFineCompact) {
        e.fine_bytes = 80u + align4(fkf * key_stride(fcodec));
        total = fine_off + e.fine_bytes;
    }
    uint32_t active = 0;
    if (total > bytes) {
        status = kErrLeafShort;
    } else if (mode == kModeFineCompact) {
        flags |= kFlagOccClamp;
        // occupancy: u64 mask[8] at fine_off, u16 prefix[8] at fine_off + 64
        const uint64_t ob = 4ull * wb + fine_off;
        uint32_t pc = 0, pref = 0;
        if (lane < 8) {
            const uint32_t m0 = ldw(pw, (uint32_t)((ob + 8u * lane) >> 2));
            const uint32_t m1 = ldw(pw, (uint32_t)((ob + 8u * lane + 4u) >> 2));
            pc = __popc(m0) + __popc(m1);
            pref = (ldw(pw, (uint32_t)((ob + 64u + 2u * lane) >> 2)) >> ((lane & 1) * 16)) & 0xFFFFu;
        }
        // exclusive scan of the 8 group popcounts
        uint32_t incl = pc;
        for (int o = 1; o < 8; o <<= 1) {
            const uint32_t v = __shfl_up_sync(0xFFFFFFFFu, incl, o);
            if (lane >= o) incl += v;
        }
        const uint32_t excl = incl - pc;
        const unsigned bad = __ballot_sync(0xFFFFFFFFu, lane < 8 && pref != excl);
        active = __shfl_sync(0xFFFFFFFFu, incl, 7);
        if (bad) {
            status = kErrShellGroupPrefix;
        } else if (active == 0u) {
            status = kErrShellNoActive;
        } else {
            const uint64_t res_off = fine_off + 80u;   // fine_off is 4-aligned
            const uint64_t res_bytes = 4ull * active + 4ull * active + (uint64_t)align4(fkf * key_stride(fcodec));
            if (res_off > bytes || res_bytes > bytes - res_off) status = kErrShellResidualOob;
            else if (res_off + res_bytes != bytes) status = kErrShellTrailing;
            e.shell_off = (uint32_t)res_off;
            e.shell_bytes = (uint32_t)res_bytes;
        }
    }
    if (status == kOk) {
        // coarse controls: keyStart + keyCount must stay inside the keyframe pool
        const uint64_t cbase = 4ull * wb + 8u;
        bool bad = false;
        for (uint32_t c = lane; c < cc; c += 32) {
            const uint32_t dsc = ldw(pw, (uint32_t)((cbase + 4ull * c) >> 2));
            const uint32_t kc = (dsc >> 16) & 0xFFu;
            bad |= kc != 0u && (dsc & 0xFFFFu) + kc > ckf;
        }
        if (__any_sync(0xFFFFFFFFu, bad)) status = kErrKeyRangeOob;
    }
    const bool has_fine = fres > 0u && e.fine_bytes > 0u && mode != kModeGrid4;
    if (status == kOk && has_fine) {
        flags |= kFlagFine;
        if (stream_bytes(fc, 8u, fkf, fcodec) > e.fine_bytes) {
            status = kErrStreamOob;
        } else {
            const uint64_t fbase = 4ull * wb + fine_off;
            bool bad = false;
            for (uint32_t c = lane; c < fc; c += 32) {
                const uint32_t dsc = ldw(pw, (uint32_t)((fbase + 4ull * c) >> 2));
                const uint32_t kc = (dsc >> 16) & 0xFFu;
                bad |= kc != 0u && (dsc & 0xFFFFu) + kc > fkf;
            }
            if (__any_sync(0xFFFFFFFFu, bad)) status = kErrKeyRangeOob;
        }
    }
    if (status == kOk && mode == kModeFineCompact && !has_fine && fkf > 0u) {
        flags |= kFlagShell;
        // Only occupied voxels inside the leaf extent are ever decoded, so only their descriptors
        // are checked (src/render_temporal_decode.cpp:404-450 per voxel of the cropped extent).
        uint32_t bx, by, bz;
        int w, h, d;
        leaf_extent(a.g, leaf, bx, by, bz, w, h, d);
        const uint64_t ob = 4ull * wb + fine_off;
        const uint64_t sbase = 4ull * wb + e.shell_off;
        bool bad = false;
        for (uint32_t v = lane; v < 512u; v += 32) {
            const int lx = v & 7, ly = (v >> 3) & 7, lz = v >> 6;
            if (lx >= w || ly >= h || lz >= d) continue;
            const uint32_t g = v >> 6, bit = v & 63u;
            const uint32_t mw = ldw(pw, (uint32_t)((ob + 8u * g + (bit >= 32 ? 4u : 0u)) >> 2));
            if (((mw >> (bit & 31u)) & 1u) == 0u) continue;
            const uint32_t m0 = ldw(pw, (uint32_t)((ob + 8u * g) >> 2));
            const uint32_t m1 = ldw(pw, (uint32_t)((ob + 8u * g + 4u) >> 2));
            const uint64_t mask = ((uint64_t)m1 << 32) | m0;
            const uint32_t pref = (ldw(pw, (uint32_t)((ob + 64u + 2u * g) >> 2)) >> ((g & 1u) * 16u)) & 0xFFFFu;
            const uint32_t di = (pref + __popcll(mask & ((1ull << bit) - 1ull))) & 0xFFFFu;
            const uint32_t dsc = ldw(pw, (uint32_t)((sbase + 4ull * di) >> 2));
            const uint32_t kc = (dsc >> 16) & 0xFFu;
            bad |= kc != 0u && (dsc & 0xFFFFu) + kc > fkf;
        }
        if (__any_sync(0xFFFFFFFFu, bad)) status = kErrKeyRangeOob;
    }
    if (status == kOk && (a.key_sorted[leaf] & 1u)) flags |= kFlagSorted;
    if (status == kOk && (a.key_sorted[leaf] & 2u)) flags |= kFlagHalfPlain;
    e.info = (active & 0x3FFu) | flags | (status << 16);
    return e;
}

// Key-order analysis of one leaf (one warp): are the key frames of every control the decoders
// read strictly increasing (key_sorted bit 0, kFlagSorted)?  And is no FP16 key value of those
// controls a NaN (bit 1, kFlagHalfPlain: the hardware half conversion then equals the reference's
// bit for bit)?  Controls with an out-of-pool key range are never decoded (see decode_control) and
// are skipped.
__global__ void __launch_bounds__(256) key_order_kernel(DeviceAsset a)
{
    const int lane = threadIdx.x & 31;
    const uint32_t leaf = blockIdx.x * 8u + (threadIdx.x >> 5);
    if (leaf >= a.g.leaf_count) return;
    LeafEntry& e = a.entries[leaf];
    const uint32_t info = e.info;
    bool sorted = entry_status(e) == kOk && (info & kFlagActive) && a.g.profile != 2u;
    bool plain = sorted;
    if (sorted) {
        const uint32_t* __restrict__ pw = a.payload;
        const uint64_t base = 4ull * e.word_off;
        const uint32_t cres = (e.header >> 6) & 7u, fres = (e.header >> 9) & 7u;
        StreamRef st[3];
        int ns = 0;
        st[ns++] = StreamRef{base + 8u, cres * cres * cres, 8u, e.kf & 0xFFFFu, (e.header >> 2) & 3u};
        if (info & kFlagFine)
            st[ns++] = StreamRef{base + 8u + e.coarse_bytes, fres * fres * fres, 8u, e.kf >> 16, (e.header >> 4) & 3u};
        if (info & kFlagShell)
            st[ns++] = StreamRef{base + e.shell_off, entry_shell_active(e), 4u, e.kf >> 16, (e.header >> 4) & 3u};
        bool ok = true, no_nan = true;
        for (int si = 0; si < ns; ++si) {
            const StreamRef& s = st[si];
            const uint64_t kb = stream_key_base(s);
            for (uint32_t c = lane; c < s.controls; c += 32) {
                const uint32_t desc = ldw(pw, (uint32_t)((s.base + 4ull * c) >> 2));
                const uint32_t ks = desc & 0xFFFFu, kc = (desc >> 16) & 0xFFu;
                if (kc == 0u || ks + kc > s.kf) continue;
                int prev = -1;
                for (uint32_t i = 0; i < kc; ++i) {
                    int f;
                    if (s.codec == 1u) {
                        f = key_frame(pw, kb, s.codec, ks + i);
                    } else {
                        const uint32_t k24 = ld_key24(pw, kb + 3ull * (ks + i));
                        f = (int)(k24 & 0xFFu);
                        const uint32_t h = k24 >> 8;
                        no_nan &= !((h & 0x7C00u) == 0x7C00u && (h & 0x3FFu) != 0u);
                    }
                    ok &= i == 0u || f > prev;
                    prev = f;
                }
            }
        }
        sorted = __all_sync(0xFFFFFFFFu, ok);
        plain = __all_sync(0xFFFFFFFFu, no_nan);
    }
    if (lane == 0) {
        a.key_sorted[leaf] = (sorted ? 1 : 0) | (plain ? 2 : 0);
        e.info = info | (sorted ? kFlagSorted : 0u) | (plain ? kFlagHalfPlain : 0u);
    }
}

static void launch_sci_event_order(const DeviceAsset& a, cudaStream_t s);

void launch_key_order(const DeviceAsset& a, cudaStream_t s)
{
    if (a.g.profile == 2u) launch_sci_event_order(a, s);
    else key_order_kernel<<<(a.g.leaf_count + 7) / 8, 256, 0, s>>>(a);
}

// Scientific leaves: every leaf is active.  The decoder reads through bounds-checked accessors
// (the reference reads through std::vector::at, render/src/scientific_decode.cpp:41-58); here the
// walker only checks that every AC scale the leaf's keep needs exists (the reference's
// coarseAcScales.at(k - 1), :91).
__device__ LeafEntry walk_sci_leaf(const DeviceAsset& a, uint32_t leaf)
{
    LeafEntry e{};
    e.word_off = __ldg(a.offsets + leaf);
    e.header = e.word_off < a.g.payload_words ? ldw(a.payload, e.word_off) : 0u;
    const uint32_t keep = ((e.header >> 2) & 0x3Fu) + 1u;
    uint32_t status = kOk;
    if (e.word_off >= a.g.payload_words || keep - 1u > a.g.scale_count) status = kErrDecodeOob;
    e.info = kFlagActive | (status << 16);
    return e;
}

// Page-table compaction of one tile of kWalkTile leaves (one flag per thread): ballot/popc within
// warps, a serial scan over the tile's warps, and a single-pass decoupled look-back across tiles
// (epoch-tagged descriptors, bounded spin).  Writes compact[], active_list[] and, from the last
// tile, the active count.
__device__ __forceinline__ void compact_tile(const DeviceAsset& a, uint32_t epoch, uint32_t tile, bool flag,
                                             uint32_t* s_warp, uint32_t& s_base)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t leaf0 = tile * kWalkTile;
    const uint32_t L = a.g.leaf_count;
    const uint32_t leaf = leaf0 + threadIdx.x;
    const unsigned bal = __ballot_sync(0xFFFFFFFFu, flag);
    const uint32_t in_warp = __popc(bal & ((1u << lane) - 1u));
    if (lane == 0) s_warp[warp] = __popc(bal);
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t run = 0;
        for (int w = 0; w < kWalkThreads / 32; ++w) {
            const uint32_t c = s_warp[w];
            s_warp[w] = run;
            run += c;
        }
        // decoupled look-back: descriptor = epoch[63:34] | flag[33:32] (1 aggregate, 2 prefix) | count
        cuda::atomic_ref<unsigned long long, cuda::thread_scope_device> self(a.tile_state[tile]);
        const unsigned long long ep = (unsigned long long)(epoch & 0x3FFFFFFFu) << 34;
        uint32_t excl = 0;
        if (tile == 0) {
            self.store(ep | (2ull << 32) | run, cuda::memory_order_release);
        } else {
            self.store(ep | (1ull << 32) | run, cuda::memory_order_release);
            int j = (int)tile - 1;
            uint32_t spins = 0;
            while (j >= 0) {
                cuda::atomic_ref<unsigned long long, cuda::thread_scope_device> st(a.tile_state[j]);
                const unsigned long long v = st.load(cuda::memory_order_acquire);
                if ((v >> 34) != (unsigned long long)(epoch & 0x3FFFFFFFu) || ((v >> 32) & 3ull) == 0ull) {
                    if (++spins > (1u << 22)) {   // bounded wait: report and stop, never hang
                        atomicOr(a.counters + 1, 1u);
                        record_error(a.err, leaf0, kErrWaitTimeout);
                        break;
                    }
                    __nanosleep(64);
                    continue;
                }
                excl += (uint32_t)(v & 0xFFFFFFFFull);
                if (((v >> 32) & 3ull) == 2ull) break;
                --j;
            }
            self.store(ep | (2ull << 32) | (excl + run), cuda::memory_order_release);
        }
        s_base = excl;
        if (leaf0 + kWalkTile >= L) a.counters[0] = excl + run;   // last tile: total active count
    }
    __syncthreads();
    if (leaf < L) {
        const uint32_t rank = s_base + s_warp[warp] + in_warp;
        a.compact[leaf] = flag ? rank : kNoRank;
        if (flag) a.active_list[rank] = leaf;
    }
}

__global__ void __launch_bounds__(kWalkThreads) walk_kernel(DeviceAsset a, uint32_t epoch)
{
    __shared__ uint8_t s_flag[kWalkTile];
    __shared__ uint32_t s_warp[kWalkThreads / 32];
    __shared__ uint32_t s_base;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t tile = blockIdx.x;
    const uint32_t leaf0 = tile * kWalkTile;
    const uint32_t L = a.g.leaf_count;

    // phase 1: one warp per leaf, 32 leaves per warp
    for (int j = 0; j < kWalkTile / (kWalkThreads / 32); ++j) {
        const uint32_t local = warp * (kWalkTile / (kWalkThreads / 32)) + j;
        const uint32_t leaf = leaf0 + local;
        if (leaf >= L) break;
        const LeafEntry e = a.g.profile == 2u ? walk_sci_leaf(a, leaf) : walk_rt_leaf(a, leaf, lane);
        if (lane == 0) {
            a.entries[leaf] = e;
            s_flag[local] = (e.info & kFlagActive) ? 1 : 0;
        }
    }
    __syncthreads();

    // phase 2: compaction of the tile's active flags
    const uint32_t leaf = leaf0 + threadIdx.x;
    compact_tile(a, epoch, tile, leaf < L && s_flag[threadIdx.x] != 0, s_warp, s_base);
}

// Per-frame page table of an asset whose leaf table is already built: the active flag of each
// leaf's 32-byte row (the walker's predicate: offsets inside the payload, route tag not EMPTY, or
// any scientific leaf), compacted as the walker compacts it.
__global__ void __launch_bounds__(kWalkThreads) page_table_kernel(DeviceAsset a, uint32_t epoch)
{
    __shared__ uint32_t s_warp[kWalkThreads / 32];
    __shared__ uint32_t s_base;
    const uint32_t tile = blockIdx.x;
    const uint32_t leaf = tile * kWalkTile + threadIdx.x;
    const bool flag = leaf < a.g.leaf_count && (__ldg(&a.entries[leaf].info) & kFlagActive) != 0u;
    compact_tile(a, epoch, tile, flag, s_warp, s_base);
}

void launch_walk(const DeviceAsset& a, uint32_t epoch, cudaStream_t s)
{
    const uint32_t tiles = (a.g.leaf_count + kWalkTile - 1) / kWalkTile;
    walk_kernel<<<tiles, kWalkThreads, 0, s>>>(a, epoch);
}

void launch_page_table(const DeviceAsset& a, uint32_t epoch, cudaStream_t s)
{
    const uint32_t tiles = (a.g.leaf_count + kWalkTile - 1) / kWalkTile;
    // Inside a stream capture the epoch is frozen into the graph, so every replay would find the
    // previous replay's descriptors carrying its own tag: clear them first in the graph.
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cs) == cudaSuccess && cs == cudaStreamCaptureStatusActive)
        cudaMemsetAsync(a.tile_state, 0, 8ull * tiles, s);
    page_table_kernel<<<tiles, kWalkThreads, 0, s>>>(a, epoch);
}

// ---------------------------------------------------------------------------------------------
// (b) render-temporal leaf decode (one warp)

__device__ __forceinline__ float trilinear_rt(const float* __restrict__ g, int res, const AxisWeight& ax,
                                              const AxisWeight& ay, const AxisWeight& az)
{
    if (res <= 0) return 0.0f;   // no controls (the reference dereferences an empty grid here)
    if (res == 1) return g[0];   // one control (the reference reads past its coordinate vector)
    const int r = res;
    const float* gz0 = g + (az.i0 * r) * r;
    const float* gz1 = g + (az.i1 * r) * r;
    const float c00 = lerp_ref(gz0[ay.i0 * r + ax.i0], gz0[ay.i0 * r + ax.i1], ax.t, ax.omt);
    const float c01 = lerp_ref(gz1[ay.i0 * r + ax.i0], gz1[ay.i0 * r + ax.i1], ax.t, ax.omt);
    const float c10 = lerp_ref(gz0[ay.i1 * r + ax.i0], gz0[ay.i1 * r + ax.i1], ax.t, ax.omt);
    const float c11 = lerp_ref(gz1[ay.i1 * r + ax.i0], gz1[ay.i1 * r + ax.i1], ax.t, ax.omt);
    const float c0 = lerp_ref(c00, c10, ay.t, ay.omt);
    const float c1 = lerp_ref(c01, c11, ay.t, ay.omt);
    return lerp_ref(c0, c1, az.t, az.omt);
}

// Decode the controls of one leaf at one frame into s_ctrl (coarse at [0, 343), fine or shell
// at [343, 855)).  Returns false when the leaf cannot be decoded (status recorded).
__device__ __forceinline__ void rt_decode_controls(const DeviceAsset& a, const LeafEntry& e, int frame,
                                                   float* __restrict__ s_ctrl, int lane, int nl = 32)
{
    const uint32_t* __restrict__ pw = a.payload;
    const uint64_t base = 4ull * e.word_off;
    const uint32_t cres = (e.header >> 6) & 7u, fres = (e.header >> 9) & 7u;
    const int total = (int)a.g.frames;
    const uint32_t bin8 = time_bin(frame, 8u, total);
    StreamRef cs{base + 8u, cres * cres * cres, 8u, e.kf & 0xFFFFu, (e.header >> 2) & 3u};
    for (uint32_t c = lane; c < cs.controls; c += nl) s_ctrl[c] = decode_control(pw, cs, c, frame, bin8);
    if (e.info & kFlagFine) {
        StreamRef fs{base + 8u + e.coarse_bytes, fres * fres * fres, 8u, e.kf >> 16, (e.header >> 4) & 3u};
        for (uint32_t c = lane; c < fs.controls; c += nl) s_ctrl[343 + c] = decode_control(pw, fs, c, frame, bin8);
    } else if (e.info & kFlagShell) {
        const uint32_t bin4 = time_bin(frame, 4u, total);
        StreamRef ss{base + e.shell_off, entry_shell_active(e), 4u, e.kf >> 16, (e.header >> 4) & 3u};
        for (uint32_t c = lane; c < ss.controls; c += nl) s_ctrl[343 + c] = decode_control(pw, ss, c, frame, bin4);
    }
}

// Reconstruct one row (ly, lz) of 8 voxels from the decoded controls.  Voxels outside the leaf
// extent come out as 0 (they are not part of the frame; in the cache they are defined as 0).
__device__ __forceinline__ void rt_row(const DeviceAsset& a, const LeafEntry& e, const float* __restrict__ s_ctrl,
                                       int w, int h, int d, int ly, int lz, float out[8])
{
    const uint32_t cres = (e.header >> 6) & 7u, fres = (e.header >> 9) & 7u;
    const AxisWeight ay = g_axis[axis_index(cres, h, ly)], az = g_axis[axis_index(cres, d, lz)];
    AxisWeight fy{}, fz{};
    const bool fine = (e.info & kFlagFine) != 0u;
    if (fine) {
        fy = g_axis[axis_index(fres, h, ly)];
        fz = g_axis[axis_index(fres, d, lz)];
    }
    uint64_t mask = 0;
    uint32_t pref = 0;
    const bool occ = (e.info & kFlagOccClamp) != 0u;
    if (occ) {
        const uint64_t ob = 4ull * e.word_off + 8u + e.coarse_bytes;
        const uint32_t g = (uint32_t)lz;   // 64 voxels per group = one z layer
        const uint32_t m0 = ldw(a.payload, (uint32_t)((ob + 8u * g) >> 2));
        const uint32_t m1 = ldw(a.payload, (uint32_t)((ob + 8u * g + 4u) >> 2));
        mask = ((uint64_t)m1 << 32) | m0;
        pref = (ldw(a.payload, (uint32_t)((ob + 64u + 2u * g) >> 2)) >> ((g & 1u) * 16u)) & 0xFFFFu;
    }
    const bool shell = (e.info & kFlagShell) != 0u;
#pragma unroll
    for (int lx = 0; lx < 8; ++lx) {
        float v = 0.0f;
        if (lx < w && ly < h && lz < d) {
            v = trilinear_rt(s_ctrl, (int)cres, c_axis[axis_index(cres, w, lx)], ay, az);
            const uint32_t bit = (uint32_t)(ly * 8 + lx);
            const bool in_occ = occ && ((mask >> bit) & 1ull);
            if (fine) {
                v = __fadd_rn(v, trilinear_rt(s_ctrl + 343, (int)fres, c_axis[axis_index(fres, w, lx)], fy, fz));
            } else if (shell && in_occ) {
                const uint32_t di = (pref + __popcll(mask & ((1ull << bit) - 1ull))) & 0xFFFFu;
                v = __fadd_rn(v, s_ctrl[343 + di]);
            }
            if (occ && !in_occ && v < 0.0f) v = 0.0f;
        }
        out[lx] = v;
    }
}

// ---------------------------------------------------------------------------------------------
// (b') scientific leaf decode (one warp): render/src/scientific_decode.cpp:82-359

struct SciReader {
    const uint32_t* __restrict__ pw;
    uint64_t words;
    bool oob;
    __device__ __forceinline__ uint32_t byte(uint64_t b)
    {
        const uint64_t w = b >> 2;
        if (w >= words) {
            oob = true;
            return 0u;
        }
        return (ldw(pw, (uint32_t)w) >> ((uint32_t)(b & 3u) * 8u)) & 0xFFu;
    }
    __device__ __forceinline__ uint32_t u16(uint64_t b) { return byte(b) | (byte(b + 1) << 8); }
    __device__ __forceinline__ uint32_t u32(uint64_t b)
    {
        if ((b & 3u) == 0u) {
            const uint64_t w = b >> 2;
            if (w >= words) {
                oob = true;
                return 0u;
            }
            return ldw(pw, (uint32_t)w);
        }
        return u16(b) | (u16(b + 2) << 16);
    }
};

// Error-free transforms for the compensated sum.
__device__ __forceinline__ void two_prod(float a, float b, float& p, float& e)
{
    p = __fmul_rn(a, b);
    e = __fmaf_rn(a, b, -p);
}
__device__ __forceinline__ void ff_add(float& hi, float& lo, float ph, float pl)
{
    const float s = __fadd_rn(hi, ph);
    const float bb = __fsub_rn(s, hi);
    const float err = __fadd_rn(__fsub_rn(hi, __fsub_rn(s, bb)), __fsub_rn(ph, bb));
    const float t = __fadd_rn(__fadd_rn(err, lo), pl);
    hi = __fadd_rn(s, t);
    lo = __fsub_rn(t, __fsub_rn(hi, s));
}

// 32 bits of the payload from byte b, b unaligned (two word reads; the payload's 16-byte tail
// padding keeps the second word inside the allocation).
__device__ __forceinline__ uint32_t pay_u32(const uint32_t* __restrict__ pw, uint64_t b)
{
    const uint32_t w = (uint32_t)(b >> 2);
    return __funnelshift_r(ldw(pw, w), ldw(pw, w + 1u), (uint32_t)(b & 3u) * 8u);
}

// The basis row b_k(t) and the AC scales of a leaf with keep <= 7, read once for several controls.
struct SciTerms {
    float b[7], sc[6];
    __device__ __forceinline__ SciTerms(const DeviceAsset& a, uint32_t t, int keep)
    {
        const float* brow = a.basis + (uint64_t)t * 64u;
#pragma unroll
        for (int k = 0; k < 7; ++k) b[k] = k < keep ? __ldg(brow + k) : 0.0f;
#pragma unroll
        for (int k = 0; k < 6; ++k) sc[k] = k + 1 < keep ? __ldg(a.scales + k) : 0.0f;
    }
};

// sci_control for a control record at byte cb of at most 8 bytes (keep <= 7) that lies inside the
// payload: the same products and compensated sum in the same order, the record read as two 32-bit
// windows (DC half in bytes 0-1, AC byte k at byte k + 1).
__device__ __forceinline__ float sci_control_fast(const uint32_t* __restrict__ pw, uint64_t cb, int keep,
                                                  const SciTerms& tm)
{
    const uint32_t w0 = pay_u32(pw, cb), w1 = keep > 3 ? pay_u32(pw, cb + 4u) : 0u;
    float hi, lo;
    two_prod(half_bits_to_float(w0 & 0xFFFFu), tm.b[0], hi, lo);
#pragma unroll
    for (int k = 1; k < 7; ++k) {
        if (k < keep) {
            const uint32_t byte = k + 1 < 4 ? (w0 >> (8 * (k + 1))) : (w1 >> (8 * (k - 3)));
            const float coeff = __fmul_rn((float)(int8_t)(byte & 0xFFu), tm.sc[k - 1]);
            float ph, pl;
            two_prod(coeff, tm.b[k], ph, pl);
            ff_add(hi, lo, ph, pl);
        }
    }
    return __fadd_rn(hi, lo);
}

// Coarse control ci at frame t: DC * b0(t) + sum_k (i8 * acScale[k-1]) * bk(t).
__device__ __forceinline__ float sci_control(const DeviceAsset& a, SciReader& rd, uint64_t base, int keep, int ci,
                                             const float* __restrict__ brow)
{
    const uint64_t cb = base + 4u + (uint64_t)ci * (keep + 1);
    float hi, lo;
    two_prod(half_bits_to_float(rd.u16(cb)), __ldg(brow), hi, lo);
    for (int k = 1; k < keep; ++k) {
        const float coeff = __fmul_rn((float)(int8_t)rd.byte(cb + 2u + (k - 1)), __ldg(a.scales + k - 1));
        float ph, pl;
        two_prod(coeff, __ldg(brow + k), ph, pl);
        ff_add(hi, lo, ph, pl);
    }
    return __fadd_rn(hi, lo);
}

__device__ __forceinline__ float decode_bfp(uint32_t q, float scale, int bits)
{
    if (bits <= 2) {
        const float lv = q == 0u ? -1.0f : q == 1u ? -0.3333333f : q == 2u ? 0.3333333f : 1.0f;
        return __fmul_rn(lv, scale);
    }
    const int levels = (1 << bits) - 1;
    const float norm = __fsub_rn(__fmul_rn(__fdiv_rn((float)q, (float)levels), 2.0f), 1.0f);
    return __fmul_rn(norm, scale);
}

__device__ __forceinline__ float bfp_sample(SciReader& rd, uint64_t data, int res, int bits, float scale, int ci)
{
    const int bo = ci * bits;
    const uint64_t bi = data + (uint64_t)(bo / 8);
    const int sh = bo % 8;
    uint32_t packed = rd.byte(bi);
    if (sh + bits > 8) packed |= rd.byte(bi + 1) << 8;
    return decode_bfp((packed >> sh) & ((1u << bits) - 1u), scale, bits);
}

__device__ __forceinline__ float tri_small(const float* __restrict__ g, int r, const AxisWeight& ax,
                                           const AxisWeight& ay, const AxisWeight& az)
{
    const float* gz0 = g + (az.i0 * r) * r;
    const float* gz1 = g + (az.i1 * r) * r;
    const float c00 = lerp_ref(gz0[ay.i0 * r + ax.i0], gz0[ay.i0 * r + ax.i1], ax.t, ax.omt);
    const float c01 = lerp_ref(gz1[ay.i0 * r + ax.i0], gz1[ay.i0 * r + ax.i1], ax.t, ax.omt);
    const float c10 = lerp_ref(gz0[ay.i1 * r + ax.i0], gz0[ay.i1 * r + ax.i1], ax.t, ax.omt);
    const float c11 = lerp_ref(gz1[ay.i1 * r + ax.i0], gz1[ay.i1 * r + ax.i1], ax.t, ax.omt);
    return lerp_ref(lerp_ref(c00, c10, ay.t, ay.omt), lerp_ref(c01, c11, ay.t, ay.omt), az.t, az.omt);
}

// Sparse-event residual for local voxel li at frame t (render/src/scientific_decode.cpp:235-295).
__device__ __forceinline__ float sci_sparse(SciReader& rd, uint64_t base, uint32_t hdr, int keep, uint32_t li, uint32_t t)
{
    const uint32_t count = (hdr >> 16) & 0x0FFFu;
    if (count == 0u) return 0.0f;
    const uint32_t tier = (hdr >> 8) & 3u;
    const uint32_t cap = tier == 0u ? 64u : tier == 1u ? 256u : tier == 2u ? 768u : 1024u;
    const uint32_t fpb = ((hdr >> 10) & 0xFu) + 1u;
    const uint32_t bin = t / fpb < 15u ? t / fpb : 15u;
    const uint32_t lt = (t - bin * fpb) & 0xFFu;
    const uint64_t sb = base + 4u + (uint64_t)(64 * (keep + 1));
    const float es = __uint_as_float(rd.u32(sb));
    if (!(es > 0.0f)) return 0.0f;
    const uint32_t mw = rd.u32(sb + 4u + (li >> 5) * 4u);
    if ((mw & (1u << (li & 31u))) == 0u) return 0.0f;
    const uint64_t bb = sb + 68u;
    const uint32_t start = rd.u16(bb + bin * 2u);
    const uint32_t end = bin + 1u < 16u ? rd.u16(bb + (bin + 1u) * 2u) : (count & 0xFFFFu);
    if (start >= end) return 0.0f;
    const uint64_t cb = bb + 32u, rb = cb + cap * 2u;
    const uint32_t target = ((lt << 9) | (li & 0x1FFu)) & 0xFFFFu;
    int left = (int)start, right = (int)end - 1;
    while (left <= right) {
        const int mid = (left + right) >> 1;
        const uint32_t key = rd.u16(cb + (uint32_t)mid * 2u);
        if (key == target) {
            const uint32_t byte = rd.byte(rb + (uint32_t)(mid >> 1));
            int q = (int)((mid & 1) == 0 ? (byte & 0xFu) : ((byte >> 4) & 0xFu));
            if (q & 8) q -= 16;
            return __fmul_rn((float)q, es);
        }
        if (key < target) left = mid + 1;
        else right = mid - 1;
    }
    return 0.0f;
}

// The frame-independent part of a SparseEvents leaf's residual (the same reads and checks as
// sci_sparse, split so that a caller decoding many frames of one voxel reads them once).
struct SparseLeaf {
    uint64_t sb, bb;        // section base, bin table
    float es;               // event scale (residuals are 0 unless es > 0)
    uint32_t count, cap, fpb;
    bool inside;            // the whole section lies inside the payload: reads need no checks
};

__device__ __forceinline__ SparseLeaf sparse_leaf(SciReader& rd, uint64_t base, uint32_t hdr, int keep)
{
    SparseLeaf s{};
    s.count = (hdr >> 16) & 0x0FFFu;
    const uint32_t tier = (hdr >> 8) & 3u;
    s.cap = tier == 0u ? 64u : tier == 1u ? 256u : tier == 2u ? 768u : 1024u;
    s.fpb = ((hdr >> 10) & 0xFu) + 1u;
    s.sb = base + 4u + (uint64_t)(64 * (keep + 1));
    s.bb = s.sb + 68u;
    s.es = s.count ? __uint_as_float(rd.u32(s.sb)) : 0.0f;
    // es, mask, bins, 16-bit keys, 4-bit residuals (and the 4 bytes a 32-bit window reads past)
    s.inside = s.sb + 100u + 2u * s.cap + s.cap / 2u + 4u <= 4ull * rd.words;
    return s;
}

// Mask word w (voxels 32w .. 32w+31) of a sparse leaf.
__device__ __forceinline__ uint32_t sparse_mask_word(SciReader& rd, const SparseLeaf& s, uint32_t w)
{
    return rd.u32(s.sb + 4u + w * 4u);
}

// Residual of voxel li at frame t, for a voxel whose mask bit is set in a leaf with count > 0
// and es > 0 (sci_sparse's remaining steps: bin range, binary search of the 16-bit keys).
__device__ __forceinline__ float sparse_at(SciReader& rd, const SparseLeaf& s, uint32_t li, uint32_t t)
{
    const uint32_t bin = t / s.fpb < 15u ? t / s.fpb : 15u;
    const uint32_t lt = (t - bin * s.fpb) & 0xFFu;
    // inside the payload, the 16-bit fields are read as 32-bit windows (one or two word reads
    // instead of two checked byte reads); the values are the same
    auto u16 = [&](uint64_t b) { return s.inside ? (pay_u32(rd.pw, b) & 0xFFFFu) : rd.u16(b); };
    const uint32_t start = u16(s.bb + bin * 2u);
    const uint32_t end = bin + 1u < 16u ? u16(s.bb + (bin + 1u) * 2u) : (s.count & 0xFFFFu);
    if (start >= end) return 0.0f;
    const uint64_t cb = s.bb + 32u, rb = cb + s.cap * 2u;
    const uint32_t target = ((lt << 9) | (li & 0x1FFu)) & 0xFFFFu;
    int left = (int)start, right = (int)end - 1;
    while (left <= right) {
        const int mid = (left + right) >> 1;
        const uint32_t key = u16(cb + (uint32_t)mid * 2u);
        if (key == target) {
            const uint32_t byte = s.inside ? (pay_u32(rd.pw, rb + (uint32_t)(mid >> 1)) & 0xFFu)
                                           : rd.byte(rb + (uint32_t)(mid >> 1));
            int q = (int)((mid & 1) == 0 ? (byte & 0xFu) : ((byte >> 4) & 0xFu));
            if (q & 8) q -= 16;
            return __fmul_rn((float)q, s.es);
        }
        if (key < target) left = mid + 1;
        else right = mid - 1;
    }
    return 0.0f;
}

// Scientific leaves: kFlagSorted marks a SparseEvents leaf whose bin ranges follow one another
// (start <= end, inside the key table), whose event keys strictly increase within every range and
// whose events all sit on voxels with their mask bit set.  The reference finds an event by binary
// search per voxel and frame, after the mask test (render/src/scientific_decode.cpp:235-295); on
// such a leaf the search finds a key exactly when it is present, so decoders may instead visit the
// events of a frame's bin and add each to its voxel.  One warp per leaf, at load and upload.
__global__ void __launch_bounds__(256) sci_event_order_kernel(DeviceAsset a)
{
    const int lane = threadIdx.x & 31;
    const uint32_t leaf = blockIdx.x * 8u + (threadIdx.x >> 5);
    if (leaf >= a.g.leaf_count) return;
    LeafEntry& e = a.entries[leaf];
    const uint32_t info = e.info, hdr = e.header;
    bool sorted = entry_status(e) == kOk && (hdr & 3u) == 1u;
    if (sorted) {
        SciReader rd{a.payload, a.g.payload_words, false};
        const int keep = (int)((hdr >> 2) & 0x3Fu) + 1;
        const SparseLeaf sp = sparse_leaf(rd, 4ull * e.word_off, hdr, keep);
        bool ok = true;
        if (sp.count && sp.es > 0.0f) {
            for (uint32_t b = 0; b < 16u; ++b) {
                const uint32_t st0 = rd.u16(sp.bb + 2u * b);
                const uint32_t en = b < 15u ? rd.u16(sp.bb + 2u * (b + 1u)) : (sp.count & 0xFFFFu);
                if (st0 > en) ok = false;
                if (st0 >= en) continue;
                if (en > sp.cap) ok = false;
                for (uint32_t i = st0 + (uint32_t)lane; i < en && ok; i += 32u) {
                    const uint32_t key = rd.u16(sp.bb + 32u + 2u * i);
                    if (i + 1u < en) ok = key < rd.u16(sp.bb + 32u + 2u * (i + 1u));
                    ok = ok && ((sparse_mask_word(rd, sp, (key & 511u) >> 5) >> (key & 31u)) & 1u) != 0u;
                }
            }
        }
        sorted = __all_sync(0xFFFFFFFFu, ok && !rd.oob);
    }
    if (lane == 0) {
        a.key_sorted[leaf] = sorted ? 1 : 0;
        if (sorted) e.info = info | kFlagSorted;
    }
}

static void launch_sci_event_order(const DeviceAsset& a, cudaStream_t s)
{
    sci_event_order_kernel<<<(a.g.leaf_count + 7) / 8, 256, 0, s>>>(a);
}

// Add the events of frame t to the voxels of one SparseEvents leaf with kFlagSorted (one warp;
// the voxels' coarse values are already written).  dst(li) is the voxel's output address.
template <class Dst>
__device__ __forceinline__ void sci_scatter_frame(const DeviceAsset& a, const LeafEntry& e, uint32_t t, int w, int h,
                                                  int d, int lane, Dst dst, bool& oob)
{
    SciReader rd{a.payload, a.g.payload_words, false};
    const uint32_t hdr = e.header;
    const int keep = (int)((hdr >> 2) & 0x3Fu) + 1;
    const SparseLeaf sp = sparse_leaf(rd, 4ull * e.word_off, hdr, keep);
    if (sp.count && sp.es > 0.0f) {
        const uint32_t bin = t / sp.fpb < 15u ? t / sp.fpb : 15u;
        const uint32_t lt7 = (t - bin * sp.fpb) & 0x7Fu;   // the search key keeps 7 bits of it
        auto u16 = [&](uint64_t b) { return sp.inside ? (pay_u32(rd.pw, b) & 0xFFFFu) : rd.u16(b); };
        const uint32_t st0 = u16(sp.bb + bin * 2u);
        const uint32_t en = bin + 1u < 16u ? u16(sp.bb + (bin + 1u) * 2u) : (sp.count & 0xFFFFu);
        const uint64_t cb = sp.bb + 32u, rb = cb + sp.cap * 2u;
        for (uint32_t i = st0 + (uint32_t)lane; i < en; i += 32u) {
            const uint32_t key = u16(cb + 2u * i);
            if ((key >> 9) != lt7) continue;
            const uint32_t li = key & 511u;
            if ((int)(li & 7u) >= w || (int)((li >> 3) & 7u) >= h || (int)(li >> 6) >= d) continue;
            const uint32_t byte = sp.inside ? (pay_u32(rd.pw, rb + (i >> 1)) & 0xFFu) : rd.byte(rb + (i >> 1));
            int q = (int)((i & 1u) == 0u ? (byte & 0xFu) : ((byte >> 4) & 0xFu));
            if (q & 8) q -= 16;
            float* o = dst(li);
            *o = __fadd_rn(*o, __fmul_rn((float)q, sp.es));
        }
    }
    oob |= rd.oob;
}

// Warp-cooperative scientific leaf decode at frame t: controls into s_ctrl[0..64), the dense
// residual grid(s) into s_ctrl[64..) (per-frame grid, or tkeep basis grids), then row values.
__device__ void sci_decode_controls(const DeviceAsset& a, const LeafEntry& e, uint32_t t, float* __restrict__ s_ctrl,
                                    int lane, bool& oob, int nl = 32)
{
    SciReader rd{a.payload, a.g.payload_words, false};
    const uint64_t base = 4ull * e.word_off;
    const uint32_t hdr = e.header;
    const int keep = (int)((hdr >> 2) & 0x3Fu) + 1;
    const float* brow = a.basis + (uint64_t)t * 64u;
    if (keep <= 7 && base + 4u + (uint64_t)(64 * (keep + 1)) + 4u <= 4ull * a.g.payload_words) {
        // the coarse block lies inside the payload: word-window reads, terms read once per lane
        const SciTerms tm(a, t, keep);
        for (int c = lane; c < 64; c += nl) s_ctrl[c] = sci_control_fast(a.payload, base + 4u + (uint64_t)c * (keep + 1), keep, tm);
    } else {
        for (int c = lane; c < 64; c += nl) s_ctrl[c] = sci_control(a, rd, base, keep, c, brow);
    }
    const uint32_t mode = hdr & 3u;
    if (mode >= 2u) {
        const int res = mode == 2u ? 3 : 4;
        const int bits = (int)((hdr >> 8) & 0xFu);
        const uint32_t sub = (hdr >> 12) & 7u;
        const int per = res * res * res;
        const uint64_t scales = base + 4u + (uint64_t)(64 * (keep + 1));
        if (sub == 1u) {
            const int tkeep = (int)((hdr >> 15) & 0xFu) + 1;
            const int bbytes = (per * bits + 7) / 8;
            const uint64_t data = scales + (uint64_t)(tkeep * 2);
            if (bits > 0) {
                for (int i = lane; i < tkeep * per; i += nl) {
                    const int k = i / per, ci = i % per;
                    const float sc = half_bits_to_float(rd.u16(scales + (uint64_t)(k * 2)));
                    s_ctrl[64 + i] = bfp_sample(rd, data + (uint64_t)(k * bbytes), res, bits, sc, ci);
                }
            }
        } else {
            const int fbytes = (per * bits + 7) / 8;
            const uint64_t data = scales + (uint64_t)a.g.frames * 2u + (uint64_t)t * fbytes;
            const float sc = half_bits_to_float(rd.u16(scales + t * 2u));
            for (int ci = lane; ci < per; ci += nl) s_ctrl[64 + ci] = bfp_sample(rd, data, res, bits, sc, ci);
        }
    }
    oob = rd.oob;
}

// skip_events: the sparse-event residual is left out (added by sci_scatter_frame afterwards).
__device__ __forceinline__ void sci_row(const DeviceAsset& a, const LeafEntry& e, const float* __restrict__ s_ctrl,
                                        uint32_t t, int w, int h, int d, int ly, int lz, float out[8], bool& oob,
                                        bool skip_events = false)
{
    SciReader rd{a.payload, a.g.payload_words, false};
    const uint64_t base = 4ull * e.word_off;
    const uint32_t hdr = e.header;
    const int keep = (int)((hdr >> 2) & 0x3Fu) + 1;
    const uint32_t mode = hdr & 3u;
    const AxisWeight ay = c_sci_axis[0][ly], az = c_sci_axis[0][lz];
    const int res = mode == 2u ? 3 : 4;
    const AxisWeight dy = c_sci_axis[mode == 2u ? 1 : 2][ly], dz = c_sci_axis[mode == 2u ? 1 : 2][lz];
    const int bits = (int)((hdr >> 8) & 0xFu);
    const uint32_t sub = (hdr >> 12) & 7u;
    const int tkeep = (int)((hdr >> 15) & 0xFu) + 1;
    const float* brow = a.basis + (uint64_t)t * 64u;
    // sparse events: the section header and this row's mask word once (the row's 8 voxels share
    // one 32-bit mask word); per voxel only the bin range and key search remain
    SparseLeaf sp{};
    uint32_t row_mask = 0u;
    if (mode == 1u && !skip_events) {
        sp = sparse_leaf(rd, base, hdr, keep);
        if (sp.count && sp.es > 0.0f) {
            const uint32_t li0 = (uint32_t)((lz * 8 + ly) * 8);
            row_mask = (sparse_mask_word(rd, sp, li0 >> 5) >> (li0 & 31u)) & 0xFFu;
        }
    }
#pragma unroll 1
    for (int lx = 0; lx < 8; ++lx) {
        float v = 0.0f;
        if (lx < w && ly < h && lz < d) {
            const float coarse = tri_small(s_ctrl, 4, c_sci_axis[0][lx], ay, az);
            float r = 0.0f;
            if (mode == 1u) {
                if ((row_mask >> lx) & 1u) r = sparse_at(rd, sp, (uint32_t)((lz * 8 + ly) * 8 + lx), t);
            } else if (mode >= 2u) {
                const AxisWeight dx = c_sci_axis[mode == 2u ? 1 : 2][lx];
                const int per = res * res * res;
                if (sub == 1u) {
                    if (bits > 0) {
                        for (int k = 0; k < tkeep; ++k) {
                            const float tri = tri_small(s_ctrl + 64 + k * per, res, dx, dy, dz);
                            r = __fadd_rn(r, __fmul_rn(tri, __ldg(brow + k)));
                        }
                    }
                } else {
                    r = tri_small(s_ctrl + 64, res, dx, dy, dz);
                }
            }
            v = __fadd_rn(coarse, r);
        }
        out[lx] = v;
    }
    oob |= rd.oob;
}

// ---------------------------------------------------------------------------------------------
// (b) decode kernels: warp-per-(leaf, frame) over the active list; frames in the launch are
// walked innermost so a warp re-reads its leaf's bytes from L1/L2.

struct FrameList {
    int n;
    int f[kMaxLaunchFrames];
};

template <bool DENSE, bool SCI>
__global__ void __launch_bounds__(kDecodeWarps * 32, 2) decode_kernel(DeviceAsset a, FrameList fl, float* __restrict__ out,
                                                                     uint64_t frame_stride)
{
    __shared__ __align__(16) float s_ctrl_all[kDecodeWarps][kWarpSlots];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    float* s_ctrl = s_ctrl_all[warp];
    const uint32_t n_items = DENSE ? a.g.leaf_count : *(volatile const uint32_t*)a.counters;
    const uint32_t warps_total = gridDim.x * kDecodeWarps;
    for (uint32_t item = blockIdx.x * kDecodeWarps + warp; item < n_items; item += warps_total) {
        const uint32_t leaf = DENSE ? item : __ldg(a.active_list + item);
        const LeafEntry e = a.entries[leaf];
        uint32_t bx, by, bz;
        int w, h, d;
        leaf_extent(a.g, leaf, bx, by, bz, w, h, d);
        const bool empty = !SCI && (e.header & 3u) == kModeEmpty;
        const uint32_t st = entry_status(e);
        if (st != kOk && lane == 0) record_error(a.err, leaf, st);
        // scientific SparseEvents leaves with sorted keys: events are added by visiting the
        // frame's bin after the rows are written, instead of one search per voxel
        const bool scatter = SCI && st == kOk && (e.header & 3u) == 1u && (e.info & kFlagSorted) != 0u;
        for (int fi = 0; fi < fl.n; ++fi) {
            const int frame = clamp_frame(fl.f[fi], (int)a.g.frames);
            bool oob = false;
            if (!empty && st == kOk) {
                if (SCI) sci_decode_controls(a, e, (uint32_t)fl.f[fi], s_ctrl, lane, oob);
                else rt_decode_controls(a, e, frame, s_ctrl, lane);
            }
            __syncwarp();
            for (int r = lane; r < 64; r += 32) {
                const int ly = r & 7, lz = r >> 3;
                float v[8];
                if (empty || st != kOk) {
#pragma unroll
                    for (int i = 0; i < 8; ++i) v[i] = 0.0f;
                } else if (SCI) {
                    sci_row(a, e, s_ctrl, (uint32_t)fl.f[fi], w, h, d, ly, lz, v, oob, scatter);
                } else {
                    rt_row(a, e, s_ctrl, w, h, d, ly, lz, v);
                }
                if (DENSE) {
                    if (ly < h && lz < d) {
                        float* dst = out + (uint64_t)fi * frame_stride +
                                     ((uint64_t)(bz * 8 + lz) * a.g.height + (by * 8 + ly)) * a.g.width + bx * 8;
                        if (w == 8 && (((uintptr_t)dst) & 15u) == 0u) {
                            reinterpret_cast<float4*>(dst)[0] = make_float4(v[0], v[1], v[2], v[3]);
                            reinterpret_cast<float4*>(dst)[1] = make_float4(v[4], v[5], v[6], v[7]);
                        } else {
                            for (int i = 0; i < w; ++i) dst[i] = v[i];
                        }
                    }
                } else {
                    float4* dst = reinterpret_cast<float4*>(out + (uint64_t)fi * frame_stride + (uint64_t)item * 512u + r * 8);
                    dst[0] = make_float4(v[0], v[1], v[2], v[3]);
                    dst[1] = make_float4(v[4], v[5], v[6], v[7]);
                }
            }
            if (scatter && (uint32_t)fl.f[fi] < a.g.frames) {
                __syncwarp();   // the rows written by the other lanes are visible
                if (DENSE) {
                    float* fb = out + (uint64_t)fi * frame_stride;
                    sci_scatter_frame(a, e, (uint32_t)fl.f[fi], w, h, d, lane,
                                      [&](uint32_t li) {
                                          return fb + ((uint64_t)(bz * 8 + (li >> 6)) * a.g.height +
                                                       (by * 8 + ((li >> 3) & 7u))) * a.g.width + bx * 8 + (li & 7u);
                                      },
                                      oob);
                } else {
                    float* fb = out + (uint64_t)fi * frame_stride + (uint64_t)item * 512u;
                    sci_scatter_frame(a, e, (uint32_t)fl.f[fi], w, h, d, lane, [&](uint32_t li) { return fb + li; },
                                      oob);
                }
            }
            if (__any_sync(0xFFFFFFFFu, oob) && lane == 0) record_error(a.err, leaf, kErrDecodeOob);
            __syncwarp();
        }
    }
}

// Render-temporal decode kernel (TMA-staged leaf, one CTA per leaf): rt_kernel_leaf.cuh
}  // namespace vbtb
#include "rt_kernel_leaf.cuh"
namespace vbtb {

static int default_grid()
{
    static int g = 0;
    if (!g) {
        int dev = 0, sms = 0, per = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, decode_kernel<false, false>, kDecodeWarps * 32, 0);
        g = sms * (per > 0 ? per : 1);
    }
    return g;
}

void launch_decode_cache(const DeviceAsset& a, uint32_t seq, const int* frames, int nframes, float* out,
                         uint64_t stride, int grid, cudaStream_t s)
{
    FrameList fl{};
    fl.n = nframes;
    for (int i = 0; i < nframes; ++i) fl.f[i] = frames[i];
    if (a.g.profile == 2u)
        decode_kernel<false, true><<<grid > 0 ? grid : default_grid(), kDecodeWarps * 32, 0, s>>>(a, fl, out, stride);
    else
        launch_rt_leaf(a, seq, fl, out, stride, grid, false, s);
}

// The current-frame control cache of the reference Studio (VBTStudio/frontend/shaders/
// vbt_cache.comp:168-236): 576 slots per active leaf and frame -- coarse control s in slot s < 64,
// from slot 64 on the fine grid's controls (FINE6) or the Mode2 shell residual controls, 0 in every
// slot past a leaf's controls.  Values are the reference CPU decoder's (decode_control; the shader
// blends with mix(), which can differ in the last bit).  One CTA per active leaf at a time.
constexpr uint32_t kControlCacheStride = 576u;

__global__ void __launch_bounds__(256) control_cache_kernel(DeviceAsset a, FrameList fl, float* __restrict__ out,
                                                            uint64_t frame_stride)
{
    const uint32_t n_leaves = *(volatile const uint32_t*)a.counters;
    const int total = (int)a.g.frames;
    const uint32_t* __restrict__ pw = a.payload;
    for (uint32_t rank = blockIdx.x; rank < n_leaves; rank += gridDim.x) {
        const uint32_t leaf = __ldg(a.active_list + rank);
        const LeafEntry e = a.entries[leaf];
        const uint32_t st = entry_status(e);
        const bool ok = st == kOk && (e.header & 3u) != kModeEmpty;
        if (st != kOk && threadIdx.x == 0) record_error(a.err, leaf, st);
        const uint64_t base = 4ull * e.word_off;
        const uint32_t cres = (e.header >> 6) & 7u, fres = (e.header >> 9) & 7u;
        const bool fine = (e.info & kFlagFine) != 0u, shell = (e.info & kFlagShell) != 0u;
        const StreamRef cs{base + 8u, cres * cres * cres, 8u, e.kf & 0xFFFFu, (e.header >> 2) & 3u};
        const StreamRef fs{base + 8u + e.coarse_bytes, fres * fres * fres, 8u, e.kf >> 16, (e.header >> 4) & 3u};
        const StreamRef ss{base + e.shell_off, entry_shell_active(e), 4u, e.kf >> 16, (e.header >> 4) & 3u};
        for (int j = 0; j < fl.n; ++j) {
            const int t = clamp_frame(fl.f[j], total);
            const uint32_t b8 = time_bin(t, 8u, total), b4 = time_bin(t, 4u, total);
            float* o = out + (uint64_t)j * frame_stride + (uint64_t)rank * kControlCacheStride;
            for (uint32_t slot = threadIdx.x; slot < kControlCacheStride; slot += blockDim.x) {
                float v = 0.0f;
                if (ok) {
                    if (slot < 64u) {
                        if (slot < cs.controls) v = decode_control(pw, cs, slot, t, b8);
                    } else {
                        const uint32_t ci = slot - 64u;
                        if (fine && ci < fs.controls) v = decode_control(pw, fs, ci, t, b8);
                        else if (shell && ci < ss.controls) v = decode_control(pw, ss, ci, t, b4);
                    }
                }
                o[slot] = v;
            }
        }
    }
}

void launch_control_cache(const DeviceAsset& a, const int* frames, int nframes, float* out, uint64_t stride,
                          cudaStream_t s)
{
    FrameList fl{};
    fl.n = nframes;
    for (int i = 0; i < nframes; ++i) fl.f[i] = frames[i];
    control_cache_kernel<<<default_grid(), 256, 0, s>>>(a, fl, out, stride);
}

void launch_decode_dense(const DeviceAsset& a, uint32_t seq, const int* frames, int nframes, float* out, int grid,
                         cudaStream_t s)
{
    FrameList fl{};
    fl.n = nframes;
    for (int i = 0; i < nframes; ++i) fl.f[i] = frames[i];
    const uint64_t stride = (uint64_t)a.g.width * a.g.height * a.g.depth;
    if (a.g.profile == 2u)
        decode_kernel<true, true><<<grid > 0 ? grid : default_grid(), kDecodeWarps * 32, 0, s>>>(a, fl, out, stride);
    else
        launch_rt_leaf(a, seq, fl, out, stride, grid, true, s);
}

// Leaf-per-warp cache decode (8 warps per CTA, each warp one leaf at a time, frames in turn):
// the alternative shape the autotuner weighs against the leaf-per-CTA kernel.
void launch_decode_cache_warp(const DeviceAsset& a, const int* frames, int nframes, float* out, uint64_t stride,
                              int grid, cudaStream_t s)
{
    FrameList fl{};
    fl.n = nframes;
    for (int i = 0; i < nframes; ++i) fl.f[i] = frames[i];
    const int g = grid > 0 ? grid : default_grid();
    if (a.g.profile == 2u) decode_kernel<false, true><<<g, kDecodeWarps * 32, 0, s>>>(a, fl, out, stride);
    else decode_kernel<false, false><<<g, kDecodeWarps * 32, 0, s>>>(a, fl, out, stride);
}

int decode_warp_grid() { return default_grid(); }

// Plain per-leaf launch: grid = the whole leaf grid, one 64-thread CTA per leaf (EMPTY leaves
// return at once), controls decoded by both warps' lanes, one frame.  This is the reference
// Studio's cache dispatch shape and serves as the baseline the batched path is measured against.
__global__ void __launch_bounds__(64) decode_plain_kernel(DeviceAsset a, int frame_index, float* __restrict__ out)
{
    __shared__ __align__(16) float s_ctrl[kWarpSlots];
    const uint32_t leaf = blockIdx.x;
    if (leaf >= a.g.leaf_count) return;
    const uint32_t rank = a.compact[leaf];
    if (rank == kNoRank) return;
    const LeafEntry e = a.entries[leaf];
    const uint32_t st = entry_status(e);
    uint32_t bx, by, bz;
    int w, h, d;
    leaf_extent(a.g, leaf, bx, by, bz, w, h, d);
    bool oob = false;
    if (st == kOk) {
        if (a.g.profile == 2u) sci_decode_controls(a, e, (uint32_t)frame_index, s_ctrl, threadIdx.x, oob, 64);
        else rt_decode_controls(a, e, clamp_frame(frame_index, (int)a.g.frames), s_ctrl, threadIdx.x, 64);
    }
    __syncthreads();
    const int r = threadIdx.x;
    float v[8];
    if (st != kOk) {
        for (int i = 0; i < 8; ++i) v[i] = 0.0f;
        if (threadIdx.x == 0) record_error(a.err, leaf, st);
    } else if (a.g.profile == 2u) {
        sci_row(a, e, s_ctrl, (uint32_t)frame_index, w, h, d, r & 7, r >> 3, v, oob);
    } else {
        rt_row(a, e, s_ctrl, w, h, d, r & 7, r >> 3, v);
    }
    float4* dst = reinterpret_cast<float4*>(out + (uint64_t)rank * 512u + r * 8);
    dst[0] = make_float4(v[0], v[1], v[2], v[3]);
    dst[1] = make_float4(v[4], v[5], v[6], v[7]);
    if (oob) record_error(a.err, leaf, kErrDecodeOob);
}

void launch_decode_cache_plain(const DeviceAsset& a, int frame, float* out, cudaStream_t s)
{
    decode_plain_kernel<<<a.g.leaf_count, 64, 0, s>>>(a, frame, out);
}

// ---------------------------------------------------------------------------------------------
// (c) point queries: one thread per query, decoding only the corner controls it needs.

__device__ __forceinline__ float rt_point(const DeviceAsset& a, const LeafEntry& e, int w, int h, int d, int lx, int ly, int lz,
                          int frame)
{
    const uint32_t* __restrict__ pw = a.payload;
    const uint64_t base = 4ull * e.word_off;
    const int total = (int)a.g.frames;
    const uint32_t cres = (e.header >> 6) & 7u, fres = (e.header >> 9) & 7u;
    const uint32_t bin8 = time_bin(frame, 8u, total);
    auto sample = [&](const StreamRef& s, uint32_t res) -> float {
        if (res == 0u) return 0.0f;
        if (res == 1u) return decode_control(pw, s, 0, frame, bin8);
        const AxisWeight ax = g_axis[axis_index(res, w, lx)], ay = g_axis[axis_index(res, h, ly)],
                         az = g_axis[axis_index(res, d, lz)];
        const uint32_t r = res;
        auto at = [&](uint32_t ix, uint32_t iy, uint32_t iz) { return decode_control(pw, s, (iz * r + iy) * r + ix, frame, bin8); };
        const float c00 = lerp_ref(at(ax.i0, ay.i0, az.i0), at(ax.i1, ay.i0, az.i0), ax.t, ax.omt);
        const float c01 = lerp_ref(at(ax.i0, ay.i0, az.i1), at(ax.i1, ay.i0, az.i1), ax.t, ax.omt);
        const float c10 = lerp_ref(at(ax.i0, ay.i1, az.i0), at(ax.i1, ay.i1, az.i0), ax.t, ax.omt);
        const float c11 = lerp_ref(at(ax.i0, ay.i1, az.i1), at(ax.i1, ay.i1, az.i1), ax.t, ax.omt);
        return lerp_ref(lerp_ref(c00, c10, ay.t, ay.omt), lerp_ref(c01, c11, ay.t, ay.omt), az.t, az.omt);
    };
    StreamRef cs{base + 8u, cres * cres * cres, 8u, e.kf & 0xFFFFu, (e.header >> 2) & 3u};
    float v = sample(cs, cres);
    const uint32_t vox = (uint32_t)((lz * 8 + ly) * 8 + lx);
    bool in_occ = false;
    uint64_t mask = 0;
    uint32_t pref = 0;
    if (e.info & kFlagOccClamp) {
        const uint64_t ob = base + 8u + e.coarse_bytes;
        const uint32_t g = vox >> 6;
        mask = ((uint64_t)ldw(pw, (uint32_t)((ob + 8u * g + 4u) >> 2)) << 32) | ldw(pw, (uint32_t)((ob + 8u * g) >> 2));
        pref = (ldw(pw, (uint32_t)((ob + 64u + 2u * g) >> 2)) >> ((g & 1u) * 16u)) & 0xFFFFu;
        in_occ = (mask >> (vox & 63u)) & 1ull;
    }
    if (e.info & kFlagFine) {
        StreamRef fs{base + 8u + e.coarse_bytes, fres * fres * fres, 8u, e.kf >> 16, (e.header >> 4) & 3u};
        v = __fadd_rn(v, sample(fs, fres));
    } else if ((e.info & kFlagShell) && in_occ) {
        StreamRef ss{base + e.shell_off, entry_shell_active(e), 4u, e.kf >> 16, (e.header >> 4) & 3u};
        const uint32_t di = (pref + __popcll(mask & ((1ull << (vox & 63u)) - 1ull))) & 0xFFFFu;
        v = __fadd_rn(v, decode_control(pw, ss, di, frame, time_bin(frame, 4u, total)));
    }
    if ((e.info & kFlagOccClamp) && !in_occ && v < 0.0f) v = 0.0f;
    return v;
}

// The point decode of a scientific leaf whose coarse block and sparse-event section lie inside the
// payload (so none of the SciReader's per-byte checks can fire) and whose keep is at most 8: the
// same arithmetic as sci_point's coarse part and sci_sparse, in the same order, with each
// control's record (at most 8 bytes: keep <= 7) read as two 32-bit windows, the basis row and AC
// scales read once per query, and the event keys as 32-bit windows.  Returns false (nothing
// decoded) when the leaf is not of that shape; sci_point then decodes it.
__device__ __forceinline__ bool sci_point_fast(const DeviceAsset& a, const LeafEntry& e, uint32_t lx, uint32_t ly,
                                               uint32_t lz, uint32_t t, float& value)
{
    const uint32_t hdr = e.header;
    const int keep = (int)((hdr >> 2) & 0x3Fu) + 1;
    const uint32_t mode = hdr & 3u;
    const uint64_t base = 4ull * e.word_off;
    const uint64_t bytes = 4ull * a.g.payload_words;
    const uint64_t sb = base + 4u + (uint64_t)(64 * (keep + 1));
    if (keep > 7 || mode >= 2u || sb + 4u > bytes) return false;
    const uint32_t* __restrict__ pw = a.payload;
    const SciTerms tm(a, t, keep);
    auto at = [&](int ci) { return sci_control_fast(pw, base + 4u + (uint64_t)ci * (keep + 1), keep, tm); };
    const AxisWeight ax = c_sci_axis[0][lx], ay = c_sci_axis[0][ly], az = c_sci_axis[0][lz];
    auto ci = [&](int cx, int cy, int cz) { return at((cz * 4 + cy) * 4 + cx); };
    const float c00 = lerp_ref(ci(ax.i0, ay.i0, az.i0), ci(ax.i1, ay.i0, az.i0), ax.t, ax.omt);
    const float c01 = lerp_ref(ci(ax.i0, ay.i0, az.i1), ci(ax.i1, ay.i0, az.i1), ax.t, ax.omt);
    const float c10 = lerp_ref(ci(ax.i0, ay.i1, az.i0), ci(ax.i1, ay.i1, az.i0), ax.t, ax.omt);
    const float c11 = lerp_ref(ci(ax.i0, ay.i1, az.i1), ci(ax.i1, ay.i1, az.i1), ax.t, ax.omt);
    const float coarse = lerp_ref(lerp_ref(c00, c10, ay.t, ay.omt), lerp_ref(c01, c11, ay.t, ay.omt), az.t, az.omt);
    float r = 0.0f;
    const uint32_t count = (hdr >> 16) & 0x0FFFu;
    if (mode == 1u && count != 0u) {   // sci_sparse
        const uint32_t tier = (hdr >> 8) & 3u;
        const uint32_t cap = tier == 0u ? 64u : tier == 1u ? 256u : tier == 2u ? 768u : 1024u;
        if (sb + 100u + 2u * cap + cap / 2u + 4u > bytes) return false;   // the section's extent
        const uint32_t li = (lz * 8u + ly) * 8u + lx;
        const uint32_t fpb = ((hdr >> 10) & 0xFu) + 1u;
        const uint32_t bin = t / fpb < 15u ? t / fpb : 15u;
        const uint32_t lt = (t - bin * fpb) & 0xFFu;
        const float es = __uint_as_float(pay_u32(pw, sb));
        const uint32_t mw = pay_u32(pw, sb + 4u + (li >> 5) * 4u);
        if (es > 0.0f && (mw & (1u << (li & 31u))) != 0u) {
            const uint64_t bb = sb + 68u;
            const uint32_t se = pay_u32(pw, bb + bin * 2u);
            const uint32_t start = se & 0xFFFFu;
            const uint32_t end = bin + 1u < 16u ? se >> 16 : (count & 0xFFFFu);
            const uint64_t cb = bb + 32u, rb = cb + cap * 2u;
            const uint32_t target = ((lt << 9) | (li & 0x1FFu)) & 0xFFFFu;
            int left = (int)start, right = (int)end - 1;
            while (left <= right) {
                const int mid = (left + right) >> 1;
                const uint32_t key = pay_u32(pw, cb + (uint32_t)mid * 2u) & 0xFFFFu;
                if (key == target) {
                    const uint32_t byte = pay_u32(pw, rb + (uint32_t)(mid >> 1)) & 0xFFu;
                    int q = (int)((mid & 1) == 0 ? (byte & 0xFu) : ((byte >> 4) & 0xFu));
                    if (q & 8) q -= 16;
                    r = __fmul_rn((float)q, es);
                    break;
                }
                if (key < target) left = mid + 1;
                else right = mid - 1;
            }
        }
    }
    value = __fadd_rn(coarse, r);
    return true;
}

__device__ __forceinline__ float sci_point(const DeviceAsset& a, const LeafEntry& e, uint32_t lx, uint32_t ly, uint32_t lz, uint32_t t,
                           bool& oob)
{
    SciReader rd{a.payload, a.g.payload_words, false};
    const uint64_t base = 4ull * e.word_off;
    const uint32_t hdr = e.header;
    const int keep = (int)((hdr >> 2) & 0x3Fu) + 1;
    const float* brow = a.basis + (uint64_t)t * 64u;
    const AxisWeight ax = c_sci_axis[0][lx], ay = c_sci_axis[0][ly], az = c_sci_axis[0][lz];
    auto at = [&](int cx, int cy, int cz) { return sci_control(a, rd, base, keep, (cz * 4 + cy) * 4 + cx, brow); };
    const float c00 = lerp_ref(at(ax.i0, ay.i0, az.i0), at(ax.i1, ay.i0, az.i0), ax.t, ax.omt);
    const float c01 = lerp_ref(at(ax.i0, ay.i0, az.i1), at(ax.i1, ay.i0, az.i1), ax.t, ax.omt);
    const float c10 = lerp_ref(at(ax.i0, ay.i1, az.i0), at(ax.i1, ay.i1, az.i0), ax.t, ax.omt);
    const float c11 = lerp_ref(at(ax.i0, ay.i1, az.i1), at(ax.i1, ay.i1, az.i1), ax.t, ax.omt);
    const float coarse = lerp_ref(lerp_ref(c00, c10, ay.t, ay.omt), lerp_ref(c01, c11, ay.t, ay.omt), az.t, az.omt);
    const uint32_t mode = hdr & 3u;
    float r = 0.0f;
    if (mode == 1u) {
        r = sci_sparse(rd, base, hdr, keep, (lz * 8u + ly) * 8u + lx, t);
    } else if (mode >= 2u) {
        const int res = mode == 2u ? 3 : 4;
        const int bits = (int)((hdr >> 8) & 0xFu);
        const uint32_t sub = (hdr >> 12) & 7u;
        const int per = res * res * res;
        const uint64_t scales = base + 4u + (uint64_t)(64 * (keep + 1));
        const int gi = mode == 2u ? 1 : 2;
        const AxisWeight dx = c_sci_axis[gi][lx], dy = c_sci_axis[gi][ly], dz = c_sci_axis[gi][lz];
        auto tri = [&](uint64_t data, float sc) {
            auto S = [&](int cx, int cy, int cz) { return bfp_sample(rd, data, res, bits, sc, (cz * res + cy) * res + cx); };
            const float d00 = lerp_ref(S(dx.i0, dy.i0, dz.i0), S(dx.i1, dy.i0, dz.i0), dx.t, dx.omt);
            const float d01 = lerp_ref(S(dx.i0, dy.i0, dz.i1), S(dx.i1, dy.i0, dz.i1), dx.t, dx.omt);
            const float d10 = lerp_ref(S(dx.i0, dy.i1, dz.i0), S(dx.i1, dy.i1, dz.i0), dx.t, dx.omt);
            const float d11 = lerp_ref(S(dx.i0, dy.i1, dz.i1), S(dx.i1, dy.i1, dz.i1), dx.t, dx.omt);
            return lerp_ref(lerp_ref(d00, d10, dy.t, dy.omt), lerp_ref(d01, d11, dy.t, dy.omt), dz.t, dz.omt);
        };
        if (sub == 1u) {
            const int tkeep = (int)((hdr >> 15) & 0xFu) + 1;
            if (bits > 0) {
                const int bbytes = (per * bits + 7) / 8;
                const uint64_t data = scales + (uint64_t)(tkeep * 2);
                for (int k = 0; k < tkeep; ++k) {
                    const float sc = half_bits_to_float(rd.u16(scales + (uint64_t)(k * 2)));
                    r = __fadd_rn(r, __fmul_rn(tri(data + (uint64_t)(k * bbytes), sc), __ldg(brow + k)));
                }
            }
        } else {
            const int fbytes = (per * bits + 7) / 8;
            const float sc = half_bits_to_float(rd.u16(scales + t * 2u));
            r = tri(scales + (uint64_t)a.g.frames * 2u + (uint64_t)t * fbytes, sc);
        }
    }
    oob |= rd.oob;
    return __fadd_rn(coarse, r);
}

// One point query (x, y, z, t) of one asset; decode errors go to `err`.
__device__ __forceinline__ float point_value(const DeviceAsset& a, uint4 qq, unsigned long long* err)
{
    const uint32_t x = qq.x, y = qq.y, z = qq.z, t = qq.w;
    // leaf lookup as render/src/vbt_file.cpp:250-262 leafIndexForVoxel (clamped leaf coordinates)
    const uint32_t bx = min(a.g.lcx - 1u, x >> 3), by = min(a.g.lcy - 1u, y >> 3), bz = min(a.g.lcz - 1u, z >> 3);
    const uint32_t leaf = (bz * a.g.lcy + by) * a.g.lcx + bx;
    const LeafEntry e = a.entries[leaf];
    const uint32_t st = entry_status(e);
    if (st != kOk) {
        record_error(err, leaf, st);
        return 0.0f;
    }
    if (a.g.profile == 2u) {
        if (t >= a.g.frames) {   // the reference indexes its per-frame tables out of range here
            record_error(err, leaf, kErrDecodeOob);
            return 0.0f;
        }
        float fv;
        if (sci_point_fast(a, e, x & 7u, y & 7u, z & 7u, t, fv)) return fv;
        bool oob = false;
        const float v = sci_point(a, e, x & 7u, y & 7u, z & 7u, t, oob);
        if (oob) record_error(err, leaf, kErrDecodeOob);
        return v;
    }
    if ((e.header & 3u) == kModeEmpty) return 0.0f;
    uint32_t gx, gy, gz;
    int w, h, d;
    leaf_extent(a.g, leaf, gx, gy, gz, w, h, d);
    const int lx = (int)(x - bx * 8u), ly = (int)(y - by * 8u), lz = (int)(z - bz * 8u);
    if (lx >= w || ly >= h || lz >= d) return 0.0f;   // outside the volume: no such voxel in any frame
    return rt_point(a, e, w, h, d, lx, ly, lz, clamp_frame((int)t, (int)a.g.frames));
}

// True when point_value returns 0 without decoding anything and without recording an error: a
// render-temporal query in an EMPTY leaf or outside the volume.
__device__ __forceinline__ bool point_trivial(const DeviceAsset& a, uint4 qq)
{
    if (a.g.profile == 2u) return false;
    const uint32_t bx = min(a.g.lcx - 1u, qq.x >> 3), by = min(a.g.lcy - 1u, qq.y >> 3), bz = min(a.g.lcz - 1u, qq.z >> 3);
    const uint32_t leaf = (bz * a.g.lcy + by) * a.g.lcx + bx;
    const uint32_t info = __ldg(&a.entries[leaf].info), header = __ldg(&a.entries[leaf].header);
    if (((info >> 16) & 0xFFu) != kOk) return false;   // point_value records the status
    if ((header & 3u) == kModeEmpty) return true;
    uint32_t gx, gy, gz;
    int w, h, d;
    leaf_extent(a.g, leaf, gx, gy, gz, w, h, d);
    return (int)(qq.x - bx * 8u) >= w || (int)(qq.y - by * 8u) >= h || (int)(qq.z - bz * 8u) >= d;
}

// Point queries in chunks of `per` x 128 per CTA.  In a chunk of a sparse volume a first pass
// answers the trivial queries (EMPTY leaf, outside the volume) and passes the others to a
// shared-memory list that the CTA's warps then decode with every lane busy -- most random queries
// there are trivial, and a warp that decoded its few non-trivial lanes in place would leave the
// rest idle.  Chunks of other volumes decode every query in place.  Values are point_value's
// either way.  `per` is chosen on the host so that the grid still fills the GPU.
constexpr int kPqThreads = 128, kPqMaxPer = 8, kPqMaxChunk = kPqThreads * kPqMaxPer;

template <class Resolve>
__device__ __forceinline__ void query_chunk(uint64_t n, int per, const uint4* __restrict__ q, const Resolve& resolve)
{
    __shared__ uint32_t s_list[kPqMaxChunk];
    __shared__ uint32_t s_count;
    const int tid = threadIdx.x, lane = tid & 31;
    const uint64_t base = (uint64_t)blockIdx.x * (uint64_t)(per * kPqThreads);
    if (!resolve.sparse(base)) {   // a chunk of a mostly active volume: each thread its own queries
        for (int r = 0; r < per; ++r) {
            const uint64_t i = base + (uint64_t)(r * kPqThreads + tid);
            if (i < n) resolve.second(i, q[i]);
        }
        return;
    }
    if (tid == 0) s_count = 0u;
    __syncthreads();
    for (int r = 0; r < per; ++r) {
        const uint32_t j = (uint32_t)(r * kPqThreads + tid);
        const uint64_t i = base + j;
        bool need = false;
        uint4 qq = make_uint4(0u, 0u, 0u, 0u);
        if (i < n) {
            qq = q[i];
            need = resolve.first(i, qq);
        }
        const unsigned m = __ballot_sync(0xFFFFFFFFu, need);
        uint32_t wbase = 0u;
        if (lane == 0 && m) wbase = atomicAdd(&s_count, (uint32_t)__popc(m));
        wbase = __shfl_sync(0xFFFFFFFFu, wbase, 0);
        if (need) s_list[wbase + (uint32_t)__popc(m & ((1u << lane) - 1u))] = j;
    }
    __syncthreads();
    const uint32_t cnt = s_count;
    for (uint32_t k = (uint32_t)tid; k < cnt; k += kPqThreads) {
        const uint64_t i = base + s_list[k];
        resolve.second(i, q[i]);
    }
}

// Queries per thread: the largest of 8, 4, 2, 1 that still gives four CTAs per SM.
static int query_per_thread(uint64_t n)
{
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const uint64_t want = 4ull * (uint64_t)(sms > 0 ? sms : 1);
    int per = kPqMaxPer;
    while (per > 1 && (n + (uint64_t)per * kPqThreads - 1) / ((uint64_t)per * kPqThreads) < want) per >>= 1;
    return per;
}

struct OneAssetQueries {
    const DeviceAsset& a;
    float* __restrict__ out;
    __device__ __forceinline__ bool sparse(uint64_t) const { return a.g.sparse != 0u; }
    __device__ __forceinline__ bool first(uint64_t i, uint4 qq) const
    {
        if (!point_trivial(a, qq)) return true;
        out[i] = 0.0f;
        return false;
    }
    __device__ __forceinline__ void second(uint64_t i, uint4 qq) const { out[i] = point_value(a, qq, a.err); }
};

// One thread per query: the shape for volumes whose leaves are mostly active.
__global__ void __launch_bounds__(128) query_points_kernel(DeviceAsset a, const uint32_t* __restrict__ q, uint64_t n,
                                                           float* __restrict__ out)
{
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] = point_value(a, reinterpret_cast<const uint4*>(q)[i], a.err);
}

// Compacted chunks: the shape for sparse volumes.
__global__ void __launch_bounds__(kPqThreads) query_points_compact_kernel(const __grid_constant__ DeviceAsset a,
                                                                          const uint32_t* __restrict__ q, uint64_t n,
                                                                          int per, float* __restrict__ out)
{
    query_chunk(n, per, reinterpret_cast<const uint4*>(q), OneAssetQueries{a, out});
}

// Point queries of several requests over several resident assets in one launch.  The segment
// table holds starts[0..k] (each request's first query; starts[k] = n), asset[k] (request r reads
// assets[asset[r]]) and, 8-byte aligned after them, outs[k] (request r's result array).  Request
// r's decode errors go to errs[r].
struct BatchQueries {
    const DeviceAsset* __restrict__ assets;
    const uint32_t* __restrict__ seg;
    uint32_t k;
    unsigned long long* errs;
    __device__ __forceinline__ int request(uint64_t i) const
    {
        int lo = 0, hi = (int)k - 1;
        while (lo < hi) {   // the last request whose first query is at or before i
            const int mid = (lo + hi + 1) >> 1;
            if (__ldg(seg + mid) <= (uint32_t)i) lo = mid;
            else hi = mid - 1;
        }
        return lo;
    }
    // the chunk starting at query i takes the compacting path when its first query's asset is sparse
    __device__ __forceinline__ bool sparse(uint64_t i) const
    {
        return assets[__ldg(seg + k + 1 + request(i))].g.sparse != 0u;
    }
    __device__ __forceinline__ void put(int r, uint64_t i, float v) const
    {
        const unsigned long long* outs = reinterpret_cast<const unsigned long long*>(seg + ((2u * k + 2u) & ~1u));
        reinterpret_cast<float*>(__ldg(outs + r))[i - __ldg(seg + r)] = v;
    }
    __device__ __forceinline__ bool first(uint64_t i, uint4 qq) const
    {
        const int r = request(i);
        if (!point_trivial(assets[__ldg(seg + k + 1 + r)], qq)) return true;
        put(r, i, 0.0f);
        return false;
    }
    __device__ __forceinline__ void second(uint64_t i, uint4 qq) const
    {
        const int r = request(i);
        put(r, i, point_value(assets[__ldg(seg + k + 1 + r)], qq, errs + r));
    }
};

__global__ void __launch_bounds__(128) query_points_batch_kernel(const DeviceAsset* __restrict__ assets,
                                                                 const uint32_t* __restrict__ seg, uint32_t k,
                                                                 const uint4* __restrict__ q, uint64_t n,
                                                                 unsigned long long* errs)
{
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int lo = 0, hi = (int)k - 1;
    while (lo < hi) {   // the last request whose first query is at or before i
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(seg + mid) <= (uint32_t)i) lo = mid;
        else hi = mid - 1;
    }
    const unsigned long long* outs = reinterpret_cast<const unsigned long long*>(seg + ((2u * k + 2u) & ~1u));
    float* o = reinterpret_cast<float*>(__ldg(outs + lo));
    o[i - __ldg(seg + lo)] = point_value(assets[__ldg(seg + k + 1 + lo)], q[i], errs + lo);
}

__global__ void __launch_bounds__(kPqThreads) query_points_batch_compact_kernel(
    const DeviceAsset* __restrict__ assets, const uint32_t* __restrict__ seg, uint32_t k, const uint4* __restrict__ q,
    uint64_t n, int per, unsigned long long* errs)
{
    query_chunk(n, per, q, BatchQueries{assets, seg, k, errs});
}

void launch_query_points_batch(const DeviceAsset* assets, const uint32_t* seg, uint32_t k, const uint4* q, uint64_t n,
                               unsigned long long* errs, int sparse, cudaStream_t s)
{
    if (n == 0 || k == 0) return;
    if (sparse == 0) {
        query_points_batch_kernel<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(assets, seg, k, q, n, errs);
        return;
    }
    // with requests on mostly active volumes in the launch, one query per thread for their chunks
    const int per = sparse == 2 ? query_per_thread(n) : 1;
    const uint64_t chunk = (uint64_t)per * kPqThreads;
    query_points_batch_compact_kernel<<<(unsigned)((n + chunk - 1) / chunk), kPqThreads, 0, s>>>(assets, seg, k, q, n,
                                                                                                   per, errs);
}

void launch_query_points(const DeviceAsset& a, const uint32_t* q, uint64_t n, float* out, bool sparse, cudaStream_t s)
{
    if (n == 0) return;
    if (!sparse) {
        query_points_kernel<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(a, q, n, out);
        return;
    }
    const int per = query_per_thread(n);
    const uint64_t chunk = (uint64_t)per * kPqThreads;
    query_points_compact_kernel<<<(unsigned)((n + chunk - 1) / chunk), kPqThreads, 0, s>>>(a, q, n, per, out);
}

// Z-slice over [t0, t1): one warp per (leaf of the z layer, frame); lanes 0..7 produce rows.
__global__ void __launch_bounds__(kDecodeWarps * 32) query_slice_kernel(DeviceAsset a, uint32_t z, int t0, int t1,
                                                                        float* __restrict__ out)
{
    __shared__ __align__(16) float s_ctrl_all[kDecodeWarps][kWarpSlots];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    float* s_ctrl = s_ctrl_all[warp];
    const uint32_t bz = min(a.g.lcz - 1u, z >> 3);
    const int lz = (int)(z - bz * 8u);
    const uint32_t layer = a.g.lcx * a.g.lcy;
    const uint32_t n_items = layer * (uint32_t)(t1 - t0);
    for (uint32_t item = blockIdx.x * kDecodeWarps + warp; item < n_items; item += gridDim.x * kDecodeWarps) {
        const uint32_t li = item % layer;
        const int t = t0 + (int)(item / layer);
        const uint32_t leaf = bz * layer + li;
        const LeafEntry e = a.entries[leaf];
        uint32_t bx, by, bzz;
        int w, h, d;
        leaf_extent(a.g, leaf, bx, by, bzz, w, h, d);
        const uint32_t st = entry_status(e);
        const bool empty = a.g.profile != 2u && (e.header & 3u) == kModeEmpty;
        bool oob = false;
        const bool in_range = lz < d && (a.g.profile != 2u || (uint32_t)t < a.g.frames);
        if (st != kOk && lane == 0) record_error(a.err, leaf, st);
        if (in_range && !empty && st == kOk) {
            if (a.g.profile == 2u) sci_decode_controls(a, e, (uint32_t)t, s_ctrl, lane, oob);
            else rt_decode_controls(a, e, clamp_frame(t, (int)a.g.frames), s_ctrl, lane);
        }
        __syncwarp();
        if (lane < 8 && lane < h) {
            float v[8];
            if (!in_range || empty || st != kOk) {
                for (int i = 0; i < 8; ++i) v[i] = 0.0f;
            } else if (a.g.profile == 2u) {
                sci_row(a, e, s_ctrl, (uint32_t)t, w, h, d, lane, lz, v, oob);
            } else {
                rt_row(a, e, s_ctrl, w, h, d, lane, lz, v);
            }
            float* dst = out + (uint64_t)(t - t0) * a.g.width * a.g.height + (uint64_t)(by * 8 + lane) * a.g.width + bx * 8;
            for (int i = 0; i < w; ++i) dst[i] = v[i];
        }
        if (__any_sync(0xFFFFFFFFu, oob) && lane == 0) record_error(a.err, leaf, kErrDecodeOob);
        __syncwarp();
    }
}

void launch_query_slice(const DeviceAsset& a, uint32_t z, int t0, int t1, float* out, cudaStream_t s)
{
    if (t1 <= t0) return;
    query_slice_kernel<<<default_grid(), kDecodeWarps * 32, 0, s>>>(a, z, t0, t1, out);
}

}  // namespace vbtb
#include "serve_mixed.cuh"
namespace vbtb {

uint64_t mixed_request_tiles(const MixedReq& r, const AssetGeom& g) { return mixed_tiles(r, g); }

int launch_serve_mixed(const DeviceAsset* assets, const MixedReq* reqs, uint32_t k, uint64_t n_tiles,
                       unsigned long long* counter, unsigned long long* errs, MixedStepGraph* graph, cudaStream_t s)
{
    if (k == 0 || n_tiles == 0) return 0;
    if (k > kMaxMixedReqs) return (int)cudaErrorInvalidValue;
    int grid = mixed_grid(n_tiles);
    if (!graph) {
        cudaMemsetAsync(counter, 0, sizeof(unsigned long long), s);
        serve_mixed_kernel<<<grid, kMixedWarps * 32, 0, s>>>(assets, reqs, k, n_tiles, counter, errs);
        return (int)cudaGetLastError();
    }
    void* args[] = {(void*)&assets, (void*)&reqs, (void*)&k, (void*)&n_tiles, (void*)&counter, (void*)&errs};
    cudaKernelNodeParams kp{};
    kp.func = (void*)serve_mixed_kernel;
    kp.gridDim = dim3((unsigned)grid);
    kp.blockDim = dim3(kMixedWarps * 32);
    kp.sharedMemBytes = 0;
    kp.kernelParams = args;
    cudaError_t e = cudaSuccess;
    if (!graph->exec) {
        cudaMemsetParams mp{};
        mp.dst = counter;
        mp.value = 0;
        mp.elementSize = 4;
        mp.width = 2;
        mp.height = 1;
        cudaGraphNode_t memset_node = nullptr;
        if ((e = cudaGraphCreate(&graph->graph, 0)) != cudaSuccess ||
            (e = cudaGraphAddMemsetNode(&memset_node, graph->graph, nullptr, 0, &mp)) != cudaSuccess ||
            (e = cudaGraphAddKernelNode(&graph->kernel, graph->graph, &memset_node, 1, &kp)) != cudaSuccess ||
            (e = cudaGraphInstantiate(&graph->exec, graph->graph, 0)) != cudaSuccess) {
            release_mixed_graph(*graph);
            return (int)e;
        }
    } else if ((e = cudaGraphExecKernelNodeSetParams(graph->exec, graph->kernel, &kp)) != cudaSuccess) {
        return (int)e;
    }
    return (int)cudaGraphLaunch(graph->exec, s);
}

void release_mixed_graph(MixedStepGraph& g)
{
    if (g.exec) cudaGraphExecDestroy(g.exec);
    if (g.graph) cudaGraphDestroy(g.graph);
    g = MixedStepGraph{};
}

// Exhaustive check of div_small_rn (the render decode's interval quotient) against IEEE division:
// every pair 0 < a < b <= b_max, with RN(1/b) as the decode forms it.  Counts mismatches and keeps
// the smallest failing (b << 16 | a).
__global__ void key_division_check_kernel(uint32_t b_max, unsigned long long* bad, unsigned long long* first)
{
    unsigned long long local = 0;
    for (uint32_t b = 2u + blockIdx.x; b <= b_max; b += gridDim.x) {
        const float bf = (float)b;
        const float y = __frcp_rn(bf);
        for (uint32_t a = 1u + threadIdx.x; a < b; a += blockDim.x) {
            const float q = div_small_rn((float)a, bf, y);
            if (__float_as_uint(q) != __float_as_uint(__fdiv_rn((float)a, bf))) {
                ++local;
                atomicMin(first, ((unsigned long long)b << 16) | a);
            }
        }
    }
    if (local) atomicAdd(bad, local);
}

void launch_key_division_check(uint32_t b_max, unsigned long long* d_out, cudaStream_t s)
{
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    key_division_check_kernel<<<8 * (sms > 0 ? sms : 1), 256, 0, s>>>(b_max, d_out, d_out + 1);
}

}  // namespace vbtb

// (d) window decode of scientific leaves on the tensor cores: sci_window.cuh
#include <cuda_bf16.h>

#include "sci_window.cuh"
#include "render_window.cuh"
