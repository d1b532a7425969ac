// serve.cu -- the serving loop (vbt_server_* / vbt_serve_* in include/vbt_b200.h).
//
// One scheduler thread per server issues every CUDA call on the server's streams.  Each pass:
//   1. completions: a unit (one launch group) whose event has fired is finalised: error words are
//      turned into request statuses, results bound for pageable host buffers are copied out of
//      pinned staging, arena blocks are returned, and waiting clients are woken;
//   2. admission: pending requests are taken in arrival order while a launch stream is free and
//      the device arena (the HBM budget) has room for their inputs and results.  A request that
//      does not fit may be passed over by later ones at most kMaxBypass times; after that the
//      server admits nothing behind it until it fits;
//   3. batching: the requests admitted in one pass -- points, slices and frames of any assets --
//      become units of up to max_batch_queries values each (a larger request is a unit of its own:
//      measured, a single frame of a large volume decodes faster as the mixed launch's leaf tiles,
//      which read only the keys the frame needs, than on the dense frame kernel, which stages
//      each whole leaf).
//      A unit is at most two launches: its point requests, across assets, in one multi-asset point
//      launch, and its slices and frames in ONE persistent launch (serve_mixed_kernel) whose warps
//      take tiles of all of them from a work counter, replayed from a per-stream CUDA graph with
//      the unit's parameters.  With separate_kinds, only point requests merge and slices and
//      frames run on their own kernels, a unit each.
// Units run on `slots` streams, so requests that arrive while others are on the GPU overlap
// with them.  In plain mode the server admits one request per unit, keeps one unit in flight, and
// runs each on its kind's own kernel.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "asset.h"
#include "kernels.cuh"

namespace vbtb {
int set_last_error(int status, const std::string& msg);
}

using namespace vbtb;

namespace {

using Clock = std::chrono::steady_clock;

constexpr uint32_t kMaxAssets = 64;
constexpr uint32_t kMaxUnitRequests = 256;   // requests merged into one launch
static_assert(kMaxUnitRequests <= kMaxMixedReqs, "a unit's requests fit the mixed kernel's table");
constexpr uint32_t kMaxSlots = 32;
constexpr int kMaxBypass = 64;
constexpr uint64_t kAlign = 256;

int fail(int status, const std::string& msg) { return set_last_error(status, msg); }

// First-fit allocator over one contiguous region (offsets), kAlign granules, coalescing frees.
class Arena {
  public:
    void reset(uint64_t size)
    {
        free_.clear();
        if (size) free_[0] = size;
        size_ = size;
        used_ = peak_ = 0;
    }
    static uint64_t round(uint64_t b) { return b ? (b + kAlign - 1) & ~(kAlign - 1) : kAlign; }
    bool alloc(uint64_t bytes, uint64_t* off)
    {
        bytes = round(bytes);
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < bytes) continue;
            *off = it->first;
            const uint64_t rest = it->second - bytes, start = it->first + bytes;
            free_.erase(it);
            if (rest) free_[start] = rest;
            used_ += bytes;
            peak_ = std::max(peak_, used_);
            return true;
        }
        return false;
    }
    void release(uint64_t off, uint64_t bytes)
    {
        bytes = round(bytes);
        used_ -= bytes;
        auto it = free_.emplace(off, bytes).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_.erase(nx);
        }
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_.erase(it);
            }
        }
    }
    uint64_t size() const { return size_; }
    uint64_t peak() const { return peak_; }
    void clear_peak() { peak_ = used_; }

  private:
    std::map<uint64_t, uint64_t> free_;
    uint64_t size_ = 0, used_ = 0, peak_ = 0;
};

struct Block {
    uint64_t off = 0, bytes = 0;
    bool valid = false;
};

struct Req {
    uint64_t ticket = 0;
    vbt_request r{};
    std::vector<int32_t> frames;
    uint64_t result_floats = 0;
    int state = 0;   // 0 pending, 1 being admitted or in flight, 2 done
    int status = VBT_STATUS_OK;
    uint32_t bad_leaf = 0;
    double t_submit = 0, t_start = 0, t_done = 0;
    Block dev_result;          // result in the device arena
    Block stage_out;           // pinned staging for a pageable host_out
    bool pinned_in = false, pinned_out = false;
    int bypassed = 0;
};

struct Unit {
    std::vector<Req*> reqs;
    Block dev_in;     // error words, segment or request table, point inputs
    Block stage_in;   // pinned staging of the table and pageable point inputs
    uint64_t points = 0;
    uint64_t frames = 0;   // frame indices of the unit's frame requests (mixed units)
    bool mixed = false;    // one serve_mixed_kernel launch over all of its requests
};

// Memory the copy engines reach directly: pinned host memory, or device (or managed) memory of
// a GPU -- a client that keeps its query batches and results on the GPU.  Pageable host memory
// goes through the server's pinned staging.
bool is_pinned(const void* p)
{
    if (!p) return false;
    cudaPointerAttributes at{};
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return at.type == cudaMemoryTypeHost || at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}

// Segment table of a k-request point unit: starts[k+1], asset[k], 8-byte aligned outs[k].
uint64_t seg_bytes(uint32_t k) { return ((4ull * (2 * k + 1) + 7) & ~7ull) + 8ull * k; }
// Error words of a unit, padded so that what follows starts on a 16-byte boundary.
uint64_t err_bytes(uint32_t k) { return (8ull * k + 15) & ~15ull; }
// Device input block of a point unit: [errs][segment table][queries 16N], each part 16-byte
// aligned (the queries are read as uint4, the output addresses as 64-bit words).
uint64_t points_in_bytes(uint32_t k, uint64_t n) { return err_bytes(k) + ((seg_bytes(k) + 15) & ~15ull) + 16ull * n; }
uint64_t a16(uint64_t b) { return (b + 15) & ~15ull; }
// Tables of a mixed unit with kp point requests and km slice / frame requests holding nf frame
// indices in all: [point segment table][MixedReq km][int32 nf], staged on the host and copied as
// one block.
uint64_t mixed_table_bytes(uint32_t kp, uint32_t km, uint64_t nf)
{
    return a16(seg_bytes(kp)) + a16(sizeof(MixedReq) * km) + a16(4ull * nf);
}
// Device input block of a mixed unit: [errs][tables][queries 16N], each part 16-byte aligned.
uint64_t mixed_in_bytes(uint32_t kp, uint32_t km, uint64_t nf, uint64_t n)
{
    return err_bytes(kp + km) + mixed_table_bytes(kp, km, nf) + 16ull * n;
}

}  // namespace

struct vbt_server {
    vbt_server_config cfg{};
    Clock::time_point t0 = Clock::now();
    // assets
    std::vector<vbt_asset*> assets;
    DeviceAsset* d_assets = nullptr;
    uint64_t resident_bytes = 0;
    // memory (the arenas are touched by the scheduler thread only)
    uint8_t* d_arena = nullptr;
    uint8_t* h_stage = nullptr;
    Arena arena, stage;
    unsigned long long* h_err = nullptr;   // pinned error words: [slot][kMaxUnitRequests]
    // streams
    cudaStream_t streams[kMaxSlots]{};
    cudaEvent_t events[kMaxSlots]{};
    Unit* busy[kMaxSlots]{};
    unsigned long long* d_counters = nullptr;   // the mixed launch's work counter, one per stream
    MixedStepGraph graphs[kMaxSlots];           // the mixed step as a graph, one per stream
    // requests
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Req*> pending;
    std::unordered_map<uint64_t, Req*> tickets;
    std::vector<Block> to_free;   // device results released by clients
    uint64_t next_ticket = 1;
    bool stop = false;
    bool dead = false;   // the device reported a fault; no further work is launched
    std::thread worker;
    // stats (guarded by mu)
    std::vector<double> latencies;
    uint64_t requests_done = 0, points_done = 0, voxels_done = 0, launches = 0, units = 0;
    double busy_ms = 0;

    double now_ms() const { return std::chrono::duration<double, std::milli>(Clock::now() - t0).count(); }
    void run();
    bool reserve_result(Req* r);
    void unreserve_result(Req* r);
    bool fill_points(Unit* u);
    bool fill_mixed(Unit* u);
    void admit(std::vector<Unit*>& out, int free_slots);
    void launch(Unit* u, int slot);
    void finalize(Unit* u, int slot);
};

// ------------------------------------------------------------------------------ admission

static uint64_t result_floats(const vbt_request& r, const vbt_asset* a)
{
    const uint64_t X = a->hdr.width, Y = a->hdr.height, Z = a->hdr.depth;
    switch (r.kind) {
    case VBT_REQ_POINTS: return r.n_points;
    case VBT_REQ_SLICE: return r.t1 > r.t0 ? (uint64_t)(r.t1 - r.t0) * X * Y : 0;
    case VBT_REQ_FRAMES: return (uint64_t)r.n_frames * X * Y * Z;
    }
    return 0;
}

// Reserve a request's own result block (and pinned staging for a pageable host buffer).
// Returns false, holding nothing, when they do not fit.
bool vbt_server::reserve_result(Req* r)
{
    Block d;
    d.bytes = 4ull * r->result_floats;
    if (!arena.alloc(d.bytes, &d.off)) return false;
    d.valid = true;
    r->pinned_out = r->r.host_out && is_pinned(r->r.host_out);
    if (r->r.host_out && !r->pinned_out) {
        Block h;
        h.bytes = d.bytes;
        if (!stage.alloc(h.bytes, &h.off)) {
            arena.release(d.off, d.bytes);
            return false;
        }
        h.valid = true;
        r->stage_out = h;
    }
    r->dev_result = d;
    return true;
}

void vbt_server::unreserve_result(Req* r)
{
    if (r->dev_result.valid) arena.release(r->dev_result.off, r->dev_result.bytes);
    if (r->stage_out.valid) stage.release(r->stage_out.off, r->stage_out.bytes);
    r->dev_result.valid = r->stage_out.valid = false;
}

// Reserve a point unit's input blocks, returning requests from the back to the queue until they fit.
bool vbt_server::fill_points(Unit* u)
{
    while (!u->reqs.empty()) {
        const uint32_t k = (uint32_t)u->reqs.size();
        uint64_t n = 0, pageable = 0;
        for (Req* r : u->reqs) {
            n += r->r.n_points;
            if (!r->pinned_in) pageable += 16ull * r->r.n_points;
        }
        Block d, h;
        d.bytes = points_in_bytes(k, n);
        h.bytes = seg_bytes(k) + pageable;
        if (arena.alloc(d.bytes, &d.off)) {
            d.valid = true;
            if (stage.alloc(h.bytes, &h.off)) {
                h.valid = true;
                u->dev_in = d;
                u->stage_in = h;
                u->points = n;
                return true;
            }
            arena.release(d.off, d.bytes);
        }
        Req* last = u->reqs.back();
        u->reqs.pop_back();
        unreserve_result(last);
        last->state = 0;
    }
    return false;
}

// Reserve a mixed unit's input blocks, returning requests from the back to the queue until they fit.
bool vbt_server::fill_mixed(Unit* u)
{
    while (!u->reqs.empty()) {
        uint32_t kp = 0;
        uint64_t n = 0, nf = 0, pageable = 0;
        for (Req* r : u->reqs) {
            if (r->r.kind == VBT_REQ_POINTS) {
                ++kp;
                n += r->r.n_points;
                if (!r->pinned_in) pageable += 16ull * r->r.n_points;
            } else if (r->r.kind == VBT_REQ_FRAMES) {
                nf += r->frames.size();
            }
        }
        const uint32_t km = (uint32_t)u->reqs.size() - kp;
        Block d, h;
        d.bytes = mixed_in_bytes(kp, km, nf, n);
        h.bytes = mixed_table_bytes(kp, km, nf) + pageable;
        if (arena.alloc(d.bytes, &d.off)) {
            d.valid = true;
            if (stage.alloc(h.bytes, &h.off)) {
                h.valid = true;
                u->dev_in = d;
                u->stage_in = h;
                u->points = n;
                u->frames = nf;
                u->mixed = true;
                // point requests first: the point launch reports into errs[0, kp), the mixed one
                // into errs[kp, k)
                std::stable_partition(u->reqs.begin(), u->reqs.end(),
                                      [](const Req* r) { return r->r.kind == VBT_REQ_POINTS; });
                return true;
            }
            arena.release(d.off, d.bytes);
        }
        Req* last = u->reqs.back();
        u->reqs.pop_back();
        unreserve_result(last);
        last->state = 0;
    }
    return false;
}

// Build the units of this pass (called with mu held).
void vbt_server::admit(std::vector<Unit*>& out, int free_slots)
{
    const bool mixed = !cfg.plain && !cfg.separate_kinds;
    while (free_slots > 0 && !pending.empty()) {
        Unit* u = new Unit();
        bool points_unit = false;
        uint64_t points = 0, values = 0;
        size_t scanned = 0;
        Req* blocked = nullptr;   // the oldest request of this pass that did not fit
        for (auto it = pending.begin(); it != pending.end(); ++it, ++scanned) {
            Req* r = *it;
            if (r->state != 0) continue;
            if (cfg.plain && scanned > 0) break;
            const bool pts = r->r.kind == VBT_REQ_POINTS;
            if (!u->reqs.empty()) {
                if (u->reqs.size() >= kMaxUnitRequests) continue;
                if (mixed) {
                    if (values + r->result_floats > cfg.max_batch_queries) continue;
                } else {
                    if (!points_unit || !pts) continue;   // only point requests merge
                    if (points + r->r.n_points > cfg.max_batch_queries) continue;
                }
            }
            if (blocked && blocked->bypassed >= kMaxBypass) break;   // hold the line for it
            if (pts) r->pinned_in = is_pinned(r->r.points);
            if (!reserve_result(r)) {
                if (!blocked) blocked = r;
                continue;
            }
            if (blocked) ++blocked->bypassed;
            r->state = 1;
            u->reqs.push_back(r);
            values += r->result_floats;
            if (pts) {
                points_unit = true;
                points += r->r.n_points;
            }
            if (cfg.plain) break;
            if (mixed) continue;
            if (!pts) break;   // slices and frames run alone
        }
        bool ok = !u->reqs.empty();
        if (ok && mixed) {
            ok = fill_mixed(u);
        } else if (ok && points_unit) {
            ok = fill_points(u);
        } else if (ok) {
            Block d;
            d.bytes = 8;
            ok = arena.alloc(d.bytes, &d.off);
            if (ok) {
                d.valid = true;
                u->dev_in = d;
            } else {
                unreserve_result(u->reqs[0]);
                u->reqs[0]->state = 0;
                u->reqs.clear();
            }
        }
        if (!ok) {
            delete u;
            break;
        }
        for (Req* r : u->reqs) pending.erase(std::find(pending.begin(), pending.end(), r));
        out.push_back(u);
        --free_slots;
        if (cfg.plain) break;
    }
}

// ------------------------------------------------------------------------------ launch

void vbt_server::launch(Unit* u, int slot)
{
    cudaStream_t st = streams[slot];
    uint8_t* din = d_arena + u->dev_in.off;
    unsigned long long* d_err = reinterpret_cast<unsigned long long*>(din);
    const uint32_t k = (uint32_t)u->reqs.size();
    const double t = now_ms();
    for (Req* r : u->reqs) r->t_start = t;
    cudaMemsetAsync(d_err, 0xFF, 8ull * k, st);
    uint64_t nl = 0;
    Req* r0 = u->reqs[0];
    int launch_err = 0;
    if (u->mixed) {
        // tables staged and copied as one block: [point segment table][MixedReq][frame lists];
        // the point inputs after them
        uint32_t kp = 0;
        while (kp < k && u->reqs[kp]->r.kind == VBT_REQ_POINTS) ++kp;
        const uint32_t km = k - kp;
        uint8_t* hs = h_stage + u->stage_in.off;
        uint32_t* starts = reinterpret_cast<uint32_t*>(hs);
        uint64_t* outs = reinterpret_cast<uint64_t*>(hs + ((4ull * (2 * kp + 1) + 7) & ~7ull));
        MixedReq* tab = reinterpret_cast<MixedReq*>(hs + a16(seg_bytes(kp)));
        int32_t* hfr = reinterpret_cast<int32_t*>(reinterpret_cast<uint8_t*>(tab) + a16(sizeof(MixedReq) * km));
        uint8_t* dseg = din + err_bytes(k);
        uint8_t* dtab = dseg + a16(seg_bytes(kp));
        uint8_t* dfr = dtab + a16(sizeof(MixedReq) * km);
        const uint64_t tables = mixed_table_bytes(kp, km, u->frames);
        uint8_t* dq = dseg + tables;
        uint8_t* hpage = hs + tables;
        uint64_t q = 0, f = 0, tiles = 0, sparse_points = 0;
        for (uint32_t i = 0; i < kp; ++i) {
            Req* r = u->reqs[i];
            starts[i] = (uint32_t)q;
            starts[kp + 1 + i] = r->r.asset;
            outs[i] = reinterpret_cast<uint64_t>(d_arena + r->dev_result.off);
            const uint64_t b = 16ull * r->r.n_points;
            if (b) {
                if (r->pinned_in) {
                    cudaMemcpyAsync(dq + 16ull * q, r->r.points, b, cudaMemcpyDefault, st);
                } else {
                    std::memcpy(hpage, r->r.points, b);
                    cudaMemcpyAsync(dq + 16ull * q, hpage, b, cudaMemcpyHostToDevice, st);
                    hpage += b;
                }
            }
            if (assets[r->r.asset]->sparse) sparse_points += r->r.n_points;
            q += r->r.n_points;
        }
        starts[kp] = (uint32_t)q;
        for (uint32_t i = 0; i < km; ++i) {
            Req* r = u->reqs[kp + i];
            MixedReq m{};
            m.asset = r->r.asset;
            m.first = tiles;
            m.out = reinterpret_cast<uint64_t>(d_arena + r->dev_result.off);
            if (r->r.kind == VBT_REQ_SLICE) {
                m.kind = kMixedSlice;
                m.a0 = r->r.z;
                m.t0 = r->r.t0;
                m.t1 = r->r.t1;
            } else {
                m.kind = kMixedFrames;
                m.n = (uint32_t)r->frames.size();
                m.in = reinterpret_cast<uint64_t>(dfr + 4ull * f);
                if (m.n) std::memcpy(hfr + f, r->frames.data(), 4ull * m.n);
                f += m.n;
            }
            tab[i] = m;
            tiles += mixed_request_tiles(m, assets[r->r.asset]->dev.g);
        }
        cudaMemcpyAsync(dseg, hs, tables, cudaMemcpyHostToDevice, st);
        if (q) {
            launch_query_points_batch(d_assets, reinterpret_cast<const uint32_t*>(dseg), kp,
                                      reinterpret_cast<const uint4*>(dq), q, d_err,
                                      sparse_points == 0u ? 0 : (sparse_points == q ? 2 : 1), st);
            ++nl;
        }
        if (tiles) {
            launch_err = launch_serve_mixed(d_assets, reinterpret_cast<const MixedReq*>(dtab), km, tiles,
                                            d_counters + slot, d_err + kp, &graphs[slot], st);
            ++nl;
        }
    } else if (r0->r.kind == VBT_REQ_POINTS) {
        uint8_t* hseg = h_stage + u->stage_in.off;
        uint32_t* starts = reinterpret_cast<uint32_t*>(hseg);
        uint64_t* outs = reinterpret_cast<uint64_t*>(hseg + ((4ull * (2 * k + 1) + 7) & ~7ull));
        uint64_t run = 0;
        for (uint32_t i = 0; i < k; ++i) {
            starts[i] = (uint32_t)run;
            starts[k + 1 + i] = u->reqs[i]->r.asset;
            outs[i] = reinterpret_cast<uint64_t>(d_arena + u->reqs[i]->dev_result.off);
            run += u->reqs[i]->r.n_points;
        }
        starts[k] = (uint32_t)run;
        uint8_t* dseg = din + err_bytes(k);
        uint8_t* dq = dseg + ((seg_bytes(k) + 15) & ~15ull);
        cudaMemcpyAsync(dseg, hseg, seg_bytes(k), cudaMemcpyHostToDevice, st);
        uint8_t* hpage = hseg + seg_bytes(k);
        uint64_t q = 0;
        for (Req* r : u->reqs) {
            const uint64_t b = 16ull * r->r.n_points;
            if (b) {
                if (r->pinned_in) {
                    cudaMemcpyAsync(dq + 16ull * q, r->r.points, b, cudaMemcpyDefault, st);
                } else {
                    std::memcpy(hpage, r->r.points, b);
                    cudaMemcpyAsync(dq + 16ull * q, hpage, b, cudaMemcpyHostToDevice, st);
                    hpage += b;
                }
            }
            q += r->r.n_points;
        }
        uint64_t sparse_points = 0;
        for (Req* r : u->reqs)
            if (assets[r->r.asset]->sparse) sparse_points += r->r.n_points;
        launch_query_points_batch(d_assets, reinterpret_cast<const uint32_t*>(dseg), k,
                                  reinterpret_cast<const uint4*>(dq), u->points, d_err,
                                  sparse_points == 0u ? 0 : (sparse_points == u->points ? 2 : 1),
                                  st);
        nl = 1;
    } else {
        vbt_asset* a = assets[r0->r.asset];
        DeviceAsset dv = a->dev;
        dv.err = d_err;   // this request's own error word
        float* out = reinterpret_cast<float*>(d_arena + r0->dev_result.off);
        if (r0->r.kind == VBT_REQ_SLICE) {
            launch_query_slice(dv, r0->r.z, r0->r.t0, r0->r.t1, out, st);
            nl = 1;
        } else {
            const uint64_t vox = (uint64_t)a->hdr.width * a->hdr.height * a->hdr.depth;
            for (size_t i = 0; i < r0->frames.size(); i += 64) {
                const int n = (int)std::min<size_t>(64, r0->frames.size() - i);
                launch_decode_dense(dv, a->launch_seq.fetch_add(1), r0->frames.data() + i, n, out + i * vox, 0, st);
                ++nl;
            }
        }
    }
    for (uint32_t i = 0; i < k; ++i) {
        Req* r = u->reqs[i];
        const uint64_t b = 4ull * r->result_floats;
        if (r->r.host_out && b) {
            void* dst = r->pinned_out ? static_cast<void*>(r->r.host_out) : static_cast<void*>(h_stage + r->stage_out.off);
            cudaMemcpyAsync(dst, d_arena + r->dev_result.off, b, cudaMemcpyDefault, st);
        }
    }
    cudaMemcpyAsync(h_err + (size_t)slot * kMaxUnitRequests, d_err, 8ull * k, cudaMemcpyDeviceToHost, st);
    cudaEventRecord(events[slot], st);
    const cudaError_t e = cudaGetLastError();
    busy[slot] = u;
    std::lock_guard<std::mutex> lk(mu);
    launches += nl;
    ++units;
    if (e != cudaSuccess || launch_err != 0)
        for (Req* r : u->reqs) r->status = VBT_STATUS_CUDA;
}

void vbt_server::finalize(Unit* u, int slot)
{
    const double t = now_ms();
    const unsigned long long* errs = h_err + (size_t)slot * kMaxUnitRequests;
    for (size_t i = 0; i < u->reqs.size(); ++i) {
        Req* r = u->reqs[i];
        if (r->status == VBT_STATUS_OK && errs[i] != ~0ull) {
            r->status = (int)(errs[i] & 0xFFull);
            r->bad_leaf = (uint32_t)(errs[i] >> 8);
        }
        if (r->r.host_out && !r->pinned_out && r->result_floats)
            std::memcpy(r->r.host_out, h_stage + r->stage_out.off, 4ull * r->result_floats);
        if (r->stage_out.valid) stage.release(r->stage_out.off, r->stage_out.bytes);
        r->stage_out.valid = false;
        if (r->r.host_out && r->dev_result.valid) {
            arena.release(r->dev_result.off, r->dev_result.bytes);
            r->dev_result.valid = false;
        }
    }
    if (u->dev_in.valid) arena.release(u->dev_in.off, u->dev_in.bytes);
    if (u->stage_in.valid) stage.release(u->stage_in.off, u->stage_in.bytes);
    busy[slot] = nullptr;
    {
        std::lock_guard<std::mutex> lk(mu);
        for (Req* r : u->reqs) {
            r->t_done = t;
            r->state = 2;
            latencies.push_back(t - r->t_submit);
            ++requests_done;
            if (r->r.kind == VBT_REQ_POINTS) points_done += r->r.n_points;
            else voxels_done += r->result_floats;
        }
    }
    cv_done.notify_all();
    delete u;
}

void vbt_server::run()
{
    cudaSetDevice(cfg.device);
    double busy_since = -1.0;
    for (;;) {
        bool progressed = false;
        int in_flight = 0;
        for (uint32_t s = 0; s < cfg.slots; ++s) {
            if (!busy[s]) continue;
            const cudaError_t q = cudaEventQuery(events[s]);
            if (q == cudaSuccess) {
                finalize(busy[s], (int)s);
                progressed = true;
            } else if (q == cudaErrorNotReady) {
                cudaGetLastError();   // not sticky; clear it
                ++in_flight;
            } else {
                // the device reported a fault: the unit's requests fail, and so does all later work
                dead = true;
                for (Req* r : busy[s]->reqs) r->status = VBT_STATUS_CUDA;
                finalize(busy[s], (int)s);
                progressed = true;
            }
        }
        std::vector<Unit*> ready;
        {
            std::unique_lock<std::mutex> lk(mu);
            for (const Block& b : to_free) arena.release(b.off, b.bytes);
            to_free.clear();
            if (dead) {   // complete everything pending with the device error
                const double t = now_ms();
                for (Req* r : pending) {
                    r->status = VBT_STATUS_CUDA;
                    r->t_done = t;
                    r->state = 2;
                }
                pending.clear();
                cv_done.notify_all();
            }
            int free_slots = 0;
            for (uint32_t s = 0; s < cfg.slots; ++s) free_slots += busy[s] ? 0 : 1;
            if (cfg.plain && in_flight > 0) free_slots = 0;
            admit(ready, free_slots);
            if (ready.empty() && in_flight == 0) {
                if (busy_since >= 0.0) {
                    busy_ms += now_ms() - busy_since;
                    busy_since = -1.0;
                }
                if (stop && pending.empty()) break;
                if (!progressed)
                    cv_work.wait_for(lk, std::chrono::milliseconds(2),
                                     [&] { return stop || !to_free.empty() || !pending.empty(); });
                continue;
            }
        }
        for (Unit* u : ready) {
            int slot = 0;
            while (busy[slot]) ++slot;   // admit() never returns more units than free slots
            if (busy_since < 0.0) busy_since = now_ms();
            launch(u, slot);
        }
        if (ready.empty() && !progressed) std::this_thread::yield();
    }
}

// ------------------------------------------------------------------------------ C-ABI

static void fill_result(const vbt_server* s, const Req* r, vbt_request_result* res)
{
    if (!res) return;
    res->status = r->status;
    res->bad_leaf = r->bad_leaf;
    res->result_floats = r->result_floats;
    res->device_result =
        (!r->r.host_out && r->dev_result.valid) ? reinterpret_cast<const float*>(s->d_arena + r->dev_result.off) : nullptr;
    res->submit_ms = r->t_submit;
    res->start_ms = r->t_start;
    res->done_ms = r->t_done;
}

extern "C" {

int vbt_server_create(const vbt_server_config* config, vbt_server** out)
{
    if (!config || !out) return fail(VBT_STATUS_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    vbt_server_config c = *config;
    if (c.slots == 0 || c.slots > kMaxSlots) return fail(VBT_STATUS_INVALID_ARGUMENT, "slots must be 1..32");
    if (c.hbm_budget_bytes < 4096) return fail(VBT_STATUS_INVALID_ARGUMENT, "hbm_budget_bytes below 4 KiB");
    if (c.max_batch_queries == 0) c.max_batch_queries = 4u << 20;
    if (c.max_batch_queries > (1u << 31)) return fail(VBT_STATUS_INVALID_ARGUMENT, "max_batch_queries above 2^31");
    if (c.host_staging_bytes < 65536) c.host_staging_bytes = 65536;
    if (c.plain) c.slots = 1;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0)
        return fail(VBT_STATUS_CUDA, "no usable CUDA device for the VBT decode path");
    if (c.device < 0 || c.device >= n) return fail(VBT_STATUS_INVALID_ARGUMENT, "device index out of range");
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(c.device);
    auto* s = new vbt_server();
    s->cfg = c;
    cudaError_t e = cudaMalloc(&s->d_arena, c.hbm_budget_bytes);
    if (e == cudaSuccess) e = cudaMalloc(&s->d_assets, sizeof(DeviceAsset) * kMaxAssets);
    if (e == cudaSuccess) e = cudaHostAlloc(&s->h_stage, c.host_staging_bytes, cudaHostAllocDefault);
    if (e == cudaSuccess) e = cudaHostAlloc(&s->h_err, 8ull * kMaxSlots * kMaxUnitRequests, cudaHostAllocDefault);
    if (e == cudaSuccess) e = cudaMalloc(&s->d_counters, 8ull * kMaxSlots);
    for (uint32_t i = 0; e == cudaSuccess && i < c.slots; ++i) {
        e = cudaStreamCreateWithFlags(&s->streams[i], cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->events[i], cudaEventDisableTiming);
    }
    if (e != cudaSuccess) {
        const std::string msg = std::string("server allocation: ") + cudaGetErrorString(e);
        cudaGetLastError();
        for (uint32_t i = 0; i < c.slots; ++i) {
            if (s->streams[i]) cudaStreamDestroy(s->streams[i]);
            if (s->events[i]) cudaEventDestroy(s->events[i]);
        }
        cudaFree(s->d_arena);
        cudaFree(s->d_assets);
        cudaFree(s->d_counters);
        cudaFreeHost(s->h_stage);
        cudaFreeHost(s->h_err);
        delete s;
        cudaSetDevice(prev);
        return fail(VBT_STATUS_CUDA, msg);
    }
    s->arena.reset(c.hbm_budget_bytes);
    s->stage.reset(c.host_staging_bytes);
    s->worker = std::thread([s] { s->run(); });
    cudaSetDevice(prev);
    *out = s;
    return VBT_STATUS_OK;
}

int vbt_server_add_asset(vbt_server* s, vbt_asset* a, uint32_t* id)
{
    if (!s || !a || !id) return fail(VBT_STATUS_INVALID_ARGUMENT, "null argument");
    if (a->device != s->cfg.device) return fail(VBT_STATUS_INVALID_ARGUMENT, "asset is on another device");
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->assets.size() >= kMaxAssets) return fail(VBT_STATUS_LIMIT, "a server holds at most 64 assets");
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(s->cfg.device);
    const cudaError_t e =
        cudaMemcpy(s->d_assets + s->assets.size(), &a->dev, sizeof(DeviceAsset), cudaMemcpyHostToDevice);
    cudaSetDevice(prev);
    if (e != cudaSuccess) return fail(VBT_STATUS_CUDA, std::string("asset table: ") + cudaGetErrorString(e));
    *id = (uint32_t)s->assets.size();
    s->assets.push_back(a);
    s->resident_bytes += a->device_bytes;
    return VBT_STATUS_OK;
}

int vbt_serve_submit(vbt_server* s, const vbt_request* rq, uint64_t* ticket)
{
    if (!s || !rq || !ticket) return fail(VBT_STATUS_INVALID_ARGUMENT, "null argument");
    const vbt_asset* a = nullptr;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (rq->asset >= s->assets.size()) return fail(VBT_STATUS_INVALID_ARGUMENT, "unknown asset id");
        a = s->assets[rq->asset];
    }
    auto* r = new Req();
    r->r = *rq;
    int st = VBT_STATUS_OK;
    std::string msg;
    switch (rq->kind) {
    case VBT_REQ_POINTS:
        if (rq->n_points && !rq->points) st = VBT_STATUS_INVALID_ARGUMENT, msg = "null points";
        else if (rq->n_points >= (1ull << 31)) st = VBT_STATUS_LIMIT, msg = "more than 2^31 - 1 points in one request";
        break;
    case VBT_REQ_SLICE:
        if (rq->t1 < rq->t0 || rq->z >= a->hdr.depth)
            st = VBT_STATUS_INVALID_ARGUMENT, msg = "slice outside the volume or t1 < t0";
        break;
    case VBT_REQ_FRAMES:
        if (rq->n_frames && !rq->frames) {
            st = VBT_STATUS_INVALID_ARGUMENT, msg = "null frames";
        } else {
            r->frames.assign(rq->frames, rq->frames + rq->n_frames);
            r->r.frames = nullptr;
        }
        break;
    default: st = VBT_STATUS_INVALID_ARGUMENT, msg = "unknown request kind";
    }
    if (st == VBT_STATUS_OK) {
        r->result_floats = result_floats(r->r, a);
        const uint64_t np = rq->kind == VBT_REQ_POINTS ? rq->n_points : 0, nf = r->frames.size();
        const uint32_t kp = rq->kind == VBT_REQ_POINTS ? 1u : 0u;
        const uint64_t need = Arena::round(4ull * r->result_floats) +
                              Arena::round(std::max(points_in_bytes(1, np), mixed_in_bytes(kp, 1u - kp, nf, np)));
        const uint64_t staged = (rq->host_out && !is_pinned(rq->host_out) ? 4ull * r->result_floats : 0) +
                                (rq->kind == VBT_REQ_POINTS && !is_pinned(rq->points) ? 16ull * rq->n_points : 0) +
                                std::max(seg_bytes(1), mixed_table_bytes(kp, 1u - kp, nf));
        if (need > s->cfg.hbm_budget_bytes)
            st = VBT_STATUS_LIMIT, msg = "request needs more device memory than the server's budget";
        else if (Arena::round(staged) + kAlign > s->cfg.host_staging_bytes)
            st = VBT_STATUS_LIMIT, msg = "pageable host buffers larger than the server's pinned staging";
    }
    if (st != VBT_STATUS_OK) {
        delete r;
        return fail(st, msg);
    }
    {
        std::lock_guard<std::mutex> lk(s->mu);
        r->ticket = s->next_ticket++;
        r->t_submit = s->now_ms();
        s->tickets[r->ticket] = r;
        s->pending.push_back(r);
        *ticket = r->ticket;
    }
    s->cv_work.notify_one();
    return VBT_STATUS_OK;
}

int vbt_serve_poll(vbt_server* s, uint64_t ticket, int* done, vbt_request_result* res)
{
    if (!s || !done) return fail(VBT_STATUS_INVALID_ARGUMENT, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->tickets.find(ticket);
    if (it == s->tickets.end()) return fail(VBT_STATUS_INVALID_ARGUMENT, "unknown ticket");
    *done = it->second->state == 2;
    if (*done) fill_result(s, it->second, res);
    return VBT_STATUS_OK;
}

int vbt_serve_wait(vbt_server* s, uint64_t ticket, vbt_request_result* res)
{
    if (!s) return fail(VBT_STATUS_INVALID_ARGUMENT, "null argument");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->tickets.find(ticket);
    if (it == s->tickets.end()) return fail(VBT_STATUS_INVALID_ARGUMENT, "unknown ticket");
    Req* r = it->second;
    s->cv_done.wait(lk, [&] { return r->state == 2; });
    fill_result(s, r, res);
    return VBT_STATUS_OK;
}

int vbt_serve_release(vbt_server* s, uint64_t ticket)
{
    if (!s) return fail(VBT_STATUS_INVALID_ARGUMENT, "null argument");
    {
        std::lock_guard<std::mutex> lk(s->mu);
        auto it = s->tickets.find(ticket);
        if (it == s->tickets.end()) return fail(VBT_STATUS_INVALID_ARGUMENT, "unknown ticket");
        Req* r = it->second;
        if (r->state != 2) return fail(VBT_STATUS_INVALID_ARGUMENT, "request not done");
        if (r->dev_result.valid) s->to_free.push_back(r->dev_result);
        s->tickets.erase(it);
        delete r;
    }
    s->cv_work.notify_one();
    return VBT_STATUS_OK;
}

int vbt_server_get_stats(vbt_server* s, vbt_server_stats* o)
{
    if (!s || !o) return fail(VBT_STATUS_INVALID_ARGUMENT, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    *o = vbt_server_stats{};
    o->requests_done = s->requests_done;
    o->points_done = s->points_done;
    o->voxels_done = s->voxels_done;
    o->launches = s->launches;
    o->units = s->units;
    o->arena_peak_bytes = s->arena.peak();
    o->arena_bytes = s->arena.size();
    o->resident_asset_bytes = s->resident_bytes;
    o->busy_ms = s->busy_ms;
    if (!s->latencies.empty()) {
        std::vector<double> v = s->latencies;
        auto pct = [&](double p) {
            const size_t i = std::min(v.size() - 1, (size_t)(p * (double)(v.size() - 1) + 0.5));
            std::nth_element(v.begin(), v.begin() + (long)i, v.end());
            return v[i];
        };
        o->p50_ms = pct(0.50);
        o->p99_ms = pct(0.99);
        o->max_ms = *std::max_element(v.begin(), v.end());
    }
    return VBT_STATUS_OK;
}

int vbt_server_reset_stats(vbt_server* s)
{
    if (!s) return fail(VBT_STATUS_INVALID_ARGUMENT, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    s->latencies.clear();
    s->requests_done = s->points_done = s->voxels_done = s->launches = s->units = 0;
    s->busy_ms = 0;
    s->arena.clear_peak();
    return VBT_STATUS_OK;
}

int vbt_server_destroy(vbt_server* s)
{
    if (!s) return fail(VBT_STATUS_INVALID_ARGUMENT, "null argument");
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    s->worker.join();
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(s->cfg.device);
    for (uint32_t i = 0; i < s->cfg.slots; ++i) {
        cudaStreamSynchronize(s->streams[i]);
        release_mixed_graph(s->graphs[i]);
        cudaStreamDestroy(s->streams[i]);
        cudaEventDestroy(s->events[i]);
    }
    for (auto& kv : s->tickets) delete kv.second;
    cudaFree(s->d_arena);
    cudaFree(s->d_assets);
    cudaFree(s->d_counters);
    cudaFreeHost(s->h_stage);
    cudaFreeHost(s->h_err);
    cudaSetDevice(prev);
    delete s;
    return VBT_STATUS_OK;
}

}  // extern "C"
