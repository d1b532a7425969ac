// tune.cu -- the batched cache timeline: per-asset launch-shape autotuner and CUDA-graph replay
// (vbt_autotune_cache, vbt_set_tuning, vbt_get_tuning, vbt_decode_cache_timeline).
//
// A timeline is a page-table build followed by ceil(n / frames_per_launch) cache-decode launches.
// The autotuner times every candidate shape on the caller's own output buffer with CUDA events
// and keeps the fastest: leaf per CTA (the TMA-staged kernel; 16, 24, 32, 48, 64, 96 or 128
// frames per launch) or leaf per warp (8 leaves per CTA; 16, 32 or 64 frames, one or two waves).  All shapes
// write identical values.
#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <vector>

#include "asset.h"
#include "kernels.cuh"

namespace vbtb {
int set_last_error(int status, const std::string& msg);

void release_timeline_graphs(vbt_asset* a)
{
    std::lock_guard<std::mutex> lk(a->graph_mu);
    for (auto& kv : a->graphs) cudaGraphExecDestroy(kv.second);
    a->graphs.clear();
}
}  // namespace vbtb

using namespace vbtb;

namespace {

struct Guard {
    int prev = -1;
    explicit Guard(int dev)
    {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~Guard()
    {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

int cuda_fail(cudaError_t e, const char* what)
{
    return set_last_error(VBT_STATUS_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// Enqueue one timeline with tuning `t` on stream `s` (no synchronisation).
void enqueue_timeline(vbt_asset* a, const vbt_tuning& t, int t0, int n, float* out, uint64_t stride, cudaStream_t s)
{
    launch_page_table(a->dev, ++a->epoch, s);
    int fr[kMaxLaunchFrames];
    const int fpl = (int)std::max<uint32_t>(1u, std::min<uint32_t>((uint32_t)kMaxLaunchFrames, t.frames_per_launch));
    for (int i = 0; i < n; i += fpl) {
        const int m = std::min(fpl, n - i);
        for (int j = 0; j < m; ++j) fr[j] = t0 + i + j;
        if (t.variant == 1u)
            launch_decode_cache_warp(a->dev, fr, m, out + (uint64_t)i * stride, stride, t.grid, s);
        else
            launch_decode_cache(a->dev, a->launch_seq.fetch_add(1), fr, m, out + (uint64_t)i * stride, stride, t.grid,
                                s);
    }
}

// Mean milliseconds of one timeline (one warm-up, then `reps` timed runs).
float time_timeline(vbt_asset* a, const vbt_tuning& t, int n, float* out, uint64_t stride, cudaStream_t s, int reps)
{
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    enqueue_timeline(a, t, 0, n, out, stride, s);
    cudaEventRecord(e0, s);
    for (int r = 0; r < reps; ++r) enqueue_timeline(a, t, 0, n, out, stride, s);
    cudaEventRecord(e1, s);
    cudaEventSynchronize(e1);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return ms / (float)reps;
}

}  // namespace

extern "C" {

int vbt_autotune_cache(vbt_asset* a, int nframes, float* d_out, uint64_t stride, vbt_tuning* out, void* stream)
{
    if (!a || !d_out) return set_last_error(VBT_STATUS_INVALID_ARGUMENT, "null argument");
    if (nframes <= 0) return set_last_error(VBT_STATUS_INVALID_ARGUMENT, "nframes must be positive");
    Guard guard(a->device);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int wave = decode_warp_grid();
    std::vector<vbt_tuning> cands;
    for (uint32_t f : {16u, 24u, 32u, 48u, 64u, 96u, 128u}) cands.push_back(vbt_tuning{0u, f, 0, 0.f, 0.f});
    for (uint32_t f : {16u, 32u, 64u})
        for (int g : {0, 2 * wave}) cands.push_back(vbt_tuning{1u, f, g, 0.f, 0.f});
    // two rounds over the candidates, four timed timelines each, and per candidate the faster
    // round: a shape is not picked or dropped on one noisy measurement (clock ramp, a neighbour)
    std::vector<float> cand_ms(cands.size(), 0.0f);
    for (int round = 0; round < 2; ++round)
        for (size_t i = 0; i < cands.size(); ++i) {
            const float ms = time_timeline(a, cands[i], nframes, d_out, stride, s, 4);
            const cudaError_t e = cudaGetLastError();
            if (e != cudaSuccess) return cuda_fail(e, "autotune launch");
            if (round == 0 || ms < cand_ms[i]) cand_ms[i] = ms;
        }
    vbt_tuning best{0u, 48u, 0, 0.f, 0.f};
    float best_ms = 0.0f, default_ms = 0.0f;
    for (size_t i = 0; i < cands.size(); ++i) {
        const vbt_tuning& c = cands[i];
        const float ms = cand_ms[i];
        if (c.variant == 0u && c.frames_per_launch == 48u && c.grid == 0) default_ms = ms;
        if (best_ms == 0.0f || ms < best_ms) {
            best_ms = ms;
            best = c;
        }
    }
    best.ms_per_frame = best_ms / (float)nframes;
    best.ms_per_frame_default = default_ms / (float)nframes;
    vbtb::release_timeline_graphs(a);
    a->tuning = best;
    if (out) *out = best;
    return VBT_STATUS_OK;
}

int vbt_set_tuning(vbt_asset* a, const vbt_tuning* t)
{
    if (!a || !t) return set_last_error(VBT_STATUS_INVALID_ARGUMENT, "null argument");
    if (t->variant > 1u || t->frames_per_launch == 0u || t->frames_per_launch > (uint32_t)kMaxLaunchFrames || t->grid < 0)
        return set_last_error(VBT_STATUS_INVALID_ARGUMENT, "tuning out of range");
    Guard guard(a->device);
    vbtb::release_timeline_graphs(a);
    a->tuning = *t;
    return VBT_STATUS_OK;
}

int vbt_get_tuning(vbt_asset* a, vbt_tuning* out)
{
    if (!a || !out) return set_last_error(VBT_STATUS_INVALID_ARGUMENT, "null argument");
    *out = a->tuning;
    return VBT_STATUS_OK;
}

int vbt_decode_cache_timeline(vbt_asset* a, int t0, int n, float* d_out, uint64_t stride, int use_graph, void* stream)
{
    if (!a || !d_out) return set_last_error(VBT_STATUS_INVALID_ARGUMENT, "null argument");
    if (n <= 0) return set_last_error(VBT_STATUS_INVALID_ARGUMENT, "n must be positive");
    if ((reinterpret_cast<uintptr_t>(d_out) & 15u) != 0u || (stride & 3u) != 0u)
        return set_last_error(VBT_STATUS_INVALID_ARGUMENT, "cache output must be 16-byte aligned, stride a multiple of 4");
    Guard guard(a->device);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (!use_graph) {
        enqueue_timeline(a, a->tuning, t0, n, d_out, stride, s);
        const cudaError_t e = cudaGetLastError();
        return e == cudaSuccess ? VBT_STATUS_OK : cuda_fail(e, "timeline launch");
    }
    if (s == nullptr)
        return set_last_error(VBT_STATUS_INVALID_ARGUMENT, "graph replay needs a non-default stream (capture)");
    std::lock_guard<std::mutex> lk(a->graph_mu);
    const auto key = std::make_tuple(t0, n, reinterpret_cast<uintptr_t>(d_out), stride);
    auto it = a->graphs.find(key);
    if (it == a->graphs.end()) {
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed);
        if (e != cudaSuccess) return cuda_fail(e, "cudaStreamBeginCapture");
        enqueue_timeline(a, a->tuning, t0, n, d_out, stride, s);
        e = cudaStreamEndCapture(s, &g);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return cuda_fail(e, "timeline capture");
        }
        cudaGraphExec_t x = nullptr;
        e = cudaGraphInstantiate(&x, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGraphInstantiate");
        it = a->graphs.emplace(key, x).first;
    }
    const cudaError_t e = cudaGraphLaunch(it->second, s);
    return e == cudaSuccess ? VBT_STATUS_OK : cuda_fail(e, "cudaGraphLaunch");
}

}  // extern "C"
