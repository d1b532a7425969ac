// facade_test.cpp -- GPU checks of how the C++ decoder API (include/vbt/*.h) keeps its device
// copies of VbtFile objects, and the per-call latency of its scalar calls.
//
// Built and run by tests/test_cpp_api.py on a CUDA device.
//  - lifetime: 1,000 VbtFile objects loaded, decoded and destroyed without releaseDeviceCopy (as
//    the reference's own callers do) leave at most the cache's bound of copies and no growth of
//    used device memory;
//  - contents: a payload changed in place, and a different file loaded into the same VbtFile
//    object, decode their current bytes (compared with a fresh object holding the same bytes);
//  - latency: microseconds per call of decodeRenderTemporalLeafControlValue and of
//    decodeScientificValueAtCpu, printed as "LATENCY <name> <us>".
// usage: facade_test <render asset> <scientific asset>
#include <cuda_runtime.h>

#include <chrono>
#include <cstring>
#include <functional>
#include <iostream>
#include <string>
#include <vector>

#include "check.h"
#include "vbt/query_patterns.h"
#include "vbt/render_temporal_decode.h"
#include "vbt/render_temporal_payload.h"
#include "vbt/scientific_decode.h"
#include "vbt/vbt_file.h"

using namespace check;
using namespace vbt;
using namespace vbt::render;

namespace {

VbtFile load(const std::string& path)
{
    VbtFile f;
    std::string err;
    require(loadVbtFile(path, f, err), "load " + path + ": " + err);
    return f;
}

size_t used_device_bytes()
{
    size_t free_b = 0, total_b = 0;
    require(cudaMemGetInfo(&free_b, &total_b) == cudaSuccess, "cudaMemGetInfo");
    return total_b - free_b;
}

std::vector<Query4D> queries(const VbtFile& f, int n, uint32_t seed)
{
    Rng rng(seed);
    std::vector<Query4D> q(n);
    for (auto& x : q) {
        x.x = rng.below(f.header.width);
        x.y = rng.below(f.header.height);
        x.z = rng.below(f.header.depth);
        x.t = rng.below(f.header.frames);
        x.leafIndex = leafIndexForVoxel(f.header, x.x, x.y, x.z);
    }
    return q;
}

bool same(const std::vector<float>& a, const std::vector<float>& b)
{
    return a.size() == b.size() && std::memcmp(a.data(), b.data(), 4 * a.size()) == 0;
}

void lifetime_test(const std::string& path)
{
    const VbtFile proto = load(path);
    const auto q = queries(proto, 64, 5);
    const auto want = decodeValuesGpu(proto, q);
    releaseDeviceCopy(proto);
    size_t base = 0;
    for (int i = 0; i < 1000; ++i) {
        auto* f = new VbtFile(proto);
        require(same(decodeValuesGpu(*f, q), want), "values of a copied file");
        delete f;   // no releaseDeviceCopy, as the reference's callers
        require(deviceCopyCount() <= 8, "device copies beyond the bound");
        if (i == 20) base = used_device_bytes();
    }
    const size_t end = used_device_bytes();
    require(end <= base + (16u << 20), "device memory grew by " + std::to_string((end - base) >> 20) + " MiB");
    std::cout << "lifetime: 1000 files, " << deviceCopyCount() << " copies kept, device memory "
              << (base >> 20) << " -> " << (end >> 20) << " MiB\n";
}

void contents_test(const std::string& sci_path, const std::string& render_path)
{
    // a payload changed in place: every leaf's first payload word after its header (a coarse DC
    // value for scientific leaves) is changed
    VbtFile f = load(sci_path);
    const auto q = queries(f, 512, 9);
    const auto before = decodeValuesGpu(f, q);
    const auto frame_before = reconstructScientificFrameCpu(f, 1);
    for (uint32_t l = 0; l < f.header.leafCount; ++l) {
        const uint32_t w = f.offsetsWords[l] + 1;
        if (w < f.offsetsWords[l + 1]) f.payloadWords[w] ^= 0x00001C00u;   // a different fp16 DC
    }
    const VbtFile fresh = f;   // another object with the same bytes: decoded from its own copy
    const auto after = decodeValuesGpu(f, q);
    require(same(after, decodeValuesGpu(fresh, q)), "in-place change: point values are not the current bytes'");
    require(!same(after, before), "in-place change: point values did not change");
    const auto frame_after = reconstructScientificFrameCpu(f, 1);
    require(same(frame_after, reconstructScientificFrameCpu(fresh, 1)), "in-place change: frame is stale");
    require(!same(frame_after, frame_before), "in-place change: frame did not change");
    // a different file loaded into the same object (its vectors may keep their addresses)
    VbtFile g = load(sci_path);
    (void)decodeValuesGpu(g, queries(g, 16, 1));
    std::string err;
    require(loadVbtFile(render_path, g, err), err);
    const VbtFile r = load(render_path);
    const auto rq = queries(r, 256, 3);
    require(same(decodeValuesGpu(g, rq), decodeValuesGpu(r, rq)), "reloaded object decodes the old file");
    require(same(decodeRenderTemporalFrame(g, 2), decodeRenderTemporalFrame(r, 2)), "reloaded object: stale frame");
    std::cout << "contents: in-place change and reload decode the current bytes\n";
}

double us_per_call(int n, const std::function<void()>& fn)
{
    fn();   // warm: copies and staging made
    const auto t0 = std::chrono::steady_clock::now();
    for (int i = 0; i < n; ++i) fn();
    const auto t1 = std::chrono::steady_clock::now();
    return std::chrono::duration<double, std::micro>(t1 - t0).count() / n;
}

void latency_test(const std::string& render_path, const std::string& sci_path)
{
    const VbtFile r = load(render_path);
    // the first non-EMPTY leaf's coarse stream
    uint32_t leaf = 0;
    while (leaf < r.header.leafCount && (r.payloadWords[r.offsetsWords[leaf]] & 3u) == 0u) ++leaf;
    require(leaf < r.header.leafCount, "no active leaf");
    const auto* base = reinterpret_cast<const uint8_t*>(r.payloadWords.data() + r.offsetsWords[leaf]);
    const size_t bytes = 4ull * (r.offsetsWords[leaf + 1] - r.offsetsWords[leaf]);
    const auto view = parseRenderTemporalPackedLeaf(base, bytes, true);
    int k = 0;
    volatile float sink = 0.0f;
    const double ctrl = us_per_call(2000, [&] {
        sink = decodeRenderTemporalLeafControlValue(base, view.header, view.prefix, view.layout, false, true,
                                                    int(r.header.frames), uint16_t(k % 64), k % int(r.header.frames));
        ++k;
    });
    const VbtFile s = load(sci_path);
    const auto q = queries(s, 2000, 4);
    size_t i = 0;
    const double sci = us_per_call(2000, [&] { sink = decodeScientificValueAtCpu(s, q[i++ % q.size()]); });
    (void)sink;
    std::cout << "LATENCY decodeRenderTemporalLeafControlValue " << ctrl << "\n";
    std::cout << "LATENCY decodeScientificValueAtCpu " << sci << "\n";
}

}  // namespace

int main(int argc, char** argv)
{
    if (argc < 3) {
        std::cerr << "usage: facade_test <render asset> <scientific asset>\n";
        return 2;
    }
    try {
        lifetime_test(argv[2]);
        contents_test(argv[2], argv[1]);
        latency_test(argv[1], argv[2]);
        std::cout << "facade_test: PASS\n";
    } catch (const std::exception& e) {
        std::cerr << "facade_test: FAIL: " << e.what() << "\n";
        return 1;
    }
    return 0;
}
