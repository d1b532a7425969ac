// ref_shim.cpp -- C-ABI shim over the reference VBT decoder, compiled from the reference's own
// sources by oracle/Makefile into oracle/_ref/libvbtref.so.
//
// TEST INFRASTRUCTURE ONLY: it pins the C restatement (vbt_oracle.c) to the reference and
// serves as the "reference" CPU baseline in bench.py.  It calls only the reference's public API
// (render_temporal_decode.h, render_temporal_payload.h, vbt_file.h, scientific_decode.h).  The
// full-frame composition lives in a Vulkan translation unit of the reference
// (render/src/render_smoke_vbt_bench_main.cpp:201-452, anonymous namespace), so it is restated
// here over the same public calls, in the same order.
#include "dct_codec.h"
#include "render_temporal_decode.h"
#include "render_temporal_payload.h"
#include "scientific_decode.h"
#include "vbt_file.h"

#include <algorithm>
#include <array>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

using namespace vbt;
using vbt::render::VbtFile;

namespace {

thread_local std::string g_err;

int fail(const std::exception& e)
{
    g_err = e.what();
    return 1;
}

std::vector<float> controlCoords(int resolution)
{
    std::vector<float> coords(static_cast<size_t>(resolution), 0.0f);
    if (resolution <= 1) return coords;
    const float scale = 7.0f / static_cast<float>(resolution - 1);
    for (int i = 0; i < resolution; ++i) coords[static_cast<size_t>(i)] = static_cast<float>(i) * scale;
    return coords;
}

// render/src/render_smoke_vbt_bench_main.cpp:212-219 coordsForResolution caches the coordinates per
// resolution; here they are built once for every 3-bit resolution (thread-safe static init).
const std::vector<float>& coordsForResolution(int resolution)
{
    static const std::array<std::vector<float>, 8> cache = [] {
        std::array<std::vector<float>, 8> c;
        for (int r = 0; r < 8; ++r) c[size_t(r)] = controlCoords(r);
        return c;
    }();
    return cache[size_t(resolution & 7)];
}

// render/src/render_smoke_vbt_bench_main.cpp:221-234 locateCoord
std::array<float, 3> locateCoord(float p, int extent, int resolution)
{
    const auto& coords = coordsForResolution(resolution);
    const float maxP = static_cast<float>(std::max(0, extent - 1));
    p = std::clamp(p, 0.0f, maxP);
    int i1 = 1;
    while (i1 < resolution - 1 && coords[static_cast<size_t>(i1)] < p) ++i1;
    const int i0 = std::max(0, i1 - 1);
    const float c0 = coords[static_cast<size_t>(i0)];
    const float c1 = coords[static_cast<size_t>(i1)];
    const float w = (c1 > c0) ? ((p - c0) / (c1 - c0)) : 0.0f;
    return {static_cast<float>(i0), static_cast<float>(i1), w};
}

// render/src/render_smoke_vbt_bench_main.cpp:236-267 sampleControlGrid
float sampleControlGrid(const std::vector<float>& grid, int resolution, int w, int h, int d, float fx, float fy,
                        float fz)
{
    const auto lx = locateCoord(fx, w, resolution);
    const auto ly = locateCoord(fy, h, resolution);
    const auto lz = locateCoord(fz, d, resolution);
    auto at = [&](int ix, int iy, int iz) { return grid[static_cast<size_t>((iz * resolution + iy) * resolution + ix)]; };
    const int x0 = static_cast<int>(lx[0]), x1 = static_cast<int>(lx[1]);
    const int y0 = static_cast<int>(ly[0]), y1 = static_cast<int>(ly[1]);
    const int z0 = static_cast<int>(lz[0]), z1 = static_cast<int>(lz[1]);
    const float tx = lx[2], ty = ly[2], tz = lz[2];
    const float c00 = at(x0, y0, z0) * (1.0f - tx) + at(x1, y0, z0) * tx;
    const float c01 = at(x0, y0, z1) * (1.0f - tx) + at(x1, y0, z1) * tx;
    const float c10 = at(x0, y1, z0) * (1.0f - tx) + at(x1, y1, z0) * tx;
    const float c11 = at(x0, y1, z1) * (1.0f - tx) + at(x1, y1, z1) * tx;
    const float c0 = c00 * (1.0f - ty) + c10 * ty;
    const float c1 = c01 * (1.0f - ty) + c11 * ty;
    return c0 * (1.0f - tz) + c1 * tz;
}

// render/src/render_smoke_vbt_bench_main.cpp:277-387 decodeLeafFrameValues
void decodeLeafFrameValues(const uint8_t* leafBase, size_t leafBytes, int frames, int frameIndex, int w, int h,
                           int d, std::vector<float>& outLeaf)
{
    const auto leafView = parseRenderTemporalPackedLeaf(leafBase, leafBytes, true);
    if (leafView.header.mode == TemporalFirstPackedMode::EMPTY) {
        std::fill(outLeaf.begin(), outLeaf.end(), 0.0f);
        return;
    }
    const int cres = leafView.header.coarseResolution, fres = leafView.header.fineResolution;
    const uint16_t cc = static_cast<uint16_t>(cres * cres * cres);
    std::vector<float> coarseGrid(cc, 0.0f);
    for (uint16_t i = 0; i < cc; ++i)
        coarseGrid[i] = decodeRenderTemporalLeafControlValue(leafBase, leafView.header, leafView.prefix, leafView.layout,
                                                             false, true, frames, i, frameIndex);
    std::vector<float> fineGrid;
    const bool hasFine = fres > 0 && leafView.layout.fine.totalBytes > 0 &&
                         leafView.header.mode != TemporalFirstPackedMode::TEMPORAL_GRID4;
    if (hasFine) {
        const uint16_t fc = static_cast<uint16_t>(fres * fres * fres);
        fineGrid.resize(fc, 0.0f);
        for (uint16_t i = 0; i < fc; ++i)
            fineGrid[i] = decodeRenderTemporalLeafControlValue(leafBase, leafView.header, leafView.prefix,
                                                               leafView.layout, true, true, frames, i, frameIndex);
    }
    RenderTemporalShellOccupancySection occ{};
    const bool hasOcc = leafView.header.mode == TemporalFirstPackedMode::TEMPORAL_FINE_COMPACT;
    if (hasOcc)
        occ = unpackRenderTemporalShellOccupancySection(leafBase + leafView.layout.fine.descriptorOffset,
                                                        leafView.layout.fine.descriptorBytes);
    for (int lz = 0; lz < d; ++lz)
        for (int ly = 0; ly < h; ++ly)
            for (int lx = 0; lx < w; ++lx) {
                const uint16_t vi = renderTemporalLeafVoxelIndex(lx, ly, lz, 8);
                float value = sampleControlGrid(coarseGrid, cres, w, h, d, float(lx), float(ly), float(lz));
                if (!fineGrid.empty()) {
                    value += sampleControlGrid(fineGrid, fres, w, h, d, float(lx), float(ly), float(lz));
                } else if (leafView.header.mode == TemporalFirstPackedMode::TEMPORAL_FINE_COMPACT) {
                    value += decodeRenderTemporalLeafShellVoxelValue(leafBase, leafView, true, frames, vi, frameIndex);
                }
                if (hasOcc && ((occ.shellMask[vi >> 6u] >> (vi & 63u)) & 1ull) == 0ull && value < 0.0f) value = 0.0f;
                outLeaf[static_cast<size_t>((lz * h + ly) * w + lx)] = value;
            }
}

struct Handle {
    VbtFile file;
};

} // namespace

extern "C" {

const char* vr_last_error() { return g_err.c_str(); }

void* vr_load(const char* path, char* err, size_t errLen)
{
    auto* h = new Handle();
    std::string e;
    if (!vbt::render::loadVbtFile(path, h->file, e)) {
        if (err && errLen) std::snprintf(err, errLen, "%s", e.c_str());
        delete h;
        return nullptr;
    }
    return h;
}

void vr_free(void* h) { delete static_cast<Handle*>(h); }

// render/src/render_smoke_vbt_bench_main.cpp:389-452 decodeFrameToDense, OpenMP over leaves.
int vr_decode_frame(void* hp, int frame, float* out, int threads)
{
    const VbtFile& file = static_cast<Handle*>(hp)->file;
    const int lcx = (int(file.header.width) + 7) / 8, lcy = (int(file.header.height) + 7) / 8,
              lcz = (int(file.header.depth) + 7) / 8;
    const uint8_t* payload = reinterpret_cast<const uint8_t*>(file.payloadWords.data());
    int failed = 0;
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 16)
#endif
    for (int64_t li = 0; li < int64_t(lcx) * lcy * lcz; ++li) {
        const int bx = int(li % lcx), by = int((li / lcx) % lcy), bz = int(li / (int64_t(lcx) * lcy));
        const uint32_t wb = file.offsetsWords[li], we = file.offsetsWords[li + 1];
        const int w = std::min(8, int(file.header.width) - bx * 8), h = std::min(8, int(file.header.height) - by * 8),
                  d = std::min(8, int(file.header.depth) - bz * 8);
        std::vector<float> vals(size_t(w) * h * d, 0.0f);
        try {
            decodeLeafFrameValues(payload + size_t(wb) * 4, size_t(we - wb) * 4, int(file.header.frames), frame, w, h,
                                  d, vals);
        } catch (const std::exception& e) {
#ifdef _OPENMP
#pragma omp critical
#endif
            {
                g_err = e.what();
                failed = 1;
            }
            continue;
        }
        for (int lz = 0; lz < d; ++lz)
            for (int ly = 0; ly < h; ++ly)
                std::memcpy(out + (size_t(bz * 8 + lz) * file.header.height + size_t(by * 8 + ly)) * file.header.width + bx * 8,
                            vals.data() + size_t(lz * h + ly) * w, sizeof(float) * size_t(w));
    }
    return failed;
}

// Current-frame cache over the same composition: only non-EMPTY leaves (route tag != 0) are
// decoded, into cache[rank * 512 + (lz*8 + ly)*8 + lx] with rank the ascending active rank.
int vr_decode_cache(void* hp, int frame, float* cache, int threads)
{
    const VbtFile& file = static_cast<Handle*>(hp)->file;
    const int lcx = (int(file.header.width) + 7) / 8, lcy = (int(file.header.height) + 7) / 8,
              lcz = (int(file.header.depth) + 7) / 8;
    const uint8_t* payload = reinterpret_cast<const uint8_t*>(file.payloadWords.data());
    const int64_t L = int64_t(lcx) * lcy * lcz;
    std::vector<uint32_t> rank(size_t(L), 0xFFFFFFFFu);
    uint32_t n = 0;
    for (int64_t li = 0; li < L; ++li)
        if ((file.payloadWords[file.offsetsWords[li]] & 3u) != 0u) rank[li] = n++;
    int failed = 0;
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 4)
#endif
    for (int64_t li = 0; li < L; ++li) {
        if (rank[li] == 0xFFFFFFFFu) continue;
        const int bx = int(li % lcx), by = int((li / lcx) % lcy), bz = int(li / (int64_t(lcx) * lcy));
        const uint32_t wb = file.offsetsWords[li], we = file.offsetsWords[li + 1];
        const int w = std::min(8, int(file.header.width) - bx * 8), h = std::min(8, int(file.header.height) - by * 8),
                  d = std::min(8, int(file.header.depth) - bz * 8);
        std::vector<float> vals(size_t(w) * h * d, 0.0f);
        try {
            decodeLeafFrameValues(payload + size_t(wb) * 4, size_t(we - wb) * 4, int(file.header.frames), frame, w, h,
                                  d, vals);
        } catch (const std::exception& e) {
            failed = 1;
            continue;
        }
        float* dst = cache + size_t(rank[li]) * 512u;
        for (int lz = 0; lz < d; ++lz)
            for (int ly = 0; ly < h; ++ly)
                for (int lx = 0; lx < w; ++lx) dst[(lz * 8 + ly) * 8 + lx] = vals[size_t(lz * h + ly) * w + lx];
    }
    return failed;
}

// render/src/scientific_decode.cpp:361-409, called as is.
int vr_sci_frame(void* hp, uint32_t frame, float* out)
{
    try {
        const auto v = vbt::render::reconstructScientificFrameCpu(static_cast<Handle*>(hp)->file, frame);
        std::memcpy(out, v.data(), v.size() * sizeof(float));
        return 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

// render/src/scientific_decode.cpp:335-359, called as is; leaf indices as render/src/query_patterns.cpp
// fillLeafIndices fills them.  q holds (x,y,z,t) quadruples.
int vr_sci_query(void* hp, const uint32_t* q, uint64_t n, float* out, int threads)
{
    const VbtFile& file = static_cast<Handle*>(hp)->file;
    int failed = 0;
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(static)
#endif
    for (int64_t i = 0; i < int64_t(n); ++i) {
        vbt::render::Query4D qq{q[4 * i], q[4 * i + 1], q[4 * i + 2], q[4 * i + 3], 0};
        qq.leafIndex = vbt::render::leafIndexForVoxel(file.header, qq.x, qq.y, qq.z);
        try {
            out[i] = vbt::render::decodeScientificValueAtCpu(file, qq);
        } catch (const std::exception& e) {
            failed = 1;
        }
    }
    return failed;
}

int vr_decode_control(const uint8_t* stream, uint32_t codec, uint32_t cc, uint32_t bins, uint32_t kf,
                      uint32_t streamBytes, int align, int total, uint32_t ci, int frame, float* out)
{
    try {
        *out = decodeRenderTemporalControlValue(stream, RenderTemporalSequenceCodec(codec), uint16_t(cc), uint8_t(bins),
                                                0, kf, streamBytes, align != 0, total, uint16_t(ci), frame);
        return 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

// Parse a leaf; fills out[0..15] with the view's integers (header fields, counts, layout, shell).
int vr_parse_leaf(const uint8_t* leaf, size_t bytes, uint32_t* out)
{
    try {
        const auto v = parseRenderTemporalPackedLeaf(leaf, bytes, true);
        const uint32_t vals[16] = {uint32_t(v.header.mode), uint32_t(v.header.coarseCodec), uint32_t(v.header.fineCodec),
                                   v.header.coarseResolution, v.header.fineResolution, v.prefix.coarseKeyframeCount,
                                   v.prefix.fineKeyframeCount, v.layout.coarseOffset, v.layout.coarse.totalBytes,
                                   v.layout.fineOffset, v.layout.fine.totalBytes, v.layout.totalBytes,
                                   v.shellActiveVoxelCount, v.shellResidualOffset, v.shellResidualBytes, 0u};
        std::memcpy(out, vals, sizeof vals);
        return 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

int vr_shell_voxel(const uint8_t* leaf, size_t bytes, int total, uint32_t voxel, int frame, float* out)
{
    try {
        const auto v = parseRenderTemporalPackedLeaf(leaf, bytes, true);
        *out = decodeRenderTemporalLeafShellVoxelValue(leaf, v, true, total, uint16_t(voxel), frame);
        return 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

int vr_decode_leaf(const uint8_t* leaf, size_t bytes, int total, int frame, int w, int h, int d, float* out)
{
    try {
        std::vector<float> vals(size_t(w) * h * d, 0.0f);
        decodeLeafFrameValues(leaf, bytes, total, frame, w, h, d, vals);
        std::memcpy(out, vals.data(), vals.size() * sizeof(float));
        return 0;
    } catch (const std::exception& e) {
        return fail(e);
    }
}

uint16_t vr_float_to_half(float v) { return renderTemporalFloatToHalfBits(v); }
float vr_half_to_float(uint16_t b) { return renderTemporalHalfBitsToFloat(b); }

// packRenderTemporalControlStream (src/render_temporal_decode.cpp:225-268) over flat arrays.
// desc: controlCount x (keyStart, keyCount, reserved); keys: (frame, value) pairs.
// Returns the byte count written to out (or -1 with vr_last_error()).
long vr_pack_stream(uint32_t codec, uint32_t cc, uint32_t bins, uint32_t maxLocal, const uint32_t* desc,
                    const uint8_t* binIndex, const uint32_t* keyFrames, const float* keyValues, uint32_t nkeys,
                    int align, uint8_t* out, size_t outCap)
{
    try {
        RenderTemporalControlStreamData s;
        s.codec = RenderTemporalSequenceCodec(codec);
        s.controlCount = uint16_t(cc);
        s.timeBinCount = uint8_t(bins);
        s.maxBinLocalKeys = uint8_t(maxLocal);
        for (uint32_t c = 0; c < cc; ++c)
            s.descriptors.push_back({uint16_t(desc[3 * c]), uint8_t(desc[3 * c + 1]), uint8_t(desc[3 * c + 2])});
        s.binIndex.assign(binIndex, binIndex + size_t(cc) * bins);
        for (uint32_t k = 0; k < nkeys; ++k) s.keyframes.push_back({uint16_t(keyFrames[k]), keyValues[k]});
        const auto bytes = packRenderTemporalControlStream(s, align != 0);
        if (bytes.size() > outCap) throw std::runtime_error("output buffer too small");
        std::memcpy(out, bytes.data(), bytes.size());
        return long(bytes.size());
    } catch (const std::exception& e) {
        fail(e);
        return -1;
    }
}

// buildRenderTemporalPackedLeafBytes, both overloads (src/render_temporal_payload.cpp:199-232, :348-386).
// occ == nullptr selects the 5-argument overload.
long vr_build_leaf(uint32_t packedHeader, uint32_t coarseKf, uint32_t fineKf, const uint8_t* coarse, size_t coarseLen,
                   const uint8_t* fine, size_t fineLen, const uint8_t* occ, size_t occLen, int align, uint8_t* out,
                   size_t outCap)
{
    try {
        const auto header = unpackRenderTemporalHeader(packedHeader);
        const auto prefix = makeRenderTemporalLeafPrefix(header.mode, coarseKf, fineKf);
        std::vector<uint8_t> c(coarse, coarse + coarseLen), f(fine, fine + fineLen);
        std::vector<uint8_t> bytes;
        if (occ) {
            std::vector<uint8_t> o(occ, occ + occLen);
            bytes = buildRenderTemporalPackedLeafBytes(header, prefix, c, o, f, align != 0);
        } else {
            bytes = buildRenderTemporalPackedLeafBytes(header, prefix, c, f, align != 0);
        }
        if (bytes.size() > outCap) throw std::runtime_error("output buffer too small");
        std::memcpy(out, bytes.data(), bytes.size());
        return long(bytes.size());
    } catch (const std::exception& e) {
        fail(e);
        return -1;
    }
}

// The encoder's leaf packing and payload assembly over many leaves, from the stream arrays that
// vbt_pack_leaves reads (32-byte records: header word, prefix counts, first control row / keyframe
// of the coarse and fine streams, occupancy row, maxBinLocalKeys of both streams): per leaf the
// reference's packRenderTemporalControlStream and buildRenderTemporalPackedLeafBytes on OpenMP
// threads, then the offsets and padded payload as writeRenderTemporalProbeFile concatenates them
// (src/render_temporal_kf_probe_main.cpp:2561-2585).  Returns the payload words, or -1.
long vr_pack_leaves(const uint8_t* records, uint32_t n, const uint32_t* desc, const uint8_t* bins,
                    const uint16_t* keyFrames, const float* keyValues, const uint8_t* occupancy, uint32_t* offsets,
                    uint32_t* payload, size_t capWords, int threads)
{
    struct Rec {
        uint32_t header;
        uint16_t ckf, fkf;
        uint32_t cc, ck, fc, fk, occ;
        uint8_t cml, fml, pad[2];
    };
    static_assert(sizeof(Rec) == 32, "record layout");
    std::vector<std::vector<uint8_t>> leaves(n);
    bool failed = false;
    auto stream = [&](uint32_t codec, uint32_t controls, uint32_t nb, uint32_t maxLocal, uint32_t firstControl,
                      uint32_t firstKey, uint32_t keys) {
        RenderTemporalControlStreamData s;
        s.codec = RenderTemporalSequenceCodec(codec);
        s.controlCount = uint16_t(controls);
        s.timeBinCount = uint8_t(nb);
        s.maxBinLocalKeys = uint8_t(maxLocal);
        for (uint32_t c = 0; c < controls; ++c) {
            const uint32_t d = desc[firstControl + c];
            s.descriptors.push_back({uint16_t(d & 0xFFFFu), uint8_t((d >> 16) & 0xFFu), uint8_t(d >> 24)});
            for (uint32_t b = 0; b < nb; ++b) s.binIndex.push_back(bins[size_t(firstControl + c) * 8u + b]);
        }
        for (uint32_t k = 0; k < keys; ++k) s.keyframes.push_back({keyFrames[firstKey + k], keyValues[firstKey + k]});
        return packRenderTemporalControlStream(s, true);
    };
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 64)
#endif
    for (long long i = 0; i < (long long)n; ++i) {
        try {
            Rec r;
            std::memcpy(&r, records + size_t(i) * 32u, 32);
            const auto header = unpackRenderTemporalHeader(r.header);
            if (header.mode == TemporalFirstPackedMode::EMPTY) {
                leaves[i] = buildRenderTemporalPackedLeafBytes(header, {}, {}, {}, true);
                continue;
            }
            const auto prefix = makeRenderTemporalLeafPrefix(header.mode, r.ckf, r.fkf);
            const uint32_t cres = header.coarseResolution, fres = header.fineResolution;
            const auto coarse = stream(uint32_t(header.coarseCodec), cres * cres * cres, 8, r.cml, r.cc, r.ck, r.ckf);
            if (header.mode == TemporalFirstPackedMode::TEMPORAL_FINE6) {
                const auto fine = stream(uint32_t(header.fineCodec), fres * fres * fres, 8, r.fml, r.fc, r.fk, r.fkf);
                leaves[i] = buildRenderTemporalPackedLeafBytes(header, prefix, coarse, fine, true);
            } else if (header.mode == TemporalFirstPackedMode::TEMPORAL_FINE_COMPACT) {
                const std::vector<uint8_t> occ(occupancy + size_t(r.occ) * 80u, occupancy + size_t(r.occ) * 80u + 80u);
                const auto section = unpackRenderTemporalShellOccupancySection(occ.data(), occ.size());
                const uint32_t active = renderTemporalShellActiveVoxelCount(section);
                const auto residual = stream(uint32_t(header.fineCodec), active, kRenderTemporalShellPackedTimeBinCount,
                                             r.fml, r.fc, r.fk, r.fkf);
                leaves[i] = buildRenderTemporalPackedLeafBytes(header, prefix, coarse, occ, residual, true);
            } else {
                leaves[i] = buildRenderTemporalPackedLeafBytes(header, prefix, coarse, {}, true);
            }
        } catch (const std::exception& e) {
#ifdef _OPENMP
#pragma omp critical
#endif
            {
                failed = true;
                g_err = e.what();
            }
        }
    }
    if (failed) return -1;
    size_t words = 0;
    for (uint32_t i = 0; i < n; ++i) {
        offsets[i] = uint32_t(words);
        const size_t w = (leaves[i].size() + 3u) / 4u;
        if (words + w > capWords) {
            g_err = "payload buffer too small";
            return -1;
        }
        payload[words + w - 1] = 0u;
        std::memcpy(payload + words, leaves[i].data(), leaves[i].size());
        words += w;
    }
    offsets[n] = uint32_t(words);
    return long(words);
}

// generateQueries + fillLeafIndices (render/src/query_patterns.cpp:29-90) into out[count][5]
// (x, y, z, t, leafIndex); sorted[count][5] receives the same queries after sortQueriesByLeaf.
int vr_generate_queries(uint32_t w, uint32_t h, uint32_t d, uint32_t frames, int pattern, uint32_t count,
                        uint32_t seed, uint32_t* out, uint32_t* sorted)
{
    vbt::render::VbtFileHeader hdr{};
    hdr.width = w;
    hdr.height = h;
    hdr.depth = d;
    hdr.frames = frames;
    hdr.leafSize = 8;
    auto q = vbt::render::generateQueries(hdr, vbt::render::QueryPattern(pattern), count, seed);
    vbt::render::fillLeafIndices(hdr, q);
    auto put = [&](const std::vector<vbt::render::Query4D>& v, uint32_t* dst) {
        for (size_t i = 0; i < v.size(); ++i) {
            dst[5 * i] = v[i].x;
            dst[5 * i + 1] = v[i].y;
            dst[5 * i + 2] = v[i].z;
            dst[5 * i + 3] = v[i].t;
            dst[5 * i + 4] = v[i].leafIndex;
        }
    };
    put(q, out);
    vbt::render::sortQueriesByLeaf(q);
    put(q, sorted);
    return 0;
}

// dctEncodeKeep / dctEncodeKeepWeighted (weights == nullptr selects the former) and dctDecodeAt
// (src/dct_codec.cpp:63-122): coeffs[keep'] and decoded[n] = dctDecodeAt(coeffs, n, i).
int vr_dct(const float* series, const float* weights, int n, int keep, float* coeffs, float* decoded)
{
    const std::vector<float> s(series, series + n);
    std::vector<float> c;
    if (weights) c = dctEncodeKeepWeighted(s, std::vector<float>(weights, weights + n), keep);
    else c = dctEncodeKeep(s, keep);
    std::memcpy(coeffs, c.data(), 4 * c.size());
    for (int i = 0; i < n; ++i) decoded[i] = dctDecodeAt(c, n, i);
    return static_cast<int>(c.size());
}

} // extern "C"
