// host_api_test.cpp -- host-side checks of the C++ decoder API (include/vbt/*.h).
//
// Built and run by tests/test_cpp_api.py; needs no GPU.  It restates the reference's own tests
// (tests/render_temporal_payload_tests.cpp, tests/vbt_file_tests.cpp) against this library,
// compares the format functions bit for bit with the C oracle (oracle/liboracle.so), and answers
// a case file whose results the Python side compares with golden fixtures produced by the
// reference:
//   S codec bins frames dense hint        -> packed stream of the reference test's makeStream
//   Q w h d frames pattern seed count     -> generated and sorted queries (x, y, z, t, leaf)
//   D n keep weighted s[n] (w[n])         -> dct coefficients and dctDecodeAt at 0..n-1
//   P hexbytes                            -> parse verdict: message, 16 view integers
// usage: host_api_test <scratch dir> [<case file> <output file>]
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <filesystem>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "check.h"
#include "vbt/dct_codec.h"
#include "vbt/query_patterns.h"
#include "vbt/render_temporal_decode.h"
#include "vbt/render_temporal_payload.h"
#include "vbt/vbt_file.h"
#include "vbt_b200.h"
#include "vbt_oracle.h"

using namespace check;
namespace fs = std::filesystem;

namespace {

// ------------------------------------------------ tests/render_temporal_payload_tests.cpp

vbt::RenderTemporalShellOccupancySection two_voxel_occupancy()
{
    vbt::RenderTemporalShellOccupancySection occ{};
    occ.shellMask[0] = 1ull;
    occ.shellMask[2] = 1ull << 5u;
    occ.groupPrefix = {0u, 1u, 1u, 2u, 2u, 2u, 2u, 2u};
    return occ;
}

std::vector<uint8_t> two_voxel_mode2_leaf()
{
    vbt::RenderTemporalPackedHeaderFields h;
    h.mode = vbt::TemporalFirstPackedMode::TEMPORAL_FINE_COMPACT;
    h.coarseResolution = 1u;
    h.fineResolution = 0u;
    const auto prefix = vbt::makeRenderTemporalLeafPrefix(h.mode, 0u, 2u);
    const auto layout = vbt::computeRenderTemporalLeafLayout(h, prefix, true);
    const std::vector<uint8_t> coarse(layout.coarse.totalBytes, 0u);
    const auto occ = vbt::packRenderTemporalShellOccupancySection(two_voxel_occupancy());
    const uint32_t active = 2u;
    const std::vector<uint8_t> residual(active * vbt::kRenderTemporalControlDescriptorBytes +
                                            active * vbt::kRenderTemporalShellPackedTimeBinCount + 8u,
                                        0u);
    return vbt::buildRenderTemporalPackedLeafBytes(h, prefix, coarse, occ, residual, true);
}

void payload_tests()
{
    require(vbt::renderTemporalLeafVoxelIndex(0u, 0u, 1u) == 64u, "voxel index keeps the 8x8x8 stride");
    require(vbt::renderTemporalLeafVoxelIndex(2u, 2u, 1u) == 82u, "boundary voxel index uses the full stride");

    const auto valid = two_voxel_mode2_leaf();
    const auto view = vbt::parseRenderTemporalPackedLeaf(valid.data(), valid.size(), true);
    require(view.header.mode == vbt::TemporalFirstPackedMode::TEMPORAL_FINE_COMPACT, "Mode2 header lost");
    require(view.shellActiveVoxelCount == 2u, "Mode2 active voxel count");
    require(view.shellResidualOffset + view.shellResidualBytes == valid.size(), "Mode2 residual bounds");

    auto bad_prefix = valid;
    const size_t group1 = view.layout.fine.descriptorOffset + 64u + 2u;
    bad_prefix[group1] = bad_prefix[group1 + 1] = 0u;
    expect_throw([&] { vbt::parseRenderTemporalPackedLeaf(bad_prefix.data(), bad_prefix.size(), true); },
                 "group prefix");
    auto truncated = valid;
    truncated.resize(truncated.size() - 4u);
    expect_throw([&] { vbt::parseRenderTemporalPackedLeaf(truncated.data(), truncated.size(), true); },
                 "residual stream");
    auto trailing = valid;
    trailing.resize(trailing.size() + 4u, 0u);
    expect_throw([&] { vbt::parseRenderTemporalPackedLeaf(trailing.data(), trailing.size(), true); },
                 "trailing bytes");
    auto none = valid;
    std::fill(none.begin() + view.layout.fine.descriptorOffset, none.begin() + view.layout.fine.descriptorOffset + 80,
              uint8_t{0});
    expect_throw([&] { vbt::parseRenderTemporalPackedLeaf(none.data(), none.size(), true); }, "no active voxels");

    // the remaining parser errors
    expect_throw([&] { vbt::parseRenderTemporalPackedLeaf(valid.data(), 3u, true); }, "leaf bytes too small");
    expect_throw([&] { vbt::parseRenderTemporalPackedLeaf(nullptr, 64u, true); }, "leaf bytes too small");
    expect_throw([&] { vbt::parseRenderTemporalPackedLeaf(valid.data(), 4u, true); }, "prefix missing");
    expect_throw([&] { vbt::parseRenderTemporalPackedLeaf(valid.data(), 20u, true); }, "shorter than computed layout");
    expect_throw([] { vbt::makeRenderTemporalLeafPrefix(vbt::TemporalFirstPackedMode::TEMPORAL_GRID4, 65536u, 0u); },
                 "exceeds uint16");

    vbt::RenderTemporalPackedHeaderFields fine6;
    fine6.mode = vbt::TemporalFirstPackedMode::TEMPORAL_FINE6;
    fine6.coarseResolution = 2;
    fine6.fineResolution = 3;
    const auto p6 = vbt::makeRenderTemporalLeafPrefix(fine6.mode, 3u, 5u);
    const auto l6 = vbt::computeRenderTemporalLeafLayout(fine6, p6, true);
    expect_throw([&] { vbt::buildRenderTemporalPackedLeafBytes(fine6, p6, {1, 2, 3}, {}, true); },
                 "coarse stream bytes do not match");
    expect_throw(
        [&] {
            vbt::buildRenderTemporalPackedLeafBytes(fine6, p6, std::vector<uint8_t>(l6.coarse.totalBytes, 0u), {1},
                                                    true);
        },
        "fine stream bytes do not match");
    const auto leaf6 = vbt::buildRenderTemporalPackedLeafBytes(
        fine6, p6, std::vector<uint8_t>(l6.coarse.totalBytes, 7u), std::vector<uint8_t>(l6.fine.totalBytes, 9u), true);
    require(leaf6.size() == l6.totalBytes && leaf6[l6.coarseOffset] == 7u && leaf6[l6.fineOffset] == 9u,
            "FINE6 leaf assembly");

    vbt::TemporalFirstEncoderOptions opts;
    require(vbt::validateRenderTemporalLeafPrefix(p6, fine6, opts), "valid prefix rejected");
    opts.timeBinCount = 4;
    require(!vbt::validateRenderTemporalLeafPrefix(p6, fine6, opts), "time bin count must be 8");
    opts.timeBinCount = 8;
    vbt::RenderTemporalPackedHeaderFields nores = fine6;
    nores.fineResolution = 0;
    require(!vbt::validateRenderTemporalLeafPrefix(p6, nores, opts), "fine keys without fine controls");
    require(std::string(vbt::toString(vbt::TemporalFirstPackedMode::TEMPORAL_FINE_COMPACT)) == "TemporalFineCompact",
            "route tag names");
}

// ------------------------------------------------ header, layout and parse against the oracle

void same_stream(const vbt::RenderTemporalStreamLayout& a, const vo_stream_layout& b, const std::string& what)
{
    require(a.descriptorOffset == b.desc_off && a.descriptorBytes == b.desc_bytes && a.binIndexOffset == b.bin_off &&
                a.binIndexBytes == b.bin_bytes && a.keyframeOffset == b.key_off && a.keyframeBytes == b.key_bytes &&
                a.totalBytes == b.total,
            what + ": stream layout differs from the oracle");
}

void header_layout_tests()
{
    const uint32_t kf[][2] = {{0, 0}, {1, 0}, {3, 7}, {17, 2}, {200, 999}, {65535, 65535}};
    for (uint32_t p = 0; p < 4096; ++p) {
        const auto h = vbt::unpackRenderTemporalHeader(p);
        require(vbt::packRenderTemporalHeader(h) == p, "header round trip " + std::to_string(p));
        vo_header oh;
        vo_unpack_header(p, &oh);
        require(uint32_t(h.mode) == oh.mode && uint32_t(h.coarseCodec) == oh.coarse_codec &&
                    uint32_t(h.fineCodec) == oh.fine_codec && h.coarseResolution == oh.coarse_res &&
                    h.fineResolution == oh.fine_res,
                "header fields differ from the oracle");
        require(vo_pack_header(&oh) == p, "oracle header round trip");
        for (const auto& k : kf)
            for (int align = 0; align < 2; ++align) {
                vbt::RenderTemporalPackedLeafPrefix pre;
                pre.coarseKeyframeCount = uint16_t(k[0]);
                pre.fineKeyframeCount = uint16_t(k[1]);
                const auto l = vbt::computeRenderTemporalLeafLayout(h, pre, align != 0);
                vo_leaf_view ov{};
                vo_leaf_layout(&oh, k[0], k[1], align, &ov);
                const std::string what = "layout " + std::to_string(p);
                require(l.coarseOffset == ov.coarse_off && l.fineOffset == ov.fine_off && l.totalBytes == ov.total,
                        what + ": offsets differ from the oracle");
                same_stream(l.coarse, ov.coarse, what + " coarse");
                same_stream(l.fine, ov.fine, what + " fine");
            }
    }
    // clamped resolutions
    vbt::RenderTemporalPackedHeaderFields big;
    big.coarseResolution = 200;
    big.fineResolution = 9;
    require(vbt::unpackRenderTemporalHeader(vbt::packRenderTemporalHeader(big)).coarseResolution == 7u,
            "resolution clamps to 7");
}

void parse_vs_oracle()
{
    Rng rng(12345);
    int checked = 0;
    for (int it = 0; it < 4000; ++it) {
        vbt::RenderTemporalPackedHeaderFields h;
        h.mode = static_cast<vbt::TemporalFirstPackedMode>(rng.below(4));
        h.coarseCodec = static_cast<vbt::RenderTemporalSequenceCodec>(rng.below(2));
        h.fineCodec = static_cast<vbt::RenderTemporalSequenceCodec>(rng.below(2));
        h.coarseResolution = uint8_t(rng.below(8));
        h.fineResolution = uint8_t(rng.below(8));
        const uint32_t ck = rng.below(40), fk = rng.below(40);
        const auto pre = vbt::makeRenderTemporalLeafPrefix(h.mode, ck, fk);
        std::vector<uint8_t> leaf;
        if (h.mode == vbt::TemporalFirstPackedMode::TEMPORAL_FINE_COMPACT) {
            vbt::RenderTemporalShellOccupancySection occ{};
            uint16_t run = 0;
            for (int g = 0; g < 8; ++g) {
                occ.groupPrefix[size_t(g)] = run;
                occ.shellMask[size_t(g)] = rng.below(3) == 0 ? rng.next() : (rng.next() & rng.next() & rng.next());
                run = uint16_t(run + __builtin_popcountll(occ.shellMask[size_t(g)]));
            }
            if (rng.below(8) == 0) occ.groupPrefix[rng.below(8)] ^= 1u;
            const uint32_t active = vbt::renderTemporalShellActiveVoxelCount(occ);
            const uint32_t res = active * 4u + ((active * 4u + 3u) & ~3u) +
                                 ((fk * vbt::renderTemporalKeyframeBytes(h.fineCodec) + 3u) & ~3u);
            const auto l = vbt::computeRenderTemporalLeafLayout(h, pre, true);
            std::vector<uint8_t> coarse(l.coarse.totalBytes), residual(res);
            for (auto& b : coarse) b = uint8_t(rng.next());
            for (auto& b : residual) b = uint8_t(rng.next());
            leaf = vbt::buildRenderTemporalPackedLeafBytes(h, pre, coarse,
                                                           vbt::packRenderTemporalShellOccupancySection(occ), residual,
                                                           true);
        } else {
            const auto l = vbt::computeRenderTemporalLeafLayout(h, pre, true);
            std::vector<uint8_t> coarse(l.coarse.totalBytes), fine;
            if (h.mode == vbt::TemporalFirstPackedMode::TEMPORAL_FINE6) fine.resize(l.fine.totalBytes);
            for (auto& b : coarse) b = uint8_t(rng.next());
            for (auto& b : fine) b = uint8_t(rng.next());
            leaf = vbt::buildRenderTemporalPackedLeafBytes(h, pre, coarse, fine, true);
        }
        // size perturbations exercise every length check
        const int delta = rng.below(3) == 0 ? int(rng.below(17)) - 8 : 0;
        const size_t n = size_t(std::max<int>(0, int(leaf.size()) + delta));
        leaf.resize(std::max(leaf.size(), n) + 8u, 0u);
        vo_leaf_view ov{};
        const int ost = vo_parse_leaf(leaf.data(), n, 1, &ov);
        std::string err;
        vbt::RenderTemporalPackedLeafView v;
        try {
            v = vbt::parseRenderTemporalPackedLeaf(leaf.data(), n, true);
        } catch (const std::runtime_error& e) {
            err = e.what();
        }
        if (ost != VO_OK) {
            require(err == vbt_status_string(ost), "parse error '" + err + "' vs oracle status " + std::to_string(ost));
        } else {
            require(err.empty(), "parse failed where the oracle accepts: " + err);
            require(v.shellActiveVoxelCount == ov.shell_active && v.shellResidualOffset == ov.shell_residual_off &&
                        v.shellResidualBytes == ov.shell_residual_bytes && v.layout.totalBytes == ov.total &&
                        v.prefix.coarseKeyframeCount == ov.coarse_kf && v.prefix.fineKeyframeCount == ov.fine_kf,
                    "parsed view differs from the oracle");
            ++checked;
        }
    }
    require(checked > 1000, "too few accepted leaves in the parse sweep");
}

// ------------------------------------------------ half conversion and streams

void half_tests()
{
    for (uint32_t h = 0; h < 65536u; ++h) {
        const float a = vbt::renderTemporalHalfBitsToFloat(uint16_t(h));
        require(bits(a) == bits(vo_half_to_float(uint16_t(h))), "half->float differs from the oracle at " +
                                                                     std::to_string(h));
        const bool nan = ((h >> 10) & 31u) == 31u && (h & 1023u) != 0u;
        if (!nan) require(vbt::renderTemporalFloatToHalfBits(a) == h, "half round trip at " + std::to_string(h));
    }
    for (uint64_t b = 0; b < (1ull << 32); b += 65521ull) {
        const float f = from_bits(uint32_t(b));
        require(vbt::renderTemporalFloatToHalfBits(f) == vo_float_to_half(f), "float->half differs at bits " +
                                                                                  std::to_string(b));
    }
    for (float f : {0.0f, -0.0f, 65504.0f, 65519.99f, 65520.0f, 1e-8f, 5.96e-8f, 2.98e-8f, 6.1e-5f, INFINITY, -INFINITY})
        require(vbt::renderTemporalFloatToHalfBits(f) == vo_float_to_half(f), "float->half edge value");
}

vbt::RenderTemporalControlStreamData make_stream(int frames, int bins, int codec, bool dense,
                                                 const std::vector<float>* series = nullptr)
{
    // the construction of the reference's tests/temporal_decode_tests.cpp:17-38
    vbt::RenderTemporalControlStreamData s;
    s.codec = static_cast<vbt::RenderTemporalSequenceCodec>(codec);
    s.controlCount = 1;
    s.timeBinCount = uint8_t(bins);
    s.maxBinLocalKeys = 255;
    for (int t = 0; t < frames; ++t) {
        if (!(dense || t == 0 || t == frames - 1 || t % 13 == 7)) continue;
        float value = series ? (*series)[size_t(t)] : std::sin(static_cast<float>(t) * .19f);
        if (codec == 0) value = vbt::renderTemporalHalfBitsToFloat(vbt::renderTemporalFloatToHalfBits(value));
        s.keyframes.push_back({uint16_t(t), value});
    }
    s.descriptors.push_back({0, uint8_t(s.keyframes.size()), 1});
    for (int b = 0; b < bins; ++b) {
        const int boundary = b * frames / bins;
        size_t i = 0;
        while (i < s.keyframes.size() && s.keyframes[i].frame < boundary) ++i;
        s.binIndex.push_back(uint8_t(i == 0 ? 0 : i - 1));
    }
    return s;
}

void stream_tests()
{
    Rng rng(99);
    for (int it = 0; it < 300; ++it) {
        vbt::RenderTemporalControlStreamData s;
        s.codec = static_cast<vbt::RenderTemporalSequenceCodec>(rng.below(2));
        s.controlCount = uint16_t(1 + rng.below(40));
        s.timeBinCount = rng.below(2) ? 8 : 4;
        s.maxBinLocalKeys = 255;
        for (uint32_t c = 0; c < s.controlCount; ++c) {
            const uint32_t n = rng.below(20);
            s.descriptors.push_back({uint16_t(s.keyframes.size()), uint8_t(n), uint8_t(rng.below(3))});
            uint32_t t = rng.below(5);
            for (uint32_t k = 0; k < n; ++k, t += 1 + rng.below(12)) {
                float v = (rng.uniform() - 0.5f) * 8.0f;
                if (s.codec == vbt::RenderTemporalSequenceCodec::DP_KEYFRAME_FP16)
                    v = vbt::renderTemporalHalfBitsToFloat(vbt::renderTemporalFloatToHalfBits(v));
                s.keyframes.push_back({uint16_t(std::min<uint32_t>(t, 255u)), v});
            }
            for (int b = 0; b < s.timeBinCount; ++b) s.binIndex.push_back(uint8_t(rng.below(20)));
        }
        require(vbt::validateRenderTemporalControlStreamData(s), "generated stream must validate");
        const bool align = rng.below(2) != 0;
        const auto packed = vbt::packRenderTemporalControlStream(s, align);
        const auto u = vbt::unpackRenderTemporalControlStream(packed.data(), s.codec, s.controlCount, s.timeBinCount,
                                                              s.maxBinLocalKeys, uint32_t(s.keyframes.size()),
                                                              uint32_t(packed.size()), align);
        require(u.binIndex == s.binIndex, "bin index round trip");
        for (size_t c = 0; c < s.descriptors.size(); ++c)
            require(u.descriptors[c].keyStart == s.descriptors[c].keyStart &&
                        u.descriptors[c].keyCount == s.descriptors[c].keyCount &&
                        u.descriptors[c].reserved == s.descriptors[c].reserved,
                    "descriptor round trip");
        for (size_t k = 0; k < s.keyframes.size(); ++k)
            require(u.keyframes[k].frame == s.keyframes[k].frame && bits(u.keyframes[k].value) == bits(s.keyframes[k].value),
                    "keyframe round trip");
        if (packed.size() > 0)
            expect_throw(
                [&] {
                    vbt::unpackRenderTemporalControlStream(packed.data(), s.codec, s.controlCount, s.timeBinCount,
                                                           s.maxBinLocalKeys, uint32_t(s.keyframes.size()),
                                                           uint32_t(packed.size() - 1), align);
                },
                "stream bytes too small");
    }
    auto bad = make_stream(20, 8, 0, true);
    bad.descriptors[0].keyCount = uint8_t(bad.keyframes.size() + 1);
    require(!vbt::validateRenderTemporalControlStreamData(bad), "key range past the pool must not validate");
    expect_throw([&] { vbt::packRenderTemporalControlStream(bad, true); }, "invalid render temporal control stream");
    auto far = make_stream(20, 8, 0, true);
    far.keyframes.back().frame = 300;
    expect_throw([&] { vbt::packRenderTemporalControlStream(far, true); }, "exceeds uint8 range");
    auto zero = make_stream(20, 8, 0, true);
    zero.maxBinLocalKeys = 0;
    require(!vbt::validateRenderTemporalControlStreamData(zero), "maxBinLocalKeys 0 must not validate");

    // A keyframe count whose byte size wraps the reference's 32-bit extent (2^29 FP32 keys of 8
    // bytes = 2^32 = 0): the reference's check passes and it would read keys past the stream.
    // The value decode refuses it on the host, before any device work, with the extent message;
    // a control without keys still decodes to 0, and an out-of-range descriptor or key range keeps
    // the reference's own message.
    {
        std::vector<uint8_t> st(64, 0u);
        st[0] = 0u, st[1] = 0u, st[2] = 2u;   // control 0: keyStart 0, keyCount 2
        const uint32_t wrap_kf = 1u << 29;
        const auto fp32 = vbt::RenderTemporalSequenceCodec::DP_KEYFRAME_FP32;
        expect_throw([&] { vbt::decodeRenderTemporalControlValue(st.data(), fp32, 2, 8, 0, wrap_kf, 64, true, 10, 0, 3); },
                     "render temporal stream decode out of bounds");
        expect_throw(
            [&] { vbt::decodeRenderTemporalControlValues(st.data(), fp32, 2, 8, wrap_kf, 64, true, 10, {1, 0}, {0, 3}); },
            "render temporal stream decode out of bounds");
        require(vbt::decodeRenderTemporalControlValue(st.data(), fp32, 2, 8, 0, wrap_kf, 64, true, 10, 1, 3) == 0.0f,
                "a control without keys decodes to 0 without reading keys");
        st[2] = 0u;
        const auto zeros = vbt::decodeRenderTemporalControlValues(st.data(), fp32, 2, 8, wrap_kf, 64, true, 10, {0, 1}, {0, 5});
        require(zeros.size() == 2 && zeros[0] == 0.0f && zeros[1] == 0.0f, "controls without keys decode to 0");
        st[0] = 1u, st[2] = 1u;   // keyStart 1 + keyCount 1 > keyframeCount 1
        expect_throw([&] { vbt::decodeRenderTemporalControlValue(st.data(), fp32, 2, 8, 0, 1, 64, true, 10, 0, 3); },
                     "render temporal keyframe range out of bounds");
        expect_throw([&] { vbt::decodeRenderTemporalControlValue(st.data(), fp32, 2, 8, 0, 1, 64, true, 10, 2, 3); },
                     "render temporal control index out of range");
    }
}

// ------------------------------------------------ tests/vbt_file_tests.cpp

struct FileSpec {
    uint32_t version = 4, width = 8, height = 8, depth = 8, frames = 4, leafSize = 8, coarseResolution = 4,
             maxCoarseKeep = 0, leafCount = 1, profileType = 1;
    std::vector<float> scales;
    std::vector<uint32_t> offsets{0, 1};
    std::vector<uint32_t> payload{0};
    bool trailingByte = false;
};

void write_spec(const fs::path& path, const FileSpec& f)
{
    std::ofstream out(path, std::ios::binary);
    out.write("VBTPACK4", 8);
    const uint32_t words[11] = {f.version,          f.width,         f.height,    f.depth,
                                f.frames,           f.leafSize,      f.coarseResolution,
                                f.maxCoarseKeep,    f.leafCount,     f.profileType,
                                uint32_t(f.scales.size())};
    out.write(reinterpret_cast<const char*>(words), sizeof(words));
    out.write(reinterpret_cast<const char*>(f.scales.data()), std::streamsize(4 * f.scales.size()));
    out.write(reinterpret_cast<const char*>(f.offsets.data()), std::streamsize(4 * f.offsets.size()));
    out.write(reinterpret_cast<const char*>(f.payload.data()), std::streamsize(4 * f.payload.size()));
    if (f.trailingByte) out.put('\0');
}

void expect_load_failure(const fs::path& path, const std::string& fragment)
{
    vbt::render::VbtFile f;
    std::string error;
    require(!vbt::render::loadVbtFile(path, f, error), "load must fail: " + path.string());
    require(error.find(fragment) != std::string::npos, "reader error '" + error + "', wanted '" + fragment + "'");
}

void file_tests(const fs::path& root)
{
    fs::create_directories(root);
    FileSpec valid;
    write_spec(root / "valid.vbtp", valid);
    vbt::render::VbtFile loaded;
    std::string error;
    require(vbt::render::loadVbtFile(root / "valid.vbtp", loaded, error), "valid file rejected: " + error);
    require(loaded.header.version == 4 && loaded.header.leafCount == 1, "valid header");
    require(loaded.offsetsWords == valid.offsets && loaded.payloadWords == valid.payload, "valid tables");

    FileSpec f = valid;
    f.version = 3;
    write_spec(root / "bad_version.vbtp", f);
    expect_load_failure(root / "bad_version.vbtp", "Unsupported VBTPACK4 version");
    f = valid;
    f.width = 16;
    write_spec(root / "bad_leaf_count.vbtp", f);
    expect_load_failure(root / "bad_leaf_count.vbtp", "leafCount does not match");
    f.leafCount = 2;
    f.offsets = {0, 2, 1};
    write_spec(root / "non_monotonic.vbtp", f);
    expect_load_failure(root / "non_monotonic.vbtp", "strictly increasing");
    f = valid;
    f.offsets = {0, 0};
    f.payload.clear();
    write_spec(root / "empty_leaf.vbtp", f);
    expect_load_failure(root / "empty_leaf.vbtp", "strictly increasing");
    f = valid;
    f.trailingByte = true;
    write_spec(root / "trailing.vbtp", f);
    expect_load_failure(root / "trailing.vbtp", "trailing bytes");
    f = valid;
    f.offsets = {0, 2};
    write_spec(root / "truncated.vbtp", f);
    expect_load_failure(root / "truncated.vbtp", "truncated");
    expect_load_failure(root / "missing.vbtp", "Failed to query file size");
    {
        std::ofstream(root / "short.vbtp", std::ios::binary).write("VBTPACK4", 8);
    }
    expect_load_failure(root / "short.vbtp", "Invalid VBTPACK4 file size");

    // accessors
    require(vbt::render::readPackedHeaderWord(loaded, 0) == 0u && vbt::render::readPackedHeaderWord(loaded, 5) == 0u,
            "readPackedHeaderWord");
    vbt::render::VbtFileHeader hdr{};
    hdr.width = 20;
    hdr.height = 12;
    hdr.depth = 17;
    hdr.leafSize = 8;
    for (uint32_t z = 0; z < 30; ++z)
        for (uint32_t y = 0; y < 20; ++y)
            for (uint32_t x = 0; x < 30; ++x) {
                const uint32_t bx = std::min(2u, x / 8), by = std::min(1u, y / 8), bz = std::min(2u, z / 8);
                require(vbt::render::leafIndexForVoxel(hdr, x, y, z) == (bz * 2 + by) * 3 + bx, "leafIndexForVoxel");
            }
    hdr.leafSize = 0;
    require(vbt::render::leafIndexForVoxel(hdr, 5, 5, 5) == 0u, "leafIndexForVoxel with leafSize 0");
    Rng rng(3);
    for (int i = 0; i < 10000; ++i) {
        const uint32_t w = uint32_t(rng.next());
        const auto d = vbt::render::decodeScientificHeaderV2(w);
        require(uint32_t(d.mode) == (w & 3u) && d.coarseKeepMinus1 == ((w >> 2) & 63u), "scientific header mode/keep");
        if (d.mode == vbt::render::ScientificMode::SparseEvents)
            require(d.tierId == ((w >> 8) & 3u) && d.framesPerBinMinus1 == ((w >> 10) & 15u) &&
                        d.eventQuantCode == ((w >> 14) & 3u) && d.packedEventCount == ((w >> 16) & 0xFFFu) &&
                        d.sparseSubtype == (w >> 28),
                    "sparse header fields");
        else if (d.mode == vbt::render::ScientificMode::CoarseOnly)
            require(d.coarseQuantClass == ((w >> 8) & 7u) && d.denseQuantBits == 0u, "coarse-only header fields");
        else
            require(d.denseQuantBits == ((w >> 8) & 15u) && d.denseSubtype == ((w >> 12) & 7u) &&
                        d.denseTemporalKeepMinus1 == ((w >> 15) & 15u),
                    "dense header fields");
    }
    vbt::render::QueryPattern qp;
    require(vbt::render::parseQueryPattern("coherent", qp) && qp == vbt::render::QueryPattern::CoherentTiles &&
                !vbt::render::parseQueryPattern("diagonal", qp),
            "parseQueryPattern");
}

// A real asset through loadVbtFile equals the oracle's own reader.
void asset_load_test(const std::string& path)
{
    vbt::render::VbtFile f;
    std::string error;
    require(vbt::render::loadVbtFile(path, f, error), "asset rejected: " + error);
    vo_file of{};
    char err[256];
    require(vo_load_file(path.c_str(), &of, err, sizeof err) == 0, std::string("oracle reader: ") + err);
    require(f.header.width == of.width && f.header.frames == of.frames && f.header.profileType == of.profile_type &&
                f.coarseAcScales.size() == of.scale_count && f.payloadWords.size() == of.payload_words,
            "asset header differs from the oracle reader");
    require(std::equal(f.offsetsWords.begin(), f.offsetsWords.end(), of.offsets) &&
                std::equal(f.payloadWords.begin(), f.payloadWords.end(), of.payload) &&
                std::memcmp(f.coarseAcScales.data(), of.scales, 4 * of.scale_count) == 0,
            "asset tables differ from the oracle reader");
    vo_free_file(&of);
}

// ------------------------------------------------ case file

void put32(std::vector<uint32_t>& out, uint32_t v) { out.push_back(v); }

void answer_cases(const std::string& in_path, const std::string& out_path)
{
    std::ifstream in(in_path);
    std::vector<uint32_t> out;
    std::string line;
    while (std::getline(in, line)) {
        std::istringstream ls(line);
        std::string kind;
        ls >> kind;
        if (kind == "S") {
            int codec, bins, frames, dense, hint;
            ls >> codec >> bins >> frames >> dense >> hint;
            // per-frame series values (hex float bits) replace sin(0.19 t), so that both packers
            // see identical inputs whatever the libm of the fixture generator
            std::vector<float> series(static_cast<size_t>(frames), 0.0f);
            for (auto& v : series) {
                uint32_t b;
                ls >> std::hex >> b >> std::dec;
                v = from_bits(b);
            }
            auto s = make_stream(frames, bins, codec, dense != 0, &series);
            if (hint >= 0) std::fill(s.binIndex.begin(), s.binIndex.end(), uint8_t(hint));
            const auto packed = vbt::packRenderTemporalControlStream(s, true);
            put32(out, uint32_t(packed.size()));
            std::vector<uint32_t> words((packed.size() + 3) / 4, 0u);
            std::memcpy(words.data(), packed.data(), packed.size());
            out.insert(out.end(), words.begin(), words.end());
        } else if (kind == "Q") {
            vbt::render::VbtFileHeader h{};
            uint32_t pattern, seed, count;
            ls >> h.width >> h.height >> h.depth >> h.frames >> pattern >> seed >> count;
            h.leafSize = 8;
            auto q = vbt::render::generateQueries(h, vbt::render::QueryPattern(pattern), count, seed);
            vbt::render::fillLeafIndices(h, q);
            for (int pass = 0; pass < 2; ++pass) {
                if (pass == 1) vbt::render::sortQueriesByLeaf(q);
                for (const auto& r : q) {
                    put32(out, r.x);
                    put32(out, r.y);
                    put32(out, r.z);
                    put32(out, r.t);
                    put32(out, r.leafIndex);
                }
            }
        } else if (kind == "D") {
            int n, keep, weighted;
            ls >> n >> keep >> weighted;
            std::vector<float> s(static_cast<size_t>(n), 0.0f), w;
            for (auto& v : s) {
                uint32_t b;
                ls >> std::hex >> b >> std::dec;
                v = from_bits(b);
            }
            if (weighted) {
                w.resize(size_t(n));
                for (auto& v : w) {
                    uint32_t b;
                    ls >> std::hex >> b >> std::dec;
                    v = from_bits(b);
                }
            }
            const auto c = weighted ? vbt::dctEncodeKeepWeighted(s, w, keep) : vbt::dctEncodeKeep(s, keep);
            put32(out, uint32_t(c.size()));
            for (float v : c) put32(out, bits(v));
            for (int i = 0; i < n; ++i) put32(out, bits(vbt::dctDecodeAt(c, n, i)));
        } else if (kind == "P") {
            std::string hex;
            ls >> hex;
            std::vector<uint8_t> leaf(hex.size() / 2);
            for (size_t i = 0; i < leaf.size(); ++i) leaf[i] = uint8_t(std::stoul(hex.substr(2 * i, 2), nullptr, 16));
            std::string msg;
            uint32_t vals[16] = {};
            try {
                const auto v = vbt::parseRenderTemporalPackedLeaf(leaf.data(), leaf.size(), true);
                const uint32_t f[16] = {uint32_t(v.header.mode), uint32_t(v.header.coarseCodec),
                                        uint32_t(v.header.fineCodec), v.header.coarseResolution,
                                        v.header.fineResolution, v.prefix.coarseKeyframeCount,
                                        v.prefix.fineKeyframeCount, v.layout.coarseOffset, v.layout.coarse.totalBytes,
                                        v.layout.fineOffset, v.layout.fine.totalBytes, v.layout.totalBytes,
                                        v.shellActiveVoxelCount, v.shellResidualOffset, v.shellResidualBytes, 0u};
                std::memcpy(vals, f, sizeof f);
            } catch (const std::runtime_error& e) {
                msg = e.what();
            }
            put32(out, uint32_t(msg.size()));
            std::vector<uint32_t> words((msg.size() + 3) / 4, 0u);
            std::memcpy(words.data(), msg.data(), msg.size());
            out.insert(out.end(), words.begin(), words.end());
            out.insert(out.end(), vals, vals + 16);
        } else if (!kind.empty()) {
            throw std::runtime_error("unknown case kind " + kind);
        }
    }
    std::ofstream o(out_path, std::ios::binary);
    o.write(reinterpret_cast<const char*>(out.data()), std::streamsize(4 * out.size()));
}

}  // namespace

int main(int argc, char** argv)
{
    if (argc < 2) {
        std::cerr << "usage: host_api_test <scratch dir> [<case file> <output file>] [<asset>...]\n";
        return 2;
    }
    try {
        payload_tests();
        header_layout_tests();
        parse_vs_oracle();
        half_tests();
        stream_tests();
        file_tests(fs::path(argv[1]) / "reader");
        int next = 2;
        if (argc >= 4) {
            answer_cases(argv[2], argv[3]);
            next = 4;
        }
        for (int i = next; i < argc; ++i) asset_load_test(argv[i]);
    } catch (const std::exception& e) {
        std::cerr << "host_api_test: FAIL: " << e.what() << "\n";
        return 1;
    }
    std::cout << "host_api_test: PASS\n";
    return 0;
}
