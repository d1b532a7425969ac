// decode_api_test.cpp -- GPU checks of the C++ decoder API's decode calls (include/vbt/*.h).
//
// Built and run by tests/test_cpp_api.py on a CUDA device.  It restates the reference's
// tests/temporal_decode_tests.cpp (dense and sparse streams, 4 and 8 bins, built / zero / 255
// bin hints, frames 1..255 at t = -2..T+2, and the Mode2 shell leaf on voxels {0, 63, 64, 255,
// 511}) with its 2e-6 lerp tolerance, and additionally requires every decoded value to be
// bit-identical to the C oracle (vo_decode_control).  Then the VbtFile calls (frame decode,
// point queries, scientific reconstruction) are compared with the oracle on real assets.
// usage: decode_api_test <render asset>... --sci <scientific asset>...
#include <algorithm>
#include <cmath>
#include <iostream>
#include <string>
#include <vector>

#include "check.h"
#include "vbt/query_patterns.h"
#include "vbt/render_temporal_decode.h"
#include "vbt/render_temporal_payload.h"
#include "vbt/scientific_decode.h"
#include "vbt/vbt_file.h"
#include "vbt_oracle.h"

using namespace check;
using namespace vbt;

namespace {

void near(float actual, float expected, const std::string& what)
{
    if (!std::isfinite(actual) || std::abs(actual - expected) > 2e-6f)
        throw std::runtime_error(what + ": " + std::to_string(actual) + " vs " + std::to_string(expected));
}

RenderTemporalControlStreamData make_stream(int frames, int bins, int codec, bool dense)
{
    RenderTemporalControlStreamData s;
    s.codec = static_cast<RenderTemporalSequenceCodec>(codec);
    s.controlCount = 1;
    s.timeBinCount = uint8_t(bins);
    s.maxBinLocalKeys = 255;
    for (int t = 0; t < frames; ++t) {
        if (!(dense || t == 0 || t == frames - 1 || t % 13 == 7)) continue;
        float value = std::sin(static_cast<float>(t) * .19f);
        if (codec == 0) value = renderTemporalHalfBitsToFloat(renderTemporalFloatToHalfBits(value));
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

// lower_bound + lerp over the keyframes: the expectation the reference's test uses.
float lerp_expectation(const RenderTemporalControlStreamData& s, int frames, int frame)
{
    frame = std::clamp(frame, 0, frames - 1);
    const auto& keys = s.keyframes;
    auto hi = std::lower_bound(keys.begin(), keys.end(), frame, [](const auto& k, int t) { return k.frame < t; });
    if (hi == keys.end()) return keys.back().value;
    if (hi == keys.begin() || hi->frame == frame) return hi->value;
    const auto lo = hi - 1;
    const float alpha = static_cast<float>(frame - lo->frame) / (hi->frame - lo->frame);
    return lo->value * (1.0f - alpha) + hi->value * alpha;
}

long g_values = 0;

void check_stream(RenderTemporalControlStreamData s, int frames, int hint)
{
    if (hint >= 0) std::fill(s.binIndex.begin(), s.binIndex.end(), uint8_t(hint));
    const auto packed = packRenderTemporalControlStream(s, true);
    const uint32_t kf = uint32_t(s.keyframes.size()), bytes = uint32_t(packed.size());
    std::vector<uint16_t> ci;
    std::vector<int> ts;
    for (int t = -2; t <= frames + 2; ++t) {
        ci.push_back(0);
        ts.push_back(t);
    }
    const auto got = decodeRenderTemporalControlValues(packed.data(), s.codec, 1, s.timeBinCount, kf, bytes, true,
                                                       frames, ci, ts);
    const std::string what = "codec " + std::to_string(int(s.codec)) + " bins " + std::to_string(s.timeBinCount) +
                             " frames " + std::to_string(frames) + " hint " + std::to_string(hint);
    for (size_t i = 0; i < ts.size(); ++i) {
        near(got[i], lerp_expectation(s, frames, ts[i]), what + " t " + std::to_string(ts[i]));
        float want = 0.0f;
        require(vo_decode_control(packed.data(), uint32_t(s.codec), 1, s.timeBinCount, kf, bytes, 1, frames, 0, ts[i],
                                  &want) == VO_OK,
                "oracle decode failed");
        require(bits(got[i]) == bits(want), what + ": not bit-identical to the oracle at t " + std::to_string(ts[i]));
    }
    for (int t : {-2, 0, frames / 2, frames - 1, frames + 2}) {
        const float one = decodeRenderTemporalControlValue(packed.data(), s.codec, 1, s.timeBinCount, 1, kf, bytes,
                                                           true, frames, 0, t);
        require(bits(one) == bits(got[size_t(t + 2)]), what + ": single and batched decode differ");
    }
    g_values += long(ts.size());
}

void shell_test()
{
    auto coarse = make_stream(101, 8, 0, false);
    coarse.controlCount = 64;
    coarse.descriptors.resize(64, coarse.descriptors.front());
    coarse.binIndex.resize(64 * 8);
    for (int c = 1; c < 64; ++c) std::copy_n(coarse.binIndex.begin(), 8, coarse.binIndex.begin() + c * 8);
    auto residual = make_stream(101, 4, 1, true);
    const std::vector<int> voxels{0, 63, 64, 255, 511};
    residual.controlCount = uint16_t(voxels.size());
    residual.descriptors.resize(voxels.size(), residual.descriptors.front());
    residual.binIndex.resize(voxels.size() * 4);
    for (size_t c = 1; c < voxels.size(); ++c)
        std::copy_n(residual.binIndex.begin(), 4, residual.binIndex.begin() + c * 4);
    RenderTemporalShellOccupancySection occ{};
    for (int v : voxels) occ.shellMask[size_t(v / 64)] |= 1ull << (v % 64);
    for (int g = 0; g < 8; ++g)
        occ.groupPrefix[size_t(g)] =
            uint16_t(std::count_if(voxels.begin(), voxels.end(), [g](int v) { return v < g * 64; }));
    RenderTemporalPackedHeaderFields header;
    header.mode = TemporalFirstPackedMode::TEMPORAL_FINE_COMPACT;
    header.fineCodec = residual.codec;
    const auto prefix = makeRenderTemporalLeafPrefix(header.mode, uint32_t(coarse.keyframes.size()),
                                                     uint32_t(residual.keyframes.size()));
    const auto leaf = buildRenderTemporalPackedLeafBytes(header, prefix, packRenderTemporalControlStream(coarse, true),
                                                         packRenderTemporalShellOccupancySection(occ),
                                                         packRenderTemporalControlStream(residual, true), true);
    const auto view = parseRenderTemporalPackedLeaf(leaf.data(), leaf.size(), true);
    vo_leaf_view ov{};
    require(vo_parse_leaf(leaf.data(), leaf.size(), 1, &ov) == VO_OK, "oracle parse of the shell leaf");
    for (int t = -1; t <= 101; ++t) {
        for (int v = 0; v < 512; ++v) {
            const bool active = std::find(voxels.begin(), voxels.end(), v) != voxels.end();
            const float got = decodeRenderTemporalLeafShellVoxelValue(leaf.data(), view, true, 101, uint16_t(v), t);
            near(got, active ? lerp_expectation(residual, 101, t) : 0.0f, "shell voxel " + std::to_string(v));
            float want = 0.0f;
            require(vo_decode_shell_voxel(leaf.data(), &ov, 101, uint32_t(v), t, &want) == VO_OK, "oracle shell voxel");
            require(bits(got) == bits(want), "shell voxel not bit-identical to the oracle");
        }
        for (uint16_t c = 0; c < 64; c += 9) {
            const float got = decodeRenderTemporalLeafControlValue(leaf.data(), view.header, view.prefix, view.layout,
                                                                   false, true, 101, c, t);
            near(got, lerp_expectation(coarse, 101, t), "coarse control");
        }
    }
}

void error_tests()
{
    auto s = make_stream(40, 8, 1, false);
    const auto packed = packRenderTemporalControlStream(s, true);
    const uint32_t kf = uint32_t(s.keyframes.size()), bytes = uint32_t(packed.size());
    expect_throw([&] { decodeRenderTemporalControlValue(packed.data(), s.codec, 1, 8, 1, kf, bytes, true, 40, 1, 3); },
                 "render temporal control index out of range");
    expect_throw(
        [&] { decodeRenderTemporalControlValue(packed.data(), s.codec, 1, 8, 1, kf, bytes - 4, true, 40, 0, 3); },
        "render temporal stream decode out of bounds");
    auto bad = packed;
    bad[2] = uint8_t(kf + 1);   // descriptor keyCount past the keyframe pool
    expect_throw([&] { decodeRenderTemporalControlValue(bad.data(), s.codec, 1, 8, 1, kf, bytes, true, 40, 0, 3); },
                 "render temporal keyframe range out of bounds");
    expect_throw(
        [&] {
            decodeRenderTemporalControlValues(bad.data(), s.codec, 1, 8, kf, bytes, true, 40, {0, 0}, {1, 2});
        },
        "render temporal keyframe range out of bounds");
    bad[2] = 0;   // keyCount 0 decodes to 0
    require(decodeRenderTemporalControlValue(bad.data(), s.codec, 1, 8, 1, kf, bytes, true, 40, 0, 3) == 0.0f,
            "empty control decodes to 0");
}

void render_file_test(const std::string& path)
{
    render::VbtFile file;
    std::string error;
    require(render::loadVbtFile(path, file, error), "load: " + error);
    vo_file of{};
    char err[256];
    require(vo_load_file(path.c_str(), &of, err, sizeof err) == 0, err);
    const size_t voxels = size_t(of.width) * of.height * of.depth;
    std::vector<float> want(voxels);
    for (int t = -1; t <= int(of.frames); ++t) {
        const auto got = render::decodeRenderTemporalFrame(file, t);
        require(vo_decode_frame(&of, t, want.data(), 0, nullptr) == 0, "oracle frame");
        require(got.size() == voxels && std::memcmp(got.data(), want.data(), 4 * voxels) == 0,
                path + ": frame " + std::to_string(t) + " not bit-identical to the oracle");
    }
    auto q = render::generateQueries(file.header, render::QueryPattern::RandomFull, 4096, 11);
    const auto got = render::decodeValuesGpu(file, q);
    std::vector<uint32_t> flat;
    for (const auto& r : q) flat.insert(flat.end(), {r.x, r.y, r.z, r.t});
    std::vector<float> qw(q.size());
    require(vo_query_points(&of, flat.data(), q.size(), qw.data(), 0) == 0, "oracle queries");
    require(std::memcmp(got.data(), qw.data(), 4 * q.size()) == 0, path + ": point queries differ from the oracle");
    render::releaseDeviceCopy(file);
    const auto again = render::decodeRenderTemporalFrame(file, 0);
    require(vo_decode_frame(&of, 0, want.data(), 0, nullptr) == 0 &&
                std::memcmp(again.data(), want.data(), 4 * voxels) == 0,
            "decode after releaseDeviceCopy");
    render::releaseDeviceCopy(file);
    vo_free_file(&of);
}

void sci_file_test(const std::string& path)
{
    render::VbtFile file;
    std::string error;
    require(render::loadVbtFile(path, file, error), "load: " + error);
    vo_file of{};
    char err[256];
    require(vo_load_file(path.c_str(), &of, err, sizeof err) == 0, err);
    const size_t voxels = size_t(of.width) * of.height * of.depth;
    std::vector<float> want(voxels);
    double lo = 1e300, hi = -1e300;
    std::vector<std::vector<float>> frames;
    for (uint32_t t = 0; t < of.frames; ++t) {
        vo_sci_frame(&of, t, want.data(), 0);
        for (float v : want) {
            lo = std::min(lo, double(v));
            hi = std::max(hi, double(v));
        }
        frames.push_back(want);
    }
    const double tol = 1e-6 * std::max(hi - lo, 1e-30);
    for (uint32_t t = 0; t < of.frames; ++t) {
        const auto got = render::reconstructScientificFrameCpu(file, t);
        for (size_t i = 0; i < voxels; ++i)
            require(std::abs(double(got[i]) - double(frames[t][i])) <= tol,
                    path + ": scientific frame " + std::to_string(t) + " outside 1e-6 of the field range");
    }
    auto q = render::generateQueries(file.header, render::QueryPattern::RandomFull, 512, 5);
    render::fillLeafIndices(file.header, q);
    for (size_t i = 0; i < q.size(); i += 37) {
        const float got = render::decodeScientificValueAtCpu(file, q[i]);
        const float w = frames[q[i].t][(size_t(q[i].z) * of.height + q[i].y) * of.width + q[i].x];
        require(std::abs(double(got) - double(w)) <= tol, "scientific point value");
    }
    auto wrong = q[0];
    wrong.leafIndex += 1;
    expect_throw<std::invalid_argument>([&] { render::decodeScientificValueAtCpu(file, wrong); }, "leafIndex");
    auto late = q[0];
    late.t = of.frames;
    expect_throw<std::out_of_range>([&] { render::decodeScientificValueAtCpu(file, late); }, "frame");
    render::releaseDeviceCopy(file);
    vo_free_file(&of);
}

}  // namespace

int main(int argc, char** argv)
{
    try {
        for (int codec : {0, 1})
            for (int bins : {4, 8})
                for (int frames = 1; frames <= 255; ++frames) {
                    check_stream(make_stream(frames, bins, codec, true), frames, -1);
                    for (int hint : {-1, 0, 255}) check_stream(make_stream(frames, bins, codec, false), frames, hint);
                }
        shell_test();
        error_tests();
        bool sci = false;
        int files = 0;
        for (int i = 1; i < argc; ++i) {
            const std::string a = argv[i];
            if (a == "--sci") {
                sci = true;
                continue;
            }
            if (sci) sci_file_test(a);
            else render_file_test(a);
            ++files;
        }
        std::cout << "decode_api_test: PASS (" << g_values << " stream values, " << files << " files)\n";
    } catch (const std::exception& e) {
        std::cerr << "decode_api_test: FAIL: " << e.what() << "\n";
        return 1;
    }
    return 0;
}
