// kf_ref_shim.cpp -- C-ABI over the reference encoder's per-voxel keyframe detector, compiled by
// oracle/Makefile into oracle/_ref/libkfref.so.
//
// TEST INFRASTRUCTURE ONLY: it pins the C restatement (vbt_keyframe_oracle.c) to the reference and
// serves as the "reference" CPU baseline of the keyframe pass in bench.py.
//
// detectDensityKeyFrames and reconstructFromKeys (src/render_temporal_kf_probe_main.cpp:2080-2201)
// sit in an anonymous namespace of the reference's encoder translation unit, so they have no
// external symbol.  This shim therefore makes that unmodified source file part of its own
// translation unit: the #include below reads it from the reference tree at build time (nothing is
// copied into this repository), and the extern "C" functions after it call the two functions
// directly.  The encoder's own main() stays out (it is behind VBT_RENDER_TEMPORAL_PROBE_STANDALONE).
#include "render_temporal_kf_probe_main.cpp"

#include <cstring>

extern "C" {

// Layout of vo_keyframe_profile (vbt_oracle.h) and vbt_keyframe_profile (include/vbt_b200.h).
struct vr_keyframe_profile {
    float eps_abs, eps_rel, gamma_delta, render_cutoff, cutoff_band;
    uint32_t cutoff_temporal_protect, iso_surface_protect;
    float iso_value, iso_band;
    double bg_threshold;
};

static DensityTemporalProfile to_profile(const vr_keyframe_profile* p)
{
    DensityTemporalProfile q;
    q.epsAbs = p->eps_abs;
    q.epsRel = p->eps_rel;
    q.gammaDelta = p->gamma_delta;
    q.renderCutoff = p->render_cutoff;
    q.cutoffBand = p->cutoff_band;
    q.cutoffTemporalProtect = p->cutoff_temporal_protect != 0;
    q.isoSurfaceProtect = p->iso_surface_protect != 0;
    q.isoValue = p->iso_value;
    q.isoBand = p->iso_band;
    return q;
}

// detectDensityKeyFrames on one series: writes the sorted keys, returns their count.
int vbtref_detect_keyframes(const float* values, int n, const vr_keyframe_profile* p, int* keys, int* used_protect)
{
    const std::vector<float> v(values, values + n);
    bool used = false;
    const std::vector<int> k = detectDensityKeyFrames(v, to_profile(p), &used);
    if (!k.empty()) std::memcpy(keys, k.data(), k.size() * sizeof(int));
    if (used_protect) *used_protect = used ? 1 : 0;
    return static_cast<int>(k.size());
}

// reconstructFromKeys on one series.
void vbtref_reconstruct(const float* values, int n, const int* keys, int key_count, float* out)
{
    const std::vector<float> v(values, values + n);
    const std::vector<int> k(keys, keys + key_count);
    std::vector<float> r;
    reconstructFromKeys(v, k, r);
    std::memcpy(out, r.data(), r.size() * sizeof(float));
}

// The per-voxel temporal pass of the encoder's leaf loop (src/render_temporal_kf_probe_main.cpp:
// 619-659) over `series` independent series, series s at values[t * frame_stride + s]: the
// background test on the running max, detectDensityKeyFrames, reconstructFromKeys and the squared
// error, on `threads` OpenMP threads (0: all).  key_count[s] is the number of keys the encoder
// counts for the series (1 for a background-zeroed one); err2 the summed squared error.
int vbtref_temporal_pass(const float* values, uint64_t series, int frames, uint64_t frame_stride,
                         const vr_keyframe_profile* p, uint32_t* key_count, double* err2, int threads)
{
    const DensityTemporalProfile prof = to_profile(p);
    const double bg = p->bg_threshold;
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel
#endif
    {
        std::vector<float> series_v(static_cast<size_t>(frames)), recon;
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 256)
#endif
        for (long long s = 0; s < static_cast<long long>(series); ++s) {
            float vmax = 0.0f;
            for (int t = 0; t < frames; ++t) {
                const float v = values[static_cast<uint64_t>(t) * frame_stride + static_cast<uint64_t>(s)];
                series_v[static_cast<size_t>(t)] = v;
                vmax = std::max(vmax, v);
            }
            double e2 = 0.0;
            if (bg >= 0.0 && static_cast<double>(vmax) < bg) {
                for (int t = 0; t < frames; ++t) {
                    const double d = static_cast<double>(series_v[static_cast<size_t>(t)]);
                    e2 += d * d;
                }
                key_count[s] = 1;
            } else {
                const auto keys = detectDensityKeyFrames(series_v, prof, nullptr);
                reconstructFromKeys(series_v, keys, recon);
                for (int t = 0; t < frames; ++t) {
                    const double d = static_cast<double>(series_v[static_cast<size_t>(t)]) -
                                     static_cast<double>(recon[static_cast<size_t>(t)]);
                    e2 += d * d;
                }
                key_count[s] = static_cast<uint32_t>(keys.size());
            }
            if (err2) err2[s] = e2;
        }
    }
    return 0;
}

// The coarse control fitting of the encoder's leaf loop (src/render_temporal_kf_probe_main.cpp:
// 705-729) for one leaf: the 4^3 controls sampled from the leaf's reconstruction (leafTemporal,
// voxel (lz*8 + ly)*8 + lx, frames fastest) at controlCoords(4), detectDensityKeyFrames with the
// control profile, appendControlSequenceToStream (8 time bins) and reconstructFromKeys.  Outputs the
// stream's descriptor words (keyStart | keyCount << 16 | reserved << 24), bin rows (8 bytes per
// control), keyframes, requiredMaxBinLocalKeys and the fitted grid [64][frames].  Returns the key
// count, or -1 when keyCap is too small.
int vbtref_coarse_fit(const float* leafTemporal, int frames, int width, int height, int depth,
                      const vr_keyframe_profile* p, uint32_t* desc, uint8_t* bins, uint16_t* keyFrames,
                      float* keyValues, int keyCap, int* requiredMaxLocal, float* grid)
{
    const std::vector<float> lt(leafTemporal, leafTemporal + size_t(512) * size_t(frames));
    const DensityTemporalProfile prof = to_profile(p);
    const auto coords = controlCoords(kCoarseRes);
    BuiltControlStream stream;
    stream.data.controlCount = uint16_t(kCoarseRes * kCoarseRes * kCoarseRes);
    stream.data.timeBinCount = 8;
    std::vector<float> series(static_cast<size_t>(frames)), recon;
    for (int gz = 0; gz < kCoarseRes; ++gz)
        for (int gy = 0; gy < kCoarseRes; ++gy)
            for (int gx = 0; gx < kCoarseRes; ++gx) {
                const int ctrl = (gz * kCoarseRes + gy) * kCoarseRes + gx;
                for (int t = 0; t < frames; ++t)
                    series[size_t(t)] = sampleLeafBufferAtFractional(lt, frames, t, width, height, depth,
                                                                     coords[size_t(gx)], coords[size_t(gy)],
                                                                     coords[size_t(gz)]);
                const auto keys = detectDensityKeyFrames(series, prof, nullptr);
                appendControlSequenceToStream(stream.data, stream.requiredMaxBinLocalKeys, series, keys, frames, 8);
                reconstructFromKeys(series, keys, recon);
                for (int t = 0; t < frames; ++t) grid[size_t(ctrl) * size_t(frames) + size_t(t)] = recon[size_t(t)];
            }
    const auto& d = stream.data;
    if (int(d.keyframes.size()) > keyCap) return -1;
    for (size_t c = 0; c < d.descriptors.size(); ++c)
        desc[c] = uint32_t(d.descriptors[c].keyStart) | (uint32_t(d.descriptors[c].keyCount) << 16) |
                  (uint32_t(d.descriptors[c].reserved) << 24);
    std::memcpy(bins, d.binIndex.data(), d.binIndex.size());
    for (size_t k = 0; k < d.keyframes.size(); ++k) {
        keyFrames[k] = d.keyframes[k].frame;
        keyValues[k] = d.keyframes[k].value;
    }
    *requiredMaxLocal = stream.requiredMaxBinLocalKeys;
    return int(d.keyframes.size());
}

}  // extern "C"
