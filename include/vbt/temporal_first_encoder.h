// vbt/temporal_first_encoder.h -- the render-temporal route tags and the decode-relevant encoder
// options, as declared by the reference's src/temporal_first_encoder.h:15-44.  Only what the
// payload/decode API needs is declared here (the encoder itself is not part of this library).
#pragma once

#include <cstdint>

namespace vbt {

enum class TemporalFirstPackedMode : uint8_t {
    EMPTY = 0,
    TEMPORAL_GRID4 = 1,
    TEMPORAL_FINE_COMPACT = 2,   // Mode2: shell-voxel residual
    TEMPORAL_FINE6 = 3,
};

// Decode-relevant subset of the reference's TemporalFirstEncoderOptions
// (src/temporal_first_encoder.h:25-44): the fields validateRenderTemporalLeafPrefix reads and the
// packing constraints.
struct TemporalFirstEncoderOptions {
    float cutoff = 0.0f;
    float cutoffBand = 0.0f;
    float temporalEpsAbs = 1e-5f;
    float temporalEpsRel = 0.02f;
    float temporalGammaDelta = 0.2f;
    bool cutoffProtect = true;
    int timeBinCount = 8;
    int maxBinLocalKeys = 8;
    bool useGlobalOffsetTable = true;
    bool alignPayloadTo4Bytes = true;
};

const char* toString(TemporalFirstPackedMode mode);

}  // namespace vbt
