// vbt/scientific_decode.h -- scientific (Grid4 DCT) decode, drop-in for the reference's
// render/src/scientific_decode.h:11-12, plus the render-temporal frame decode and batched calls.
// Despite the reference's "Cpu" names, every call here decodes on the GPU: the file is uploaded
// once and kept resident (keyed by the VbtFile object and its buffers); call
// releaseDeviceCopy(file) after modifying a VbtFile's contents in place.
#pragma once

#include <cstdint>
#include <vector>

#include "query_patterns.h"
#include "vbt_file.h"

namespace vbt::render {

// decodeScientificValueAtCpu: query.leafIndex must equal leafIndexForVoxel(x, y, z) (as
// fillLeafIndices sets it; std::invalid_argument otherwise) and query.t must be a frame of the
// file (std::out_of_range otherwise; the reference reads past its per-frame tables there).
// A device copy must not be released (releaseDeviceCopy) while another thread decodes from it.
float decodeScientificValueAtCpu(const VbtFile& file, const Query4D& query);
std::vector<float> reconstructScientificFrameCpu(const VbtFile& file, uint32_t frameIndex);

// Batched point queries (any family): one value per query.
std::vector<float> decodeValuesGpu(const VbtFile& file, const std::vector<Query4D>& queries);
// Dense frame [z][y][x] of a render-temporal file, equal to the reference smoke bench's
// decodeFrameToDense (render/src/render_smoke_vbt_bench_main.cpp:389-452).
std::vector<float> decodeRenderTemporalFrame(const VbtFile& file, int frameIndex);

void releaseDeviceCopy(const VbtFile& file);

}  // namespace vbt::render
