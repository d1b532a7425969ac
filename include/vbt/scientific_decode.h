// vbt/scientific_decode.h -- scientific (Grid4 DCT) decode, drop-in for the reference's
// render/src/scientific_decode.h:11-12, plus the render-temporal frame decode and batched calls.
// Despite the reference's "Cpu" names, every call here decodes on the GPU from a device copy of the
// file, kept resident between calls for the most recently used files (8 files and 2 GiB of device
// memory at most; older copies are dropped).  Each call first compares the bytes it will decode
// (header, AC scales, and the offsets and payload of every leaf it reads) with the copy and
// uploads the file again when they differ, so a VbtFile changed in place, or a new one at a freed
// one's address, decodes its current contents.  releaseDeviceCopy frees a file's copy at once.
#pragma once

#include <cstddef>
#include <cstdint>
#include <vector>

#include "query_patterns.h"
#include "vbt_file.h"

namespace vbt::render {

// decodeScientificValueAtCpu: query.leafIndex must equal leafIndexForVoxel(x, y, z) (as
// fillLeafIndices sets it; std::invalid_argument otherwise) and query.t must be a frame of the
// file (std::out_of_range otherwise; the reference reads past its per-frame tables there).
// Calls on one file from several threads run one at a time.
float decodeScientificValueAtCpu(const VbtFile& file, const Query4D& query);
std::vector<float> reconstructScientificFrameCpu(const VbtFile& file, uint32_t frameIndex);

// Batched point queries (any family): one value per query.
std::vector<float> decodeValuesGpu(const VbtFile& file, const std::vector<Query4D>& queries);
// Dense frame [z][y][x] of a render-temporal file, equal to the reference smoke bench's
// decodeFrameToDense (render/src/render_smoke_vbt_bench_main.cpp:389-452).
std::vector<float> decodeRenderTemporalFrame(const VbtFile& file, int frameIndex);

void releaseDeviceCopy(const VbtFile& file);
// Number of files that currently have a device copy.
size_t deviceCopyCount();

}  // namespace vbt::render
