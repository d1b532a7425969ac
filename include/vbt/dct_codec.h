// vbt/dct_codec.h -- orthonormal DCT-II keep-K helpers, drop-in for the reference's
// src/dct_codec.h:7-11.  In the reference these are called only by the scientific encoder
// (src/spatial_first_encoder.cpp:1337-2959); the B200 decode path evaluates its basis from
// a host-built table instead, so these remain host functions.
#pragma once

#include <vector>

namespace vbt {

std::vector<float> dctEncodeKeep(const std::vector<float>& series, int keepCount);
std::vector<float> dctEncodeKeepWeighted(const std::vector<float>& series, const std::vector<float>& weights,
                                         int keepCount);
float dctDecodeAt(const std::vector<float>& coeffs, int totalLength, int index);

}  // namespace vbt
