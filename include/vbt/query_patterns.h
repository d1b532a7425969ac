// vbt/query_patterns.h -- point-query records and generators, drop-in for the reference's
// render/src/query_patterns.h:11-31.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "vbt_file.h"

namespace vbt::render {

struct Query4D {
    uint32_t x = 0;
    uint32_t y = 0;
    uint32_t z = 0;
    uint32_t t = 0;
    uint32_t leafIndex = 0;
};

enum class QueryPattern {
    RandomFull,
    SameT,
    SameXYZ,
    CoherentTiles,
};

bool parseQueryPattern(const std::string& text, QueryPattern& outPattern);
std::vector<Query4D> generateQueries(const VbtFileHeader& header, QueryPattern pattern, uint32_t count, uint32_t seed);
void fillLeafIndices(const VbtFileHeader& header, std::vector<Query4D>& queries);
void sortQueriesByLeaf(std::vector<Query4D>& queries);

}  // namespace vbt::render
