// vbt_format.cuh -- VBTPACK4 leaf format, shared by host and device code of the CUDA path.
//
// Layout facts (all little-endian, byte offsets inside one leaf block):
//   word 0      packed header: route tag [1:0], coarse codec [3:2], fine codec [5:4],
//               coarse resolution [8:6], fine resolution [11:9]
//               (src/render_temporal_payload.cpp:87-107)
//   bytes 4..7  u16 coarse keyframe count, u16 fine keyframe count (render_temporal_payload.h:32-38)
//   byte 8      coarse stream: desc[C] (u16 keyStart, u8 keyCount, u8 localMax) | u8 bins[C*8] pad4
//               | keyframes pad4 (render_temporal_payload.cpp:62-78)
//   FINE6:      fine stream (C = fineRes^3, 8 bins) right after the coarse stream
//   Mode2:      80-byte occupancy (u64 mask[8], u16 groupPrefix[8]) then the shell residual
//               stream (C = popcount, 4 bins), which ends exactly at the leaf end (:234-311)
//   keyframe    codec 1: u16 frame, u16 pad, f32 value (8 B); other codecs: u8 frame, fp16 (3 B)
//               (src/render_temporal_decode.cpp:11-15, 33-77)
#pragma once
#include <cstdint>

#ifdef __CUDACC__
#define VBT_HD __host__ __device__ __forceinline__
#else
#define VBT_HD inline
#endif

namespace vbtb {

constexpr uint32_t kModeEmpty = 0, kModeGrid4 = 1, kModeFineCompact = 2, kModeFine6 = 3;
constexpr uint32_t kNoRank = 0xFFFFFFFFu;

// Status codes (same numbering as VBT_STATUS_* in include/vbt_b200.h).
enum : uint32_t {
    kOk = 0,
    kErrLeafTooSmall = 1,
    kErrPrefixMissing = 2,
    kErrLeafShort = 3,
    kErrShellOccOob = 4,
    kErrShellGroupPrefix = 5,
    kErrShellNoActive = 6,
    kErrShellResidualOob = 7,
    kErrShellTrailing = 8,
    kErrControlIndex = 9,
    kErrStreamOob = 10,
    kErrDecodeOob = 11,
    kErrKeyRangeOob = 12,
    kErrKeyIndex = 13,
    kErrWaitTimeout = 30,
    kErrUnsupported = 44,   // a leaf mode the call does not cover
};

// One 32-byte leaf-table row, written by the payload walker (kernel a) and read by every decode
// kernel, so that no decode kernel re-parses or re-validates a leaf.
struct __align__(16) LeafEntry {
    uint32_t word_off;     // payload word offset of the leaf block
    uint32_t header;       // packed header word (0 for EMPTY leaves)
    uint32_t kf;           // coarse keyframe count | fine keyframe count << 16
    uint32_t coarse_bytes; // coarse stream bytes (stream starts at byte 8)
    uint32_t fine_bytes;   // fine stream bytes (FINE6) or 80 + keyframe bytes (Mode2), at 8 + coarse_bytes
    uint32_t shell_off;    // Mode2 residual stream byte offset
    uint32_t shell_bytes;  // Mode2 residual stream bytes
    uint32_t info;         // [9:0] shell active count, [15:10] flags, [23:16] status
};
static_assert(sizeof(LeafEntry) == 32, "LeafEntry is one 32-byte sector");

// info flags
constexpr uint32_t kFlagActive = 1u << 10;    // route tag != EMPTY (page-table membership)
constexpr uint32_t kFlagFine = 1u << 11;      // decode the fine stream and add its trilinear sample
constexpr uint32_t kFlagShell = 1u << 12;     // decode the Mode2 shell residual per occupied voxel
constexpr uint32_t kFlagOccClamp = 1u << 13;  // Mode2: clamp negatives outside the occupancy to 0
constexpr uint32_t kFlagSorted = 1u << 14;    // every decoded control's key frames strictly increase
constexpr uint32_t kFlagHalfPlain = 1u << 15; // no FP16 key value of the leaf is a NaN (the hardware conversion is exact)

VBT_HD uint32_t entry_status(const LeafEntry& e) { return (e.info >> 16) & 0xFFu; }
VBT_HD uint32_t entry_shell_active(const LeafEntry& e) { return e.info & 0x3FFu; }

VBT_HD uint32_t align4(uint32_t b) { return (b + 3u) & ~3u; }
VBT_HD uint32_t key_stride(uint32_t codec) { return codec == 1u ? 8u : 3u; }

// Bytes of one control stream: desc + aligned bins + aligned keyframes, in 32-bit arithmetic as
// src/render_temporal_decode.cpp:316-326 computes them.
VBT_HD uint32_t stream_bytes(uint32_t controls, uint32_t bins, uint32_t kf, uint32_t codec)
{
    return controls * 4u + align4(controls * bins) + align4(kf * key_stride(codec));
}

// IEEE binary16 bits -> binary32, exact, including subnormals, infinities and NaN payloads
// (the same mapping as src/render_temporal_decode.cpp:167-199).
VBT_HD float half_bits_to_float(uint32_t h)
{
    const uint32_t sign = (h & 0x8000u) << 16;
    uint32_t e = (h >> 10) & 0x1Fu;
    uint32_t m = h & 0x3FFu;
    uint32_t bits;
    if (e == 0u) {
        if (m == 0u) {
            bits = sign;
        } else {
            // normalise: shift the leading one of the 10-bit mantissa up to bit 10
#ifdef __CUDA_ARCH__
            const int lz = __clz(m) - 21;   // leading zeros inside the 11-bit field
#else
            int lz = 0;
            while (((m << lz) & 0x400u) == 0u) ++lz;
#endif
            m = (m << lz) & 0x3FFu;
            bits = sign | ((uint32_t)(113 - lz) << 23) | (m << 13);
        }
    } else if (e == 31u) {
        bits = sign | 0x7F800000u | (m << 13);
    } else {
        bits = sign | ((e + 112u) << 23) | (m << 13);
    }
#ifdef __CUDA_ARCH__
    return __uint_as_float(bits);
#else
    float f;
    __builtin_memcpy(&f, &bits, 4);
    return f;
#endif
}

// Trilinear axis table: for control resolution r (2..7), leaf extent e (1..8) and voxel p (0..7):
// control indices i0, i1 and the weights t and 1-t, computed on the host exactly as
// render/src/render_smoke_vbt_bench_main.cpp:201-234 (controlCoords + locateCoord) computes them.
struct AxisWeight {
    uint8_t i0, i1, pad0, pad1;
    float t, omt;
};
constexpr int kAxisRes = 8, kAxisExt = 9, kAxisPos = 8;
VBT_HD int axis_index(int res, int ext, int p) { return (res * kAxisExt + ext) * kAxisPos + p; }

}  // namespace vbtb
