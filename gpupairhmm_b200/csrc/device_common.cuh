// Device-side data layout and constants shared by all kernels.
//
// HBM layout of a batch (written by the packing kernels in prep_kernels.cu):
//   read_pack  uint32 per read position: base code | bq<<8 | iq<<16 | dq<<24.
//              Each read starts at a multiple of 4 positions (16 bytes), so a
//              lane fetches its R positions with R/4 aligned 16-byte loads.
//   hap_code   one byte per haplotype position, codes 0..4 (A,C,G,T,N).  Each
//              haplotype starts at a multiple of 16 bytes and is padded with 4;
//              the arena ends with kHapSlack bytes of 4 so a group may read a
//              few words past the end of its haplotype.
//   tasks      16-byte work items (read, hap, output slot), sorted by
//              (length bucket, haplotype length descending).
#pragma once

#include <cfloat>
#include <cstdint>

namespace phmm {

// pairhmm_kernels.cuh:1195-1196 (eps, beta fixed on the GPU path) and :1201
// (initial scale FLT_MAX/16).
constexpr float kBeta = 0.9f;
constexpr float kEps = 0.1f;
constexpr float kScale = FLT_MAX / 16.0f;

// Scaled FP32 sums below this are treated as underflowed and recomputed in
// FP64: every cell value whose rounding could matter is then a normal float.
constexpr float kRescueThreshold = 0x1p-100f;

// The FP32 kernel divides by alpha = 1 - (delta + sigma); pairs with a smaller
// |alpha| anywhere go to the FP64 pass instead.
constexpr float kMinAlpha = 0x1p-8f;

constexpr int kHapSlack = 256;    // bytes of code-4 padding after the last haplotype
constexpr int kReadSlackPos = 2048;  // uint32 positions of padding after the last read
constexpr unsigned kFullMask = 0xffffffffu;

struct Task {
    int32_t read;  // global read index in the batch
    int32_t hap;   // global haplotype index in the batch
    int64_t out;   // output slot
};
static_assert(sizeof(Task) == 16, "Task must be 16 bytes");

struct DevView {
    const uint32_t* read_pack;
    const int64_t* read_start;  // in positions, multiple of 4
    const int32_t* read_len;
    const uint8_t* hap_code;
    const int64_t* hap_start;  // in bytes, multiple of 16
    const int32_t* hap_len;
    float* scores;
    Task* rescue[3];            // flagged pairs by read-length class (fp64_class)
    unsigned long long* rescue_count;  // [3]
    int rescue_enabled;
    const float* ph2pr;         // 128 floats in global memory
};

__device__ __forceinline__ uint32_t code_of(uint8_t c) {
    // utility_kernels.cuh:6-23
    return c == 'A' ? 0u : c == 'C' ? 1u : c == 'G' ? 2u : c == 'T' ? 3u : 4u;
}

__device__ __forceinline__ int min_i(int a, int b) { return a < b ? a : b; }

// FP64 pass classes: reads up to 64 and 128 positions run 4 and 2 pairs per
// warp (single tile); longer reads one pair per warp, multi-tile.
constexpr int kFp64ClassMax0 = 64;
constexpr int kFp64ClassMax1 = 128;
__host__ __device__ __forceinline__ int fp64_class(int L) {
    return L <= kFp64ClassMax0 ? 0 : (L <= kFp64ClassMax1 ? 1 : 2);
}

}  // namespace phmm
