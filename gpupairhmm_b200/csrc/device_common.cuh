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
//   items      32-byte work items (one or two reads x one haplotype, output
//              slots), sorted by (length bucket, haplotype length descending);
//              the FP64 pass takes 16-byte single-pair tasks.
#pragma once

#include <cfloat>
#include <cstdint>

namespace phmm {

// pairhmm_kernels.cuh:1195-1196 (eps, beta fixed on the GPU path) and :1201
// (initial scale FLT_MAX/16).
constexpr float kBeta = 0.9f;
constexpr float kEps = 0.1f;
constexpr float kScale = FLT_MAX / 16.0f;

// FP64 recompute threshold.  Each path reaches the last read row at most
// once and transitions never exceed 1, so a value's share of the result is at
// most the value itself; cells that round in the denormal range (absolute
// error <= 2^-150 each, 3 states per cell) therefore move the scaled sum S by
// at most 3*L*H*2^-150.  S >= 3*L*H*2^-127 keeps that below 2^-23 relative;
// smaller sums go to the FP64 pass.
__host__ __device__ __forceinline__ float rescue_threshold(int L, int H) {
    return 3.0f * (float)L * (float)H * 0x1p-127f;
}

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

// Work item of the FP32 pass: a unit (one read, or two reads of the same
// record and length bucket for the packed kernel) against one haplotype.
struct Item {
    int32_t read0;
    int32_t read1;  // -1 when the unit holds one read
    int32_t hap;
    int32_t pad;
    int64_t out0;   // output slot of (read0, hap)
    int64_t out1;   // output slot of (read1, hap), -1 when absent
};
static_assert(sizeof(Item) == 32, "Item must be 32 bytes");

// Where the FP64 pass's scaled tier sends the pairs beyond its range: the
// extended tier's class lists (same class offsets as the rescue lists) and
// their counts.
struct ExtList {
    Task* base;
    const long long* off;        // [kFp64Classes]
    unsigned long long* count;   // [kFp64Classes]
};

struct DevView;
__device__ __forceinline__ void append_rescue(const DevView& v, int cls, const Task& t);

struct DevView {
    const uint32_t* read_pack;
    const int64_t* read_start;  // in positions, multiple of 4
    const int32_t* read_len;
    const uint8_t* hap_code;
    const int64_t* hap_start;  // in bytes, multiple of 16
    const int32_t* hap_len;
    float* scores;
    Task* rescue_base;          // flagged pairs, one list per read-length class (fp64_class)
    const long long* rescue_off;  // [kFp64Classes] start of each class list in rescue_base
    unsigned long long* rescue_count;  // [kFp64Classes]
    int rescue_enabled;
    const float* ph2pr;         // 128 floats in global memory
    // gcp mode only (else null): the gcp quality of each read's first position,
    // clamped to 127.  eps = p(gcp), beta = 1 - eps for all of the read's pairs,
    // as the reference's CPU recurrence takes them (gpuworker.cuh:1009, 1048-1049).
    const uint8_t* read_gcp;
};

__device__ __forceinline__ uint32_t code_of(uint8_t c) {
    // utility_kernels.cuh:6-23
    return c == 'A' ? 0u : c == 'C' ? 1u : c == 'G' ? 2u : c == 'T' ? 3u : 4u;
}

__device__ __forceinline__ int min_i(int a, int b) { return a < b ? a : b; }

// FP64 pass length classes (tile = G x R): 64 = 4x16, 96 = 8x12, 128 = 8x16,
// 160 = 16x10, 192 = 16x12, 256 = 16x16, then 32x16 multi-tile for longer reads.
constexpr int kFp64Classes = 7;
constexpr int kFp64ClassMax[kFp64Classes - 1] = {64, 96, 128, 160, 192, 256};
__host__ __device__ __forceinline__ int fp64_class(int L) {
    return L <= 64 ? 0 : L <= 96 ? 1 : L <= 128 ? 2 : L <= 160 ? 3 : L <= 192 ? 4 : L <= 256 ? 5 : 6;
}

// Appends a flagged pair to its FP64 class list (rare: one global load for the
// list start).
__device__ __forceinline__ void append_rescue(const DevView& v, int cls, const Task& t) {
    const unsigned long long slot = atomicAdd(v.rescue_count + cls, 1ull);
    v.rescue_base[v.rescue_off[cls] + (long long)slot] = t;
}

}  // namespace phmm
