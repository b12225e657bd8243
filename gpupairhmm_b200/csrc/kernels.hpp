// Host-visible registry of the compiled kernel configurations.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <vector>

#include "device_common.cuh"
#include "prep_kernels.cuh"

namespace phmm {

constexpr int kBlockThreads = 64;  // 2 warps per CTA: register-bound configs reach 10 warps/SM
constexpr int kWarpsPerBlock = kBlockThreads / 32;

struct Fp32LaunchArgs {
    DevView view;
    const Item* items;
    const Schedule* sched;
    int rank;                       // bucket rank this launch serves
    int persistent;                 // 1: warps loop on an atomic task counter
    unsigned long long* counter;    // per-rank task counter (persistent)
    void* scratch;                  // multi-tile border storage
    int64_t rows;                   // border rows per buffer
    int grid;
    cudaStream_t stream;
};

struct Fp64LaunchArgs {
    DevView view;
    int cls;                         // length class (fp64_class)
    bool gcp;                        // gcp mode kernel
    bool ext;                        // extended-range tier (per-lane exponents)
    ExtList ext_list;                // scaled tier: where pairs beyond its range go
    bool fuse = false;               // multi-tile scaled tier: run the extended form in the same warp
    const Task* items;               // that class's rescue list
    const unsigned long long* count; // number of items (device)
    unsigned long long* counter;     // task counter
    void* scratch;                   // border storage (class 2 only)
    int64_t rows;
    int grid;
    cudaStream_t stream;
};

struct ConfigInfo {
    int G;
    int R;
    bool multi_tile;
    bool packed;                     // two reads per group with packed FP32 (single tile)
    bool gcp;                        // eps/beta per read (gcp mode)
    int tile() const { return G * R; }
    int per_warp() const { return 32 / G; }   // items per warp task
    size_t smem_bytes;               // dynamic shared memory per CTA
    size_t scratch_bytes_per_row;    // per warp, per border row (both buffers)
    const void* kernel;
    cudaError_t (*launch)(const Fp32LaunchArgs&);
};

// All compiled FP32 configurations.
const std::vector<ConfigInfo>& fp32_configs();
const ConfigInfo* find_fp32_config(int G, int R, bool multi_tile, bool packed = false, bool gcp = false);

// FP64 pass, one kernel per length class and tier (misc_kernels.cu): the
// scaled tier (ext = false) recomputes every flagged pair, the extended tier
// (ext = true) the pairs beyond the scaled tier's range.  gcp selects the
// gcp-mode kernels (eps/beta per read).
cudaError_t launch_fp64_rescue(const Fp64LaunchArgs& a);
size_t fp64_smem_bytes(int cls, bool ext);
size_t fp64_scratch_bytes_per_row(int cls, bool ext);  // per warp, per border row
const void* fp64_kernel(int cls, bool gcp, bool ext, bool fuse = false);
int fp64_per_warp(int cls);

// Preparation kernels.
cudaError_t launch_pack(const PrepArgs& a, int grid, cudaStream_t s);
// byte fills of n <= kFillRanges device ranges in one kernel launch
cudaError_t launch_fill(uint8_t* const* ptr, const long long* bytes, const int* value, int n, cudaStream_t s);
// FP64 class lists sorted by haplotype length (count, scan, scatter)
cudaError_t launch_rescue_sort(const RescueSortArgs& a, int grid, cudaStream_t s);
cudaError_t launch_binning(BinArgs a, int grid, cudaStream_t s, const int* per_task_dev,
                           const int* config_dev, Schedule* sched, int nranks);

// FP32 FFMA throughput probe used to measure the roofline denominator:
// `iters` dependent-chain-free FMAs per thread over grid x 256 threads.
cudaError_t launch_ffma_peak(float* out, int grid, int iters, cudaStream_t s);
// The same with double FMAs.
cudaError_t launch_dfma_peak(float* out, int grid, int iters, cudaStream_t s);

}  // namespace phmm
