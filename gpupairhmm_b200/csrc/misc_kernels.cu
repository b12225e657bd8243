// FP64 rescue kernel, preparation launchers, configuration registry and the
// FFMA throughput probe.
#include <algorithm>
#include <mutex>

#define PHMM_PREP_KERNELS_IMPL
#include "kernels.hpp"
#include "prep_kernels.cuh"
#include "wavefront_fp64.cuh"

namespace phmm {

void register_fp32_g4(std::vector<ConfigInfo>& out);
void register_fp32_g8(std::vector<ConfigInfo>& out);
void register_fp32_g16(std::vector<ConfigInfo>& out);
void register_fp32_g32(std::vector<ConfigInfo>& out);
void register_fp32_gcp(std::vector<ConfigInfo>& out);
void register_fp32_geven(std::vector<ConfigInfo>& out);

const std::vector<ConfigInfo>& fp32_configs() {
    static std::vector<ConfigInfo> all;
    static std::once_flag once;
    std::call_once(once, [] {
        register_fp32_g4(all);
        register_fp32_g8(all);
        register_fp32_g16(all);
        register_fp32_g32(all);
        register_fp32_geven(all);
        register_fp32_gcp(all);
    });
    return all;
}

const ConfigInfo* find_fp32_config(int G, int R, bool multi_tile, bool packed, bool gcp) {
    for (const auto& c : fp32_configs())
        if (c.G == G && c.R == R && c.multi_tile == multi_tile && c.packed == packed && c.gcp == gcp) return &c;
    return nullptr;
}

// ---------------------------------------------------------------- FP64 pass
// Tiles per length class.  A step's cost is mostly per lane (hand-off, scale
// conversion, renormalisation), so the single-tile classes take 12-16
// positions per lane where the registers allow (2 warps per scheduler at
// 216-255 registers beat 4 warps at 8 positions: FP64 pass of the uneven
// workload -6%, of 250-bp reads -9%); 160 keeps 16 x 10 at 168 registers.
// Multi-tile: 512-row tiles (32 x 16) halve the tiles of a long pair against
// 32 x 8 (long-read workload's FP64 pass 38.3 -> 26.9 ms; one long-read
// region's 11.5 -> 7.3 ms).  Both tiers use the same tiles: the scaled tier
// (EXT = false) takes every flagged pair, the extended tier (EXT = true) the
// few the scaled tier hands on.
template <bool EXT> using W64c0 = Fp64Wavefront<4, 16, false, false, EXT>;
template <bool EXT> using W64c1 = Fp64Wavefront<8, 12, false, false, EXT>;
template <bool EXT> using W64c2 = Fp64Wavefront<8, 16, false, false, EXT>;
template <bool EXT> using W64c3 = Fp64Wavefront<16, 10, false, false, EXT>;
template <bool EXT> using W64c4 = Fp64Wavefront<16, 12, false, false, EXT>;
template <bool EXT> using W64c5 = Fp64Wavefront<16, 16, false, false, EXT>;
template <bool EXT> using W64c6 = Fp64Wavefront<32, 16, true, false, EXT>;
static_assert(W64c0<true>::T == kFp64ClassMax[0] && W64c1<true>::T == kFp64ClassMax[1] &&
                  W64c2<true>::T == kFp64ClassMax[2] && W64c3<true>::T == kFp64ClassMax[3] &&
                  W64c4<true>::T == kFp64ClassMax[4] && W64c5<true>::T == kFp64ClassMax[5],
              "class bounds follow the tiles");

// The multi-tile class's scaled tier runs the extended form of a pair right
// after it in the same warp when the pair needs it, so the border ring and the
// scratch rows are sized for the extended form's 32-byte rows.
template <class W>
using Fp64ExtOf = Fp64Wavefront<W::G_, W::R_, W::kMT, W::kGCP, true>;
template <class W>
constexpr size_t fp64_ring_entry() { return W::kMT ? sizeof(Border64) : sizeof(typename W::Border); }

// FUSE (multi-tile scaled tier): a pair that needs the extended tier runs it
// right away in the same warp, instead of waiting in the extended tier's list
// for a launch of its own; for batches of a few long regions (one long pair is
// a long serial wavefront) that takes the second pass off their latency.
template <class W, bool FUSE>
__global__ void __launch_bounds__(kBlockThreads, W::kMinCtas)
fp64_rescue_kernel(DevView v, const Task* __restrict__ items, const unsigned long long* count,
                   unsigned long long* counter, void* scratch, int64_t rows, ExtList ext) {
    using Border = typename W::Border;
    extern __shared__ double2 smem64[];
    float* ph = reinterpret_cast<float*>(smem64);  // 128 floats = 32 double2
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    double2* wtab = smem64 + 32 + warp * W::kTableDouble2;
    char* ring_bytes = reinterpret_cast<char*>(smem64 + 32 + kWarpsPerBlock * W::kTableDouble2) +
                       (size_t)warp * W::kRing * fp64_ring_entry<W>();
    for (int i = threadIdx.x; i < 128; i += blockDim.x) ph[i] = v.ph2pr[i];
    __syncthreads();
    const unsigned long long n = *count;
    const unsigned long long ntasks = (n + W::NG - 1) / W::NG;
    const long long gwarp = (long long)blockIdx.x * kWarpsPerBlock + warp;
    char* wscratch = scratch ? static_cast<char*>(scratch) + (size_t)gwarp * rows * fp64_ring_entry<W>() : nullptr;
    while (true) {
        unsigned long long x = 0;
        if (lane == 0) x = atomicAdd(counter, 1ull);
        x = __shfl_sync(kFullMask, x, 0);
        if (x >= ntasks) break;
        const unsigned long long first = x * W::NG;
        const int ntask = (int)((n - first) < (unsigned long long)W::NG ? (n - first) : W::NG);
        const bool to_ext = W::run(v, items + first, ntask, ph, wtab, reinterpret_cast<Border*>(ring_bytes),
                                   reinterpret_cast<Border*>(wscratch), rows, ext, FUSE);
        if constexpr (FUSE) {
            if (to_ext) {  // warp-uniform: one pair per warp
                using WE = Fp64ExtOf<W>;
                __syncwarp();
                WE::run(v, items + first, ntask, ph, wtab, reinterpret_cast<typename WE::Border*>(ring_bytes),
                        reinterpret_cast<typename WE::Border*>(wscratch), rows, ext, false);
                if (lane == 0) atomicAdd(ext.count + (kFp64Classes - 1), 1ull);  // counted with the extended tier
            }
        }
    }
}

template <class W>
size_t fp64_smem_for() {
    return (32 + (size_t)kWarpsPerBlock * W::kTableDouble2) * sizeof(double2) +
           (size_t)kWarpsPerBlock * W::kRing * fp64_ring_entry<W>();
}

// gcp-mode twins of the class kernels (same tiles, eps/beta per read)
template <class W>
struct WithGcp;
template <int G, int R, bool MT, bool EXT>
struct WithGcp<Fp64Wavefront<G, R, MT, false, EXT>> {
    using type = Fp64Wavefront<G, R, MT, true, EXT>;
};

#define PHMM_FP64_DISPATCH_T(cls, X, EXPR)    \
    switch (cls) {                             \
        case 0: { using W = W64c0<X>; EXPR; }  \
        case 1: { using W = W64c1<X>; EXPR; }  \
        case 2: { using W = W64c2<X>; EXPR; }  \
        case 3: { using W = W64c3<X>; EXPR; }  \
        case 4: { using W = W64c4<X>; EXPR; }  \
        case 5: { using W = W64c5<X>; EXPR; }  \
        default: { using W = W64c6<X>; EXPR; } \
    }
#define PHMM_FP64_DISPATCH(cls, ext, EXPR)                               \
    do {                                                                 \
        if (ext) { PHMM_FP64_DISPATCH_T(cls, true, EXPR) }               \
        else { PHMM_FP64_DISPATCH_T(cls, false, EXPR) }                  \
    } while (0)

// the gcp twin has the same tables and ring, so the same shared memory
size_t fp64_smem_bytes(int cls, bool ext) { PHMM_FP64_DISPATCH(cls, ext, return fp64_smem_for<W>()); }
// one border buffer per warp, shared by all tile boundaries of its pair
size_t fp64_scratch_bytes_per_row(int cls, bool) {
    return cls == kFp64Classes - 1 ? sizeof(Border64) : 0;  // both forms of the multi-tile class
}
// the kernel of a class and tier; fuse picks the multi-tile scaled tier's fused form
template <class W>
const void* fp64_kernel_of(bool gcp, bool fuse) {
    using WG = typename WithGcp<W>::type;
    if constexpr (W::kMT && !W::kEXT) {
        if (fuse)
            return gcp ? reinterpret_cast<const void*>(&fp64_rescue_kernel<WG, true>)
                       : reinterpret_cast<const void*>(&fp64_rescue_kernel<W, true>);
    }
    return gcp ? reinterpret_cast<const void*>(&fp64_rescue_kernel<WG, false>)
               : reinterpret_cast<const void*>(&fp64_rescue_kernel<W, false>);
}
const void* fp64_kernel(int cls, bool gcp, bool ext, bool fuse) {
    PHMM_FP64_DISPATCH(cls, ext, return fp64_kernel_of<W>(gcp, fuse));
}
int fp64_per_warp(int cls) { PHMM_FP64_DISPATCH(cls, true, return W::NG); }

template <class K>
cudaError_t fp64_launch_as(const Fp64LaunchArgs& a, void* scr, size_t smem) {
    K::launch(a, scr, smem);
    return cudaGetLastError();
}
template <class W, bool FUSE>
struct Fp64Launch {
    static void launch(const Fp64LaunchArgs& a, void* scr, size_t smem) {
        fp64_rescue_kernel<W, FUSE><<<a.grid, kBlockThreads, smem, a.stream>>>(a.view, a.items, a.count, a.counter,
                                                                              scr, a.rows, a.ext_list);
    }
};
template <class W>
cudaError_t fp64_launch_of(const Fp64LaunchArgs& a, void* scr, size_t smem) {
    using WG = typename WithGcp<W>::type;
    if constexpr (W::kMT && !W::kEXT) {
        if (a.fuse)
            return a.gcp ? fp64_launch_as<Fp64Launch<WG, true>>(a, scr, smem)
                         : fp64_launch_as<Fp64Launch<W, true>>(a, scr, smem);
    }
    return a.gcp ? fp64_launch_as<Fp64Launch<WG, false>>(a, scr, smem)
                 : fp64_launch_as<Fp64Launch<W, false>>(a, scr, smem);
}

cudaError_t launch_fp64_rescue(const Fp64LaunchArgs& a) {
    void* scr = a.cls == kFp64Classes - 1 ? a.scratch : nullptr;
    const size_t smem = fp64_smem_bytes(a.cls, a.ext);
    PHMM_FP64_DISPATCH(a.cls, a.ext, return fp64_launch_of<W>(a, scr, smem));
}

// ---------------------------------------------------------------- preparation
cudaError_t launch_pack(const PrepArgs& a, int grid, cudaStream_t s) {
    // a warp per read / haplotype with every warp resident at once where the batch
    // allows: each warp's work is short, so latency is hidden by warps in flight
    auto warps_grid = [&](int64_t n) {
        const int64_t g = (n + 7) / 8;  // 8 warps per 256-thread block
        return (int)std::max<int64_t>(grid, std::min<int64_t>(g, int64_t(1) << 20));
    };
    pack_reads_kernel<<<warps_grid(a.num_reads), 256, 0, s>>>(a);
    pack_haps_kernel<<<warps_grid(a.num_haps), 256, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_fill(uint8_t* const* ptr, const long long* bytes, const int* value, int n, cudaStream_t s) {
    FillArgs a{};
    long long most = 0;
    for (int k = 0; k < kFillRanges; ++k) {
        a.ptr[k] = k < n ? ptr[k] : nullptr;
        a.bytes[k] = k < n ? bytes[k] : 0;
        a.value[k] = k < n ? value[k] : 0;
        most = a.bytes[k] > most ? a.bytes[k] : most;
    }
    if (most == 0) return cudaSuccess;
    const long long blocks = (most + 255) / 256;
    fill_kernel<<<(int)(blocks < 1024 ? blocks : 1024), 256, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_rescue_sort(const RescueSortArgs& a, int grid, cudaStream_t s) {
    rescue_count_kernel<<<grid, 256, 0, s>>>(a);
    rescue_scan_kernel<<<1, 32 * kFp64Classes, 0, s>>>(a);
    rescue_scatter_kernel<<<grid, 256, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_binning(BinArgs a, int grid, cudaStream_t s, const int* per_task_dev,
                           const int* config_dev, Schedule* sched, int nranks) {
    const int nbins = a.nbuckets * a.hbins;
    bin_count_kernel<<<grid, 256, 0, s>>>(a);
    hist_scan_kernel<<<1, kHistScanThreads, 0, s>>>(a.hist, a.cursor, nbins);
    schedule_kernel<<<1, 32, 0, s>>>(a.cursor, a.hist, nranks, a.hbins, per_task_dev, config_dev, sched);
    bin_scatter_kernel<<<grid, 256, 0, s>>>(a);
    return cudaGetLastError();
}

// ---------------------------------------------------------------- FFMA probe
// 8 independent FMA chains per thread; 2 FLOP per FMA.
__global__ void __launch_bounds__(256) ffma_peak_kernel(float* out, int iters) {
    float a0 = threadIdx.x * 1e-3f, a1 = a0 + 1.f, a2 = a0 + 2.f, a3 = a0 + 3.f;
    float a4 = a0 + 4.f, a5 = a0 + 5.f, a6 = a0 + 6.f, a7 = a0 + 7.f;
    const float b = 0.9999f, c = 1e-7f;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 16; ++u) {
            a0 = fmaf(a0, b, c); a1 = fmaf(a1, b, c); a2 = fmaf(a2, b, c); a3 = fmaf(a3, b, c);
            a4 = fmaf(a4, b, c); a5 = fmaf(a5, b, c); a6 = fmaf(a6, b, c); a7 = fmaf(a7, b, c);
        }
    }
    const float s = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
    if (s == 12345.678f) out[0] = s;  // keeps the chains live
}

cudaError_t launch_ffma_peak(float* out, int grid, int iters, cudaStream_t s) {
    ffma_peak_kernel<<<grid, 256, 0, s>>>(out, iters);
    return cudaGetLastError();
}

// The same with double FMAs (the FP64 pass's roofline denominator).
__global__ void __launch_bounds__(256) dfma_peak_kernel(float* out, int iters) {
    double a0 = threadIdx.x * 1e-3, a1 = a0 + 1.0, a2 = a0 + 2.0, a3 = a0 + 3.0;
    double a4 = a0 + 4.0, a5 = a0 + 5.0, a6 = a0 + 6.0, a7 = a0 + 7.0;
    const double b = 0.9999, c = 1e-7;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 16; ++u) {
            a0 = fma(a0, b, c); a1 = fma(a1, b, c); a2 = fma(a2, b, c); a3 = fma(a3, b, c);
            a4 = fma(a4, b, c); a5 = fma(a5, b, c); a6 = fma(a6, b, c); a7 = fma(a7, b, c);
        }
    }
    const double s = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
    if (s == 12345.678) out[0] = (float)s;  // keeps the chains live
}

cudaError_t launch_dfma_peak(float* out, int grid, int iters, cudaStream_t s) {
    dfma_peak_kernel<<<grid, 256, 0, s>>>(out, iters);
    return cudaGetLastError();
}

}  // namespace phmm
