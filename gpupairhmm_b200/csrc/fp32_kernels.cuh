// __global__ wrapper around Fp32Wavefront and its registration.
#pragma once

#include <type_traits>

#include "kernels.hpp"
#include "wavefront_fp32.cuh"
#include "wavefront_fp32x2.cuh"

namespace phmm {

// One kernel per configuration.  persistent = 1: every warp repeatedly takes
// the next warp task of its bucket from an atomic counter (items are sorted
// longest first, so this is longest-processing-time-first scheduling).
// persistent = 0: warp w of the grid runs task w once (one launch per
// partition, the reference's execution form).
template <int G, int R, bool MT, bool PK, bool GCP = false>
using WavefrontOf = typename std::conditional<PK, Fp32x2Wavefront<G, R>, Fp32Wavefront<G, R, MT, GCP>>::type;

// Resident CTAs per SM asked of the register allocator for configurations whose
// natural allocation sits just above an occupancy step (64-thread CTAs: 6 CTAs
// at <= 170 registers); 1 leaves the allocator free.
constexpr int fp32_min_ctas(int R, bool MT, bool PK) {
    return PK ? (R <= 10 ? 6 : 1) : (!MT && R <= 20 ? 6 : 1);
}

template <int G, int R, bool MT, bool PK, bool GCP = false>
__global__ void __launch_bounds__(kBlockThreads, fp32_min_ctas(R, MT, PK))
fp32_bucket_kernel(DevView v, const Item* __restrict__ items, const Schedule* __restrict__ s, int rank,
                   int persistent, unsigned long long* counter, float4* scratch, int64_t rows) {
    static_assert(!(MT && PK), "the packed kernel is single tile");
    static_assert(!(GCP && PK), "gcp mode runs the scalar kernel");
    using W = WavefrontOf<G, R, MT, PK, GCP>;
    extern __shared__ float4 smem[];
    float* ph = reinterpret_cast<float*>(smem);
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    float4* wtab = smem + 32 + warp * W::kTableFloat4;
    for (int i = threadIdx.x; i < 128; i += blockDim.x) ph[i] = v.ph2pr[i];
    __syncthreads();

    const long long ib = s->item_begin[rank];
    const long long ie = s->item_begin[rank + 1];
    const int per = W::NG;
    const long long ntasks = (ie - ib + per - 1) / per;
    const long long gwarp = (long long)blockIdx.x * kWarpsPerBlock + warp;
    float4* wscratch = MT ? scratch + gwarp * (long long)per * 2 * rows : nullptr;

    long long tsk = gwarp;
    while (true) {
        if (persistent) {
            unsigned long long x = 0;
            if (lane == 0) x = atomicAdd(counter, 1ull);
            tsk = (long long)__shfl_sync(kFullMask, x, 0);
        }
        if (tsk >= ntasks) break;
        const long long first = ib + tsk * per;
        const int n = (int)((ie - first) < per ? (ie - first) : per);
        if constexpr (PK) W::run(v, items + first, n, wtab, ph);
        else W::run(v, items + first, n, wtab, ph, wscratch, rows);
        if (!persistent) break;
    }
}

template <int G, int R, bool MT, bool PK, bool GCP = false>
cudaError_t launch_fp32_bucket(const Fp32LaunchArgs& a) {
    using W = WavefrontOf<G, R, MT, PK, GCP>;
    const size_t smem = (32 + (size_t)kWarpsPerBlock * W::kTableFloat4) * sizeof(float4);
    fp32_bucket_kernel<G, R, MT, PK, GCP><<<a.grid, kBlockThreads, smem, a.stream>>>(
        a.view, a.items, a.sched, a.rank, a.persistent, a.counter, static_cast<float4*>(a.scratch), a.rows);
    return cudaGetLastError();
}

template <int G, int R, bool MT, bool PK = false, bool GCP = false>
ConfigInfo make_fp32_config() {
    using W = WavefrontOf<G, R, MT, PK, GCP>;
    ConfigInfo c{};
    c.G = G;
    c.R = R;
    c.multi_tile = MT;
    c.packed = PK;
    c.gcp = GCP;
    c.smem_bytes = (32 + (size_t)kWarpsPerBlock * W::kTableFloat4) * sizeof(float4);
    c.scratch_bytes_per_row = MT ? (size_t)W::NG * 2 * sizeof(float4) : 0;
    c.kernel = reinterpret_cast<const void*>(&fp32_bucket_kernel<G, R, MT, PK, GCP>);
    c.launch = &launch_fp32_bucket<G, R, MT, PK, GCP>;
    return c;
}

}  // namespace phmm
