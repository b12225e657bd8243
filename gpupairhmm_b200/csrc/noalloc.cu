// Allocation-free forward: pairhmm_forward_pairs_noalloc.
//
// Some callers cannot allocate device memory at all: code running inside a
// host that owns every device allocation itself (a pre-sized arena, a
// framework allocator it must not bypass), or code called from a context where
// cudaMalloc/cudaFree are forbidden because they synchronise the device.  This
// entry point serves them.  The caller passes device buffers it already owns
// (read and haplotype bytes, a flat list of pairs, the score array) and the
// call allocates nothing: no cudaMalloc, no cudaFree, no allocating library
// routine, no host heap either.
//
// The kernel is a variant of the multi-tile FP32 wavefront (G = 32 lanes,
// R = 16 positions per lane, tiles of 512 read positions) that reads the
// caller's bytes directly instead of a packed copy.  Its only scratch, the
// per-warp border between read tiles, lives in kScratchBytes of statically
// allocated device memory defined below: every GPU that loads this library
// holds that much memory until the process exits.  Limits: haplotype length
// up to kMaxHapLength; any read length.  Results are FP32 only, with no FP64
// recompute of pairs whose FP32 result underflows (those return what FP32
// gives, possibly -inf, as the reference does).
//
// Every call shares the one scratch array and it keeps the last call's
// contents.  Nothing in it has to start at zero: within a pair each border row
// is written by one tile before the next tile reads it.  Calls whose work
// overlaps on the GPU (two streams, or two host threads) race on the scratch
// and must be serialised by the caller.
#include <cuda_runtime.h>

#include <atomic>
#include <cfloat>
#include <cstdint>
#include <mutex>

#include "../../include/pairhmm_b200.h"
#include "device_common.cuh"

namespace phmm {
namespace noalloc {

constexpr int kG = 32;
constexpr int kR = 16;
constexpr int kT = kG * kR;
constexpr int kMaxHapLength = 16384;
constexpr size_t kScratchBytes = size_t(64) << 20;  // 64 MiB
constexpr int kThreads = 64;                        // 2 warps per block
constexpr int kMaxDevices = 64;

// Border scratch: per resident warp, 2 buffers x rows x float4.
static __device__ __align__(256) float4 g_scratch[kScratchBytes / sizeof(float4)];

// probability table p(q) = float(10^(-q/10)) (gpuworker.cuh:473-486), in
// constant memory of this module, initialised in the module image itself: no
// upload, so a context that is torn down and created again has it too
static __constant__ float c_ph2pr[128] = {
#include "ph2pr_table.inc"
};

__device__ __forceinline__ uint32_t encode(uint8_t c) {
    return c == 'A' ? 0u : c == 'C' ? 1u : c == 'G' ? 2u : c == 'T' ? 3u : 4u;
}

__device__ __forceinline__ float ph_of(const float* ph, uint8_t q) { return ph[q > 127 ? 127 : q]; }

// One pair per warp, read tiles of kT positions, beta absorbed into I and D
// (M keeps alpha, so no division and no degenerate-alpha case):
//   M(j,c)  = lambda*(alpha_c*M(j-1,c-1) + It(j-1,c-1) + Dt(j-1,c-1))
//   It(j,c) = eps_c*It(j,c-1) + beta*delta_c*M(j,c-1)
//   Dt(j,c) = beta*sigma_c*M(j-1,c) + eps*Dt(j-1,c)
__global__ void __launch_bounds__(kThreads)
forward_pairs_kernel(const uint8_t* __restrict__ read_bases, const uint8_t* __restrict__ base_quals,
                     const uint8_t* __restrict__ ins_quals, const uint8_t* __restrict__ del_quals,
                     const uint8_t* __restrict__ hap_bases, const pairhmm_pair_t* __restrict__ pairs,
                     int64_t num_pairs, float* __restrict__ scores, float4* scratch, int64_t rows,
                     int64_t nwarps, int max_h) {
    __shared__ float ph[128];
    for (int i = threadIdx.x; i < 128; i += blockDim.x) ph[i] = c_ph2pr[i];
    __syncthreads();
    const int t = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (warp >= nwarps) return;  // the scratch holds borders for nwarps warps only
    float4* const wscr = scratch + warp * 2 * rows;

    for (int64_t pi = warp; pi < num_pairs; pi += nwarps) {  // warp-uniform
        const pairhmm_pair_t pr = pairs[pi];
        const int L = pr.read_length, H = pr.hap_length;
        if (L < 1 || H < 1 || H > max_h) {  // H beyond the declared bound would overrun the border rows
            if (t == 0) scores[pi] = NAN;
            continue;
        }
        const uint8_t* rb = read_bases + pr.read_offset;
        const uint8_t* bq = base_quals + pr.read_offset;
        const uint8_t* iq = ins_quals + pr.read_offset;
        const uint8_t* dq = del_quals + pr.read_offset;
        const uint8_t* hb = hap_bases + pr.hap_offset;
        const int ntiles = (L + kT - 1) / kT;
        const float Dbound = kBeta * (kScale / (float)H);
        double acc = 0.0;  // summed in double: up to 16384 rows of similar size
        int rlane = -1;
        for (int tile = 0; tile < ntiles; ++tile) {  // (pair loop strides by nwarps)
            const bool last = tile == ntiles - 1;
            const int p0 = tile * kT + t * kR;
            float lm[kR], lx[kR], alpha[kR], dlt[kR], sig[kR], eps[kR], M[kR], D[kR];
            uint32_t xc[kR];
#pragma unroll
            for (int r = 0; r < kR; ++r) {
                const int c = p0 + r;
                const bool in = c < L;
                const float p = in ? ph_of(ph, bq[c]) : 1.0f;
                const float d = in ? ph_of(ph, iq[c]) : 0.0f;
                const float sg = in ? ph_of(ph, dq[c]) : 0.0f;
                xc[r] = in ? encode(rb[c]) : 4u;
                lm[r] = in ? 1.0f - p : 0.0f;
                lx[r] = in ? p / 3.0f : 0.0f;
                alpha[r] = 1.0f - (d + sg);
                dlt[r] = in ? kBeta * d : (c == L ? kBeta : 0.0f);
                sig[r] = kBeta * sg;
                eps[r] = in ? kEps : 1.0f;
                M[r] = 0.f;
                D[r] = 0.f;
            }
            int t_res = 0, r_res = 0;
            if (last) {
                const int rel = L - 1 - tile * kT;
                t_res = rel / kR;
                r_res = rel - t_res * kR;
            }
            const int kg = last ? H + t_res : H + kG - 1;
            const bool res_lane = last && t == t_res;
            const bool addM = r_res == kR - 1;
            if (res_lane) rlane = t;
            float4* ein = wscr + ((tile - 1) & 1) * rows;
            float4* eout = wscr + (tile & 1) * rows;
            const bool writer = !last && t == kG - 1;
            float Ml = 0.f, Dl = 0.f, Mul = 0.f, Dul = 0.f, Iul = 0.f;
            if (t == 0 && tile == 0) { Dl = Dbound; Dul = Dbound; }
            uint32_t h = 4u;
            for (int k = 0; k <= kg; ++k) {
                uint32_t hn = __shfl_up_sync(kFullMask, h, 1);
                if (t == 0) hn = k < H ? encode(hb[k]) : 4u;
                h = hn;
                float Mdiag = Mul, Idiag = Iul, Xdiag = Iul + Dul;
#pragma unroll
                for (int r = 0; r < kR; ++r) {
                    const float lam = (xc[r] == 4u || h == 4u || xc[r] == h) ? lm[r] : lx[r];
                    const float Mold = M[r];
                    const float Dold = D[r];
                    M[r] = lam * fmaf(alpha[r], Mdiag, Xdiag);
                    D[r] = fmaf(sig[r], Mold, kEps * Dold);
                    const float In = fmaf(eps[r], Idiag, dlt[r] * Mdiag);
                    Mdiag = Mold;
                    Idiag = In;
                    Xdiag = In + Dold;
                }
                if (res_lane) {
                    float a = Idiag;
                    if (addM && k < kg) a = fmaf(kBeta, M[kR - 1], a);
                    acc += (double)a;
                }
                if (writer) {
                    const int j = k - (kG - 1);
                    if (j >= 0 && j < H) *reinterpret_cast<float2*>(eout + j) = make_float2(M[kR - 1], D[kR - 1]);
                    if (j >= 1 && j - 1 < H) reinterpret_cast<float*>(eout + (j - 1))[2] = Idiag;
                }
                Mul = Ml;
                Dul = Dl;
                Ml = __shfl_up_sync(kFullMask, M[kR - 1], 1);
                Dl = __shfl_up_sync(kFullMask, D[kR - 1], 1);
                Iul = __shfl_up_sync(kFullMask, Idiag, 1);
                if (t == 0) {
                    if (tile > 0) {
                        // the border is indexed by row and feeds the next diagonal directly
                        if (k < H) {
                            const float4 b = __ldcg(ein + k);
                            Mul = b.x;
                            Dul = b.y;
                            Iul = b.z;
                        } else {
                            Mul = 0.f;
                            Dul = 0.f;
                            Iul = 0.f;
                        }
                    } else {
                        Ml = 0.f;
                        Dl = Dbound;
                        Iul = 0.f;
                    }
                }
            }
            __syncwarp();
        }
        if (t == rlane) scores[pi] = (float)(log10(acc) - (log10((double)kScale) + log10((double)kBeta)));
    }
}

// per-device set-up: the scratch array's device address and the grid size
struct DeviceState {
    std::atomic<int> ready{0};
    std::atomic<float4*> scratch{nullptr};
    int max_warps = 0;
};
DeviceState g_state[kMaxDevices];
std::mutex g_setup_mutex;

// Runs once per device, with that device current (the caller makes it so):
// looks up the scratch array's device address (in host code the array's name
// is only a host-side stand-in) and sizes the grid from the SM count and the
// kernel's occupancy.  Nothing here allocates.
pairhmm_status_t setup(int device, DeviceState& st) {
    std::lock_guard<std::mutex> lk(g_setup_mutex);
    if (st.ready.load()) return PAIRHMM_OK;
    float4* addr = nullptr;
    if (cudaGetSymbolAddress(reinterpret_cast<void**>(&addr), g_scratch) != cudaSuccess || addr == nullptr)
        return PAIRHMM_ERR_CUDA;
    st.scratch.store(addr);
    int sms = 0, per_sm = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return PAIRHMM_ERR_CUDA;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, forward_pairs_kernel, kThreads, 0) != cudaSuccess ||
        per_sm < 1)
        per_sm = 1;
    st.max_warps = sms * per_sm * (kThreads / 32);
    st.ready.store(1);
    return PAIRHMM_OK;
}

}  // namespace noalloc
}  // namespace phmm

extern "C" pairhmm_status_t pairhmm_forward_pairs_noalloc(
    int32_t device, const uint8_t* read_bases, const uint8_t* base_quals, const uint8_t* ins_quals,
    const uint8_t* del_quals, const uint8_t* hap_bases, const pairhmm_pair_t* pairs, int64_t num_pairs,
    int32_t max_hap_length, float* scores, void* stream) {
    using namespace phmm::noalloc;
    if (num_pairs < 0 || device < 0 || device >= kMaxDevices) return PAIRHMM_ERR_INVALID_ARGUMENT;
    if (max_hap_length > kMaxHapLength) return PAIRHMM_ERR_LIMIT;  // the scratch is sized for 16384
    if (max_hap_length < 1) return PAIRHMM_ERR_INVALID_ARGUMENT;
    if (num_pairs == 0) return PAIRHMM_OK;
    if (!read_bases || !base_quals || !ins_quals || !del_quals || !hap_bases || !pairs || !scores)
        return PAIRHMM_ERR_INVALID_ARGUMENT;
    int prev = -1;
    if (cudaGetDevice(&prev) != cudaSuccess) return PAIRHMM_ERR_CUDA;
    if (prev != device && cudaSetDevice(device) != cudaSuccess) return PAIRHMM_ERR_CUDA;
    DeviceState& st = g_state[device];
    pairhmm_status_t status = st.ready.load() ? PAIRHMM_OK : setup(device, st);
    // the set-up's address is checked against a fresh lookup on every call (a
    // symbol lookup, no allocation): after the context was torn down and created
    // again the module, and the array with it, may sit elsewhere
    float4* scratch = nullptr;
    if (status == PAIRHMM_OK &&
        (cudaGetSymbolAddress(reinterpret_cast<void**>(&scratch), g_scratch) != cudaSuccess || !scratch))
        status = PAIRHMM_ERR_CUDA;
    if (status == PAIRHMM_OK && scratch != st.scratch.load()) st.scratch.store(scratch);
    if (status == PAIRHMM_OK) {
        // border rows per buffer for this call, and how many warps the scratch holds
        const int64_t rows = ((int64_t)max_hap_length + 2 * kG + 8 + 63) / 64 * 64;
        const int64_t per_warp = 2 * rows * (int64_t)sizeof(float4);
        int64_t warps = (int64_t)(kScratchBytes / (size_t)per_warp);
        if (warps > st.max_warps) warps = st.max_warps;
        if (warps > num_pairs) warps = num_pairs;
        const int64_t warps_per_block = kThreads / 32;
        const int grid = (int)((warps + warps_per_block - 1) / warps_per_block);
        // cudaLaunchKernel returns this launch's own status, so an error the caller
        // left pending is neither reported as ours nor cleared
        int max_h = max_hap_length;
        int64_t np = num_pairs;
        void* args[] = {(void*)&read_bases, (void*)&base_quals, (void*)&ins_quals, (void*)&del_quals,
                        (void*)&hap_bases, (void*)&pairs, &np, &scores, &scratch, (void*)&rows, &warps, &max_h};
        const cudaError_t le = cudaLaunchKernel(reinterpret_cast<const void*>(&forward_pairs_kernel), dim3(grid),
                                                dim3(kThreads), args, 0, static_cast<cudaStream_t>(stream));
        if (le != cudaSuccess) {
            cudaGetLastError();  // the failed launch's own error, recorded by the runtime as well
            status = PAIRHMM_ERR_CUDA;
        }
    }
    if (prev != device) cudaSetDevice(prev);
    return status;
}
