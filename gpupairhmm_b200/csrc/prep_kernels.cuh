// Batch preparation kernels: pack reads and haplotypes into the HBM layout
// of device_common.cuh, then build the sorted work list.
//
// Work list: every item (a unit of one or two reads of a record, placed in a
// length bucket by the host, against one haplotype) gets a bin
// (bucket rank, 4095 - min(H, 4095)) so that an exclusive scan over bins
// followed by an atomic scatter sorts the items by tile bucket (largest tiles
// first) and, inside a bucket, by haplotype length descending.  Warps of the persistent kernel then take consecutive items, so
// the groups of a warp have nearly equal haplotype lengths (little idle work)
// and the longest pairs start first (short tail).  The order of pairs with the
// same bin is not deterministic; each pair still writes its own output slot,
// so results are.
#pragma once

#include "device_common.cuh"

namespace phmm {

constexpr int kHBins = 4096;     // haplotype-length classes per bucket
constexpr int kMaxBuckets = 48;

struct PrepArgs {
    // caller arrays (device)
    const uint8_t* read_bases;
    const uint8_t* base_quals;
    const uint8_t* ins_quals;
    const uint8_t* del_quals;
    const int64_t* read_offsets;
    const int32_t* read_lengths;
    const uint8_t* hap_bases;
    const int64_t* hap_offsets;
    const int32_t* hap_lengths;
    const uint8_t* gcp_quals;       // gcp mode only (else null)
    // index arrays (device, computed on the host)
    const int32_t* read_record;     // [num_reads]
    const int32_t* read_local;      // [num_reads] read index inside its record
    const int32_t* rec_haps;        // [num_records] H
    const int64_t* rec_hap_base;    // [num_records]
    const int64_t* rec_pair_base;   // [num_records]
    const int64_t* read_start;      // [num_reads] packed start (positions)
    const int64_t* hap_start;       // [num_haps] packed start (bytes)
    int64_t num_reads;
    int64_t num_haps;
    // outputs
    uint32_t* read_pack;
    uint8_t* hap_code;
    uint8_t* read_gcp;              // [num_reads], gcp mode only (else null)
};

#ifdef PHMM_PREP_KERNELS_IMPL
__device__ __forceinline__ uint32_t pack_position(uint32_t base, uint32_t bq, uint32_t iq, uint32_t dq) {
    bq = bq > 127u ? 127u : bq;
    iq = iq > 127u ? 127u : iq;
    dq = dq > 127u ? 127u : dq;
    return code_of((uint8_t)base) | (bq << 8) | (iq << 16) | (dq << 24);
}

// Warp per read; a lane packs 4 consecutive positions and stores them as one
// 16-byte word group.  Where the four source arrays are 4-byte aligned at the
// read's offset, whole groups inside the read are read with one 4-byte load
// per array; the read's ragged end (and unaligned sources) go byte by byte.
__global__ void pack_reads_kernel(PrepArgs a) {
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int lane = threadIdx.x & 31;
    for (int64_t i = warp; i < a.num_reads; i += nwarps) {
        const int L = a.read_lengths[i];
        const int Lp = (L + 3) & ~3;
        const int64_t src = a.read_offsets[i];
        const uint8_t* rb = a.read_bases + src;
        const uint8_t* bq = a.base_quals + src;
        const uint8_t* iq = a.ins_quals + src;
        const uint8_t* dq = a.del_quals + src;
        const bool aligned = ((reinterpret_cast<uintptr_t>(rb) | reinterpret_cast<uintptr_t>(bq) |
                               reinterpret_cast<uintptr_t>(iq) | reinterpret_cast<uintptr_t>(dq)) & 3u) == 0;
        uint4* dst = reinterpret_cast<uint4*>(a.read_pack + a.read_start[i]);  // 16-byte aligned
        if (a.read_gcp && lane == 0) {
            const uint32_t g = L > 0 ? a.gcp_quals[src] : 10u;
            a.read_gcp[i] = (uint8_t)(g > 127u ? 127u : g);
        }
        for (int c = lane * 4; c < Lp; c += 128) {
            uint32_t w[4];
            if (aligned && c + 3 < L) {
                const uint32_t r4 = *reinterpret_cast<const uint32_t*>(rb + c);
                const uint32_t b4 = *reinterpret_cast<const uint32_t*>(bq + c);
                const uint32_t i4 = *reinterpret_cast<const uint32_t*>(iq + c);
                const uint32_t d4 = *reinterpret_cast<const uint32_t*>(dq + c);
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    w[j] = pack_position((r4 >> (8 * j)) & 0xffu, (b4 >> (8 * j)) & 0xffu, (i4 >> (8 * j)) & 0xffu,
                                         (d4 >> (8 * j)) & 0xffu);
            } else {
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    w[j] = c + j < L ? pack_position(rb[c + j], bq[c + j], iq[c + j], dq[c + j]) : 4u;
            }
            dst[c >> 2] = make_uint4(w[0], w[1], w[2], w[3]);
        }
    }
}

// Warp per haplotype; a lane encodes 16 consecutive positions (4-byte loads
// where the source is 4-byte aligned and the 16 positions are inside the
// haplotype) and stores them as one 16-byte word; the padding to 16 bytes is
// code 4.
__global__ void pack_haps_kernel(PrepArgs a) {
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int lane = threadIdx.x & 31;
    for (int64_t i = warp; i < a.num_haps; i += nwarps) {
        const int H = a.hap_lengths[i];
        const int Hp = (H + 15) & ~15;
        const uint8_t* hb = a.hap_bases + a.hap_offsets[i];
        const bool aligned = (reinterpret_cast<uintptr_t>(hb) & 3u) == 0;
        uint4* dst = reinterpret_cast<uint4*>(a.hap_code + a.hap_start[i]);  // 16-byte aligned
        for (int c = lane * 16; c < Hp; c += 512) {
            uint32_t w[4];
            if (aligned && c + 15 < H) {
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const uint32_t v = *reinterpret_cast<const uint32_t*>(hb + c + 4 * q);
                    w[q] = code_of(v & 0xffu) | (code_of((v >> 8) & 0xffu) << 8) | (code_of((v >> 16) & 0xffu) << 16) |
                           (code_of(v >> 24) << 24);
                }
            } else {
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    uint32_t v = 0;
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        const int cc = c + 4 * q + j;
                        v |= (cc < H ? code_of(hb[cc]) : 4u) << (8 * j);
                    }
                    w[q] = v;
                }
            }
            dst[c >> 4] = make_uint4(w[0], w[1], w[2], w[3]);
        }
    }
}

#endif  // PHMM_PREP_KERNELS_IMPL

struct BinArgs {
    const int32_t* hap_lengths;
    const int32_t* read_record;
    const int32_t* read_local;
    const int32_t* rec_haps;
    const int64_t* rec_hap_base;
    const int64_t* rec_pair_base;
    const int32_t* unit_read0;      // [num_units]
    const int32_t* unit_read1;      // [num_units], -1 for a one-read unit
    const int32_t* unit_bucket;     // [num_units]
    int64_t num_units;
    int nbuckets;
    int hbins;                      // kHBins (engine) or 1 (plain)
    const int32_t* bucket_rank;     // [nbuckets] bin-major position of each bucket
    unsigned int* hist;             // [nbuckets * hbins]
    unsigned long long* cursor;     // [nbuckets * hbins] scatter positions
    Item* items;
};

__device__ __forceinline__ int bin_of(const BinArgs& a, int bucket, int H) {
    const int hc = a.hbins > 1 ? (a.hbins - 1 - (H < a.hbins - 1 ? H : a.hbins - 1)) : 0;
    return a.bucket_rank[bucket] * a.hbins + hc;
}

#ifdef PHMM_PREP_KERNELS_IMPL
// warp-aggregated increment: lanes that hit the same counter share one atomic
template <class T>
__device__ __forceinline__ T aggregated_add(T* counter, unsigned key) {
    const unsigned active = __activemask();
    const unsigned peers = __match_any_sync(active, key);
    const int leader = __ffs(peers) - 1;
    const int lane = threadIdx.x & 31;
    T base = 0;
    if (lane == leader) base = atomicAdd(counter, (T)__popc(peers));
    base = __shfl_sync(peers, base, leader);
    return base + (T)__popc(peers & ((1u << lane) - 1u));
}

// thread per unit: histogram of (bucket, H class)
__global__ void bin_count_kernel(BinArgs a) {
    for (int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; u < a.num_units;
         u += (int64_t)gridDim.x * blockDim.x) {
        const int g = a.read_record[a.unit_read0[u]];
        const int nh = a.rec_haps[g];
        const int64_t hb = a.rec_hap_base[g];
        const int b = a.unit_bucket[u];
        for (int h = 0; h < nh; ++h) {
            const int bin = bin_of(a, b, a.hap_lengths[hb + h]);
            aggregated_add(&a.hist[bin], (unsigned)bin);
        }
    }
}

// thread per unit: scatter items into their sorted slots
__global__ void bin_scatter_kernel(BinArgs a) {
    for (int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; u < a.num_units;
         u += (int64_t)gridDim.x * blockDim.x) {
        const int r0 = a.unit_read0[u], r1 = a.unit_read1[u];
        const int g = a.read_record[r0];
        const int nh = a.rec_haps[g];
        const int64_t hb = a.rec_hap_base[g];
        const int b = a.unit_bucket[u];
        const int64_t ob0 = a.rec_pair_base[g] + (int64_t)a.read_local[r0] * nh;
        const int64_t ob1 = r1 >= 0 ? a.rec_pair_base[g] + (int64_t)a.read_local[r1] * nh : -1;
        for (int h = 0; h < nh; ++h) {
            const int bin = bin_of(a, b, a.hap_lengths[hb + h]);
            const unsigned long long pos = aggregated_add(&a.cursor[bin], (unsigned)bin);
            a.items[pos] = Item{r0, r1, (int32_t)(hb + h), 0, ob0 + h, r1 >= 0 ? ob1 + h : -1};
        }
    }
}

// Byte fills of up to kFillRanges device ranges in one launch.  Used instead of
// cudaMemsetAsync inside the captured stages: a memset node may be run by a
// copy engine, where it queues behind other streams' pending copies.
constexpr int kFillRanges = 4;
struct FillArgs {
    uint8_t* ptr[kFillRanges];
    long long bytes[kFillRanges];
    int value[kFillRanges];
};
__global__ void fill_kernel(FillArgs a) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (int k = 0; k < kFillRanges; ++k)
        for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < a.bytes[k]; i += stride)
            a.ptr[k][i] = (uint8_t)a.value[k];
}

// single-block exclusive scan of the histogram into cursor (n up to a few 1e5).
// The block is kept small (kHistScanThreads) so that it finds room on an SM
// next to the long-running blocks of another engine's kernels.
constexpr int kHistScanThreads = 256;
__global__ void __launch_bounds__(kHistScanThreads)
hist_scan_kernel(const unsigned int* hist, unsigned long long* cursor, int n) {
    __shared__ unsigned long long part[kHistScanThreads];
    const int tid = threadIdx.x;
    const int per = (n + blockDim.x - 1) / blockDim.x;
    const int b = tid * per;
    const int e = b + per < n ? b + per : n;
    unsigned long long s = 0;
    for (int i = b; i < e; ++i) s += hist[i];
    part[tid] = s;
    __syncthreads();
    if (tid == 0) {
        unsigned long long run = 0;
        for (int i = 0; i < (int)blockDim.x; ++i) { const unsigned long long x = part[i]; part[i] = run; run += x; }
    }
    __syncthreads();
    unsigned long long run = part[tid];
    for (int i = b; i < e; ++i) { cursor[i] = run; run += hist[i]; }
}

#endif  // PHMM_PREP_KERNELS_IMPL

// Per-rank item ranges and warp-task ranges for the persistent kernel.
struct Schedule {
    int nranks;
    int total_tasks_hi;                       // unused padding
    long long total_tasks;
    long long item_begin[kMaxBuckets + 1];    // by rank
    long long task_begin[kMaxBuckets + 1];    // by rank
    int per_task[kMaxBuckets];                // items per warp task, by rank
    int config[kMaxBuckets];                  // kernel config id, by rank
};

#ifdef PHMM_PREP_KERNELS_IMPL
// one thread: cursor holds bin starts (before scatter); derive the schedule
__global__ void schedule_kernel(const unsigned long long* bin_start, const unsigned int* hist, int nranks,
                                int hbins, const int* per_task, const int* config, Schedule* s) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    long long tasks = 0;
    s->nranks = nranks;
    for (int r = 0; r < nranks; ++r) {
        const long long b0 = (long long)bin_start[r * hbins];
        const long long last = (long long)bin_start[(r + 1) * hbins - 1] + hist[(r + 1) * hbins - 1];
        s->item_begin[r] = b0;
        s->task_begin[r] = tasks;
        s->per_task[r] = per_task[r];
        s->config[r] = config[r];
        const long long n = last - b0;
        tasks += (n + per_task[r] - 1) / per_task[r];
        if (r == nranks - 1) s->item_begin[nranks] = last;
    }
    s->task_begin[nranks] = tasks;
    s->total_tasks = tasks;
}
#endif  // PHMM_PREP_KERNELS_IMPL

// ---------------------------------------------------------------- FP64 list order
// The FP32 pass appends flagged pairs to the FP64 class lists in completion
// order, so the pairs of one FP64 warp task (NG of them) would have unrelated
// haplotype lengths and the warp would run as long as the longest.  A counting
// sort by haplotype length (descending, 16-position classes; longer than
// 8,175 in the last class) makes consecutive pairs alike, as the FP32 work
// list is: count, per-class scan, scatter into a second list with the same
// class offsets.
constexpr int kRescueHBins = 512;
struct RescueSortArgs {
    const Task* in;                   // class lists in append order
    Task* out;                        // the same lists, sorted
    const long long* off;             // [kFp64Classes] list starts
    const unsigned long long* count;  // [kFp64Classes] list lengths
    const int32_t* hap_len;
    unsigned int* hist;               // [kFp64Classes * kRescueHBins], zeroed before the batch
    unsigned long long* cursor;       // [kFp64Classes * kRescueHBins]
};

__device__ __forceinline__ int rescue_hbin(int H) {
    const int b = H >> 4;
    return kRescueHBins - 1 - (b < kRescueHBins - 1 ? b : kRescueHBins - 1);
}

#ifdef PHMM_PREP_KERNELS_IMPL
__global__ void rescue_count_kernel(RescueSortArgs a) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (int c = 0; c < kFp64Classes; ++c) {
        const long long n = (long long)a.count[c];
        const Task* in = a.in + a.off[c];
        for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
            const int bin = c * kRescueHBins + rescue_hbin(a.hap_len[in[i].hap]);
            aggregated_add(&a.hist[bin], (unsigned)bin);
        }
    }
}

// one warp per class: exclusive scan of its bins (16 per lane) from the list start
__global__ void __launch_bounds__(32 * kFp64Classes) rescue_scan_kernel(RescueSortArgs a) {
    constexpr int kPer = kRescueHBins / 32;
    const int c = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const unsigned int* h = a.hist + c * kRescueHBins + lane * kPer;
    unsigned long long sum = 0;
#pragma unroll
    for (int i = 0; i < kPer; ++i) sum += h[i];
    unsigned long long incl = sum;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const unsigned long long y = __shfl_up_sync(kFullMask, incl, d);
        if (lane >= d) incl += y;
    }
    unsigned long long run = (unsigned long long)a.off[c] + incl - sum;
    unsigned long long* cur = a.cursor + c * kRescueHBins + lane * kPer;
#pragma unroll
    for (int i = 0; i < kPer; ++i) {
        cur[i] = run;
        run += h[i];
    }
}

__global__ void rescue_scatter_kernel(RescueSortArgs a) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (int c = 0; c < kFp64Classes; ++c) {
        const long long n = (long long)a.count[c];
        const Task* in = a.in + a.off[c];
        for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
            const Task t = in[i];
            const int bin = c * kRescueHBins + rescue_hbin(a.hap_len[t.hap]);
            a.out[aggregated_add(&a.cursor[bin], (unsigned)bin)] = t;
        }
    }
}
#endif  // PHMM_PREP_KERNELS_IMPL

}  // namespace phmm
