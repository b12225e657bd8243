// TEST INFRASTRUCTURE ONLY -- builds into oracle/_ref/, never into the product.
//
// Exposes the reference's own CPU forward recurrence, GpuPairHMMWorker::align_host
// (gpuworker.cuh:1022-1098), and its probability table generator
// (gpuworker.cuh:473-486) behind a C ABI so the tests can pin the FP64 oracle
// against the reference's code on the same inputs.  It is compiled from the
// reference sources where they lie (see oracle/Makefile); nothing is copied.
//
// align_host and generate_ph2pr use no member state, so they are invoked on
// raw storage without running the worker's constructor (the constructor would
// need a GPU for its constant-memory upload and stream creation).
#include "gpuworker.cuh"
#include "tuningconfigs.hpp"

#include <omp.h>

#include <algorithm>
#include <new>
#include <vector>

namespace {
using RefWorker = GpuPairHMMWorker<MultiConfigGpuPairHMM<PairHMMKernelConfigsSingleTile<0>>>;

RefWorker* storage_worker() {
    alignas(RefWorker) static unsigned char storage[sizeof(RefWorker)];
    return reinterpret_cast<RefWorker*>(storage);
}

const std::vector<float>& ref_table() {
    static std::vector<float> t = storage_worker()->generate_ph2pr(128);
    return t;
}
}  // namespace

extern "C" {

// read/hap: ASCII bases; quals: Phred values (ASCII - 33).  gcp is one value
// per read, as align_host takes it (gpuworker.cuh:1030).
double ref_align_host(const unsigned char* hap, int hap_length, const unsigned char* read,
                      int read_length, const unsigned char* base_quals,
                      const unsigned char* ins_quals, const unsigned char* del_quals,
                      unsigned char gcp_qual) {
    return storage_worker()->align_host(hap, hap_length, read, read_length, base_quals,
                                        ins_quals, del_quals, gcp_qual, ref_table().data());
}

float ref_ph2pr(int q) { return ref_table()[q]; }

// The loop of processBatchCPU (gpuworker.cuh:975-1020) over the same batch
// layout as the product's C ABI: OpenMP over pairs, each pair through
// align_host, results in record/read/haplotype order.  gcp is taken per read
// from its first position, as processBatchCPU does (gpuworker.cuh:1013).
long long ref_batch_align_host(long long num_records, const int* reads_per_record, const int* haps_per_record,
                               const unsigned char* read_bases, const unsigned char* base_quals,
                               const unsigned char* ins_quals, const unsigned char* del_quals,
                               const unsigned char* gcp_quals, const long long* read_offsets,
                               const int* read_lengths, const unsigned char* hap_bases,
                               const long long* hap_offsets, const int* hap_lengths, float* out, int nthreads) {
    std::vector<long long> rp(num_records + 1, 0), hp(num_records + 1, 0), pp(num_records + 1, 0);
    for (long long g = 0; g < num_records; ++g) {
        rp[g + 1] = rp[g] + reads_per_record[g];
        hp[g + 1] = hp[g] + haps_per_record[g];
        pp[g + 1] = pp[g] + (long long)reads_per_record[g] * haps_per_record[g];
    }
    const long long n = pp[num_records];
    RefWorker* w = storage_worker();
    const float* table = ref_table().data();
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 16)
    for (long long p = 0; p < n; ++p) {
        const long long g = (long long)(std::upper_bound(pp.begin() + 1, pp.end(), p) - (pp.begin() + 1));
        const long long local = p - pp[g];
        const int H = haps_per_record[g];
        const long long r = rp[g] + local / H, h = hp[g] + local % H;
        const long long ro = read_offsets[r], ho = hap_offsets[h];
        const unsigned char gcp = gcp_quals ? gcp_quals[ro] : (unsigned char)10;
        out[p] = (float)w->align_host(hap_bases + ho, hap_lengths[h], read_bases + ro, read_lengths[r],
                                      base_quals + ro, ins_quals + ro, del_quals + ro, gcp, table);
    }
    return n;
}
}
