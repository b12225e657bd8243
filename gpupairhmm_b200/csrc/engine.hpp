// Host-side engine behind the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "../../include/pairhmm_b200.h"
#include "host_upload.hpp"
#include "kernels.hpp"

namespace phmm {

// One entry of a tile table: reads with length <= max_len (and above the
// previous entry's bound) run with (G, R, multi_tile).
struct TileRule {
    int max_len;
    int G;
    int R;
    bool multi_tile;
    bool packed = false;  // two reads of a record per group, packed FP32 (single tile)
};

// Per-batch index derived on the host from the record structure.
struct BatchIndex {
    int64_t num_records = 0, num_reads = 0, num_haps = 0, num_pairs = 0, cells = 0;
    int32_t max_read_len = 0, max_hap_len = 0;
    int64_t read_bytes = 0, hap_bytes = 0;          // end of the caller's referenced byte range
    int64_t read_min = 0, hap_min = 0;              // start of that range
    int64_t pack_positions = 0, code_bytes = 0;     // packed extents
    std::vector<int32_t> read_record, read_local, rec_haps;
    std::vector<int64_t> rec_hap_base, rec_pair_base, read_start, hap_start;
    std::vector<int64_t> bucket_pairs;              // by bucket index
    std::vector<int64_t> bucket_items;              // work items (unit x haplotype) by bucket
    std::vector<int32_t> unit_read0, unit_read1, unit_bucket;  // units: 1 or 2 reads of a record
    int64_t class_pairs[kFp64Classes] = {};         // by FP64 length class (fp64_class)
    int64_t class_start[kFp64Classes] = {};         // start of each class's FP64 list
    int64_t multi_tile_pairs = 0;
};

// Sizes and referenced byte ranges of a host batch, validated (first pass,
// cheap: lets the input upload start before the index is built).
struct InputRanges {
    int64_t num_reads = 0, num_haps = 0, num_pairs = 0;
    int64_t read_min = 0, read_end = 0, hap_min = 0, hap_end = 0;
};

// Grow-only device buffer.  With a pool and a stream set (every engine
// buffer), growth is stream-ordered (cudaFreeAsync + cudaMallocFromPoolAsync
// on the engine's stream): unlike cudaFree it does not wait for the whole
// device, so one engine growing its buffers does not stall other engines'
// work (serving runs several).
struct DevBuf {
    void* ptr = nullptr;
    size_t cap = 0;
    cudaMemPool_t pool = nullptr;
    cudaStream_t stream = nullptr;
    cudaError_t ensure(size_t bytes);
    void release();
    template <class T> T* as() const { return static_cast<T*>(ptr); }
};

class Engine {
public:
    explicit Engine(const pairhmm_options_t& opts);
    ~Engine();
    Engine(const Engine&) = delete;
    Engine& operator=(const Engine&) = delete;

    pairhmm_status_t init();
    // keeps `bytes` of device memory in the engine's pool (allocated once and freed), so
    // that buffer growth up to that size maps no new memory while other work runs
    pairhmm_status_t reserve_pool(size_t bytes);
    pairhmm_status_t compute_host(const pairhmm_batch_t& b, float* scores);
    pairhmm_status_t compute_device(const pairhmm_batch_t& b, int32_t max_read_len, int32_t max_hap_len,
                                    float* scores, cudaStream_t stream);
    const pairhmm_stats_t& stats() const { return stats_; }
    const std::string& last_error() const { return last_error_; }
    pairhmm_status_t fail(pairhmm_status_t s, const std::string& msg);
    pairhmm_status_t cuda_fail(cudaError_t e, const char* what);

    // Replace the tile table of the current mode (autotuner).
    pairhmm_status_t set_tile_table(const std::vector<TileRule>& rules);
    const std::vector<TileRule>& tile_table() const { return rules_; }
    int device() const { return opts_.device; }
    bool gcp() const { return opts_.gcp != 0; }
    int64_t budget_bytes() const { return opts_.device_budget_bytes; }
    int num_sms() const { return num_sms_; }

    static pairhmm_status_t build_index(const pairhmm_batch_t& b, const std::vector<TileRule>& rules,
                                        BatchIndex& idx, std::string& err);
    // gcp: the batch must carry gcp qualities, none 0 at a read's first position
    static pairhmm_status_t scan_inputs(const pairhmm_batch_t& b, InputRanges& r, std::string& err, bool gcp);

private:
    // compute_host in two halves: everything enqueued / the wait and results
    pairhmm_status_t host_begin(const pairhmm_batch_t& b, float* scores, cudaEvent_t mark_start,
                                cudaEvent_t mark_end);
    pairhmm_status_t host_end();
    pairhmm_status_t upload_rules();
    pairhmm_status_t run_pipeline(const pairhmm_batch_t& dev_in, const BatchIndex& idx, float* d_scores,
                                  cudaStream_t s);
    struct Plan {
        int64_t rows = 0;                 // border rows per buffer
        std::vector<int> grid;            // by bucket
        std::vector<int> persistent;      // by bucket
        int fp64_grid[kFp64Classes] = {};   // by FP64 length class: scaled tier
        int fp64_ext_grid[kFp64Classes] = {};  // extended tier
        std::vector<int64_t> scratch_off;   // by bucket: multi-tile kernels run side by side
        size_t scratch_bytes = 0;
    };
    Plan make_plan(const BatchIndex& idx) const;
    // stage 0: packing + work list, 1: FP32 launches, 2: FP64 pass
    pairhmm_status_t enqueue_pipeline(const pairhmm_batch_t& dev_in, const BatchIndex& idx, const Plan& plan,
                                      float* d_scores, cudaStream_t s, int stage);
    pairhmm_status_t ensure_buffers(const BatchIndex& idx, bool host_inputs);
    pairhmm_status_t ensure_inputs(const InputRanges& r);
    pairhmm_status_t upload_index(const BatchIndex& idx, cudaStream_t s);
    int persistent_grid(const void* kernel, size_t smem) const;
    static int64_t index_bytes(const BatchIndex& x);

    pairhmm_options_t opts_;
    std::vector<TileRule> rules_;
    std::vector<const ConfigInfo*> rule_cfg_;
    int num_sms_ = 0;
    bool ready_ = false;
    cudaStream_t stream_ = nullptr;
    // the launches of one stage (bucket kernels, FP64 classes) fork onto side
    // streams so that their tails overlap and a small batch's buckets run side
    // by side; they join back into stream_ before the stage ends
    static constexpr int kSideStreams = 4;
    cudaStream_t side_[kSideStreams] = {};
    cudaEvent_t fork_ = nullptr, join_[kSideStreams] = {};
    cudaEvent_t ev0_ = nullptr, ev1_ = nullptr, ev_prep_ = nullptr, ev_fp32_ = nullptr;
    int64_t launches_ = 0, fp32_launches_ = 0;
    cudaGraphExec_t graph_exec_[3] = {nullptr, nullptr, nullptr};  // prep, FP32, FP64
    pairhmm_stats_t stats_{};
    std::string last_error_;

    // device buffers
    DevBuf ph2pr_, rules_maxlen_, rules_rank_, per_task_, config_;
    DevBuf in_read_bases_, in_bq_, in_iq_, in_dq_, in_read_off_, in_read_len_;
    DevBuf in_gq_, read_gcp_;  // gcp mode: uploaded gcp qualities, per-read gcp
    DevBuf in_hap_bases_, in_hap_off_, in_hap_len_;
    DevBuf read_record_, read_local_, rec_haps_, rec_hap_base_, rec_pair_base_, read_start_, hap_start_;
    DevBuf unit_read0_, unit_read1_, unit_bucket_;
    DevBuf read_pack_, hap_code_, hist_, cursor_, items_, rescue_, counters_, sched_, scores_, scratch_;
    DevBuf lens_tmp_, rescue_off_, rescue_ext_, rsort_;
    // host-to-device uploads (caller inputs, index) and the reused index
    HostUploader uploader_;
    BatchIndex idx_;
    // pipelined compute_host: chunks of at least kChunkPairs pairs (up to
    // kMaxChunks) alternate between this engine and its twin; only the first
    // chunk's upload is exposed (uneven workload, 10.9 M pairs: 8 chunks 185.1 ms,
    // 4 chunks 186.8 ms end to end)
    static constexpr int64_t kChunkPairs = int64_t(1) << 20;
    static constexpr int64_t kMaxChunks = 8;
    std::unique_ptr<Engine> twin_;
    cudaEvent_t span0_ = nullptr, span1_ = nullptr;
    bool pending_ = false, pend_direct_ = false;
    float* pend_scores_ = nullptr;
    int64_t pend_pairs_ = 0;
    // page-locked landing spot for the rescue counts (both FP64 tiers)
    void* host_hdr_ = nullptr;
    // device memory pool of this engine's buffers (kept, not returned to the
    // system between batches)
    cudaMemPool_t pool_ = nullptr;
    std::vector<DevBuf*> all_buffers();
};

}  // namespace phmm
