// Host-side engine: batch validation and indexing, device buffers, the
// per-batch launch sequence and its CUDA-graph replay.
//
// Launch sequence of one batch (all on one stream, replayed as one graph):
//   pack_reads / pack_haps      caller SoA -> packed HBM layout
//   bin_count, hist_scan,
//   schedule, bin_scatter       sorted work list + per-bucket task ranges
//   fp32_bucket_kernel<G,R,MT>  one launch per non-empty length bucket
//   fp64_rescue_kernel<scaled>  pairs flagged by the FP32 pass, in doubles
//   fp64_rescue_kernel<ext>     the few beyond the scaled doubles' range
// Compared with the reference executor (gpuworker.cuh:559-973) there is no
// device-to-host synchronisation inside a batch: the host derives bucket sizes
// from the record structure it already holds, and the kernels read their task
// ranges from device memory.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>
#include <thread>

#include "engine.hpp"

namespace phmm {

namespace {

constexpr int64_t kScratchBudget = int64_t(4) << 30;  // border scratch cap per batch

// Device counters of a batch (one array, zeroed by the fill kernel): bucket
// task counters, then per FP64 length class the scaled tier's list counts, the
// extended tier's list counts, and the two tiers' task counters.
constexpr int kCtrScaled = kMaxBuckets;
constexpr int kCtrExt = kMaxBuckets + kFp64Classes;
constexpr int kCtrTaskScaled = kMaxBuckets + 2 * kFp64Classes;
constexpr int kCtrTaskExt = kMaxBuckets + 3 * kFp64Classes;
constexpr int kCtrTotal = kMaxBuckets + 4 * kFp64Classes;
// multi-tile FP64 pairs up to which the two tiers run fused (about one round of
// resident warps of that class's kernel on 148 SMs)
constexpr int64_t kFuseMaxPairs = 2048;

std::vector<TileRule> engine_default_rules() {
    // Tile per read-length bucket for the persistent engine, measured on a B200
    // by gpupairhmm_b200/autotune.py (every compiled configuration timed on each
    // 16-position length class; adjacent classes with one winner merged).
    return {
#include "tuned_table.inc"
    };
}

std::vector<TileRule> plain_rules() {
    // The reference's generic single-tile table (tuningconfigs.hpp:33-57) and
    // its multi-tile configuration for longer reads (gpuworker.cuh:189-194).
    return {
        {16, 4, 4, false},     {32, 4, 8, false},     {48, 4, 12, false},    {64, 4, 16, false},
        {80, 4, 20, false},    {96, 4, 24, false},    {112, 4, 28, false},   {128, 4, 32, false},
        {160, 8, 20, false},   {192, 8, 24, false},   {224, 8, 28, false},   {256, 8, 32, false},
        {320, 16, 20, false},  {384, 16, 24, false},  {448, 16, 28, false},  {512, 16, 32, false},
        {640, 32, 20, false},  {768, 32, 24, false},  {896, 32, 28, false},  {1024, 32, 32, false},
        {1 << 30, 32, 16, true},
    };
}

std::vector<TileRule> gcp_rules() {
    // gcp mode (eps and beta per read): the scalar kernels compiled with that
    // option (fp32_gcp.cu), one per length class.
    return {
        {64, 4, 16, false},   {128, 8, 16, false},  {160, 8, 20, false},    {256, 16, 16, false},
        {512, 32, 16, false}, {1024, 32, 32, false}, {1 << 30, 32, 32, true},
    };
}

inline int64_t round_up(int64_t x, int64_t m) { return (x + m - 1) / m * m; }

int bucket_of_host(int L, const std::vector<TileRule>& rules) {
    int b = 0;
    const int nb = (int)rules.size();
    while (b < nb - 1 && L > rules[b].max_len) ++b;
    return b;
}

}  // namespace

cudaError_t DevBuf::ensure(size_t bytes) {
    if (bytes <= cap && ptr) return cudaSuccess;
    release();
    size_t want = std::max<size_t>(bytes + bytes / 4, 256);
    cudaError_t e = pool ? cudaMallocFromPoolAsync(&ptr, want, pool, stream) : cudaMalloc(&ptr, want);
    if (e != cudaSuccess) {
        ptr = nullptr;
        cap = 0;
        return e;
    }
    cap = want;
    return cudaSuccess;
}

void DevBuf::release() {
    if (ptr) {
        if (pool) cudaFreeAsync(ptr, stream);
        else cudaFree(ptr);
    }
    ptr = nullptr;
    cap = 0;
}

Engine::Engine(const pairhmm_options_t& opts) : opts_(opts) {
    rules_ = opts_.mode == PAIRHMM_MODE_PLAIN ? plain_rules() : opts_.gcp ? gcp_rules() : engine_default_rules();
}

std::vector<DevBuf*> Engine::all_buffers() {
    return {&ph2pr_, &rules_maxlen_, &rules_rank_, &per_task_, &config_, &in_read_bases_, &in_bq_,
            &in_iq_, &in_dq_, &in_read_off_, &in_read_len_, &in_hap_bases_, &in_hap_off_, &in_hap_len_,
            &read_record_, &read_local_, &rec_haps_, &rec_hap_base_, &rec_pair_base_, &read_start_,
            &hap_start_, &read_pack_, &hap_code_, &hist_, &cursor_, &items_, &rescue_, &counters_,
            &sched_, &scores_, &scratch_, &lens_tmp_, &unit_read0_, &unit_read1_, &unit_bucket_, &rescue_off_,
            &rescue_ext_, &rsort_,
            &in_gq_, &read_gcp_};
}

Engine::~Engine() {
    if (ready_) cudaSetDevice(opts_.device);
    for (cudaGraphExec_t& g : graph_exec_)
        if (g) cudaGraphExecDestroy(g);
    for (DevBuf* b : all_buffers()) b->release();
    if (stream_) cudaStreamSynchronize(stream_);
    if (pool_) cudaMemPoolDestroy(pool_);
    if (host_hdr_) cudaFreeHost(host_hdr_);
    if (ev0_) cudaEventDestroy(ev0_);
    if (ev1_) cudaEventDestroy(ev1_);
    if (ev_prep_) cudaEventDestroy(ev_prep_);
    if (ev_fp32_) cudaEventDestroy(ev_fp32_);
    for (int i = 0; i < kSideStreams; ++i) {
        if (join_[i]) cudaEventDestroy(join_[i]);
        if (side_[i]) cudaStreamDestroy(side_[i]);
    }
    if (fork_) cudaEventDestroy(fork_);
    if (span0_) cudaEventDestroy(span0_);
    if (span1_) cudaEventDestroy(span1_);
    if (stream_) cudaStreamDestroy(stream_);
}

pairhmm_status_t Engine::fail(pairhmm_status_t s, const std::string& msg) {
    last_error_ = msg;
    return s;
}

pairhmm_status_t Engine::cuda_fail(cudaError_t e, const char* what) {
    last_error_ = std::string(what) + ": " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? PAIRHMM_ERR_OUT_OF_MEMORY : PAIRHMM_ERR_CUDA;
}

#define PHMM_CUDA(call)                                   \
    do {                                                  \
        cudaError_t e_ = (call);                          \
        if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
    } while (0)

pairhmm_status_t Engine::reserve_pool(size_t bytes) {
    if (!pool_ || bytes == 0) return PAIRHMM_OK;
    PHMM_CUDA(cudaSetDevice(opts_.device));
    void* p = nullptr;
    PHMM_CUDA(cudaMallocFromPoolAsync(&p, bytes, pool_, stream_));
    PHMM_CUDA(cudaFreeAsync(p, stream_));
    PHMM_CUDA(cudaStreamSynchronize(stream_));
    return PAIRHMM_OK;
}

pairhmm_status_t Engine::init() {
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) return fail(PAIRHMM_ERR_UNSUPPORTED, "no CUDA device");
    if (opts_.device < 0 || opts_.device >= ndev) return fail(PAIRHMM_ERR_INVALID_ARGUMENT, "bad device ordinal");
    if (opts_.gcp && opts_.mode == PAIRHMM_MODE_PLAIN)
        return fail(PAIRHMM_ERR_INVALID_ARGUMENT, "gcp mode runs in the engine form, not the plain form");
    PHMM_CUDA(cudaSetDevice(opts_.device));
    cudaDeviceProp prop{};
    PHMM_CUDA(cudaGetDeviceProperties(&prop, opts_.device));
    if (prop.major < 10) return fail(PAIRHMM_ERR_UNSUPPORTED, "the kernels are built for sm_100a");
    num_sms_ = prop.multiProcessorCount;
    PHMM_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    for (int i = 0; i < kSideStreams; ++i) {
        PHMM_CUDA(cudaStreamCreateWithFlags(&side_[i], cudaStreamNonBlocking));
        PHMM_CUDA(cudaEventCreateWithFlags(&join_[i], cudaEventDisableTiming));
    }
    PHMM_CUDA(cudaEventCreateWithFlags(&fork_, cudaEventDisableTiming));
    {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = opts_.device;
        PHMM_CUDA(cudaMemPoolCreate(&pool_, &props));
        uint64_t keep = UINT64_MAX;
        PHMM_CUDA(cudaMemPoolSetAttribute(pool_, cudaMemPoolAttrReleaseThreshold, &keep));
        for (DevBuf* b : all_buffers()) {
            b->pool = pool_;
            b->stream = stream_;
        }
    }
    PHMM_CUDA(cudaMallocHost(&host_hdr_, 256));
    PHMM_CUDA(cudaEventCreate(&ev0_));
    PHMM_CUDA(cudaEventCreate(&ev1_));
    PHMM_CUDA(cudaEventCreate(&ev_prep_));
    PHMM_CUDA(cudaEventCreate(&ev_fp32_));

    // dynamic shared memory opt-in for every kernel on this device
    for (const ConfigInfo& c : fp32_configs())
        PHMM_CUDA(cudaFuncSetAttribute(c.kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)c.smem_bytes));
    for (int c = 0; c < kFp64Classes; ++c)
        for (const bool gcp : {false, true})
            for (const bool ext : {false, true})
                for (const bool fuse : {false, true})
                    PHMM_CUDA(cudaFuncSetAttribute(fp64_kernel(c, gcp, ext, fuse),
                                                   cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   (int)fp64_smem_bytes(c, ext)));

    // probability table p(q) = float(10^(-q/10)) (gpuworker.cuh:473-486)
    float table[128];
    for (int i = 0; i < 128; ++i) table[i] = (float)std::pow(10.0, (-i) / 10.0);
    PHMM_CUDA(ph2pr_.ensure(sizeof(table)));
    PHMM_CUDA(cudaMemcpy(ph2pr_.ptr, table, sizeof(table), cudaMemcpyHostToDevice));
    PHMM_CUDA(counters_.ensure(sizeof(unsigned long long) * kCtrTotal));
    // FP64 list sort: per-class histogram (uint32) then cursors (uint64)
    PHMM_CUDA(rsort_.ensure((sizeof(unsigned int) + sizeof(unsigned long long)) * kFp64Classes * kRescueHBins));
    PHMM_CUDA(sched_.ensure(sizeof(Schedule)));
    ready_ = true;
    return upload_rules();
}

pairhmm_status_t Engine::set_tile_table(const std::vector<TileRule>& rules) {
    if (twin_) {
        const pairhmm_status_t t = twin_->set_tile_table(rules);
        if (t != PAIRHMM_OK) return fail(t, twin_->last_error());
    }
    if (rules.empty() || (int)rules.size() > kMaxBuckets) return fail(PAIRHMM_ERR_INVALID_ARGUMENT, "tile table size");
    for (size_t i = 0; i < rules.size(); ++i) {
        if (rules[i].packed && rules[i].multi_tile)
            return fail(PAIRHMM_ERR_INVALID_ARGUMENT, "packed rules are single tile");
        if (!find_fp32_config(rules[i].G, rules[i].R, rules[i].multi_tile, rules[i].packed, opts_.gcp != 0))
            return fail(PAIRHMM_ERR_INVALID_ARGUMENT, "tile table names a configuration that is not compiled");
        if (i > 0 && rules[i].max_len <= rules[i - 1].max_len)
            return fail(PAIRHMM_ERR_INVALID_ARGUMENT, "tile table bounds must increase");
        if (!rules[i].multi_tile && rules[i].max_len > rules[i].G * rules[i].R)
            return fail(PAIRHMM_ERR_INVALID_ARGUMENT, "single-tile rule shorter than its bucket");
    }
    if (!rules.back().multi_tile) return fail(PAIRHMM_ERR_INVALID_ARGUMENT, "last rule must be multi-tile");
    rules_ = rules;
    for (cudaGraphExec_t& g : graph_exec_) {
        if (g) cudaGraphExecDestroy(g);
        g = nullptr;
    }
    return ready_ ? upload_rules() : PAIRHMM_OK;
}

pairhmm_status_t Engine::upload_rules() {
    const int nb = (int)rules_.size();
    rule_cfg_.assign(nb, nullptr);
    std::vector<int32_t> maxlen(nb), rank(nb), per(nb), cfg(nb);
    for (int b = 0; b < nb; ++b) {
        rule_cfg_[b] =
            find_fp32_config(rules_[b].G, rules_[b].R, rules_[b].multi_tile, rules_[b].packed, opts_.gcp != 0);
        if (!rule_cfg_[b]) return fail(PAIRHMM_ERR_INVALID_ARGUMENT, "tile rule without compiled kernel");
        maxlen[b] = rules_[b].max_len;
        rank[b] = opts_.mode == PAIRHMM_MODE_PLAIN ? b : nb - 1 - b;
    }
    for (int b = 0; b < nb; ++b) {
        per[rank[b]] = rule_cfg_[b]->per_warp();
        cfg[rank[b]] = b;
    }
    PHMM_CUDA(rules_maxlen_.ensure(sizeof(int32_t) * nb));
    PHMM_CUDA(rules_rank_.ensure(sizeof(int32_t) * nb));
    PHMM_CUDA(per_task_.ensure(sizeof(int32_t) * nb));
    PHMM_CUDA(config_.ensure(sizeof(int32_t) * nb));
    PHMM_CUDA(cudaMemcpy(rules_maxlen_.ptr, maxlen.data(), sizeof(int32_t) * nb, cudaMemcpyHostToDevice));
    PHMM_CUDA(cudaMemcpy(rules_rank_.ptr, rank.data(), sizeof(int32_t) * nb, cudaMemcpyHostToDevice));
    PHMM_CUDA(cudaMemcpy(per_task_.ptr, per.data(), sizeof(int32_t) * nb, cudaMemcpyHostToDevice));
    PHMM_CUDA(cudaMemcpy(config_.ptr, cfg.data(), sizeof(int32_t) * nb, cudaMemcpyHostToDevice));
    return PAIRHMM_OK;
}

pairhmm_status_t Engine::build_index(const pairhmm_batch_t& b, const std::vector<TileRule>& rules, BatchIndex& x,
                                     std::string& err) {
    // Scalars reset; vectors keep their storage between calls (an engine
    // reuses one index, so a batch of the same size touches no fresh pages).
    x.num_records = x.num_reads = x.num_haps = x.num_pairs = x.cells = 0;
    x.max_read_len = x.max_hap_len = 0;
    x.read_bytes = x.hap_bytes = x.read_min = x.hap_min = 0;
    x.pack_positions = x.code_bytes = 0;
    x.multi_tile_pairs = 0;
    for (int64_t& c : x.class_pairs) c = 0;
    for (int64_t& c : x.class_start) c = 0;
    x.unit_read0.clear();
    x.unit_read1.clear();
    x.unit_bucket.clear();
    x.bucket_pairs.assign(rules.size(), 0);
    x.bucket_items.assign(rules.size(), 0);
    if (b.num_records < 0) { err = "num_records < 0"; return PAIRHMM_ERR_INVALID_ARGUMENT; }
    x.num_records = b.num_records;
    if (b.num_records == 0) return PAIRHMM_OK;
    if (!b.reads_per_record || !b.haps_per_record) { err = "null record arrays"; return PAIRHMM_ERR_INVALID_ARGUMENT; }
    x.rec_haps.resize(b.num_records);
    x.rec_hap_base.resize(b.num_records);
    x.rec_pair_base.resize(b.num_records);
    for (int64_t g = 0; g < b.num_records; ++g) {
        const int32_t R = b.reads_per_record[g], H = b.haps_per_record[g];
        if (R < 0 || H < 0) { err = "negative reads/haplotypes in a record"; return PAIRHMM_ERR_INVALID_ARGUMENT; }
        x.rec_haps[g] = H;
        x.rec_hap_base[g] = x.num_haps;
        x.rec_pair_base[g] = x.num_pairs;
        x.num_reads += R;
        x.num_haps += H;
        x.num_pairs += (int64_t)R * H;
    }
    if (x.num_reads >= (int64_t(1) << 31) || x.num_haps >= (int64_t(1) << 31)) {
        err = "more than 2^31-1 reads or haplotypes in one batch";
        return PAIRHMM_ERR_INVALID_ARGUMENT;
    }
    if ((x.num_reads && (!b.read_lengths)) || (x.num_haps && !b.hap_lengths)) {
        err = "null length arrays";
        return PAIRHMM_ERR_INVALID_ARGUMENT;
    }
    x.read_record.resize(x.num_reads);
    x.read_local.resize(x.num_reads);
    x.read_start.resize(x.num_reads);
    x.hap_start.resize(x.num_haps);
    x.unit_read0.reserve(x.num_reads);
    x.unit_read1.reserve(x.num_reads);
    x.unit_bucket.reserve(x.num_reads);

    // bucket of every read length up to the longest finite rule, by table
    const int nb = (int)rules.size();
    int lut_max = 0;
    for (const TileRule& r : rules)
        if (r.max_len < (1 << 20)) lut_max = std::max(lut_max, r.max_len);
    std::vector<uint8_t> lut((size_t)lut_max + 1);
    for (int L = 0, bk = 0; L <= lut_max; ++L) {
        while (bk < nb - 1 && L > rules[bk].max_len) ++bk;
        lut[L] = (uint8_t)bk;
    }
    std::vector<uint8_t> packed(nb), multi(nb);
    for (int k = 0; k < nb; ++k) {
        packed[k] = rules[k].packed;
        multi[k] = rules[k].multi_tile;
    }

    // haplotypes: extents, packed starts, per-record length sums
    std::vector<int64_t> rec_hap_sum(b.num_records);
    {
        int64_t h = 0;
        for (int64_t g = 0; g < b.num_records; ++g) {
            int64_t sh = 0;
            for (int32_t k = 0; k < x.rec_haps[g]; ++k, ++h) {
                const int32_t H = b.hap_lengths[h];
                if (H < 1) { err = "haplotype length < 1"; return PAIRHMM_ERR_INVALID_ARGUMENT; }
                if (b.hap_offsets) {
                    const int64_t o = b.hap_offsets[h];
                    if (o < 0) { err = "negative haplotype offset"; return PAIRHMM_ERR_INVALID_ARGUMENT; }
                    x.hap_bytes = std::max<int64_t>(x.hap_bytes, o + H);
                    x.hap_min = h == 0 ? o : std::min<int64_t>(x.hap_min, o);
                }
                x.max_hap_len = std::max(x.max_hap_len, H);
                x.hap_start[h] = x.code_bytes;
                x.code_bytes += round_up(H, 16);
                sh += H;
            }
            rec_hap_sum[g] = sh;
        }
    }

    // reads, one record at a time: record/local index, packed start, bucket
    // counts, and units -- reads of a record in the same bucket, paired when
    // the bucket's kernel is packed (order inside a record does not matter:
    // output slots are per read); cells = sum over records of
    // (sum L) * (sum H) (gpuworker.cuh:495-520)
    std::vector<int32_t> pending(nb, -1);
    std::vector<int> touched;
    touched.reserve(nb);
    int64_t i = 0;
    for (int64_t g = 0; g < b.num_records; ++g) {
        const int64_t H = x.rec_haps[g];
        const int32_t R = b.reads_per_record[g];
        int64_t sl = 0;
        touched.clear();
        for (int32_t r = 0; r < R; ++r, ++i) {
            const int32_t L = b.read_lengths[i];
            if (L < 1) { err = "read length < 1"; return PAIRHMM_ERR_INVALID_ARGUMENT; }
            if (b.read_offsets) {
                const int64_t o = b.read_offsets[i];
                if (o < 0) { err = "negative read offset"; return PAIRHMM_ERR_INVALID_ARGUMENT; }
                x.read_bytes = std::max<int64_t>(x.read_bytes, o + L);
                x.read_min = i == 0 ? o : std::min<int64_t>(x.read_min, o);
            }
            x.max_read_len = std::max(x.max_read_len, L);
            x.read_record[i] = (int32_t)g;
            x.read_local[i] = r;
            x.read_start[i] = x.pack_positions;
            x.pack_positions += round_up(L, 4);
            sl += L;
            const int bk = L <= lut_max ? lut[L] : bucket_of_host(L, rules);
            x.bucket_pairs[bk] += H;
            x.class_pairs[fp64_class(L)] += H;
            if (multi[bk]) x.multi_tile_pairs += H;
            if (packed[bk]) {
                if (pending[bk] < 0) {
                    pending[bk] = (int32_t)i;
                    touched.push_back(bk);
                    continue;
                }
                x.unit_read0.push_back(pending[bk]);
                x.unit_read1.push_back((int32_t)i);
                pending[bk] = -1;
            } else {
                x.unit_read0.push_back((int32_t)i);
                x.unit_read1.push_back(-1);
            }
            x.unit_bucket.push_back(bk);
            x.bucket_items[bk] += H;
        }
        for (int bk : touched)
            if (pending[bk] >= 0) {
                x.unit_read0.push_back(pending[bk]);
                x.unit_read1.push_back(-1);
                x.unit_bucket.push_back(bk);
                x.bucket_items[bk] += H;
                pending[bk] = -1;
            }
        x.cells += sl * rec_hap_sum[g];
    }
    {
        int64_t off = 0;
        for (int c = 0; c < kFp64Classes; ++c) {
            x.class_start[c] = off;
            off += x.class_pairs[c];
        }
    }
    return PAIRHMM_OK;
}

pairhmm_status_t Engine::scan_inputs(const pairhmm_batch_t& b, InputRanges& r, std::string& err, bool gcp) {
    r = InputRanges{};
    if (b.num_records < 0) { err = "num_records < 0"; return PAIRHMM_ERR_INVALID_ARGUMENT; }
    if (b.num_records == 0) return PAIRHMM_OK;
    if (!b.reads_per_record || !b.haps_per_record) { err = "null record arrays"; return PAIRHMM_ERR_INVALID_ARGUMENT; }
    for (int64_t g = 0; g < b.num_records; ++g) {
        const int32_t R = b.reads_per_record[g], H = b.haps_per_record[g];
        if (R < 0 || H < 0) { err = "negative reads/haplotypes in a record"; return PAIRHMM_ERR_INVALID_ARGUMENT; }
        r.num_reads += R;
        r.num_haps += H;
        r.num_pairs += (int64_t)R * H;
    }
    if (r.num_reads >= (int64_t(1) << 31) || r.num_haps >= (int64_t(1) << 31)) {
        err = "more than 2^31-1 reads or haplotypes in one batch";
        return PAIRHMM_ERR_INVALID_ARGUMENT;
    }
    if (r.num_reads > 0 && (!b.read_lengths || !b.read_offsets || !b.read_bases || !b.base_quals || !b.ins_quals ||
                            !b.del_quals)) {
        err = "null read arrays";
        return PAIRHMM_ERR_INVALID_ARGUMENT;
    }
    if (r.num_haps > 0 && (!b.hap_lengths || !b.hap_offsets || !b.hap_bases)) {
        err = "null haplotype arrays";
        return PAIRHMM_ERR_INVALID_ARGUMENT;
    }
    if (gcp && r.num_reads > 0 && !b.gcp_quals) {
        err = "gcp mode needs the gcp quality array";
        return PAIRHMM_ERR_INVALID_ARGUMENT;
    }
    for (int64_t i = 0; i < r.num_reads; ++i) {
        const int32_t L = b.read_lengths[i];
        const int64_t o = b.read_offsets[i];
        if (L < 1) { err = "read length < 1"; return PAIRHMM_ERR_INVALID_ARGUMENT; }
        if (o < 0) { err = "negative read offset"; return PAIRHMM_ERR_INVALID_ARGUMENT; }
        if (gcp && b.gcp_quals[o] == 0) {
            err = "gcp quality 0 (eps = 1, beta = 0) has no gap-to-match transition to rescale by";
            return PAIRHMM_ERR_INVALID_ARGUMENT;
        }
        r.read_min = i == 0 ? o : std::min(r.read_min, o);
        r.read_end = std::max(r.read_end, o + L);
    }
    for (int64_t h = 0; h < r.num_haps; ++h) {
        const int32_t H = b.hap_lengths[h];
        const int64_t o = b.hap_offsets[h];
        if (H < 1) { err = "haplotype length < 1"; return PAIRHMM_ERR_INVALID_ARGUMENT; }
        if (o < 0) { err = "negative haplotype offset"; return PAIRHMM_ERR_INVALID_ARGUMENT; }
        r.hap_min = h == 0 ? o : std::min(r.hap_min, o);
        r.hap_end = std::max(r.hap_end, o + H);
    }
    return PAIRHMM_OK;
}

pairhmm_status_t Engine::ensure_inputs(const InputRanges& r) {
    const int64_t nr = std::max<int64_t>(r.num_reads, 1), nh = std::max<int64_t>(r.num_haps, 1);
    const int64_t rb = std::max<int64_t>(r.read_end - r.read_min, 1);
    const int64_t hb = std::max<int64_t>(r.hap_end - r.hap_min, 1);
    PHMM_CUDA(in_read_bases_.ensure(rb));
    PHMM_CUDA(in_bq_.ensure(rb));
    PHMM_CUDA(in_iq_.ensure(rb));
    PHMM_CUDA(in_dq_.ensure(rb));
    if (opts_.gcp) PHMM_CUDA(in_gq_.ensure(rb));
    PHMM_CUDA(in_read_off_.ensure(8 * nr));
    PHMM_CUDA(in_read_len_.ensure(4 * nr));
    PHMM_CUDA(in_hap_bases_.ensure(hb));
    PHMM_CUDA(in_hap_off_.ensure(8 * nh));
    PHMM_CUDA(in_hap_len_.ensure(4 * nh));
    PHMM_CUDA(scores_.ensure(4 * std::max<int64_t>(r.num_pairs, 1)));
    return PAIRHMM_OK;
}

pairhmm_status_t Engine::ensure_buffers(const BatchIndex& x, bool host_inputs) {
    const int64_t nr = std::max<int64_t>(x.num_reads, 1), nh = std::max<int64_t>(x.num_haps, 1);
    const int64_t ng = std::max<int64_t>(x.num_records, 1), np = std::max<int64_t>(x.num_pairs, 1);
    if (host_inputs) {
        const int64_t rb = std::max<int64_t>(x.read_bytes - x.read_min, 1);
        const int64_t hb = std::max<int64_t>(x.hap_bytes - x.hap_min, 1);
        PHMM_CUDA(in_read_bases_.ensure(rb));
        PHMM_CUDA(in_bq_.ensure(rb));
        PHMM_CUDA(in_iq_.ensure(rb));
        PHMM_CUDA(in_dq_.ensure(rb));
        if (opts_.gcp) PHMM_CUDA(in_gq_.ensure(rb));
        PHMM_CUDA(in_read_off_.ensure(8 * nr));
        PHMM_CUDA(in_read_len_.ensure(4 * nr));
        PHMM_CUDA(in_hap_bases_.ensure(hb));
        PHMM_CUDA(in_hap_off_.ensure(8 * nh));
        PHMM_CUDA(in_hap_len_.ensure(4 * nh));
        PHMM_CUDA(scores_.ensure(4 * np));
    }
    PHMM_CUDA(read_record_.ensure(4 * nr));
    PHMM_CUDA(read_local_.ensure(4 * nr));
    if (opts_.gcp) PHMM_CUDA(read_gcp_.ensure(nr));
    PHMM_CUDA(rec_haps_.ensure(4 * ng));
    PHMM_CUDA(rec_hap_base_.ensure(8 * ng));
    PHMM_CUDA(rec_pair_base_.ensure(8 * ng));
    PHMM_CUDA(read_start_.ensure(8 * nr));
    PHMM_CUDA(unit_read0_.ensure(4 * nr));
    PHMM_CUDA(unit_read1_.ensure(4 * nr));
    PHMM_CUDA(unit_bucket_.ensure(4 * nr));
    PHMM_CUDA(hap_start_.ensure(8 * nh));
    PHMM_CUDA(read_pack_.ensure(4 * (x.pack_positions + kReadSlackPos)));
    PHMM_CUDA(hap_code_.ensure(x.code_bytes + kHapSlack));
    const int64_t nbins = (int64_t)rules_.size() * (opts_.mode == PAIRHMM_MODE_PLAIN ? 1 : kHBins);
    PHMM_CUDA(hist_.ensure(4 * nbins));
    PHMM_CUDA(cursor_.ensure(8 * nbins));
    PHMM_CUDA(items_.ensure(sizeof(Item) * np));
    PHMM_CUDA(rescue_.ensure(sizeof(Task) * np));  // class lists laid out back to back
    PHMM_CUDA(rescue_ext_.ensure(sizeof(Task) * np));  // the extended tier's, same offsets
    PHMM_CUDA(rescue_off_.ensure(sizeof(int64_t) * kFp64Classes));
    return PAIRHMM_OK;
}

pairhmm_status_t Engine::upload_index(const BatchIndex& x, cudaStream_t s) {
    const std::vector<HostUploader::Copy> copies = {
        {read_record_.ptr, x.read_record.data(), 4 * x.read_record.size()},
        {read_local_.ptr, x.read_local.data(), 4 * x.read_local.size()},
        {rec_haps_.ptr, x.rec_haps.data(), 4 * x.rec_haps.size()},
        {rec_hap_base_.ptr, x.rec_hap_base.data(), 8 * x.rec_hap_base.size()},
        {rec_pair_base_.ptr, x.rec_pair_base.data(), 8 * x.rec_pair_base.size()},
        {read_start_.ptr, x.read_start.data(), 8 * x.read_start.size()},
        {hap_start_.ptr, x.hap_start.data(), 8 * x.hap_start.size()},
        {unit_read0_.ptr, x.unit_read0.data(), 4 * x.unit_read0.size()},
        {unit_read1_.ptr, x.unit_read1.data(), 4 * x.unit_read1.size()},
        {unit_bucket_.ptr, x.unit_bucket.data(), 4 * x.unit_bucket.size()},
        {rescue_off_.ptr, x.class_start, sizeof(x.class_start)},
    };
    PHMM_CUDA(uploader_.run(opts_.device, copies, s));
    return PAIRHMM_OK;
}

int64_t Engine::index_bytes(const BatchIndex& x) {
    return 4 * (int64_t)(x.read_record.size() + x.read_local.size() + x.rec_haps.size() + x.unit_read0.size() +
                         x.unit_read1.size() + x.unit_bucket.size()) +
           8 * (int64_t)(x.rec_hap_base.size() + x.rec_pair_base.size() + x.read_start.size() + x.hap_start.size());
}

int Engine::persistent_grid(const void* kernel, size_t smem) const {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kBlockThreads, smem) != cudaSuccess ||
        per_sm < 1)
        per_sm = 1;
    return per_sm * num_sms_;
}

pairhmm_status_t Engine::enqueue_pipeline(const pairhmm_batch_t& in, const BatchIndex& x, const Plan& plan,
                                          float* d_scores, cudaStream_t s, int stage) {
    const int nb = (int)rules_.size();
    const bool plain = opts_.mode == PAIRHMM_MODE_PLAIN;
    const int prep_grid = 4 * num_sms_;

    PrepArgs pa{};
    pa.read_bases = in.read_bases;
    pa.base_quals = in.base_quals;
    pa.ins_quals = in.ins_quals;
    pa.del_quals = in.del_quals;
    pa.read_offsets = in.read_offsets;
    pa.read_lengths = in.read_lengths;
    pa.hap_bases = in.hap_bases;
    pa.hap_offsets = in.hap_offsets;
    pa.hap_lengths = in.hap_lengths;
    pa.gcp_quals = opts_.gcp ? in.gcp_quals : nullptr;
    pa.read_gcp = opts_.gcp ? read_gcp_.as<uint8_t>() : nullptr;
    pa.read_record = read_record_.as<int32_t>();
    pa.read_local = read_local_.as<int32_t>();
    pa.rec_haps = rec_haps_.as<int32_t>();
    pa.rec_hap_base = rec_hap_base_.as<int64_t>();
    pa.rec_pair_base = rec_pair_base_.as<int64_t>();
    pa.read_start = read_start_.as<int64_t>();
    pa.hap_start = hap_start_.as<int64_t>();
    pa.num_reads = x.num_reads;
    pa.num_haps = x.num_haps;
    pa.read_pack = read_pack_.as<uint32_t>();
    pa.hap_code = hap_code_.as<uint8_t>();
    if (stage == 0) {
    launches_ = 0;
    fp32_launches_ = 0;
    // zero the histogram and the work/rescue counters, pad the haplotype codes
    // (a kernel, not memset nodes: see launch_fill)
    {
        uint8_t* const ptr[4] = {hap_code_.as<uint8_t>() + x.code_bytes, hist_.as<uint8_t>(),
                                 counters_.as<uint8_t>(), rsort_.as<uint8_t>()};
        const long long bytes[4] = {kHapSlack, (long long)sizeof(unsigned int) * nb * (plain ? 1 : kHBins),
                                    (long long)sizeof(unsigned long long) * kCtrTotal,
                                    (long long)sizeof(unsigned int) * kFp64Classes * kRescueHBins};
        const int value[4] = {4, 0, 0, 0};
        PHMM_CUDA(launch_fill(ptr, bytes, value, 4, s));
        launches_ += 1;
    }
    PHMM_CUDA(launch_pack(pa, prep_grid, s));
    launches_ += 2;
    }

    BinArgs ba{};
    ba.hap_lengths = in.hap_lengths;
    ba.read_record = pa.read_record;
    ba.read_local = pa.read_local;
    ba.rec_haps = pa.rec_haps;
    ba.rec_hap_base = pa.rec_hap_base;
    ba.rec_pair_base = pa.rec_pair_base;
    ba.unit_read0 = unit_read0_.as<int32_t>();
    ba.unit_read1 = unit_read1_.as<int32_t>();
    ba.unit_bucket = unit_bucket_.as<int32_t>();
    ba.num_units = (int64_t)x.unit_read0.size();
    ba.nbuckets = nb;
    ba.hbins = plain ? 1 : kHBins;
    ba.bucket_rank = rules_rank_.as<int32_t>();
    ba.hist = hist_.as<unsigned int>();
    ba.cursor = cursor_.as<unsigned long long>();
    ba.items = items_.as<Item>();
    if (stage == 0) {
    PHMM_CUDA(launch_binning(ba, prep_grid, s, per_task_.as<int>(), config_.as<int>(), sched_.as<Schedule>(), nb));
    launches_ += 4;
    return PAIRHMM_OK;
    }

    unsigned long long* counters = counters_.as<unsigned long long>();
    DevView v{};
    v.read_pack = pa.read_pack;
    v.read_start = pa.read_start;
    v.read_len = in.read_lengths;
    v.hap_code = pa.hap_code;
    v.hap_start = pa.hap_start;
    v.hap_len = in.hap_lengths;
    v.scores = d_scores;
    v.rescue_base = rescue_.as<Task>();
    v.rescue_off = rescue_off_.as<long long>();
    v.rescue_count = counters + kCtrScaled;
    v.rescue_enabled = (!plain && opts_.fp64_rescue) ? 1 : 0;
    v.ph2pr = ph2pr_.as<float>();
    v.read_gcp = pa.read_gcp;

    // FP64 pass: first sort each class's list by haplotype length into the
    // work-item buffer (free once the FP32 stage is done), same class offsets
    Task* const fp64_lists = items_.as<Task>();
    int64_t fp64_upper = 0;  // pairs the FP64 lists could hold
    for (int c = 0; c < kFp64Classes; ++c) fp64_upper += x.class_pairs[c];
    if (stage == 2 && fp64_upper > 0) {
        const int64_t upper = fp64_upper;
        RescueSortArgs ra{};
        ra.in = rescue_.as<Task>();
        ra.out = fp64_lists;
        ra.off = rescue_off_.as<long long>();
        ra.count = counters + kCtrScaled;
        ra.hap_len = in.hap_lengths;
        ra.hist = rsort_.as<unsigned int>();
        ra.cursor = reinterpret_cast<unsigned long long*>(rsort_.as<unsigned int>() + kFp64Classes * kRescueHBins);
        const int sort_grid = (int)std::max<int64_t>(1, std::min<int64_t>((upper + 255) / 256, 8 * (int64_t)num_sms_));
        PHMM_CUDA(launch_rescue_sort(ra, sort_grid, s));
        launches_ += 3;
    }

    // engine form: the stage's launches go round-robin onto the side streams
    // (forked from s, joined back below); the plain form keeps one stream
    const bool fork = !plain;
    int nlaunch = 0;
    auto next_stream = [&]() { return fork ? side_[nlaunch++ % kSideStreams] : s; };
    if (fork) {
        PHMM_CUDA(cudaEventRecord(fork_, s));
        for (int i = 0; i < kSideStreams; ++i) PHMM_CUDA(cudaStreamWaitEvent(side_[i], fork_, 0));
    }
    if (stage == 1) {
        for (int rank = 0; rank < nb; ++rank) {
            const int b = plain ? rank : nb - 1 - rank;
            if (x.bucket_items[b] == 0) continue;
            const ConfigInfo* c = rule_cfg_[b];
            Fp32LaunchArgs la{};
            la.view = v;
            la.items = items_.as<Item>();
            la.sched = sched_.as<Schedule>();
            la.rank = rank;
            la.persistent = plan.persistent[b];
            la.counter = counters + rank;
            la.scratch = static_cast<char*>(scratch_.ptr) + plan.scratch_off[b];
            la.rows = plan.rows;
            la.grid = plan.grid[b];
            la.stream = next_stream();
            PHMM_CUDA(c->launch(la));
            ++launches_;
            ++fp32_launches_;
        }
    } else {
        // stage 2: FP64 pass over flagged pairs (FP32 underflow, or degenerate alpha):
        // per length class the scaled tier, then on the same stream the extended
        // tier over the pairs the scaled tier handed on (for the multi-tile class of
        // a small batch, inside the scaled tier's launch); only the last class uses
        // the border scratch (the two tiers of a class run in turn, so they share it)
        const ExtList ext{rescue_ext_.as<Task>(), rescue_off_.as<long long>(), counters + kCtrExt};
        // a few long pairs (at most a round of resident warps): the multi-tile scaled tier
        // runs a pair's extended form right after it in the same warp, so the batch waits
        // for one pass instead of two
        const bool fuse_mt = x.class_pairs[kFp64Classes - 1] <= kFuseMaxPairs;
        for (int c = 0; c < kFp64Classes; ++c) {
            if (x.class_pairs[c] == 0) continue;
            const cudaStream_t sc = next_stream();
            const bool fuse = fuse_mt && c == kFp64Classes - 1;
            for (const bool tier_ext : {false, true}) {
                if (tier_ext && fuse) continue;
                Fp64LaunchArgs fa{};
                fa.fuse = fuse && !tier_ext;
                fa.view = v;
                fa.cls = c;
                fa.gcp = opts_.gcp != 0;
                fa.ext = tier_ext;
                fa.ext_list = ext;
                fa.items = (tier_ext ? rescue_ext_.as<Task>() : fp64_lists) + x.class_start[c];
                fa.count = counters + (tier_ext ? kCtrExt : kCtrScaled) + c;
                fa.counter = counters + (tier_ext ? kCtrTaskExt : kCtrTaskScaled) + c;
                fa.scratch = scratch_.ptr;
                fa.rows = plan.rows;
                fa.grid = tier_ext ? plan.fp64_ext_grid[c] : plan.fp64_grid[c];
                fa.stream = sc;
                PHMM_CUDA(launch_fp64_rescue(fa));
                ++launches_;
            }
        }
    }
    if (fork) {
        for (int i = 0; i < kSideStreams; ++i) {
            PHMM_CUDA(cudaEventRecord(join_[i], side_[i]));
            PHMM_CUDA(cudaStreamWaitEvent(s, join_[i], 0));
        }
    }
    return PAIRHMM_OK;
}

Engine::Plan Engine::make_plan(const BatchIndex& x) const {
    const int nb = (int)rules_.size();
    const bool plain = opts_.mode == PAIRHMM_MODE_PLAIN;
    Plan p;
    p.rows = round_up((int64_t)x.max_hap_len + 2 * 32 + 8, 64);
    p.grid.assign(nb, 0);
    p.persistent.assign(nb, 1);
    p.scratch_off.assign(nb, 0);
    // multi-tile buckets may run at the same time: each gets its own slice of
    // the border scratch, out of an equal share of the budget
    int n_mt = 0;
    for (int b = 0; b < nb; ++b)
        if (x.bucket_items[b] != 0 && rule_cfg_[b]->multi_tile) ++n_mt;
    const int64_t mt_budget = kScratchBudget / std::max(1, n_mt);
    int64_t scratch = 0, fp32_scratch = 0;
    for (int b = 0; b < nb; ++b) {
        if (x.bucket_items[b] == 0) continue;
        const ConfigInfo* c = rule_cfg_[b];
        const int64_t tasks = (x.bucket_items[b] + c->per_warp() - 1) / c->per_warp();
        const int64_t need_blocks = (tasks + kWarpsPerBlock - 1) / kWarpsPerBlock;
        int64_t grid = plain ? need_blocks : std::min<int64_t>(persistent_grid(c->kernel, c->smem_bytes), need_blocks);
        if (c->multi_tile) {
            const int64_t per_warp = (int64_t)c->scratch_bytes_per_row * p.rows;
            const int64_t cap_blocks = std::max<int64_t>(1, mt_budget / (per_warp * kWarpsPerBlock));
            grid = std::min(grid, cap_blocks);
            p.scratch_off[b] = fp32_scratch;
            fp32_scratch += round_up(grid * kWarpsPerBlock * per_warp, 256);
        }
        grid = std::max<int64_t>(1, std::min<int64_t>(grid, INT32_MAX));
        p.grid[b] = (int)grid;
        // the plain form runs one task per warp; a grid capped by scratch loops on the counter
        p.persistent[b] = (!plain || grid < need_blocks) ? 1 : 0;
    }
    for (int c = 0; c < kFp64Classes; ++c) {
        for (const bool tier_ext : {false, true}) {
            int64_t grid = persistent_grid(fp64_kernel(c, opts_.gcp != 0, tier_ext), fp64_smem_bytes(c, tier_ext));
            const int64_t per_warp = (int64_t)fp64_scratch_bytes_per_row(c, tier_ext) * p.rows;
            if (per_warp > 0) {
                grid = std::min<int64_t>(grid, std::max<int64_t>(1, kScratchBudget / (per_warp * kWarpsPerBlock)));
                scratch = std::max(scratch, grid * kWarpsPerBlock * per_warp);
            }
            // no more warps than flagged pairs could need
            const int64_t need = (x.class_pairs[c] + fp64_per_warp(c) - 1) / fp64_per_warp(c);
            grid = std::min<int64_t>(grid, std::max<int64_t>(1, (need + kWarpsPerBlock - 1) / kWarpsPerBlock));
            (tier_ext ? p.fp64_ext_grid : p.fp64_grid)[c] = (int)grid;
        }
    }
    p.scratch_bytes = (size_t)std::max<int64_t>(std::max(scratch, fp32_scratch), 256);
    return p;
}

pairhmm_status_t Engine::run_pipeline(const pairhmm_batch_t& in, const BatchIndex& x, float* d_scores,
                                      cudaStream_t s) {
    if (x.num_pairs == 0) return PAIRHMM_OK;
    // every buffer the launches reference exists before capture starts
    const Plan plan = make_plan(x);
    PHMM_CUDA(scratch_.ensure(plan.scratch_bytes));
    cudaEvent_t marks[3] = {ev_prep_, ev_fp32_, ev1_};
    for (int stage = 0; stage < 3; ++stage) {
        if (!opts_.use_graphs) {
            pairhmm_status_t st = enqueue_pipeline(in, x, plan, d_scores, s, stage);
            if (st != PAIRHMM_OK) return st;
        } else {
            cudaGraph_t graph = nullptr;
            PHMM_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
            pairhmm_status_t st = enqueue_pipeline(in, x, plan, d_scores, s, stage);
            cudaError_t ce = cudaStreamEndCapture(s, &graph);
            if (st != PAIRHMM_OK) {
                if (graph) cudaGraphDestroy(graph);
                return st;
            }
            if (ce != cudaSuccess) return cuda_fail(ce, "cudaStreamEndCapture");
            cudaGraphExec_t& exec = graph_exec_[stage];
            bool updated = false;
            if (exec) {
                cudaGraphExecUpdateResultInfo info{};
                if (cudaGraphExecUpdate(exec, graph, &info) == cudaSuccess) updated = true;
                else {
                    cudaGetLastError();
                    cudaGraphExecDestroy(exec);
                    exec = nullptr;
                }
            }
            if (!updated) {
                ce = cudaGraphInstantiate(&exec, graph, 0);
                if (ce != cudaSuccess) {
                    cudaGraphDestroy(graph);
                    exec = nullptr;
                    return cuda_fail(ce, "cudaGraphInstantiate");
                }
            }
            cudaGraphDestroy(graph);
            PHMM_CUDA(cudaGraphLaunch(exec, s));
        }
        PHMM_CUDA(cudaEventRecord(marks[stage], s));
    }
    return PAIRHMM_OK;
}

pairhmm_status_t Engine::host_begin(const pairhmm_batch_t& b, float* scores, cudaEvent_t mark_start,
                                    cudaEvent_t mark_end) {
    PHMM_CUDA(cudaSetDevice(opts_.device));
    // first a cheap validating pass for sizes and byte ranges, so the input
    // upload runs on helper threads while this thread builds the index
    InputRanges rg;
    std::string err;
    pairhmm_status_t st = scan_inputs(b, rg, err, opts_.gcp != 0);
    if (st != PAIRHMM_OK) return fail(st, err);
    if (rg.num_pairs > 0 && !scores) return fail(PAIRHMM_ERR_INVALID_ARGUMENT, "null scores");
    stats_ = pairhmm_stats_t{};
    pending_ = false;
    if (rg.num_pairs == 0) return PAIRHMM_OK;
    if ((st = ensure_inputs(rg)) != PAIRHMM_OK) return st;
    cudaStream_t s = stream_;
    // only the byte range the batch references is copied; device base pointers
    // are shifted so the caller's absolute offsets stay valid
    const int64_t rlo = rg.read_min, rn = rg.read_end - rg.read_min;
    const int64_t hlo = rg.hap_min, hn = rg.hap_end - rg.hap_min;
    std::vector<HostUploader::Copy> inputs = {
        {in_read_bases_.ptr, b.read_bases + rlo, (size_t)rn},
        {in_bq_.ptr, b.base_quals + rlo, (size_t)rn},
        {in_iq_.ptr, b.ins_quals + rlo, (size_t)rn},
        {in_dq_.ptr, b.del_quals + rlo, (size_t)rn},
        {in_read_off_.ptr, b.read_offsets, (size_t)(8 * rg.num_reads)},
        {in_read_len_.ptr, b.read_lengths, (size_t)(4 * rg.num_reads)},
        {in_hap_bases_.ptr, b.hap_bases + hlo, (size_t)hn},
        {in_hap_off_.ptr, b.hap_offsets, (size_t)(8 * rg.num_haps)},
        {in_hap_len_.ptr, b.hap_lengths, (size_t)(4 * rg.num_haps)},
    };
    if (opts_.gcp) inputs.push_back({in_gq_.ptr, b.gcp_quals + rlo, (size_t)rn});
    cudaError_t up = uploader_.start(opts_.device, inputs, s);
    st = build_index(b, rules_, idx_, err);
    const cudaError_t upf = uploader_.finish();
    if (up == cudaSuccess) up = upf;
    if (up != cudaSuccess) return cuda_fail(up, "input upload");
    if (st != PAIRHMM_OK) return fail(st, err);
    const BatchIndex& x = idx_;
    stats_.pairs = x.num_pairs;
    stats_.cells = x.cells;
    stats_.multi_tile_pairs = x.multi_tile_pairs;
    if ((st = ensure_buffers(x, false)) != PAIRHMM_OK) return st;
    if ((st = upload_index(x, s)) != PAIRHMM_OK) return st;

    pairhmm_batch_t dev = b;
    auto shifted = [](const DevBuf& d, int64_t lo) {
        return reinterpret_cast<const uint8_t*>(reinterpret_cast<uintptr_t>(d.ptr) - (uintptr_t)lo);
    };
    dev.read_bases = shifted(in_read_bases_, rlo);
    dev.base_quals = shifted(in_bq_, rlo);
    dev.ins_quals = shifted(in_iq_, rlo);
    dev.del_quals = shifted(in_dq_, rlo);
    dev.gcp_quals = opts_.gcp ? shifted(in_gq_, rlo) : nullptr;
    dev.read_offsets = in_read_off_.as<int64_t>();
    dev.read_lengths = in_read_len_.as<int32_t>();
    dev.hap_bases = shifted(in_hap_bases_, hlo);
    dev.hap_offsets = in_hap_off_.as<int64_t>();
    dev.hap_lengths = in_hap_len_.as<int32_t>();

    PHMM_CUDA(cudaEventRecord(ev0_, s));
    if (mark_start) PHMM_CUDA(cudaEventRecord(mark_start, s));
    if ((st = run_pipeline(dev, x, scores_.as<float>(), s)) != PAIRHMM_OK) return st;
    if (mark_end) PHMM_CUDA(cudaEventRecord(mark_end, s));
    // rescue counts and (into page-locked memory) scores come down now; scores
    // for pageable memory go through the uploader's slots in host_end
    PHMM_CUDA(cudaMemcpyAsync(host_hdr_, counters_.as<unsigned long long>() + kCtrScaled,
                              sizeof(unsigned long long) * 2 * kFp64Classes, cudaMemcpyDeviceToHost, s));
    pend_direct_ = HostUploader::is_page_locked(scores);
    if (pend_direct_)
        PHMM_CUDA(cudaMemcpyAsync(scores, scores_.ptr, 4 * (size_t)x.num_pairs, cudaMemcpyDeviceToHost, s));
    pend_scores_ = scores;
    pend_pairs_ = x.num_pairs;
    stats_.h2d_bytes = 4 * rn + hn + 12 * x.num_reads + 12 * x.num_haps + index_bytes(x);
    stats_.d2h_bytes = 4 * x.num_pairs + (int64_t)sizeof(unsigned long long) * 2 * kFp64Classes;
    stats_.launches = launches_;
    stats_.fp32_launches = fp32_launches_;
    pending_ = true;
    return PAIRHMM_OK;
}

pairhmm_status_t Engine::host_end() {
    if (!pending_) return PAIRHMM_OK;
    pending_ = false;
    PHMM_CUDA(cudaSetDevice(opts_.device));
    cudaStream_t s = stream_;
    if (!pend_direct_)
        PHMM_CUDA(uploader_.download(opts_.device, pend_scores_, scores_.ptr, 4 * (size_t)pend_pairs_, s));
    PHMM_CUDA(cudaStreamSynchronize(s));
    // per class: the scaled tier's counts, then the extended tier's
    unsigned long long rescued_by_class[2 * kFp64Classes] = {};
    static_assert(sizeof(rescued_by_class) <= 256, "rescue counts fit the landing spot");
    std::memcpy(rescued_by_class, host_hdr_, sizeof(rescued_by_class));
    float ms = 0.f, a = 0.f, b2 = 0.f, c = 0.f;
    PHMM_CUDA(cudaEventElapsedTime(&ms, ev0_, ev1_));
    PHMM_CUDA(cudaEventElapsedTime(&a, ev0_, ev_prep_));
    PHMM_CUDA(cudaEventElapsedTime(&b2, ev_prep_, ev_fp32_));
    PHMM_CUDA(cudaEventElapsedTime(&c, ev_fp32_, ev1_));
    stats_.device_ms = ms;
    stats_.prep_ms = a;
    stats_.fp32_ms = b2;
    stats_.fp64_ms = c;
    stats_.rescued = 0;
    stats_.rescued_ext = 0;
    for (int c = 0; c < kFp64Classes; ++c) {
        stats_.rescued += (int64_t)rescued_by_class[c];
        stats_.rescued_ext += (int64_t)rescued_by_class[kFp64Classes + c];
    }
    return PAIRHMM_OK;
}

pairhmm_status_t Engine::compute_host(const pairhmm_batch_t& b, float* scores) {
    const auto t0 = std::chrono::steady_clock::now();
    // large batches run as chunks of whole records on this engine and a twin
    // engine in turn, so a chunk's index build and upload overlap the previous
    // chunk's kernels
    int64_t pairs = 0;
    if (b.num_records > 0 && b.reads_per_record && b.haps_per_record)
        for (int64_t g = 0; g < b.num_records; ++g)
            pairs += (int64_t)std::max(b.reads_per_record[g], 0) * std::max(b.haps_per_record[g], 0);
    int nchunks = opts_.pipeline_chunks > 0 ? opts_.pipeline_chunks
                                             : (int)std::min<int64_t>(kMaxChunks, pairs / kChunkPairs);
    if (nchunks > b.num_records) nchunks = (int)b.num_records;
    if (nchunks < 2 || !b.read_lengths || !b.hap_lengths || !b.read_offsets || !b.hap_offsets) {
        pairhmm_status_t st = host_begin(b, scores, nullptr, nullptr);
        if (st == PAIRHMM_OK) st = host_end();
        stats_.total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        return st;
    }
    if (!twin_) {
        pairhmm_options_t o = opts_;
        o.pipeline_chunks = 1;
        twin_ = std::make_unique<Engine>(o);
        pairhmm_status_t st = twin_->init();
        if (st == PAIRHMM_OK) st = twin_->set_tile_table(rules_);
        if (st != PAIRHMM_OK) {
            last_error_ = "twin engine: " + twin_->last_error();
            twin_.reset();
            return st;
        }
    }
    PHMM_CUDA(cudaSetDevice(opts_.device));
    if (!span0_) {
        PHMM_CUDA(cudaEventCreate(&span0_));
        PHMM_CUDA(cudaEventCreate(&span1_));
    }
    // chunk boundaries: records in order, about equal pairs per chunk except the
    // first, which is half a chunk (its index build and upload are not overlapped)
    std::vector<int64_t> bound{0};
    {
        int64_t acc = 0, next = 1;
        for (int64_t g = 0; g < b.num_records && (int)bound.size() < nchunks; ++g) {
            acc += (int64_t)std::max(b.reads_per_record[g], 0) * std::max(b.haps_per_record[g], 0);
            if (acc * (2 * nchunks - 1) >= pairs * (2 * next - 1) && g + 1 < b.num_records) {
                bound.push_back(g + 1);
                ++next;
            }
        }
        bound.push_back(b.num_records);
    }
    pairhmm_stats_t sum{};
    Engine* eng[2] = {this, twin_.get()};
    pairhmm_status_t st = PAIRHMM_OK;
    int64_t read0 = 0, hap0 = 0, pair0 = 0;
    const int n = (int)bound.size() - 1;
    auto collect = [&](Engine* e) {
        const pairhmm_status_t r = e->host_end();
        if (r != PAIRHMM_OK) {
            if (e != this) last_error_ = e->last_error();
            return r;
        }
        const pairhmm_stats_t& x = e->stats_;
        sum.pairs += x.pairs;
        sum.cells += x.cells;
        sum.rescued += x.rescued;
        sum.rescued_ext += x.rescued_ext;
        sum.multi_tile_pairs += x.multi_tile_pairs;
        sum.prep_ms += x.prep_ms;
        sum.fp32_ms += x.fp32_ms;
        sum.fp64_ms += x.fp64_ms;
        sum.launches += x.launches;
        sum.fp32_launches += x.fp32_launches;
        sum.h2d_bytes += x.h2d_bytes;
        sum.d2h_bytes += x.d2h_bytes;
        return PAIRHMM_OK;
    };
    for (int i = 0; i < n && st == PAIRHMM_OK; ++i) {
        Engine* e = eng[i & 1];
        if (i >= 2) st = collect(e);  // this engine's previous chunk
        if (st != PAIRHMM_OK) break;
        const int64_t g0 = bound[i], g1 = bound[i + 1];
        int64_t reads = 0, haps = 0, cp = 0;
        for (int64_t g = g0; g < g1; ++g) {
            reads += std::max(b.reads_per_record[g], 0);
            haps += std::max(b.haps_per_record[g], 0);
            cp += (int64_t)std::max(b.reads_per_record[g], 0) * std::max(b.haps_per_record[g], 0);
        }
        pairhmm_batch_t v = b;
        v.num_records = g1 - g0;
        v.reads_per_record += g0;
        v.haps_per_record += g0;
        v.read_offsets += read0;
        v.read_lengths += read0;
        v.hap_offsets += hap0;
        v.hap_lengths += hap0;
        st = e->host_begin(v, scores + pair0, i == 0 ? span0_ : nullptr, i == n - 1 ? span1_ : nullptr);
        if (st != PAIRHMM_OK && e != this) last_error_ = e->last_error();
        read0 += reads;
        hap0 += haps;
        pair0 += cp;
    }
    // the last chunks in flight (also after an error: nothing may stay queued)
    for (int i = std::max(0, n - 2); i < n; ++i) {
        const pairhmm_status_t r = collect(eng[i & 1]);
        if (st == PAIRHMM_OK) st = r;
    }
    if (st != PAIRHMM_OK) return st;
    float span = 0.f;
    PHMM_CUDA(cudaEventElapsedTime(&span, span0_, span1_));
    sum.device_ms = span;
    sum.total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    stats_ = sum;
    return PAIRHMM_OK;
}

pairhmm_status_t Engine::compute_device(const pairhmm_batch_t& b, int32_t, int32_t, float* scores,
                                        cudaStream_t stream) {
    const auto t0 = std::chrono::steady_clock::now();
    PHMM_CUDA(cudaSetDevice(opts_.device));
    if (b.num_records < 0) return fail(PAIRHMM_ERR_INVALID_ARGUMENT, "num_records < 0");
    if (b.num_records == 0) { stats_ = pairhmm_stats_t{}; return PAIRHMM_OK; }
    if (!b.reads_per_record || !b.haps_per_record) return fail(PAIRHMM_ERR_INVALID_ARGUMENT, "null record arrays");
    if (opts_.gcp && !b.gcp_quals) return fail(PAIRHMM_ERR_INVALID_ARGUMENT, "gcp mode needs the gcp quality array");
    // the host needs the record structure and lengths to derive the index
    std::vector<int32_t> rpr(b.num_records), hpr(b.num_records);
    PHMM_CUDA(cudaMemcpyAsync(rpr.data(), b.reads_per_record, 4 * b.num_records, cudaMemcpyDeviceToHost, stream));
    PHMM_CUDA(cudaMemcpyAsync(hpr.data(), b.haps_per_record, 4 * b.num_records, cudaMemcpyDeviceToHost, stream));
    PHMM_CUDA(cudaStreamSynchronize(stream));
    int64_t nr = 0, nh = 0;
    for (int64_t g = 0; g < b.num_records; ++g) { nr += std::max(rpr[g], 0); nh += std::max(hpr[g], 0); }
    std::vector<int32_t> rl(nr), hl(nh);
    if (nr) PHMM_CUDA(cudaMemcpyAsync(rl.data(), b.read_lengths, 4 * nr, cudaMemcpyDeviceToHost, stream));
    if (nh) PHMM_CUDA(cudaMemcpyAsync(hl.data(), b.hap_lengths, 4 * nh, cudaMemcpyDeviceToHost, stream));
    PHMM_CUDA(cudaStreamSynchronize(stream));
    pairhmm_batch_t hb = b;
    hb.reads_per_record = rpr.data();
    hb.haps_per_record = hpr.data();
    hb.read_lengths = rl.data();
    hb.hap_lengths = hl.data();
    hb.read_offsets = nullptr;
    hb.hap_offsets = nullptr;
    std::string err;
    pairhmm_status_t st = build_index(hb, rules_, idx_, err);
    const BatchIndex& x = idx_;
    if (st != PAIRHMM_OK) return fail(st, err);
    stats_ = pairhmm_stats_t{};
    stats_.pairs = x.num_pairs;
    stats_.cells = x.cells;
    stats_.multi_tile_pairs = x.multi_tile_pairs;
    stats_.rescued = -1;
    stats_.rescued_ext = -1;
    if (x.num_pairs == 0) return PAIRHMM_OK;
    if (!scores) return fail(PAIRHMM_ERR_INVALID_ARGUMENT, "null scores");
    if ((st = ensure_buffers(x, false)) != PAIRHMM_OK) return st;
    cudaStream_t s = stream_;
    PHMM_CUDA(cudaEventRecord(ev0_, stream));
    PHMM_CUDA(cudaStreamWaitEvent(s, ev0_, 0));
    if ((st = upload_index(x, s)) != PAIRHMM_OK) return st;
    PHMM_CUDA(cudaEventRecord(ev0_, s));
    if ((st = run_pipeline(b, x, scores, s)) != PAIRHMM_OK) return st;
    PHMM_CUDA(cudaStreamWaitEvent(stream, ev1_, 0));
    stats_.total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    stats_.device_ms = -1.0;
    return PAIRHMM_OK;
}

}  // namespace phmm
