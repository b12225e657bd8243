// extern "C" boundary: no C++ exceptions or types cross it.
#include <cstring>
#include <memory>
#include <mutex>
#include <new>

#include "engine.hpp"
#include "records.hpp"
#include "serving.hpp"

struct pairhmm_records {
    phmm::HostBatch batch;
};

struct pairhmm_reader {
    explicit pairhmm_reader(const char* path) : reader(path) {}
    phmm::RecordReader reader;
    bool done = false;
};

namespace {
thread_local std::string t_records_error;
}

struct pairhmm_engine {
    std::unique_ptr<phmm::Engine> engine;
    std::unique_ptr<phmm::ServingQueue> serving;
    std::mutex serving_mu;  // creation of the serving queue; its calls may overlap
    std::mutex error_mu;    // error text: serving calls may come from several threads
    std::string error;
};

namespace {

void set_error(pairhmm_engine* h, std::string msg) {
    if (!h) return;
    std::lock_guard<std::mutex> lk(h->error_mu);
    h->error = std::move(msg);
}

template <class F>
pairhmm_status_t guarded(pairhmm_engine* h, F&& f) {
    try {
        return f();
    } catch (const std::bad_alloc&) {
        set_error(h, "host allocation failed");
        return PAIRHMM_ERR_OUT_OF_MEMORY;
    } catch (const std::exception& e) {
        set_error(h, e.what());
        return PAIRHMM_ERR_CUDA;
    } catch (...) {
        set_error(h, "unknown exception");
        return PAIRHMM_ERR_CUDA;
    }
}

// the serving queue of an engine, created on first use
phmm::ServingQueue* serving_of(pairhmm_engine* h, bool create) {
    std::lock_guard<std::mutex> lk(h->serving_mu);
    if (!h->serving && create) h->serving = std::make_unique<phmm::ServingQueue>(*h->engine);
    return h->serving.get();
}

pairhmm_status_t serving_result(pairhmm_engine* h, phmm::ServingQueue* q, pairhmm_status_t s) {
    if (s != PAIRHMM_OK) {
        set_error(h, q ? q->last_error() : std::string("no region was submitted to this engine"));
    }
    return s;
}

pairhmm_status_t finish(pairhmm_engine* h, pairhmm_status_t s) {
    set_error(h, s != PAIRHMM_OK ? h->engine->last_error() : std::string());
    return s;
}

}  // namespace

extern "C" {

void pairhmm_default_options(pairhmm_options_t* o) {
    if (!o) return;
    o->device = 0;
    o->mode = PAIRHMM_MODE_ENGINE;
    o->fp64_rescue = 1;
    o->use_graphs = 1;
    o->device_budget_bytes = 0;
    o->pipeline_chunks = 0;
    o->gcp = 0;
}

pairhmm_status_t pairhmm_engine_create(const pairhmm_options_t* opts, pairhmm_engine_t** out) {
    if (!out) return PAIRHMM_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    pairhmm_options_t o;
    pairhmm_default_options(&o);
    if (opts) o = *opts;
    if (o.mode != PAIRHMM_MODE_ENGINE && o.mode != PAIRHMM_MODE_PLAIN) return PAIRHMM_ERR_INVALID_ARGUMENT;
    auto* h = new (std::nothrow) pairhmm_engine;
    if (!h) return PAIRHMM_ERR_OUT_OF_MEMORY;
    pairhmm_status_t s = guarded(h, [&] {
        h->engine = std::make_unique<phmm::Engine>(o);
        return h->engine->init();
    });
    if (s != PAIRHMM_OK) {
        delete h;
        return s;
    }
    *out = h;
    return PAIRHMM_OK;
}

pairhmm_status_t pairhmm_engine_destroy(pairhmm_engine_t* h) {
    if (!h) return PAIRHMM_ERR_INVALID_ARGUMENT;
    pairhmm_status_t s = guarded(h, [&] {
        h->serving.reset();
        h->engine.reset();
        return PAIRHMM_OK;
    });
    delete h;
    return s;
}

pairhmm_status_t pairhmm_compute_host(pairhmm_engine_t* h, const pairhmm_batch_t* batch, float* scores) {
    if (!h || !batch) return PAIRHMM_ERR_INVALID_ARGUMENT;
    return guarded(h, [&] { return finish(h, h->engine->compute_host(*batch, scores)); });
}

pairhmm_status_t pairhmm_compute_device(pairhmm_engine_t* h, const pairhmm_batch_t* batch, int32_t max_read_length,
                                        int32_t max_hap_length, float* scores, void* stream) {
    if (!h || !batch) return PAIRHMM_ERR_INVALID_ARGUMENT;
    return guarded(h, [&] {
        return finish(h, h->engine->compute_device(*batch, max_read_length, max_hap_length, scores,
                                                   static_cast<cudaStream_t>(stream)));
    });
}

pairhmm_status_t pairhmm_get_stats(pairhmm_engine_t* h, pairhmm_stats_t* stats) {
    if (!h || !stats) return PAIRHMM_ERR_INVALID_ARGUMENT;
    *stats = h->engine->stats();
    return PAIRHMM_OK;
}

pairhmm_status_t pairhmm_submit(pairhmm_engine_t* h, const pairhmm_batch_t* region, uint64_t* ticket) {
    if (!h || !region || !ticket) return PAIRHMM_ERR_INVALID_ARGUMENT;
    return guarded(h, [&] {
        phmm::ServingQueue* q = serving_of(h, true);
        return serving_result(h, q, q->submit(*region, ticket));
    });
}

pairhmm_status_t pairhmm_submit_many(pairhmm_engine_t* h, const pairhmm_batch_t* regions, int64_t num_regions,
                                     uint64_t* tickets) {
    if (!h || num_regions < 0 || (num_regions > 0 && (!regions || !tickets))) return PAIRHMM_ERR_INVALID_ARGUMENT;
    return guarded(h, [&] {
        phmm::ServingQueue* q = serving_of(h, true);
        return serving_result(h, q, q->submit_many(regions, num_regions, tickets));
    });
}

pairhmm_status_t pairhmm_poll(pairhmm_engine_t* h, uint64_t ticket, int32_t* done) {
    if (!h || !done) return PAIRHMM_ERR_INVALID_ARGUMENT;
    return guarded(h, [&] {
        phmm::ServingQueue* q = serving_of(h, false);
        return serving_result(h, q, q ? q->poll(ticket, done) : PAIRHMM_ERR_NOT_FOUND);
    });
}

pairhmm_status_t pairhmm_drain(pairhmm_engine_t* h, uint64_t ticket, float* scores, int64_t num_scores,
                               int32_t timeout_ms) {
    if (!h || (!scores && num_scores > 0)) return PAIRHMM_ERR_INVALID_ARGUMENT;
    return guarded(h, [&] {
        phmm::ServingQueue* q = serving_of(h, false);
        return serving_result(h, q, q ? q->drain(ticket, scores, num_scores, timeout_ms) : PAIRHMM_ERR_NOT_FOUND);
    });
}

pairhmm_status_t pairhmm_region_latency_ms(pairhmm_engine_t* h, uint64_t ticket, double* ms) {
    if (!h || !ms) return PAIRHMM_ERR_INVALID_ARGUMENT;
    return guarded(h, [&] {
        phmm::ServingQueue* q = serving_of(h, false);
        return serving_result(h, q, q ? q->latency(ticket, ms) : PAIRHMM_ERR_NOT_FOUND);
    });
}

pairhmm_status_t pairhmm_serving_stats(pairhmm_engine_t* h, pairhmm_serving_stats_t* stats) {
    if (!h || !stats) return PAIRHMM_ERR_INVALID_ARGUMENT;
    *stats = pairhmm_serving_stats_t{};
    phmm::ServingQueue* q = serving_of(h, false);
    if (q) q->stats(stats);
    return PAIRHMM_OK;
}

const char* pairhmm_status_string(pairhmm_status_t s) {
    switch (s) {
        case PAIRHMM_OK: return "ok";
        case PAIRHMM_ERR_INVALID_ARGUMENT: return "invalid argument";
        case PAIRHMM_ERR_CUDA: return "CUDA error";
        case PAIRHMM_ERR_OUT_OF_MEMORY: return "out of memory";
        case PAIRHMM_ERR_BUDGET: return "region exceeds the device budget";
        case PAIRHMM_ERR_NOT_FOUND: return "unknown ticket";
        case PAIRHMM_ERR_TIMEOUT: return "timed out";
        case PAIRHMM_ERR_UNSUPPORTED: return "unsupported";
        case PAIRHMM_ERR_BUSY: return "busy";
        case PAIRHMM_ERR_LIMIT: return "haplotype length above the no-alloc limit of 16384";
    }
    return "unknown status";
}

const char* pairhmm_last_error(const pairhmm_engine_t* h) {
    // a copy per calling thread: serving calls on other threads may replace the text
    thread_local std::string copy;
    if (!h) return "";
    std::lock_guard<std::mutex> lk(const_cast<pairhmm_engine_t*>(h)->error_mu);
    copy = h->error;
    return copy.c_str();
}

pairhmm_status_t pairhmm_batch_counts(const pairhmm_batch_t* batch, int64_t* pairs, int64_t* cells) {
    if (!batch) return PAIRHMM_ERR_INVALID_ARGUMENT;
    phmm::BatchIndex x;
    std::string err;
    pairhmm_status_t s;
    try {
        s = phmm::Engine::build_index(*batch, {{1 << 30, 32, 32, true, false}}, x, err);
    } catch (...) {
        return PAIRHMM_ERR_OUT_OF_MEMORY;
    }
    if (s != PAIRHMM_OK) return s;
    if (pairs) *pairs = x.num_pairs;
    if (cells) *cells = x.cells;
    return PAIRHMM_OK;
}

pairhmm_status_t pairhmm_records_parse(const char* text, int64_t length, pairhmm_records_t** out) {
    t_records_error.clear();
    if (!out || (!text && length > 0) || length < 0) return PAIRHMM_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    try {
        auto r = std::make_unique<pairhmm_records>();
        if (!phmm::parse_records(text, (size_t)length, r->batch, t_records_error))
            return PAIRHMM_ERR_INVALID_ARGUMENT;
        *out = r.release();
        return PAIRHMM_OK;
    } catch (...) {
        t_records_error = "host allocation failed";
        return PAIRHMM_ERR_OUT_OF_MEMORY;
    }
}

pairhmm_status_t pairhmm_reader_open(const char* path, pairhmm_reader_t** out) {
    t_records_error.clear();
    if (!path || !out) return PAIRHMM_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    try {
        auto r = std::make_unique<pairhmm_reader>(path);
        if (!r->reader.ok()) {
            t_records_error = r->reader.error();
            return PAIRHMM_ERR_INVALID_ARGUMENT;
        }
        *out = r.release();
        return PAIRHMM_OK;
    } catch (...) {
        t_records_error = "host allocation failed";
        return PAIRHMM_ERR_OUT_OF_MEMORY;
    }
}

pairhmm_status_t pairhmm_reader_next(pairhmm_reader_t* rd, int64_t min_pairs, pairhmm_records_t** out) {
    t_records_error.clear();
    if (!rd || !out) return PAIRHMM_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    if (rd->done) return PAIRHMM_OK;
    try {
        auto r = std::make_unique<pairhmm_records>();
        bool eof = false;
        if (!rd->reader.next(r->batch, min_pairs > 0 ? min_pairs : INT64_MAX, eof)) {
            t_records_error = rd->reader.error();
            rd->done = true;
            return PAIRHMM_ERR_INVALID_ARGUMENT;
        }
        if (eof) rd->done = true;
        if (r->batch.num_records() > 0) *out = r.release();
        return PAIRHMM_OK;
    } catch (...) {
        t_records_error = "host allocation failed";
        return PAIRHMM_ERR_OUT_OF_MEMORY;
    }
}

void pairhmm_reader_close(pairhmm_reader_t* rd) { delete rd; }

const char* pairhmm_records_last_error(void) { return t_records_error.c_str(); }

void pairhmm_set_host_threads(int32_t threads) { phmm::set_host_threads(threads); }

pairhmm_status_t pairhmm_records_view(const pairhmm_records_t* r, pairhmm_batch_t* view, int64_t* num_pairs) {
    if (!r || !view) return PAIRHMM_ERR_INVALID_ARGUMENT;
    *view = r->batch.view();
    if (num_pairs) *num_pairs = r->batch.pairs;
    return PAIRHMM_OK;
}

pairhmm_status_t pairhmm_records_format(const pairhmm_records_t* r, const float* scores, char* buf,
                                        int64_t capacity, int64_t* length) {
    if (!r || !length || (!scores && r->batch.pairs > 0)) return PAIRHMM_ERR_INVALID_ARGUMENT;
    try {
        std::string text;
        phmm::format_scores(r->batch, scores, text);
        *length = (int64_t)text.size();
        if (buf && capacity > (int64_t)text.size()) {
            std::memcpy(buf, text.data(), text.size());
            buf[text.size()] = '\0';
        }
        return PAIRHMM_OK;
    } catch (...) {
        return PAIRHMM_ERR_OUT_OF_MEMORY;
    }
}

void pairhmm_records_free(pairhmm_records_t* r) { delete r; }

pairhmm_status_t pairhmm_host_register(void* ptr, size_t bytes) {
    if (!ptr || bytes == 0) return PAIRHMM_ERR_INVALID_ARGUMENT;
    const cudaError_t e = cudaHostRegister(ptr, bytes, cudaHostRegisterPortable);
    if (e == cudaErrorHostMemoryAlreadyRegistered) {
        cudaGetLastError();
        return PAIRHMM_OK;
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        return e == cudaErrorMemoryAllocation ? PAIRHMM_ERR_OUT_OF_MEMORY : PAIRHMM_ERR_CUDA;
    }
    return PAIRHMM_OK;
}

pairhmm_status_t pairhmm_host_unregister(void* ptr) {
    if (!ptr) return PAIRHMM_ERR_INVALID_ARGUMENT;
    const cudaError_t e = cudaHostUnregister(ptr);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return PAIRHMM_ERR_INVALID_ARGUMENT;
    }
    return PAIRHMM_OK;
}

const char* pairhmm_version(void) { return "pairhmm_b200 0.1.0 (sm_100a)"; }

pairhmm_status_t pairhmm_set_tile_table(pairhmm_engine_t* h, const int32_t* max_len, const int32_t* group,
                                        const int32_t* regs, const int32_t* multi_tile, int32_t n) {
    if (!h || !max_len || !group || !regs || !multi_tile || n <= 0) return PAIRHMM_ERR_INVALID_ARGUMENT;
    return guarded(h, [&] {
        std::vector<phmm::TileRule> rules(n);
        for (int i = 0; i < n; ++i) {
            if (multi_tile[i] < 0 || multi_tile[i] > 2) return PAIRHMM_ERR_INVALID_ARGUMENT;
            rules[i] = {max_len[i], group[i], regs[i], multi_tile[i] == 1, multi_tile[i] == 2};
        }
        return finish(h, h->engine->set_tile_table(rules));
    });
}

pairhmm_status_t pairhmm_get_tile_table(pairhmm_engine_t* h, int32_t* max_len, int32_t* group, int32_t* regs,
                                        int32_t* multi_tile, int32_t capacity, int32_t* n) {
    if (!h || !n) return PAIRHMM_ERR_INVALID_ARGUMENT;
    const auto& r = h->engine->tile_table();
    *n = (int32_t)r.size();
    if (capacity < (int32_t)r.size() || !max_len || !group || !regs || !multi_tile) return PAIRHMM_OK;
    for (size_t i = 0; i < r.size(); ++i) {
        max_len[i] = r[i].max_len;
        group[i] = r[i].G;
        regs[i] = r[i].R;
        multi_tile[i] = r[i].multi_tile ? 1 : (r[i].packed ? 2 : 0);
    }
    return PAIRHMM_OK;
}

}  // extern "C"

namespace {
// FMA throughput of one of the probe kernels: grow the launch until it takes
// the requested time, keep the best rate
pairhmm_status_t probe_peak(int32_t device, int32_t milliseconds, double* tflops,
                            cudaError_t (*launch)(float*, int, int, cudaStream_t)) {
    if (!tflops || milliseconds <= 0) return PAIRHMM_ERR_INVALID_ARGUMENT;
    if (cudaSetDevice(device) != cudaSuccess) return PAIRHMM_ERR_CUDA;
    cudaDeviceProp prop{};
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return PAIRHMM_ERR_CUDA;
    float* out = nullptr;
    cudaStream_t s = nullptr;
    cudaEvent_t a = nullptr, b = nullptr;
    if (cudaMalloc(&out, 16) != cudaSuccess) return PAIRHMM_ERR_OUT_OF_MEMORY;
    cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    const int grid = prop.multiProcessorCount * 8;  // 8 x 256 threads per SM
    int iters = 1000;
    double best = 0.0;
    pairhmm_status_t st = PAIRHMM_OK;
    // grow until one launch takes the requested time, then keep the best of 3
    for (int rep = 0; rep < 12 && st == PAIRHMM_OK; ++rep) {
        cudaEventRecord(a, s);
        if (launch(out, grid, iters, s) != cudaSuccess) st = PAIRHMM_ERR_CUDA;
        cudaEventRecord(b, s);
        if (cudaEventSynchronize(b) != cudaSuccess) st = PAIRHMM_ERR_CUDA;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, a, b);
        const double flops = (double)grid * 256 * (double)iters * 128.0 * 2.0;
        if (ms > 0.f) best = std::max(best, flops / (ms * 1e-3) / 1e12);
        if (ms < milliseconds && rep < 9) iters = (int)std::min<double>(iters * 2.0, 4e8);
    }
    *tflops = best;
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaStreamDestroy(s);
    cudaFree(out);
    return st;
}
}  // namespace

extern "C" {

pairhmm_status_t pairhmm_probe_fp32_peak(int32_t device, int32_t milliseconds, double* tflops) {
    return probe_peak(device, milliseconds, tflops, &phmm::launch_ffma_peak);
}

pairhmm_status_t pairhmm_probe_fp64_peak(int32_t device, int32_t milliseconds, double* tflops) {
    return probe_peak(device, milliseconds, tflops, &phmm::launch_dfma_peak);
}

}  // extern "C"
