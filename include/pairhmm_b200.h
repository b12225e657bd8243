/*
 * pairhmm_b200 -- PairHMM forward-algorithm engine for NVIDIA B200 (sm_100a).
 *
 * C ABI (plain pointers and sizes, int status codes, no exceptions across the
 * boundary).  It is the drop-in for the forward path of asbschmidt/gpuPairHMM:
 *
 *   reference                                              replaced by
 *   ------------------------------------------------------------------------------
 *   BatchOfSequenceGroups (common.cuh:109-201)             pairhmm_batch_t
 *   GpuPairHMMWorker ctor: ph2pr upload + streams
 *     (gpuworker.cuh:401-416)                              pairhmm_engine_create
 *   GpuPairHMMWorker dtor (gpuworker.cuh:418-428)          pairhmm_engine_destroy
 *   GpuPairHMMWorker::processBatch_overlapped_float_
 *     coalesced_smem (gpuworker.cuh:559-973): host batch
 *     in, h_scores out                                     pairhmm_compute_host
 *   MultiConfigGpuPairHMM::launchPairHMMSingleTileKernel
 *     (gpuworker.cuh:220-274) and ::launchPairHMMMultiTile
 *     Kernel (gpuworker.cuh:303-375): device arrays +
 *     stream, scores written on the device                 pairhmm_compute_device
 *   GpuPairHMMWorker::computeNumberOfDPCells
 *     (gpuworker.cuh:495-520) and the GCUPS print
 *     (gpuworker.cuh:426-427)                              pairhmm_get_stats
 *   (no counterpart: the reference has no serving mode)    pairhmm_submit / _submit_many /
 *                                                          _poll / _drain
 *
 * Scores: one float log10 likelihood per (read, haplotype) pair, written at
 * slot  sum_{previous records} R*H + r*H + h  (gpuworker.cuh:1002-1021,
 * pairhmm_kernels.cuh:1154).
 *
 * Threading: an engine is used by one host thread at a time (as the
 * reference's worker is), except for the serving calls (submit, submit_many,
 * poll, drain, region_latency_ms, serving_stats), which may overlap from
 * several threads (a producer submitting while a consumer drains).  Different
 * engines are independent.
 */
#ifndef PAIRHMM_B200_H
#define PAIRHMM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum pairhmm_status {
    PAIRHMM_OK = 0,
    PAIRHMM_ERR_INVALID_ARGUMENT = 1, /* null pointer, negative count, bad length */
    PAIRHMM_ERR_CUDA = 2,             /* a CUDA runtime call failed; see pairhmm_last_error */
    PAIRHMM_ERR_OUT_OF_MEMORY = 3,    /* device or pinned allocation failed */
    PAIRHMM_ERR_BUDGET = 4,           /* serving: region larger than the device budget */
    PAIRHMM_ERR_NOT_FOUND = 5,        /* serving: unknown ticket */
    PAIRHMM_ERR_TIMEOUT = 6,          /* a bounded device wait gave up */
    PAIRHMM_ERR_UNSUPPORTED = 7,      /* no sm_100 device, or feature not built */
    PAIRHMM_ERR_BUSY = 8,             /* serving: queue full, retry after draining */
    PAIRHMM_ERR_LIMIT = 9             /* no-alloc forward: max_hap_length above 16384 */
} pairhmm_status_t;

/*
 * One batch of records in the reference's structure-of-arrays layout
 * (common.cuh:109-201).  Record g has reads_per_record[g] reads and
 * haps_per_record[g] haplotypes; reads and haplotypes are numbered globally
 * in record order.  Bases are ASCII (A, C, G, T; anything else counts as N,
 * utility_kernels.cuh:6-23).  Qualities are Phred values, i.e. the file's
 * ASCII minus 33 (file_parser_worker.cu:95); values above 127 are clamped to
 * 127.  The byte arrays share one layout: read i occupies
 * [read_offsets[i], read_offsets[i] + read_lengths[i]) in read_bases and in
 * each quality array.  gcp_quals may be NULL: like the reference GPU path the
 * engine uses a fixed gap-continuation probability of 0.1
 * (pairhmm_kernels.cuh:1195-1196).
 */
typedef struct pairhmm_batch {
    int64_t num_records;
    const int32_t* reads_per_record; /* [num_records] */
    const int32_t* haps_per_record;  /* [num_records] */
    const uint8_t* read_bases;
    const uint8_t* base_quals;
    const uint8_t* ins_quals;
    const uint8_t* del_quals;
    const uint8_t* gcp_quals;    /* gcp mode (pairhmm_options_t.gcp = 1): required, the first
                                    position's quality of each read sets its eps and beta;
                                    default mode: optional and unused, as on the reference's
                                    GPU path */
    const int64_t* read_offsets; /* [num_reads] */
    const int32_t* read_lengths; /* [num_reads], each >= 1 */
    const uint8_t* hap_bases;
    const int64_t* hap_offsets; /* [num_haps] */
    const int32_t* hap_lengths; /* [num_haps], each >= 1 */
} pairhmm_batch_t;

/* Execution forms. */
enum {
    /* Persistent, length-bucketed, H-sorted work queue; tuned tile per bucket;
     * CUDA-graph launched; FP64 rescue of FP32 underflows. */
    PAIRHMM_MODE_ENGINE = 0,
    /* One launch per read-length partition with the reference's generic tile
     * table (tuningconfigs.hpp:33-57), no sorting, FP32 only.  Kept as the
     * comparison baseline. */
    PAIRHMM_MODE_PLAIN = 1
};

typedef struct pairhmm_options {
    int32_t device;       /* CUDA ordinal, default 0 */
    int32_t mode;         /* PAIRHMM_MODE_* */
    int32_t fp64_rescue;  /* 1 (default): recompute FP32 underflows in FP64 */
    int32_t use_graphs;   /* 1 (default): replay the per-batch launch sequence as a CUDA graph */
    int64_t device_budget_bytes; /* serving admission budget; 0 = 40 GiB */
    int32_t pipeline_chunks; /* compute_host: 0 (default) = batches of 2M+ pairs run as up to
                                8 chunks of at least 1M pairs whose uploads overlap the previous
                                chunk's kernels; 1 = one pass; N = N chunks */
    int32_t gcp;             /* 0 (default): eps = 0.1, beta = 0.9 for every pair, as the reference's
                                GPU path (pairhmm_kernels.cuh:1195-1196; gcp qualities unused).
                                1: eps = p(gcp), beta = 1 - eps per read, from the gcp quality
                                of its first position, as the reference's CPU path
                                (gpuworker.cuh:1009, 1048-1049); the batch must carry
                                gcp_quals, and a gcp quality of 0 (beta = 0) is rejected
                                (compute_host) or scores NaN (compute_device).  Engine form
                                only. */
} pairhmm_options_t;

typedef struct pairhmm_stats {
    int64_t pairs;           /* pairs in the last compute call */
    int64_t cells;           /* sum L*H over those pairs */
    int64_t rescued;         /* pairs recomputed in FP64 (scaled doubles) */
    int64_t multi_tile_pairs;/* pairs whose read exceeded the largest single tile */
    double device_ms;        /* device time of the last call (CUDA events, launch to scores) */
    double total_ms;         /* host wall time of the last call */
    double prep_ms;          /* of device_ms: packing and work-list construction */
    double fp32_ms;          /* of device_ms: the FP32 wavefront launches */
    double fp64_ms;          /* of device_ms: the FP64 pass */
    int64_t launches;        /* kernels launched by the last call */
    int64_t h2d_bytes;       /* host-to-device bytes copied by the last call */
    int64_t d2h_bytes;       /* device-to-host bytes copied by the last call */
    int64_t rescued_ext;     /* of those, pairs beyond the scaled doubles' range, recomputed
                                again with per-lane exponents */
    int64_t fp32_launches;   /* of launches: the FP32 wavefront launches */
} pairhmm_stats_t;

typedef struct pairhmm_engine pairhmm_engine_t;

/* Fill *opts with defaults. */
void pairhmm_default_options(pairhmm_options_t* opts);

pairhmm_status_t pairhmm_engine_create(const pairhmm_options_t* opts, pairhmm_engine_t** engine);
pairhmm_status_t pairhmm_engine_destroy(pairhmm_engine_t* engine);

/* Host arrays in, host scores out (float[sum R*H]).  Blocking. */
pairhmm_status_t pairhmm_compute_host(pairhmm_engine_t* engine, const pairhmm_batch_t* batch,
                                      float* scores);

/* Device arrays in (every pointer in *batch is device memory), device scores
 * out; work is ordered on `stream` (a cudaStream_t, NULL = legacy default)
 * and the call returns without waiting.  max_read_length / max_hap_length
 * bound the batch (0 = computed by the engine with one device-to-host read). */
pairhmm_status_t pairhmm_compute_device(pairhmm_engine_t* engine, const pairhmm_batch_t* batch,
                                        int32_t max_read_length, int32_t max_hap_length,
                                        float* scores, void* stream);

pairhmm_status_t pairhmm_get_stats(pairhmm_engine_t* engine, pairhmm_stats_t* stats);

/* Serving (continuous batching).  submit copies the region into host memory
 * owned by the queue and returns a ticket; regions submitted while others run
 * are admitted into the device work queue as memory under the budget frees
 * up.  poll reports completion without blocking; drain blocks (bounded by
 * timeout_ms, <0 = forever) and copies the scores out, releasing the ticket. */
pairhmm_status_t pairhmm_submit(pairhmm_engine_t* engine, const pairhmm_batch_t* region,
                                uint64_t* ticket);
/* num_regions regions in one call (one lock, one wake-up of the slots);
 * tickets[i] is region i's.  Every region is checked and copied before any is
 * queued: on an error none is queued and the error text names the region.
 * A region's latency counts from the start of the call. */
pairhmm_status_t pairhmm_submit_many(pairhmm_engine_t* engine, const pairhmm_batch_t* regions,
                                     int64_t num_regions, uint64_t* tickets);
pairhmm_status_t pairhmm_poll(pairhmm_engine_t* engine, uint64_t ticket, int32_t* done);
pairhmm_status_t pairhmm_drain(pairhmm_engine_t* engine, uint64_t ticket, float* scores,
                               int64_t num_scores, int32_t timeout_ms);

/* Submit-to-completion time of a finished region (valid until it is drained). */
pairhmm_status_t pairhmm_region_latency_ms(pairhmm_engine_t* engine, uint64_t ticket, double* ms);

/* Admission record of the serving queue (no counterpart in the reference):
 * regions completed, slot batches run, the most regions and estimated device
 * bytes admitted into one batch, the admission budget of a slot (device
 * budget / slots), the slot count, and the most slot batches on the device at
 * once.  All zero before the first submit. */
typedef struct pairhmm_serving_stats {
    int64_t regions;
    int64_t batches;
    int64_t max_batch_regions;
    int64_t max_batch_bytes;
    int64_t budget_per_slot;
    int32_t slots;
    int32_t max_in_flight;
} pairhmm_serving_stats_t;
pairhmm_status_t pairhmm_serving_stats(pairhmm_engine_t* engine, pairhmm_serving_stats_t* stats);

/*
 * Tile table: reads of length in (max_len[i-1], max_len[i]] run with groups of
 * group[i] lanes holding regs[i] read positions each (tile = group*regs).
 * kind[i] (the `multi_tile` argument): 0 = one tile, 1 = several tiles
 * (reads longer than the tile), 2 = one tile with two reads of a record per
 * group in packed FP32 arithmetic.  This is the run-time form of the
 * reference's compile-time tuning tables (tuningconfigs.hpp:33-269) and of its
 * partition rule "first tile size >= read length" (utility_kernels.cuh:45-57).
 * Only compiled (group, regs, kind) triples are accepted; the last entry must
 * be multi-tile.
 */
pairhmm_status_t pairhmm_set_tile_table(pairhmm_engine_t* engine, const int32_t* max_len, const int32_t* group,
                                        const int32_t* regs, const int32_t* multi_tile, int32_t n);
pairhmm_status_t pairhmm_get_tile_table(pairhmm_engine_t* engine, int32_t* max_len, int32_t* group,
                                        int32_t* regs, int32_t* multi_tile, int32_t capacity, int32_t* n);

/* Measurement utility (no counterpart in the reference): FP32 FMA throughput
 * of `device` in TFLOP/s (2 FLOP per FMA), best of several launches of about
 * `milliseconds` each.  Used as the roofline denominator. */
pairhmm_status_t pairhmm_probe_fp32_peak(int32_t device, int32_t milliseconds, double* tflops);
/* The same for FP64 FMAs: the FP64 pass's roofline denominator. */
pairhmm_status_t pairhmm_probe_fp64_peak(int32_t device, int32_t milliseconds, double* tflops);

/*
 * Record file format (README.md:41-61).  A parsed buffer owns its arrays; the
 * view points into them (valid until pairhmm_records_free).  Parsing and
 * formatting run on several host threads (pairhmm_set_host_threads); the
 * results do not depend on the thread count.
 *   pairhmm_records_parse   FileParserWorker::parseNextSequenceGroup +
 *                           convertGroupsToBatchInplace (file_parser_worker.cu:88-218):
 *                           R/H header, 5 fields per read at k*(L+1), quality - 33,
 *                           4 - len%4 bytes of 'N' padding (quality 'N'-33)
 *   pairhmm_records_format  OutputWriterWorker::run (output_writer_worker.cu:107-135):
 *                           "%d %d\n", then R lines of H "%.5f" joined by spaces,
 *                           the same text as the C library's printf gives.
 *                           With buf == NULL (or capacity too small) only *len is set.
 *   pairhmm_reader_*        FileParserWorker::run (file_parser_worker.cu:226-262): a
 *                           record file read batch by batch; next returns whole records
 *                           holding at least min_pairs pairs (<= 0: the rest of the
 *                           file), or *records = NULL at the end of the file.  A regular
 *                           file is mapped; other files are read whole at open.
 *   pairhmm_records_last_error  why the last parse or read on this thread failed
 *                           (names the 1-based line), "" if it did not.
 */
typedef struct pairhmm_records pairhmm_records_t;
pairhmm_status_t pairhmm_records_parse(const char* text, int64_t length, pairhmm_records_t** records);
pairhmm_status_t pairhmm_records_view(const pairhmm_records_t* records, pairhmm_batch_t* view,
                                      int64_t* num_pairs);
pairhmm_status_t pairhmm_records_format(const pairhmm_records_t* records, const float* scores, char* buf,
                                        int64_t capacity, int64_t* length);
void pairhmm_records_free(pairhmm_records_t* records);
typedef struct pairhmm_reader pairhmm_reader_t;
pairhmm_status_t pairhmm_reader_open(const char* path, pairhmm_reader_t** reader);
pairhmm_status_t pairhmm_reader_next(pairhmm_reader_t* reader, int64_t min_pairs, pairhmm_records_t** records);
void pairhmm_reader_close(pairhmm_reader_t* reader);
const char* pairhmm_records_last_error(void);
/* Host threads for record parsing and formatting: threads > 0 sets the count,
 * 0 returns to the default (PAIRHMM_HOST_THREADS, else all hardware threads;
 * at most 64). */
void pairhmm_set_host_threads(int32_t threads);

/*
 * No counterpart in the reference.  Allocation-free forward for callers that
 * cannot allocate device memory (a host that owns every device allocation, or
 * a context where cudaMalloc/cudaFree must not run because they synchronise
 * the device).  All arrays are the caller's device memory: the byte arrays
 * with the same meaning as in pairhmm_batch_t, `pairs` a flat list (offsets
 * into those arrays and lengths), `scores` one float per pair.  Work is
 * ordered on `stream` (a cudaStream_t, NULL = legacy default); the call does
 * not wait for it.  Nothing is allocated: the kernel's only scratch (borders
 * between 512-position read tiles) is a 64 MiB statically allocated device
 * array that every GPU loading the library keeps until exit.  Limits:
 * max_hap_length in [1, 16384] (above: PAIRHMM_ERR_LIMIT, nothing launched)
 * and every pair's hap_length <= max_hap_length (a longer pair, or an empty
 * read or haplotype, gets NaN); any read length.  FP32 only: pairs whose FP32
 * result underflows are not recomputed in FP64.  The first call on a device
 * sets it up (the scratch array's device address, the grid size); make that
 * first call before any stream capture.  Every call checks the address
 * against a fresh symbol lookup, so the entry point stays valid after the
 * device's context is torn down and created again; the probability table is
 * compiled into the module and needs no upload.  Launch errors are this
 * call's own: an error the caller left pending is neither returned nor
 * cleared.  All calls share the scratch: calls that overlap on the GPU race
 * and must be serialised by the caller.
 */
typedef struct pairhmm_pair {
    int64_t read_offset;
    int64_t hap_offset;
    int32_t read_length;
    int32_t hap_length;
} pairhmm_pair_t;
pairhmm_status_t pairhmm_forward_pairs_noalloc(int32_t device, const uint8_t* read_bases,
                                               const uint8_t* base_quals, const uint8_t* ins_quals,
                                               const uint8_t* del_quals, const uint8_t* hap_bases,
                                               const pairhmm_pair_t* pairs, int64_t num_pairs,
                                               int32_t max_hap_length, float* scores, void* stream);

const char* pairhmm_status_string(pairhmm_status_t status);
/* Message of the last failing call on this engine (empty when none). */
const char* pairhmm_last_error(const pairhmm_engine_t* engine);

/* Number of pairs and DP cells of a host batch (gpuworker.cuh:495-520). */
pairhmm_status_t pairhmm_batch_counts(const pairhmm_batch_t* batch, int64_t* pairs, int64_t* cells);

/*
 * Page-lock (and release) a caller's host buffer so that pairhmm_compute_host
 * uploads it by DMA straight from that memory; the buffer must not be freed
 * or reallocated while registered.  The reference gets the same effect by
 * allocating its batch vectors page-locked (PinnedAllocator, common.cuh:29-55).
 * Registering memory that is already page-locked is not an error.
 */
pairhmm_status_t pairhmm_host_register(void* ptr, size_t bytes);
pairhmm_status_t pairhmm_host_unregister(void* ptr);

/* Library version string. */
const char* pairhmm_version(void);

#ifdef __cplusplus
}
#endif
#endif /* PAIRHMM_B200_H */
