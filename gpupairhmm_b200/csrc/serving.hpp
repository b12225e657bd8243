// Continuous-batching request loop (no counterpart in the reference, which
// only processes whole files: gpuworker.cuh:435-471).
//
// submit() copies a region (one or more records) into host memory and queues
// it (submit_many() takes many regions per call).  kSlots worker threads each own an Engine (own stream and device
// buffers); a worker that becomes free takes every queued region that fits its
// share of the device budget, merges them into one batch, runs it, and
// completes the tickets.  While one slot's batch runs on the GPU the next slot
// is already admitting, uploading and launching, so the work of regions that
// arrive while others are on the device overlaps with them.
//
// Regions with reads longer than the largest single tile (multi-tile work,
// whose pairs each take a long serial wavefront) queue separately and run on
// their own two slots, so that a batch of short regions never waits behind
// them and a long region waits for at most one batch of long ones.
#pragma once

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "engine.hpp"

namespace phmm {

class ServingQueue {
public:
    explicit ServingQueue(Engine& parent);
    ~ServingQueue();

    pairhmm_status_t submit(const pairhmm_batch_t& region, uint64_t* ticket);
    // n regions under one lock and one wake-up; all are checked and copied
    // before any is queued, so an error queues none of them
    pairhmm_status_t submit_many(const pairhmm_batch_t* regions, int64_t n, uint64_t* tickets);
    pairhmm_status_t poll(uint64_t ticket, int32_t* done);
    pairhmm_status_t drain(uint64_t ticket, float* scores, int64_t num_scores, int32_t timeout_ms);
    pairhmm_status_t latency(uint64_t ticket, double* ms);
    void stats(pairhmm_serving_stats_t* out);
    // the last error of any call (a copy: calls may come from several threads)
    std::string last_error();

    static constexpr int kLightSlots = 2;          // regions of single-tile reads
    static constexpr int kSlots = kLightSlots + 2;  // + two slots for multi-tile regions

private:
    struct Region {
        uint64_t ticket = 0;
        // the region's inputs in one allocation: per record R and H, read and
        // haplotype lengths (int32), then the read bases, base/ins/del (and in gcp
        // mode gcp) qualities and the haplotype bases, each packed back to back
        std::unique_ptr<uint8_t[]> data;
        int64_t records = 0, reads = 0, haps = 0, read_bytes = 0, hap_bytes = 0;
        bool gcp = false;
        int64_t pairs = 0;
        int64_t device_bytes = 0;
        bool heavy = false;  // has a read beyond the largest single tile
        std::chrono::steady_clock::time_point t_submit, t_done;
        std::vector<float> scores;
        bool done = false;
        pairhmm_status_t status = PAIRHMM_OK;
        std::string error;

        const int32_t* rpr() const { return reinterpret_cast<const int32_t*>(data.get()); }
        const int32_t* hpr() const { return rpr() + records; }
        const int32_t* read_len() const { return hpr() + records; }
        const int32_t* hap_len() const { return read_len() + reads; }
        const uint8_t* read_part(int k) const {  // 0 bases, 1 base, 2 ins, 3 del, 4 gcp quals
            return data.get() + 4 * (2 * records + reads + haps) + k * read_bytes;
        }
        const uint8_t* hap_bases() const { return read_part(gcp ? 5 : 4); }
        // after the merge only the counts, pairs and results are used
        void release_inputs() { data.reset(); }
    };

    // reusable, uninitialised host buffer of a slot's merged batch
    struct MergeBuf {
        std::unique_ptr<uint8_t[]> p;
        size_t cap = 0;
        template <class T>
        T* get(int64_t n) {
            const size_t bytes = (size_t)std::max<int64_t>(n, 1) * sizeof(T);
            if (bytes > cap) {
                cap = bytes + bytes / 4;
                p.reset(new uint8_t[cap]);
            }
            return reinterpret_cast<T*>(p.get());
        }
    };

    void worker(int slot);
    // checks a region and copies it into host memory owned by the queue (no lock held)
    pairhmm_status_t prepare(const pairhmm_batch_t& b, std::shared_ptr<Region>& out, std::string& err) const;
    // gives the regions tickets and queues them (starts the slots on first use)
    pairhmm_status_t enqueue(const std::vector<std::shared_ptr<Region>>& rs,
                             std::chrono::steady_clock::time_point t_submit, uint64_t* tickets);
    static int64_t estimate_device_bytes(const Region& r);
    pairhmm_status_t set_error(pairhmm_status_t s, const char* msg);  // caller holds mu_

    Engine& parent_;
    int64_t budget_per_slot_ = 0;
    std::vector<std::unique_ptr<Engine>> engines_;
    std::vector<std::thread> threads_;
    std::mutex mu_;
    std::condition_variable cv_work_, cv_done_;
    std::deque<std::shared_ptr<Region>> light_, heavy_;
    int32_t single_tile_max_ = 0;  // longest read length without multi-tile work
    std::map<uint64_t, std::shared_ptr<Region>> tickets_;
    uint64_t next_ticket_ = 1;
    bool stop_ = false;
    std::string error_;
    // admission record (under mu_)
    int64_t batches_ = 0, regions_done_ = 0, max_batch_regions_ = 0, max_batch_bytes_ = 0;
    int32_t in_flight_ = 0, max_in_flight_ = 0;
};

}  // namespace phmm
