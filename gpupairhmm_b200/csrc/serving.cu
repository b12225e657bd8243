#include <algorithm>
#include <cstring>
#include <new>
#include <stdexcept>
#include <string>

#include "serving.hpp"

namespace phmm {

namespace {
constexpr int64_t kDefaultBudget = int64_t(40) << 30;  // 40 GiB
constexpr int64_t kMaxBatchPairs = int64_t(4) << 20;   // cap on pairs merged into one batch
constexpr int64_t kReservePerSlot = int64_t(3) << 30;  // device memory a slot keeps from its start
}  // namespace

ServingQueue::ServingQueue(Engine& parent) : parent_(parent) {
    // the parent's options carry the budget; each slot gets an equal share
    const int64_t budget = parent.budget_bytes() > 0 ? parent.budget_bytes() : kDefaultBudget;
    budget_per_slot_ = budget / kSlots;
    for (const TileRule& r : parent.tile_table())
        if (!r.multi_tile) single_tile_max_ = std::max(single_tile_max_, r.max_len);
}

ServingQueue::~ServingQueue() {
    {
        std::lock_guard<std::mutex> lk(mu_);
        stop_ = true;
    }
    cv_work_.notify_all();
    for (auto& t : threads_) t.join();
}

pairhmm_status_t ServingQueue::set_error(pairhmm_status_t s, const char* msg) {
    error_ = msg;
    return s;
}

std::string ServingQueue::last_error() {
    std::lock_guard<std::mutex> lk(mu_);
    return error_;
}

void ServingQueue::stats(pairhmm_serving_stats_t* out) {
    std::lock_guard<std::mutex> lk(mu_);
    out->regions = regions_done_;
    out->batches = batches_;
    out->max_batch_regions = max_batch_regions_;
    out->max_batch_bytes = max_batch_bytes_;
    out->budget_per_slot = budget_per_slot_;
    out->slots = kSlots;
    out->max_in_flight = max_in_flight_;
}

int64_t ServingQueue::estimate_device_bytes(const Region& r) {
    // inputs (4 byte arrays + haplotypes), packed copies, work items, rescue
    // list and scores, plus the per-read/per-haplotype index arrays
    int64_t pos = 0, hb = 0;
    for (int64_t i = 0; i < r.reads; ++i) pos += (r.read_len()[i] + 3) & ~3;
    for (int64_t h = 0; h < r.haps; ++h) hb += (r.hap_len()[h] + 15) & ~15;
    return 4 * r.read_bytes + 2 * r.hap_bytes + 4 * pos + hb + r.pairs * (16 + 16 + 4) + r.reads * 32 +
           r.haps * 24 + 4096;
}

pairhmm_status_t ServingQueue::prepare(const pairhmm_batch_t& b, std::shared_ptr<Region>& out,
                                       std::string& err) const {
    // the checks of a batch call (counts, null arrays, lengths, offsets, gcp),
    // without building its work list: the slot's merged batch builds that
    InputRanges x;
    const bool gcp = parent_.gcp();
    const pairhmm_status_t st = Engine::scan_inputs(b, x, err, gcp);
    if (st != PAIRHMM_OK) return st;
    auto r = std::make_shared<Region>();
    r->records = b.num_records;
    r->reads = x.num_reads;
    r->haps = x.num_haps;
    r->gcp = gcp;
    int32_t max_read_len = 0;
    for (int64_t i = 0; i < x.num_reads; ++i) {
        r->read_bytes += b.read_lengths[i];
        max_read_len = std::max(max_read_len, b.read_lengths[i]);
    }
    for (int64_t h = 0; h < x.num_haps; ++h) r->hap_bytes += b.hap_lengths[h];
    const int64_t ints = 2 * r->records + r->reads + r->haps;
    r->data.reset(new uint8_t[(size_t)std::max<int64_t>(4 * ints + (gcp ? 5 : 4) * r->read_bytes + r->hap_bytes, 1)]);
    int32_t* ip = reinterpret_cast<int32_t*>(r->data.get());
    auto put = [](void* dst, const void* src, int64_t bytes) {
        if (bytes > 0) std::memcpy(dst, src, (size_t)bytes);
    };
    put(ip, b.reads_per_record, 4 * r->records);
    put(ip + r->records, b.haps_per_record, 4 * r->records);
    put(ip + 2 * r->records, b.read_lengths, 4 * r->reads);
    put(ip + 2 * r->records + r->reads, b.hap_lengths, 4 * r->haps);
    // compact copy: each read/haplotype stored back to back
    uint8_t* rp = r->data.get() + 4 * ints;
    const int64_t rbytes = r->read_bytes;
    for (int64_t i = 0, d = 0; i < x.num_reads; ++i) {
        const int64_t o = b.read_offsets[i], L = b.read_lengths[i];
        put(rp + d, b.read_bases + o, L);
        put(rp + rbytes + d, b.base_quals + o, L);
        put(rp + 2 * rbytes + d, b.ins_quals + o, L);
        put(rp + 3 * rbytes + d, b.del_quals + o, L);
        if (gcp) put(rp + 4 * rbytes + d, b.gcp_quals + o, L);
        d += L;
    }
    uint8_t* hp = rp + (gcp ? 5 : 4) * rbytes;
    for (int64_t h = 0, d = 0; h < x.num_haps; ++h) {
        put(hp + d, b.hap_bases + b.hap_offsets[h], b.hap_lengths[h]);
        d += b.hap_lengths[h];
    }
    r->pairs = x.num_pairs;
    r->heavy = max_read_len > single_tile_max_;
    r->device_bytes = estimate_device_bytes(*r);
    if (r->device_bytes > budget_per_slot_) {
        err = "region needs more device memory than one batch slot's budget";
        return PAIRHMM_ERR_BUDGET;
    }
    out = std::move(r);
    return PAIRHMM_OK;
}

pairhmm_status_t ServingQueue::enqueue(const std::vector<std::shared_ptr<Region>>& rs,
                                       std::chrono::steady_clock::time_point t_submit, uint64_t* tickets) {
    {
        std::lock_guard<std::mutex> lk(mu_);
        if (engines_.empty()) {
            for (int s = 0; s < kSlots; ++s) {
                pairhmm_options_t o{};
                o.device = parent_.device();
                o.mode = PAIRHMM_MODE_ENGINE;
                o.fp64_rescue = 1;
                o.use_graphs = 1;
                o.pipeline_chunks = 1;  // merged batches stay small: one pass
                o.gcp = parent_.gcp() ? 1 : 0;
                auto e = std::make_unique<Engine>(o);
                pairhmm_status_t is = e->init();
                if (is == PAIRHMM_OK) is = e->set_tile_table(parent_.tile_table());
                // device memory for the slot's batches up front (its budget, at most
                // kReservePerSlot): a batch larger than any before then grows its buffers
                // inside the pool instead of mapping memory while the other slots run
                if (is == PAIRHMM_OK) is = e->reserve_pool((size_t)std::min(budget_per_slot_, kReservePerSlot));
                if (is != PAIRHMM_OK) {
                    error_ = e->last_error();
                    engines_.clear();
                    return is;  // mu_ is held: error_ is written under it
                }
                engines_.push_back(std::move(e));
            }
            for (int s = 0; s < kSlots; ++s) threads_.emplace_back(&ServingQueue::worker, this, s);
        }
        for (size_t i = 0; i < rs.size(); ++i) {
            const std::shared_ptr<Region>& r = rs[i];
            r->t_submit = t_submit;
            r->ticket = next_ticket_++;
            tickets_[r->ticket] = r;
            (r->heavy ? heavy_ : light_).push_back(r);
            tickets[i] = r->ticket;
        }
    }
    cv_work_.notify_all();
    return PAIRHMM_OK;
}

pairhmm_status_t ServingQueue::submit(const pairhmm_batch_t& b, uint64_t* ticket) {
    return submit_many(&b, 1, ticket);
}

pairhmm_status_t ServingQueue::submit_many(const pairhmm_batch_t* regions, int64_t n, uint64_t* tickets) {
    if (n < 0 || (n > 0 && (!regions || !tickets))) {
        std::lock_guard<std::mutex> lk(mu_);
        return set_error(PAIRHMM_ERR_INVALID_ARGUMENT, "bad region list");
    }
    const auto t_submit = std::chrono::steady_clock::now();  // latency counts the copies below
    std::vector<std::shared_ptr<Region>> rs((size_t)n);
    for (int64_t i = 0; i < n; ++i) {
        std::string err;
        const pairhmm_status_t st = prepare(regions[i], rs[(size_t)i], err);
        if (st != PAIRHMM_OK) {
            if (n > 1) err = "region " + std::to_string(i) + ": " + err;
            std::lock_guard<std::mutex> lk(mu_);
            return set_error(st, err.c_str());
        }
    }
    if (n == 0) return PAIRHMM_OK;
    return enqueue(rs, t_submit, tickets);
}

void ServingQueue::worker(int slot) {
    Engine& eng = *engines_[slot];
    std::deque<std::shared_ptr<Region>>& queue = slot < kLightSlots ? light_ : heavy_;
    // merge buffers live as long as the slot: a batch maps no new memory once
    // they have grown to the slot's usual size (uninitialised: every byte is
    // written by the merge)
    MergeBuf m_rpr, m_hpr, m_rl, m_hl, m_ro, m_ho, m_rb, m_bq, m_iq, m_dq, m_gq, m_hb;
    std::vector<float> scores;
    for (;;) {
        std::vector<std::shared_ptr<Region>> take;
        bool more = false;
        {
            std::unique_lock<std::mutex> lk(mu_);
            cv_work_.wait(lk, [&] { return stop_ || !queue.empty(); });
            if (stop_ && queue.empty()) return;
            // admission: everything queued that fits this slot's budget
            int64_t bytes = 0, pairs = 0;
            while (!queue.empty()) {
                const auto& r = queue.front();
                if (!take.empty() && (bytes + r->device_bytes > budget_per_slot_ || pairs + r->pairs > kMaxBatchPairs))
                    break;
                bytes += r->device_bytes;
                pairs += r->pairs;
                take.push_back(r);
                queue.pop_front();
            }
            more = !queue.empty();
            ++batches_;
            max_batch_regions_ = std::max<int64_t>(max_batch_regions_, (int64_t)take.size());
            max_batch_bytes_ = std::max(max_batch_bytes_, bytes);
            max_in_flight_ = std::max(max_in_flight_, ++in_flight_);
        }
        if (more) cv_work_.notify_all();
        // merge the regions into one batch and run it; a failure (host memory
        // included: this thread has no caller to throw to) fails the batch's regions
        pairhmm_status_t st = PAIRHMM_OK;
        std::string batch_error;
        try {
            int64_t nrec = 0, nreads = 0, nhaps = 0, rbytes = 0, hbytes = 0;
            bool gcp = false;
            for (const auto& r : take) {
                nrec += r->records;
                nreads += r->reads;
                nhaps += r->haps;
                rbytes += r->read_bytes;
                hbytes += r->hap_bytes;
                gcp = gcp || r->gcp;
            }
            int32_t* rpr = m_rpr.get<int32_t>(nrec);
            int32_t* hpr = m_hpr.get<int32_t>(nrec);
            int32_t* rl = m_rl.get<int32_t>(nreads);
            int32_t* hl = m_hl.get<int32_t>(nhaps);
            int64_t* ro = m_ro.get<int64_t>(nreads);
            int64_t* ho = m_ho.get<int64_t>(nhaps);
            uint8_t* rb = m_rb.get<uint8_t>(rbytes);
            uint8_t* bq = m_bq.get<uint8_t>(rbytes);
            uint8_t* iq = m_iq.get<uint8_t>(rbytes);
            uint8_t* dq = m_dq.get<uint8_t>(rbytes);
            uint8_t* gq = gcp ? m_gq.get<uint8_t>(rbytes) : nullptr;
            uint8_t* hb = m_hb.get<uint8_t>(hbytes);
            {
                int64_t g = 0, i = 0, h = 0, rp = 0, hp = 0;
                auto put = [](void* dst, const void* src, int64_t bytes) {
                    if (bytes > 0) std::memcpy(dst, src, (size_t)bytes);
                };
                for (const auto& r : take) {
                    put(rpr + g, r->rpr(), 4 * r->records);
                    put(hpr + g, r->hpr(), 4 * r->records);
                    put(rl + i, r->read_len(), 4 * r->reads);
                    put(hl + h, r->hap_len(), 4 * r->haps);
                    for (int64_t k = 0, o = rp; k < r->reads; ++k) {
                        ro[i + k] = o;
                        o += r->read_len()[k];
                    }
                    for (int64_t k = 0, o = hp; k < r->haps; ++k) {
                        ho[h + k] = o;
                        o += r->hap_len()[k];
                    }
                    put(rb + rp, r->read_part(0), r->read_bytes);
                    put(bq + rp, r->read_part(1), r->read_bytes);
                    put(iq + rp, r->read_part(2), r->read_bytes);
                    put(dq + rp, r->read_part(3), r->read_bytes);
                    if (gcp) put(gq + rp, r->read_part(4), r->read_bytes);
                    put(hb + hp, r->hap_bases(), r->hap_bytes);
                    g += r->records;
                    i += r->reads;
                    h += r->haps;
                    rp += r->read_bytes;
                    hp += r->hap_bytes;
                    // the merged copy is all the batch needs: give the region's input copy back
                    // now rather than when it is drained (a client that drains late would
                    // otherwise hold every input it submitted meanwhile)
                    r->release_inputs();
                }
            }
            pairhmm_batch_t b{};
            b.num_records = nrec;
            b.reads_per_record = rpr;
            b.haps_per_record = hpr;
            b.read_bases = rb;
            b.base_quals = bq;
            b.ins_quals = iq;
            b.del_quals = dq;
            b.gcp_quals = gq;
            b.read_offsets = ro;
            b.read_lengths = rl;
            b.hap_bases = hb;
            b.hap_offsets = ho;
            b.hap_lengths = hl;
            int64_t total_pairs = 0;
            for (const auto& r : take) total_pairs += r->pairs;
            scores.resize((size_t)std::max<int64_t>(total_pairs, 1));
            st = eng.compute_host(b, scores.data());
            if (st != PAIRHMM_OK) batch_error = eng.last_error();
        } catch (const std::bad_alloc&) {
            st = PAIRHMM_ERR_OUT_OF_MEMORY;
            batch_error = "host allocation failed while merging a batch";
        } catch (const std::exception& e) {
            st = PAIRHMM_ERR_CUDA;
            batch_error = e.what();
        }
        const auto now = std::chrono::steady_clock::now();
        {
            std::lock_guard<std::mutex> lk(mu_);
            --in_flight_;
            regions_done_ += (int64_t)take.size();
            int64_t off = 0;
            for (const auto& r : take) {
                r->status = st;
                if (st != PAIRHMM_OK) {
                    r->error = batch_error;
                } else {
                    try {
                        r->scores.assign(scores.begin() + off, scores.begin() + off + r->pairs);
                    } catch (const std::bad_alloc&) {
                        r->status = PAIRHMM_ERR_OUT_OF_MEMORY;
                        r->error = "host allocation failed for the region's scores";
                    }
                }
                off += r->pairs;
                r->t_done = now;
                r->done = true;
            }
        }
        cv_done_.notify_all();
    }
}

pairhmm_status_t ServingQueue::poll(uint64_t ticket, int32_t* done) {
    std::lock_guard<std::mutex> lk(mu_);
    auto it = tickets_.find(ticket);
    if (it == tickets_.end()) return set_error(PAIRHMM_ERR_NOT_FOUND, "unknown ticket");
    *done = it->second->done ? 1 : 0;
    return PAIRHMM_OK;
}

pairhmm_status_t ServingQueue::latency(uint64_t ticket, double* ms) {
    std::lock_guard<std::mutex> lk(mu_);
    auto it = tickets_.find(ticket);
    if (it == tickets_.end()) return set_error(PAIRHMM_ERR_NOT_FOUND, "unknown ticket");
    if (!it->second->done) return set_error(PAIRHMM_ERR_BUSY, "region not finished");
    *ms = std::chrono::duration<double, std::milli>(it->second->t_done - it->second->t_submit).count();
    return PAIRHMM_OK;
}

pairhmm_status_t ServingQueue::drain(uint64_t ticket, float* scores, int64_t num_scores, int32_t timeout_ms) {
    std::unique_lock<std::mutex> lk(mu_);
    auto it = tickets_.find(ticket);
    if (it == tickets_.end()) return set_error(PAIRHMM_ERR_NOT_FOUND, "unknown ticket");
    std::shared_ptr<Region> r = it->second;
    if (timeout_ms < 0) cv_done_.wait(lk, [&] { return r->done; });
    else if (!cv_done_.wait_for(lk, std::chrono::milliseconds(timeout_ms), [&] { return r->done; }))
        return set_error(PAIRHMM_ERR_TIMEOUT, "timed out waiting for the region");
    // the wait released mu_: another thread may have drained this ticket meanwhile,
    // so the map entry is looked up again rather than reused
    if (tickets_.find(ticket) == tickets_.end())
        return set_error(PAIRHMM_ERR_NOT_FOUND, "ticket drained by another call");
    if (r->status != PAIRHMM_OK) {
        error_ = r->error;
        tickets_.erase(ticket);
        return r->status;
    }
    if (num_scores < r->pairs)
        return set_error(PAIRHMM_ERR_INVALID_ARGUMENT, "score buffer smaller than the region's pair count");
    std::copy(r->scores.begin(), r->scores.end(), scores);
    tickets_.erase(ticket);
    return PAIRHMM_OK;
}

}  // namespace phmm
