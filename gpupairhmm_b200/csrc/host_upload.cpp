#include "host_upload.hpp"

#include <algorithm>
#include <cstring>
#include <thread>

namespace phmm {

HostUploader::~HostUploader() {
    {
        std::lock_guard<std::mutex> lk(mu_);
        stop_ = true;
    }
    cv_work_.notify_all();
    for (std::thread& th : workers_) th.join();
    for (cudaEvent_t& e : done_)
        if (e) cudaEventDestroy(e);
    if (stage_) cudaFreeHost(stage_);
}

bool HostUploader::is_page_locked(const void* p) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();  // pageable memory on older runtimes reports an error; clear it
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

cudaError_t HostUploader::ensure_staging() {
    if (stage_) return cudaSuccess;
    void* p = nullptr;
    cudaError_t e = cudaMallocHost(&p, kSlotBytes * kThreads * kSlotsPerThread);
    if (e != cudaSuccess) return e;
    stage_ = static_cast<char*>(p);
    for (cudaEvent_t& ev : done_)
        if ((e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming)) != cudaSuccess) return e;
    return cudaSuccess;
}

void HostUploader::worker_loop(int t) {
    unsigned long long seen = 0;
    for (;;) {
        {
            std::unique_lock<std::mutex> lk(mu_);
            cv_work_.wait(lk, [&] { return stop_ || job_ != seen; });
            if (stop_) return;
            seen = job_;
        }
        copy_pieces(t);
        {
            std::lock_guard<std::mutex> lk(mu_);
            --busy_;
        }
        cv_done_.notify_all();
    }
}

// copy thread t takes pieces t, t + kThreads, ... through its two slots
void HostUploader::copy_pieces(int t) {
    cudaError_t r = cudaSetDevice(device_);
    int j = 0;
    for (size_t k = (size_t)t; k < pieces_.size() && r == cudaSuccess; k += kThreads, ++j) {
        const int slot = t * kSlotsPerThread + (j % kSlotsPerThread);
        char* buf = stage_ + (size_t)slot * kSlotBytes;
        // the slot's previous DMA (this job or an earlier one) must be done
        if ((r = cudaEventSynchronize(done_[slot])) != cudaSuccess) break;
        std::memcpy(buf, pieces_[k].src, pieces_[k].bytes);
        if ((r = cudaMemcpyAsync(pieces_[k].dst, buf, pieces_[k].bytes, cudaMemcpyHostToDevice, stream_)) !=
            cudaSuccess)
            break;
        r = cudaEventRecord(done_[slot], stream_);
    }
    err_[t] = r;
}

cudaError_t HostUploader::start(int device, const std::vector<Copy>& copies, cudaStream_t s) {
    staged_ = direct_ = 0;
    pieces_.clear();
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return e;
    for (const Copy& c : copies) {
        if (c.bytes == 0) continue;
        if (is_page_locked(c.src)) {
            if ((e = cudaMemcpyAsync(c.dst, c.src, c.bytes, cudaMemcpyHostToDevice, s)) != cudaSuccess) return e;
            direct_ += c.bytes;
            continue;
        }
        for (size_t off = 0; off < c.bytes; off += kSlotBytes)
            pieces_.push_back({static_cast<char*>(c.dst) + off, static_cast<const char*>(c.src) + off,
                               std::min(kSlotBytes, c.bytes - off)});
        staged_ += c.bytes;
    }
    if (pieces_.empty()) return cudaSuccess;
    if ((e = ensure_staging()) != cudaSuccess) {
        pieces_.clear();
        return e;
    }
    if (workers_.empty())
        for (int t = 0; t < kThreads; ++t) workers_.emplace_back(&HostUploader::worker_loop, this, t);
    device_ = device;
    stream_ = s;
    {
        std::lock_guard<std::mutex> lk(mu_);
        for (cudaError_t& x : err_) x = cudaSuccess;
        busy_ = kThreads;
        ++job_;
    }
    cv_work_.notify_all();
    return cudaSuccess;
}

cudaError_t HostUploader::finish() {
    if (pieces_.empty()) return cudaSuccess;
    {
        std::unique_lock<std::mutex> lk(mu_);
        cv_done_.wait(lk, [&] { return busy_ == 0; });
    }
    pieces_.clear();
    for (cudaError_t x : err_)
        if (x != cudaSuccess) return x;
    return cudaSuccess;
}

cudaError_t HostUploader::download(int device, void* dst, const void* src, size_t bytes, cudaStream_t s) {
    if (bytes == 0) return cudaSuccess;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return e;
    if (is_page_locked(dst)) {
        if ((e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s)) != cudaSuccess) return e;
        return cudaStreamSynchronize(s);
    }
    if ((e = ensure_staging()) != cudaSuccess) return e;
    constexpr int kSlots = kThreads * kSlotsPerThread;
    const size_t n = (bytes + kSlotBytes - 1) / kSlotBytes;
    auto issue = [&](size_t k) -> cudaError_t {
        const int slot = (int)(k % kSlots);
        const size_t off = k * kSlotBytes, len = std::min(kSlotBytes, bytes - off);
        cudaError_t r = cudaEventSynchronize(done_[slot]);  // the slot's earlier use is over
        if (r == cudaSuccess)
            r = cudaMemcpyAsync(stage_ + (size_t)slot * kSlotBytes, static_cast<const char*>(src) + off, len,
                                cudaMemcpyDeviceToHost, s);
        if (r == cudaSuccess) r = cudaEventRecord(done_[slot], s);
        return r;
    };
    for (size_t k = 0; k < n && k < (size_t)kSlots; ++k)
        if ((e = issue(k)) != cudaSuccess) return e;
    for (size_t k = 0; k < n; ++k) {
        const int slot = (int)(k % kSlots);
        if ((e = cudaEventSynchronize(done_[slot])) != cudaSuccess) return e;
        const size_t off = k * kSlotBytes, len = std::min(kSlotBytes, bytes - off);
        std::memcpy(static_cast<char*>(dst) + off, stage_ + (size_t)slot * kSlotBytes, len);
        if (k + kSlots < n && (e = issue(k + kSlots)) != cudaSuccess) return e;
    }
    staged_ += bytes;
    return cudaSuccess;
}

}  // namespace phmm
