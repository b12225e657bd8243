// Host-to-device upload of caller buffers for one batch.
//
// Page-locked sources (cudaMallocHost / cudaHostAlloc / cudaHostRegister) are
// copied by DMA straight from the caller's memory.  Pageable sources go
// through a ring of page-locked staging slots: several host threads each copy
// a slot's worth out of the caller's memory and enqueue that slot's DMA, then
// reuse the slot once its DMA has completed, so the host copies run in
// parallel with one another and with the DMA of earlier slots.  (A single
// cudaMemcpyAsync from pageable memory is staged by the driver one piece at a
// time on the calling thread.)  Downloads use the same slots in the other
// direction.  The copy threads are created once and kept: a batch creates no
// threads and maps no memory.
#pragma once

#include <cuda_runtime.h>

#include <condition_variable>
#include <cstddef>
#include <mutex>
#include <thread>
#include <vector>

namespace phmm {

class HostUploader {
public:
    struct Copy {
        void* dst;        // device
        const void* src;  // host, page-locked or pageable
        size_t bytes;
    };

    HostUploader() = default;
    ~HostUploader();
    HostUploader(const HostUploader&) = delete;
    HostUploader& operator=(const HostUploader&) = delete;

    // Enqueues every copy on stream s (device `device` is made current on the
    // copy threads).  start() enqueues the page-locked copies and hands the
    // pageable ones to the copy threads; finish() returns once every copy is
    // enqueued and every pageable byte has been read: the caller may then
    // reuse its host buffers, and work enqueued on s afterwards sees the data.
    // Between the two the calling thread is free (the engine builds its index).
    cudaError_t start(int device, const std::vector<Copy>& copies, cudaStream_t s);
    cudaError_t finish();
    cudaError_t run(int device, const std::vector<Copy>& copies, cudaStream_t s) {
        const cudaError_t e = start(device, copies, s);
        const cudaError_t f = finish();
        return e != cudaSuccess ? e : f;
    }

    // Device-to-host copy of `bytes` after the work already on stream s: one
    // DMA into a page-locked `dst`, else chunks through the staging slots,
    // each copied out on the host as soon as its DMA lands.  Returns when dst
    // holds the data.
    cudaError_t download(int device, void* dst, const void* src, size_t bytes, cudaStream_t s);

    // bytes that went through staging / straight from page-locked memory in the
    // last run
    size_t staged_bytes() const { return staged_; }
    size_t direct_bytes() const { return direct_; }

    static bool is_page_locked(const void* p);

private:
    static constexpr int kThreads = 4;
    static constexpr int kSlotsPerThread = 2;
    static constexpr size_t kSlotBytes = size_t(8) << 20;
    cudaError_t ensure_staging();
    void worker_loop(int t);
    void copy_pieces(int t);

    struct Piece {
        char* dst;
        const char* src;
        size_t bytes;
    };
    char* stage_ = nullptr;
    cudaEvent_t done_[kThreads * kSlotsPerThread] = {};
    size_t staged_ = 0, direct_ = 0;

    // the current staged job, worked on by the copy threads
    std::vector<Piece> pieces_;
    int device_ = 0;
    cudaStream_t stream_ = nullptr;
    cudaError_t err_[kThreads] = {};
    std::vector<std::thread> workers_;
    std::mutex mu_;
    std::condition_variable cv_work_, cv_done_;
    unsigned long long job_ = 0;  // incremented per job
    int busy_ = 0;                // threads still on the current job
    bool stop_ = false;
};

}  // namespace phmm
