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
// direction.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
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
    // helper threads).  Returns once every copy is enqueued and every pageable
    // byte has been read: the caller may then reuse its host buffers, and work
    // enqueued on s afterwards sees the data.
    cudaError_t run(int device, const std::vector<Copy>& copies, cudaStream_t s);

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

    char* stage_ = nullptr;
    cudaEvent_t done_[kThreads * kSlotsPerThread] = {};
    size_t staged_ = 0, direct_ = 0;
};

}  // namespace phmm
