// Transfers between ordinary (pageable) host memory and the device.
//
// The reference wraps every host array in an OpenCL buffer per call
// (core/src/ocl/ocl_buffer.cpp:27-42) and reads the outputs back before
// returning (core/src/ocl/ocl_kernel.cpp:59-111); a drop-in caller therefore
// passes ordinary malloc'd memory.  A DMA engine can only read page-locked
// memory, so such a copy goes through pinned memory either way.  Here each
// handle owns two pinned bounce buffers: while the DMA engine moves one
// buffer, host threads of a process-wide pool copy the next chunk into (or
// out of) the other, so the host-side copies and the PCIe transfers overlap.
#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <vector>

#include "internal.h"

namespace iclb {
namespace {

constexpr size_t kBounceBytes = (size_t)32 << 20;   // one bounce buffer
constexpr size_t kSliceBytes = (size_t)2 << 20;     // host-copy work per thread and task

// Process-wide pool of host threads for large memcpy calls (started on first
// use).  A call splits its copy into slices, queues all but one, copies one
// itself and waits for its own slices only.
class CopyPool {
public:
    static CopyPool& get()
    {
        static CopyPool pool;
        return pool;
    }

    void copy(void* dst, const void* src, size_t bytes)
    {
        const size_t nslices = std::min<size_t>(workers_.size() + 1, (bytes + kSliceBytes - 1) / kSliceBytes);
        if (nslices <= 1) {
            std::memcpy(dst, src, bytes);
            return;
        }
        Batch b;
        b.left.store((int)nslices - 1);
        const size_t per = (bytes + nslices - 1) / nslices;
        {
            std::lock_guard<std::mutex> lock(mu_);
            for (size_t i = 1; i < nslices; ++i) {
                const size_t off = i * per;
                if (off >= bytes) {
                    b.left.fetch_sub(1);
                    continue;
                }
                q_.push_back(Task{(char*)dst + off, (const char*)src + off, std::min(per, bytes - off), &b});
            }
        }
        cv_.notify_all();
        std::memcpy(dst, src, std::min(per, bytes));
        std::unique_lock<std::mutex> lock(mu_);
        done_.wait(lock, [&] { return b.left.load() == 0; });
    }

    ~CopyPool()
    {
        {
            std::lock_guard<std::mutex> lock(mu_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto& t : workers_) t.join();
    }

private:
    struct Batch {
        std::atomic<int> left{0};
    };
    struct Task {
        char* dst;
        const char* src;
        size_t bytes;
        Batch* batch;
    };

    CopyPool()
    {
        const unsigned hw = std::max(2u, std::thread::hardware_concurrency());
        const unsigned n = std::min(8u, hw / 2);
        for (unsigned i = 0; i < n; ++i) workers_.emplace_back([this] { run(); });
    }

    void run()
    {
        std::unique_lock<std::mutex> lock(mu_);
        for (;;) {
            cv_.wait(lock, [&] { return stop_ || !q_.empty(); });
            if (stop_ && q_.empty()) return;
            Task t = q_.front();
            q_.pop_front();
            lock.unlock();
            std::memcpy(t.dst, t.src, t.bytes);
            lock.lock();
            if (t.batch->left.fetch_sub(1) == 1) done_.notify_all();
        }
    }

    std::mutex mu_;
    std::condition_variable cv_, done_;
    std::deque<Task> q_;
    std::vector<std::thread> workers_;
    bool stop_ = false;
};

cudaError_t ensure_bounce(iclblasHandle_t h)
{
    for (int b = 0; b < 2; ++b) {
        cudaError_t e;
        if (!h->bounce[b] && (e = cudaHostAlloc(&h->bounce[b], kBounceBytes, cudaHostAllocDefault)) != cudaSuccess)
            return e;
        if (!h->bounce_ev[b] && (e = cudaEventCreateWithFlags(&h->bounce_ev[b], cudaEventDisableTiming)) != cudaSuccess)
            return e;
    }
    return cudaSuccess;
}

// Waits until the copy that last used bounce buffer b has finished with it.
cudaError_t bounce_free(iclblasHandle_t h, int b)
{
    if (!h->bounce_busy[b]) return cudaSuccess;
    h->bounce_busy[b] = false;
    return cudaEventSynchronize(h->bounce_ev[b]);
}

}  // namespace

void host_copy(void* dst, const void* src, size_t bytes) { CopyPool::get().copy(dst, src, bytes); }

cudaError_t copy_pageable_h2d(iclblasHandle_t h, void* dst, const void* src, size_t bytes)
{
    cudaError_t e = ensure_bounce(h);
    if (e != cudaSuccess) return e;
    size_t off = 0;
    for (int i = 0; off < bytes; ++i) {
        const int b = i & 1;
        const size_t len = std::min(kBounceBytes, bytes - off);
        if ((e = bounce_free(h, b)) != cudaSuccess) return e;
        host_copy(h->bounce[b], (const char*)src + off, len);
        if ((e = cudaMemcpyAsync((char*)dst + off, h->bounce[b], len, cudaMemcpyHostToDevice, h->stream)) !=
            cudaSuccess)
            return e;
        if ((e = cudaEventRecord(h->bounce_ev[b], h->stream)) != cudaSuccess) return e;
        h->bounce_busy[b] = true;
        off += len;
    }
    return cudaSuccess;
}

cudaError_t copy_pageable_d2h(iclblasHandle_t h, void* dst, const void* src, size_t bytes)
{
    cudaError_t e = ensure_bounce(h);
    if (e != cudaSuccess) return e;
    const int nchunks = (int)((bytes + kBounceBytes - 1) / kBounceBytes);
    auto issue = [&](int i) -> cudaError_t {
        const int b = i & 1;
        const size_t off = (size_t)i * kBounceBytes, len = std::min(kBounceBytes, bytes - off);
        cudaError_t r = bounce_free(h, b);
        if (r != cudaSuccess) return r;
        if ((r = cudaMemcpyAsync(h->bounce[b], (const char*)src + off, len, cudaMemcpyDeviceToHost, h->stream)) !=
            cudaSuccess)
            return r;
        if ((r = cudaEventRecord(h->bounce_ev[b], h->stream)) != cudaSuccess) return r;
        h->bounce_busy[b] = true;
        return cudaSuccess;
    };
    if (nchunks > 0 && (e = issue(0)) != cudaSuccess) return e;
    for (int i = 0; i < nchunks; ++i) {
        // the DMA of chunk i + 1 runs while chunk i is copied out
        if (i + 1 < nchunks && (e = issue(i + 1)) != cudaSuccess) return e;
        const int b = i & 1;
        if ((e = cudaEventSynchronize(h->bounce_ev[b])) != cudaSuccess) return e;
        const size_t off = (size_t)i * kBounceBytes, len = std::min(kBounceBytes, bytes - off);
        host_copy((char*)dst + off, h->bounce[b], len);
        h->bounce_busy[b] = false;
    }
    return cudaSuccess;
}

cudaError_t free_bounce(iclblasHandle_t h)
{
    cudaError_t r = cudaSuccess;
    for (int b = 0; b < 2; ++b) {
        if (h->bounce_ev[b]) {
            cudaEventSynchronize(h->bounce_ev[b]);
            cudaEventDestroy(h->bounce_ev[b]);
            h->bounce_ev[b] = nullptr;
        }
        if (h->bounce[b]) {
            cudaError_t e = cudaFreeHost(h->bounce[b]);
            if (r == cudaSuccess) r = e;
            h->bounce[b] = nullptr;
        }
        h->bounce_busy[b] = false;
    }
    return r;
}

}  // namespace iclb
