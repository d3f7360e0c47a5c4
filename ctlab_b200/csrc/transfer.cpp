// Host <-> device copies of the host-pointer entry points (see transfer.h).
#include "transfer.h"

#include <algorithm>
#include <condition_variable>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

namespace ctlab {

namespace {

// A few host threads that split one memcpy between them (page-cache and
// memory bandwidth of one core cannot keep up with the DMA engine).  One job
// at a time; a caller that finds the pool busy copies alone.
class CopyPool {
public:
    CopyPool()
    {
        const unsigned hw = std::thread::hardware_concurrency();
        nworkers_ = (int)std::min(7u, hw > 2 ? hw / 2 - 1 : 0u);
        for (int i = 0; i < nworkers_; ++i) workers_.emplace_back([this, i] { run(i + 1); });
    }
    ~CopyPool()
    {
        {
            std::lock_guard<std::mutex> lk(mu_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto &t : workers_) t.join();
    }
    void copy(void *dst, const void *src, size_t n)
    {
        std::unique_lock<std::mutex> job(job_mu_, std::try_to_lock);
        if (!job.owns_lock() || nworkers_ == 0 || n < (1u << 20)) {
            std::memcpy(dst, src, n);
            return;
        }
        {
            std::lock_guard<std::mutex> lk(mu_);
            dst_ = static_cast<char *>(dst);
            src_ = static_cast<const char *>(src);
            n_ = n;
            remaining_ = nworkers_;
            ++gen_;
        }
        cv_.notify_all();
        piece(0);
        std::unique_lock<std::mutex> lk(mu_);
        done_.wait(lk, [this] { return remaining_ == 0; });
    }

private:
    void piece(int i)
    {
        const int parts = nworkers_ + 1;
        // 4 KiB-aligned pieces
        const size_t per = ((n_ / parts) + 4095) & ~size_t(4095);
        const size_t a = std::min(n_, per * (size_t)i), b = (i == parts - 1) ? n_ : std::min(n_, per * (size_t)(i + 1));
        if (b > a) std::memcpy(dst_ + a, src_ + a, b - a);
    }
    void run(int i)
    {
        unsigned long long seen = 0;
        for (;;) {
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_.wait(lk, [&] { return stop_ || gen_ != seen; });
                if (stop_) return;
                seen = gen_;
            }
            piece(i);
            std::lock_guard<std::mutex> lk(mu_);
            if (--remaining_ == 0) done_.notify_one();
        }
    }
    int nworkers_ = 0;
    std::vector<std::thread> workers_;
    std::mutex mu_, job_mu_;
    std::condition_variable cv_, done_;
    char *dst_ = nullptr;
    const char *src_ = nullptr;
    size_t n_ = 0;
    int remaining_ = 0;
    unsigned long long gen_ = 0;
    bool stop_ = false;
};

CopyPool &pool()
{
    static CopyPool p;
    return p;
}

} // namespace

bool host_pinned(const void *p)
{
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError(); // clear the sticky-free error of an unknown pointer
        return false;
    }
    return at.type == cudaMemoryTypeHost;
}

// The stagers live in static per-device contexts for the life of the
// process; their stream, events and pinned ring go with the process (CUDA
// calls from static destructors may run after the runtime has unloaded).
Stager::~Stager() {}

int Stager::init()
{
    if (!cs_) CTLAB_CUDA_TRY(cudaStreamCreateWithFlags(&cs_, cudaStreamNonBlocking));
    return CTLAB_OK;
}

int Stager::ring()
{
    if (ring_) return CTLAB_OK;
    CTLAB_CUDA_TRY(cudaHostAlloc((void **)&ring_, kSlots * kSlotBytes, cudaHostAllocDefault));
    for (cudaEvent_t &e : ev_) CTLAB_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    for (cudaEvent_t &e : ev_) CTLAB_CUDA_TRY(cudaEventRecord(e, cs_)); // every slot starts free
    return CTLAB_OK;
}

int Stager::take_slot(int *slot)
{
    const int s = next_;
    next_ = (next_ + 1) % kSlots;
    // the slot's previous piece: a device->host piece still to copy out, or
    // a host->device piece whose DMA must have read the slot
    if (!pending_.empty() && pending_.front().slot == s) {
        const Pending p = pending_.front();
        pending_.pop_front();
        CTLAB_CUDA_TRY(cudaEventSynchronize(ev_[s]));
        pool().copy(p.dst, ring_ + (size_t)s * kSlotBytes, p.bytes);
    } else {
        CTLAB_CUDA_TRY(cudaEventSynchronize(ev_[s]));
    }
    *slot = s;
    return CTLAB_OK;
}

int Stager::h2d(void *dst, const void *src, size_t bytes, cudaEvent_t after)
{
    if (after) CTLAB_CUDA_TRY(cudaStreamWaitEvent(cs_, after, 0));
    if (bytes == 0) return CTLAB_OK;
    if (host_pinned(src)) {
        CTLAB_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, cs_));
        return CTLAB_OK;
    }
    int rc = ring();
    if (rc != CTLAB_OK) return rc;
    for (size_t off = 0; off < bytes; off += kSlotBytes) {
        const size_t n = std::min(kSlotBytes, bytes - off);
        int s = 0;
        rc = take_slot(&s);
        if (rc != CTLAB_OK) return rc;
        unsigned char *slot = ring_ + (size_t)s * kSlotBytes;
        pool().copy(slot, static_cast<const unsigned char *>(src) + off, n);
        CTLAB_CUDA_TRY(cudaMemcpyAsync(static_cast<unsigned char *>(dst) + off, slot, n, cudaMemcpyHostToDevice, cs_));
        CTLAB_CUDA_TRY(cudaEventRecord(ev_[s], cs_));
    }
    return CTLAB_OK;
}

int Stager::d2h(void *dst, const void *src, size_t bytes, cudaEvent_t after)
{
    if (after) CTLAB_CUDA_TRY(cudaStreamWaitEvent(cs_, after, 0));
    if (bytes == 0) return CTLAB_OK;
    if (host_pinned(dst)) {
        CTLAB_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, cs_));
        return CTLAB_OK;
    }
    int rc = ring();
    if (rc != CTLAB_OK) return rc;
    for (size_t off = 0; off < bytes; off += kSlotBytes) {
        const size_t n = std::min(kSlotBytes, bytes - off);
        int s = 0;
        rc = take_slot(&s);
        if (rc != CTLAB_OK) return rc;
        CTLAB_CUDA_TRY(cudaMemcpyAsync(ring_ + (size_t)s * kSlotBytes, static_cast<const unsigned char *>(src) + off, n,
                                       cudaMemcpyDeviceToHost, cs_));
        CTLAB_CUDA_TRY(cudaEventRecord(ev_[s], cs_));
        pending_.push_back({s, static_cast<unsigned char *>(dst) + off, n});
    }
    return CTLAB_OK;
}

int Stager::finish()
{
    while (!pending_.empty()) {
        const Pending p = pending_.front();
        pending_.pop_front();
        CTLAB_CUDA_TRY(cudaEventSynchronize(ev_[p.slot]));
        pool().copy(p.dst, ring_ + (size_t)p.slot * kSlotBytes, p.bytes);
    }
    CTLAB_CUDA_TRY(cudaStreamSynchronize(cs_));
    return CTLAB_OK;
}

void Stager::abandon()
{
    if (cs_) cudaStreamSynchronize(cs_);
    pending_.clear();
}

} // namespace ctlab
