// Host <-> device copies of the host-pointer entry points (DD3Proj_gpu,
// DD3Back_gpu): a copy stream beside the compute stream, so that the copy of
// one chunk overlaps the compute of another, and a pinned staging ring for
// pageable host buffers (what thrust::host_vector or plain arrays give):
// this thread copies between the caller's memory and the ring's slots with
// several host threads while the DMA engine moves the slot it filled last.
#pragma once

#include <cstddef>
#include <deque>

#include "internal.h"

namespace ctlab {

// True when the CUDA runtime knows p as page-locked (cudaHostAlloc'd or
// cudaHostRegister'ed) host memory.
bool host_pinned(const void *p);

class Stager {
public:
    static constexpr int kSlots = 4;
    static constexpr size_t kSlotBytes = 16u << 20;

    ~Stager();
    // Creates the copy stream and events on the current device (once).
    int init();
    cudaStream_t stream() const { return cs_; }
    // dst (device) <- src (host), ordered on the copy stream after `after`
    // (an event on another stream, or nullptr).
    int h2d(void *dst, const void *src, size_t bytes, cudaEvent_t after);
    // dst (host) <- src (device), ordered on the copy stream after `after`.
    // For a pageable dst the bytes land when finish() returns.
    int d2h(void *dst, const void *src, size_t bytes, cudaEvent_t after);
    // Waits for every copy and finishes the staged host copies.
    int finish();
    // After a failed call: waits for the copy stream and drops the staged
    // host copies still queued, so none lands in a later call's buffers.
    void abandon();

private:
    struct Pending {
        int slot;
        void *dst;
        size_t bytes;
    };
    int ring();
    int take_slot(int *slot); // the next slot, its previous use completed
    cudaStream_t cs_ = nullptr;
    unsigned char *ring_ = nullptr;
    cudaEvent_t ev_[kSlots] = {};
    int next_ = 0;
    std::deque<Pending> pending_; // staged device->host pieces not yet copied out
};

} // namespace ctlab
