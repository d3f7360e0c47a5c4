// Allocation-free volume SAT.
//
// Some callers of this library cannot allocate device memory while they
// reconstruct: acquisition and real-time reconstruction systems that reserve
// their whole device-memory budget up front, and callers that must not let
// a cudaMalloc / cudaFree implicitly synchronise the device (stalling their
// other streams) or fail half-way through a scan.  For them this file
// provides ctlab_volume_sat_noalloc: the same decoupled-lookback SAT scan as
// the plan path, with its lookback scratch (ticket, error word, chunk flags,
// chunk aggregates and inclusive prefixes) in a fixed device array owned by
// the library instead of a cudaMalloc'd workspace.  The caller passes the
// volume, the mask and the output SAT buffer.
#include <cstdio>
#include <mutex>

#include "internal.h"

namespace {

// Scratch limit: 32 MiB.  Every GPU that loads the library holds this array
// until the process exits.
constexpr size_t kScratchBytes = 32u << 20;
constexpr int kChunk = 48;        // rows per scan chunk (the largest the scan's shared memory allows)
constexpr size_t kHeader = 256;   // ticket and error word, then the flags

__device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
unsigned char *g_scratch_addr[kMaxDevices] = {};

size_t round256(size_t n) { return (n + 255) & ~size_t(255); }

// Device address of the scratch array on the current device, looked up once
// per device.  In host code g_noalloc_scratch only names a host-side
// stand-in; passing it to a kernel would fault or touch the wrong memory.
int scratch_address(int dev, unsigned char **out)
{
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_addr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return ctlab::cuda_status(e, "cudaGetSymbolAddress(no-alloc scratch)");
        g_scratch_addr[dev] = static_cast<unsigned char *>(p);
    }
    *out = g_scratch_addr[dev];
    return CTLAB_OK;
}

} // namespace

extern "C" int ctlab_volume_sat_noalloc(const float *d_vol, const unsigned char *d_mask, int XN, int YN, int ZN,
                                        int orientation, double *d_sat, int zp, void *stream)
{
    using namespace ctlab;
    if (!d_vol || !d_sat) return set_status(CTLAB_ERR_INVALID_ARG, "null volume or SAT buffer");
    if (XN < 1 || YN < 1 || ZN < 1) return set_status(CTLAB_ERR_INVALID_ARG, "sizes must be >= 1");
    if (orientation != 0 && orientation != 1)
        return set_status(CTLAB_ERR_INVALID_ARG, "orientation must be 0 (y slices) or 1 (x slices)");
    if (zp < ZN + 1) return set_status(CTLAB_ERR_INVALID_ARG, "zp must be >= ZN + 1");
    if (ZN > 4096) return set_status(CTLAB_ERR_INVALID_ARG, "ZN beyond the scan's range (4096)");

    // scratch needed: header, one flag per (plane, chunk), aggregate and
    // inclusive-prefix vectors of ZN doubles per (plane, chunk)
    const int planes = orientation == 0 ? YN : XN, rows = orientation == 0 ? XN : YN;
    const size_t tiles = (size_t)planes * (size_t)scan_chunks(rows, ZN, kChunk, 0);
    const size_t flag_bytes = round256(sizeof(int) * tiles);
    const size_t vec_bytes = round256(sizeof(double) * tiles * (size_t)ZN);
    const size_t need = kHeader + flag_bytes + 2 * vec_bytes;
    if (need > kScratchBytes) {
        char msg[256];
        snprintf(msg, sizeof msg,
                 "volume too large for the allocation-free SAT: needs %zu bytes of scratch, the limit is %zu "
                 "(32 MiB); use ctlab_volume_sat on a plan",
                 need, kScratchBytes);
        return set_status(CTLAB_ERR_INVALID_ARG, msg);
    }

    int dev = 0;
    CTLAB_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return set_status(CTLAB_ERR_INVALID_ARG, "device index beyond 64");
    unsigned char *base = nullptr;
    int rc = scratch_address(dev, &base);
    if (rc != CTLAB_OK) return rc;

    ScanState st;
    st.ticket = reinterpret_cast<int *>(base);
    st.err = reinterpret_cast<int *>(base + sizeof(int));
    st.flags = reinterpret_cast<int *>(base + kHeader);
    st.agg = reinterpret_cast<double *>(base + kHeader + flag_bytes);
    st.pref = reinterpret_cast<double *>(base + kHeader + flag_bytes + vec_bytes);
    cudaStream_t s = (cudaStream_t)stream;
    // The array keeps the previous call's contents.  The scan launch zeroes
    // the ticket and the flags itself; the error word is left alone so that
    // a timeout stays visible until ctlab_noalloc_check reads and clears it.
    CTLAB_CUDA_TRY(launch_volume_sat(d_vol, d_mask, XN, YN, ZN, orientation, d_sat, zp, 0, st, kChunk, s));
    return ok();
}

extern "C" int ctlab_noalloc_check(void *stream)
{
    using namespace ctlab;
    int dev = 0;
    CTLAB_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return set_status(CTLAB_ERR_INVALID_ARG, "device index beyond 64");
    unsigned char *base = nullptr;
    int rc = scratch_address(dev, &base);
    if (rc != CTLAB_OK) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    int *err = reinterpret_cast<int *>(base + sizeof(int));
    int h_err = 0;
    CTLAB_CUDA_TRY(cudaMemcpyAsync(&h_err, err, sizeof(int), cudaMemcpyDeviceToHost, s));
    CTLAB_CUDA_TRY(cudaStreamSynchronize(s));
    if (h_err != 0) {
        CTLAB_CUDA_TRY(cudaMemsetAsync(err, 0, sizeof(int), s));
        CTLAB_CUDA_TRY(cudaStreamSynchronize(s));
        return set_status(CTLAB_ERR_TIMEOUT,
                          "a bounded wait in an allocation-free SAT scan timed out; its output is invalid");
    }
    return ok();
}

// Diagnostics for ctlab_noalloc_check: the lookback scan of a 2-row plane
// whose first chunk never publishes, with all of its state (and its tiny
// input and output) inside the fixed array.  The second chunk's bounded wait
// runs out after spin_limit polls and raises the array's error word.
extern "C" int ctlab_debug_noalloc_stall(unsigned spin_limit, void *stream)
{
    using namespace ctlab;
    if (spin_limit < 1 || spin_limit > (1u << 24))
        return set_status(CTLAB_ERR_INVALID_ARG, "spin_limit must be in [1, 2^24]");
    int dev = 0;
    CTLAB_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return set_status(CTLAB_ERR_INVALID_ARG, "device index beyond 64");
    unsigned char *base = nullptr;
    int rc = scratch_address(dev, &base);
    if (rc != CTLAB_OK) return rc;
    constexpr int rows = 2, nk = 8;
    // header | flags @256 | agg @512 | pref @768 | input @1024 | output @1280 (ends at 1496)
    ScanState st;
    st.ticket = reinterpret_cast<int *>(base);
    st.err = reinterpret_cast<int *>(base + sizeof(int));
    st.flags = reinterpret_cast<int *>(base + kHeader);
    st.agg = reinterpret_cast<double *>(base + 512);
    st.pref = reinterpret_cast<double *>(base + 768);
    float *vol = reinterpret_cast<float *>(base + 1024);
    double *out = reinterpret_cast<double *>(base + 1280);
    cudaStream_t s = (cudaStream_t)stream;
    CTLAB_CUDA_TRY(cudaMemsetAsync(vol, 0, sizeof(float) * rows * nk, s));
    CTLAB_CUDA_TRY(launch_scan_stall(vol, rows, nk, out, st, 1, spin_limit, s));
    return ok();
}
