// Thread-local status of the last C-ABI call and the device guard.
#include "internal.h"

namespace ctlab {

namespace {
thread_local int g_status = CTLAB_OK;
thread_local std::string g_message;
} // namespace

int set_status(int code, const std::string &msg)
{
    g_status = code;
    g_message = msg;
    return code;
}

int cuda_status(cudaError_t e, const char *what)
{
    int code = (e == cudaErrorMemoryAllocation) ? CTLAB_ERR_OOM : CTLAB_ERR_CUDA;
    return set_status(code, std::string(what) + ": " + cudaGetErrorName(e) + " (" +
                                cudaGetErrorString(e) + ")");
}

DeviceGuard::DeviceGuard(int dev)
{
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    ok = (cudaSetDevice(dev) == cudaSuccess);
}

DeviceGuard::~DeviceGuard()
{
    if (prev >= 0) cudaSetDevice(prev);
}

} // namespace ctlab

extern "C" int ctlab_last_status(void) { return ctlab::g_status; }
extern "C" const char *ctlab_last_error(void) { return ctlab::g_message.c_str(); }
