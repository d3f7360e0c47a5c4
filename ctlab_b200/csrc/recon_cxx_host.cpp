// recon_cxx.cu compiled by the host C++ compiler: the OS_SART / CG symbols
// with the host-only thrust ABI namespace, for callers built without nvcc.
#define CTLAB_RECON_HOST_COPY 1
#include "recon_cxx.cu"
