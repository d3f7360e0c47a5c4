// C++-ABI reconstruction entry points with the reference's signatures
// (thrust::host_vector arguments): OS_SART, CG and evalProjBack.  Each builds
// the scan from the reference's flat-detector description, runs the device
// solver (ctlab_os_sart / ctlab_cg) on the current device with a z-prefix
// plan, copies the image back and optionally writes it to a raw file.
//
// thrust::host_vector lives in a versioned inline namespace that differs
// between nvcc device compiles (per target architecture) and host-only
// compiles, and it is part of the mangled names.  This file is therefore
// built twice: by nvcc for sm_100a and, as recon_cxx_host.cpp, by the host
// C++ compiler, so callers of either kind link.  It uses only host APIs.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/ctlab_b200_recon.hpp"

namespace ctlab {
int set_status(int code, const std::string &msg);
int cuda_status(cudaError_t e, const char *what);
} // namespace ctlab

using namespace ctlab;

namespace {

struct DevMem {
    void *p = nullptr;
    ~DevMem()
    {
        if (p) cudaFree(p);
    }
};

// The reference's flat equal-distance detector (calSVASVB,
// src/utilities.hpp:3322-3348): source (0, sid, 0), detector plane at
// y = sid - sdd, cell centres offset by col_offset / row_offset cells.
struct FlatScan {
    std::vector<float> xds, yds, zds;
    ctlab_geometry g;
    FlatScan(float sid, float sdd, int DNU, int DNV, int PN, const float *hangs, const float *hzPos, float cx,
             float cy, float cz, int XN, int YN, int ZN, float dx, float dz, float col_size, float row_size,
             float col_offset, float row_offset)
        : xds(DNU), yds(DNU, sid - sdd), zds(DNV)
    {
        for (int u = 0; u < DNU; ++u) xds[u] = (float)((u - (DNU - 1) / 2.0 - col_offset) * col_size);
        for (int v = 0; v < DNV; ++v) zds[v] = (float)((v - (DNV - 1) / 2.0 - row_offset) * row_size);
        g = ctlab_geometry{0.f, sid, 0.f, DNU, DNV, xds.data(), yds.data(), zds.data(), cx, cy, cz, hangs, hzPos, PN,
                           XN, YN, ZN, dx, dz};
    }
};

bool write_raw(const std::string &name, const float *p, size_t n)
{
    FILE *f = std::fopen(name.c_str(), "wb");
    if (!f) return false;
    const bool ok = std::fwrite(p, sizeof(float), n, f) == n;
    return std::fclose(f) == 0 && ok;
}

enum class Solver { OsSart, Cg };

// Shared body of OS_SART and CG.
void solve(Solver which, thrust::host_vector<float> &reconImg, thrust::host_vector<float> &initImg,
           thrust::host_vector<float> &hprj, thrust::host_vector<float> &hangs, thrust::host_vector<float> &hzPos,
           thrust::host_vector<byte> &mask, const std::string &VolumeName, int osNum, int iterNum, bool outputMedRes,
           float sid, float sdd, int DNU, int DNV, int PN, float cx, float cy, float cz, int XN, int YN, int ZN,
           float dx, float dz, float col_size, float row_size, float col_offset, float row_offset, int fwd, int bwd,
           int cgm)
{
    if (fwd != PROJ_BRANCHLESS || bwd != BACK_BRANCHLESS) {
        set_status(CTLAB_ERR_UNSUPPORTED, "only the branchless projector / backprojector (mode 0) is built");
        return;
    }
    if (DNU < 1 || DNV < 1 || PN < 1 || XN < 1 || YN < 1 || ZN < 1 || iterNum < 0 || osNum < 1) {
        set_status(CTLAB_ERR_INVALID_ARG, "sizes must be >= 1, osNum >= 1, iterNum >= 0");
        return;
    }
    const size_t nv = (size_t)XN * YN * ZN, np = (size_t)PN * DNU * DNV, nc = (size_t)XN * YN;
    if (initImg.size() != nv || hprj.size() != np || hangs.size() != (size_t)PN || hzPos.size() != (size_t)PN ||
        (!mask.empty() && mask.size() != nc)) {
        set_status(CTLAB_ERR_INVALID_ARG, "array sizes do not match XN*YN*ZN, PN*DNU*DNV, PN and XN*YN");
        return;
    }
    FlatScan scan(sid, sdd, DNU, DNV, PN, hangs.data(), hzPos.data(), cx, cy, cz, XN, YN, ZN, dx, dz, col_size,
                  row_size, col_offset, row_offset);
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        set_status(CTLAB_ERR_CUDA, "no current CUDA device");
        return;
    }
    ctlab_plan *plan = nullptr;
    if (ctlab_plan_create(&scan.g, dev, CTLAB_SAT_ZPREFIX, &plan) != CTLAB_OK) return;
    DevMem d_x, d_b, d_m;
    cudaError_t e = cudaMalloc(&d_x.p, sizeof(float) * nv);
    if (e == cudaSuccess) e = cudaMalloc(&d_b.p, sizeof(float) * np);
    if (e == cudaSuccess && !mask.empty()) e = cudaMalloc(&d_m.p, nc);
    if (e == cudaSuccess) e = cudaMemcpy(d_x.p, initImg.data(), sizeof(float) * nv, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_b.p, hprj.data(), sizeof(float) * np, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && !mask.empty()) e = cudaMemcpy(d_m.p, mask.data(), nc, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        cuda_status(e, "reconstruction buffers");
        ctlab_plan_destroy(plan);
        return;
    }
    float *x = (float *)d_x.p;
    const float *b = (const float *)d_b.p;
    const unsigned char *m = (const unsigned char *)d_m.p;
    reconImg.resize(nv);
    auto run = [&](int iters) {
        return which == Solver::OsSart
                   ? ctlab_os_sart(plan, x, b, m, osNum, iters, 1.f, nullptr, 0, 0.f, 0.f, nullptr, nullptr)
                   : ctlab_cg(plan, x, b, m, iters, cgm, nullptr, nullptr);
    };
    int rc = CTLAB_OK;
    if (outputMedRes && !VolumeName.empty() && which == Solver::OsSart) {
        // one iteration per call: OS-SART restarts nothing between iterations
        for (int it = 0; it < iterNum && rc == CTLAB_OK; ++it) {
            rc = run(1);
            if (rc == CTLAB_OK && cudaMemcpy(reconImg.data(), x, sizeof(float) * nv, cudaMemcpyDeviceToHost) == cudaSuccess)
                write_raw(VolumeName + "_iter" + std::to_string(it + 1), reconImg.data(), nv);
        }
    } else {
        rc = run(iterNum);
    }
    if (rc == CTLAB_OK) {
        e = cudaMemcpy(reconImg.data(), x, sizeof(float) * nv, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) rc = cuda_status(e, "reconstruction result");
    }
    ctlab_plan_destroy(plan);
    if (rc != CTLAB_OK) return;
    if (!VolumeName.empty() && !write_raw(VolumeName, reconImg.data(), nv)) {
        set_status(CTLAB_ERR_INVALID_ARG, "could not write " + VolumeName);
        return;
    }
    set_status(CTLAB_OK, "");
}

} // namespace

void OS_SART(thrust::host_vector<float> &reconImg, thrust::host_vector<float> &initImg,
             thrust::host_vector<float> &hprj, thrust::host_vector<float> &hangs,
             thrust::host_vector<float> &hzPos, thrust::host_vector<byte> &mask, const std::string &VolumeName,
             const int osNum, const int iterNum, const bool outputMedRes, const float sid, const float sdd,
             const int DNU, const int DNV, const int PN, const float imgXCenter, const float imgYCenter,
             const float imgZCenter, const int XN, const int YN, const int ZN, const float dx, const float dz,
             const float col_size, const float row_size, const float col_offset, const float row_offset,
             const ForwardDDMethod forwardMethod, const BackwardDDMethod backwardMethod)
{
    solve(Solver::OsSart, reconImg, initImg, hprj, hangs, hzPos, mask, VolumeName, osNum, iterNum, outputMedRes, sid,
          sdd, DNU, DNV, PN, imgXCenter, imgYCenter, imgZCenter, XN, YN, ZN, dx, dz, col_size, row_size, col_offset,
          row_offset, forwardMethod, backwardMethod, 0);
}

void CG(thrust::host_vector<float> &reconImg, thrust::host_vector<float> &initImg, thrust::host_vector<float> &hprj,
        thrust::host_vector<float> &hangs, thrust::host_vector<float> &hzPos, thrust::host_vector<byte> &mask,
        const std::string &VolumeName, const int osNum, const int iterNum, const bool outputMedRes, const float sid,
        const float sdd, const int DNU, const int DNV, const int PN, const float imgXCenter, const float imgYCenter,
        const float imgZCenter, const int XN, const int YN, const int ZN, const float dx, const float dz,
        const float col_size, const float row_size, const float col_offset, const float row_offset,
        const ForwardDDMethod forwardMethod, const BackwardDDMethod backwardMethod, const CGMethod cgm)
{
    solve(Solver::Cg, reconImg, initImg, hprj, hangs, hzPos, mask, VolumeName, osNum, iterNum, outputMedRes, sid, sdd,
          DNU, DNV, PN, imgXCenter, imgYCenter, imgZCenter, XN, YN, ZN, dx, dz, col_size, row_size, col_offset,
          row_offset, forwardMethod, backwardMethod, (int)cgm);
}

#ifndef CTLAB_RECON_HOST_COPY // no thrust types in its signature: defined once
void evalProjBack(bool forwardProjection, ForwardDDMethod forwardMethod, BackwardDDMethod backwardMethod)
{
    if (forwardMethod != PROJ_BRANCHLESS || backwardMethod != BACK_BRANCHLESS) {
        set_status(CTLAB_ERR_UNSUPPORTED, "only the branchless projector / backprojector (mode 0) is built");
        return;
    }
    const int XN = 128, YN = 128, ZN = 64, PN = 360, DNU = 256, DNV = 64;
    std::vector<float> hangs(PN), hzPos(PN, 0.f);
    for (int p = 0; p < PN; ++p) hangs[p] = (float)(6.283185307179586 * p / PN);
    FlatScan scan(541.f, 949.f, DNU, DNV, PN, hangs.data(), hzPos.data(), 0.f, 0.f, 0.f, XN, YN, ZN, 0.5f, 0.5f, 1.f,
                  1.f, 0.f, 0.f);
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        set_status(CTLAB_ERR_CUDA, "no current CUDA device");
        return;
    }
    ctlab_plan *plan = nullptr;
    if (ctlab_plan_create(&scan.g, dev, CTLAB_SAT_ZPREFIX, &plan) != CTLAB_OK) return;
    const size_t nv = (size_t)XN * YN * ZN, np = (size_t)PN * DNU * DNV;
    const size_t nin = forwardProjection ? nv : np, nout = forwardProjection ? np : nv;
    DevMem d_in, d_out;
    cudaError_t e = cudaMalloc(&d_in.p, sizeof(float) * nin);
    if (e == cudaSuccess) e = cudaMalloc(&d_out.p, sizeof(float) * nout);
    std::vector<float> ones(nin, 1.f), out(nout);
    if (e == cudaSuccess) e = cudaMemcpy(d_in.p, ones.data(), sizeof(float) * nin, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        cuda_status(e, "evalProjBack buffers");
        ctlab_plan_destroy(plan);
        return;
    }
    cudaEvent_t t0, t1;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    cudaEventRecord(t0, 0);
    const int rc = forwardProjection ? ctlab_proj(plan, (float *)d_in.p, nullptr, (float *)d_out.p, nullptr)
                                     : ctlab_back(plan, (float *)d_in.p, nullptr, (float *)d_out.p, nullptr);
    cudaEventRecord(t1, 0);
    float ms = 0.f;
    if (rc == CTLAB_OK) {
        cudaEventSynchronize(t1);
        cudaEventElapsedTime(&ms, t0, t1);
        e = cudaMemcpy(out.data(), d_out.p, sizeof(float) * nout, cudaMemcpyDeviceToHost);
    }
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    ctlab_plan_destroy(plan);
    if (rc != CTLAB_OK) return;
    if (e != cudaSuccess) {
        cuda_status(e, "evalProjBack result");
        return;
    }
    double lo = out[0], hi = out[0], sum = 0.0;
    for (float v : out) {
        lo = std::min(lo, (double)v);
        hi = std::max(hi, (double)v);
        sum += v;
    }
    std::printf("%s of ones: min %.6g max %.6g sum %.10g, %.3f ms\n", forwardProjection ? "projection" : "backprojection",
                lo, hi, sum, ms);
    set_status(CTLAB_OK, "");
}
#endif
