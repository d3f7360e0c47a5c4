// Elementwise and stencil kernels of the reconstruction loops: SART
// weightings, FISTA momentum, smoothed TV gradient, residual reductions and
// the ellipsoid phantom.  All are HBM-streaming kernels with grid-stride
// loops sized to the SM count.
#include "internal.h"

namespace ctlab {

namespace {

constexpr int kT = 256;

unsigned grid_for(long long n)
{
    static int sms = 0;
    if (sms == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0)
            sms = 148;
    }
    long long want = (n + kT - 1) / kT;
    long long cap = (long long)sms * 8;
    if (want > cap) want = cap;
    if (want < 1) want = 1;
    return (unsigned)want;
}

#define GRID_STRIDE(i, n) \
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < (n); i += (long long)gridDim.x * blockDim.x)

// SART_Weighting::Proj_ptr, src/SARTWeighting.h:38-53
__global__ void sart_proj_weight_kernel(float *prj, const float *real, const float *rs, long long n)
{
    GRID_STRIDE(i, n) { prj[i] = (rs[i] > 1.0e-7f) ? (real[i] - prj[i]) / rs[i] : 0.f; }
}

// SART_Weighting::Back_ptr, src/SARTWeighting.h:74-91
__global__ void sart_back_weight_kernel(float *vol, float *recon, const float *cs, long long n)
{
    GRID_STRIDE(i, n)
    {
        const float v = (cs[i] > 1.0e-7f) ? vol[i] / cs[i] : 0.f;
        vol[i] = v;
        recon[i] += v;
    }
}

// FISTA_functor, src/FastIterativeShrinkageAlgorithm.h:17-42
__global__ void fista_kernel(const float *las, float *cur, float t1, float t2, long long n, float lo, float hi)
{
    const float c = (t1 - 1.0f) / t2;
    GRID_STRIDE(i, n)
    {
        const float r = cur[i] + c * (cur[i] - las[i]);
        cur[i] = r < lo ? lo : (r > hi ? hi : r);
    }
}

__global__ void fill_kernel(float *p, float v, long long n)
{
    GRID_STRIDE(i, n) { p[i] = v; }
}

__global__ void mask_fill_kernel(float *p, const unsigned char *mask, long long ncols, int ZN)
{
    const long long n = ncols * ZN;
    GRID_STRIDE(i, n) { p[i] = mask ? (mask[i / ZN] ? 1.f : 0.f) : 1.f; }
}

__global__ void tv_step_kernel(float *x, const float *z, const float *g, const unsigned char *mask, float lam,
                               long long n, int ZN)
{
    GRID_STRIDE(i, n)
    {
        const float m = mask ? (mask[i / ZN] ? 1.f : 0.f) : 1.f;
        x[i] = (z[i] - lam * g[i]) * m;
    }
}

__global__ void add_scaled_div_kernel(float *y, const float *q, const float *cs, long long n)
{
    GRID_STRIDE(i, n) { y[i] += (cs[i] > 1.0e-7f) ? q[i] / cs[i] : 0.f; }
}

__global__ void gather_views_kernel(const float *src, const int *list, int nv, long long per, float *dst)
{
    const long long n = (long long)nv * per;
    GRID_STRIDE(i, n)
    {
        const long long v = i / per, e = i - v * per;
        dst[i] = src[(long long)list[v] * per + e];
    }
}

__global__ void resid2_kernel(const float *meas, const float *est, long long n, double *acc)
{
    double a = 0.0, b = 0.0;
    GRID_STRIDE(i, n)
    {
        const double m = meas[i];
        const double d = m - (est ? (double)est[i] : 0.0);
        a += d * d;
        b += m * m;
    }
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, o);
        b += __shfl_down_sync(0xffffffffu, b, o);
    }
    __shared__ double sa[kT / 32], sb[kT / 32];
    if ((threadIdx.x & 31) == 0) {
        sa[threadIdx.x >> 5] = a;
        sb[threadIdx.x >> 5] = b;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double ta = 0, tb = 0;
        for (int w = 0; w < kT / 32; ++w) {
            ta += sa[w];
            tb += sb[w];
        }
        atomicAdd(acc, ta);
        atomicAdd(acc + 1, tb);
    }
}

// acc += sum a*b in FP64 (block partial sums, one atomic per block)
__global__ void dot_kernel(const float *a, const float *b, long long n, double *acc)
{
    double t = 0.0;
    GRID_STRIDE(i, n) { t += (double)a[i] * (double)b[i]; }
    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
    __shared__ double sw[kT / 32];
    if ((threadIdx.x & 31) == 0) sw[threadIdx.x >> 5] = t;
    __syncthreads();
    if (threadIdx.x == 0) {
        double tt = 0;
        for (int w = 0; w < kT / 32; ++w) tt += sw[w];
        atomicAdd(acc, tt);
    }
}

// y = alpha * x + beta * y
__global__ void axpby_kernel(float *y, float alpha, const float *x, float beta, long long n)
{
    GRID_STRIDE(i, n) { y[i] = fmaf(alpha, x[i], beta * y[i]); }
}

// Smoothed isotropic TV gradient, forward differences, replicated borders;
// the 3-D GradientOfTV_GPU of src/differentialFuncs.hpp:491-501.  One
// thread per voxel, z fastest (coalesced); neighbours come from L1/L2.
__global__ void tv_gradient_kernel(const float *__restrict__ f, float *__restrict__ g, int XN, int YN, int ZN,
                                   float eps)
{
    const long long n = (long long)XN * YN * ZN;
    GRID_STRIDE(i, n)
    {
        const int z = (int)(i % ZN);
        const long long col = i / ZN;
        const int x = (int)(col % XN), y = (int)(col / XN);
        const long long sx = ZN, sy = (long long)XN * ZN;
        auto F = [&](long long idx) { return __ldg(f + idx); };
        const float c = F(i);
        const float fxp = (x + 1 < XN) ? F(i + sx) : c;
        const float fyp = (y + 1 < YN) ? F(i + sy) : c;
        const float fzp = (z + 1 < ZN) ? F(i + 1) : c;
        float gs = ((c - fxp) + (c - fyp) + (c - fzp)) *
                   rsqrtf(eps + (fxp - c) * (fxp - c) + (fyp - c) * (fyp - c) + (fzp - c) * (fzp - c));
        if (x > 0) {
            const long long j = i - sx;
            const float nn = F(j);
            const float b = (y + 1 < YN) ? F(j + sy) : nn, d = (z + 1 < ZN) ? F(j + 1) : nn;
            gs += (c - nn) * rsqrtf(eps + (c - nn) * (c - nn) + (b - nn) * (b - nn) + (d - nn) * (d - nn));
        }
        if (y > 0) {
            const long long j = i - sy;
            const float nn = F(j);
            const float aa = (x + 1 < XN) ? F(j + sx) : nn, d = (z + 1 < ZN) ? F(j + 1) : nn;
            gs += (c - nn) * rsqrtf(eps + (aa - nn) * (aa - nn) + (c - nn) * (c - nn) + (d - nn) * (d - nn));
        }
        if (z > 0) {
            const long long j = i - 1;
            const float nn = F(j);
            const float aa = (x + 1 < XN) ? F(j + sx) : nn, b = (y + 1 < YN) ? F(j + sy) : nn;
            gs += (c - nn) * rsqrtf(eps + (aa - nn) * (aa - nn) + (b - nn) * (b - nn) + (c - nn) * (c - nn));
        }
        g[i] = gs;
    }
}

// Point-sampled ellipsoid sum; records of 10 floats (value, centre, semi
// axes, phi, theta, psi) pre-expanded by the host into 16 floats: value,
// centre (3), 1/semi-axes (3), R^T row-major (9).
__global__ void phantom_kernel(float *vol, int XN, int YN, int ZN, float dx, float dz, float cx, float cy,
                               float cz, const float *ell, int n_ell, int clamp_nonneg)
{
    extern __shared__ float s_ell[];
    for (int i = threadIdx.x; i < n_ell * 16; i += blockDim.x) s_ell[i] = ell[i];
    __syncthreads();
    const long long n = (long long)XN * YN * ZN;
    GRID_STRIDE(i, n)
    {
        const int z = (int)(i % ZN);
        const long long col = i / ZN;
        const int x = (int)(col % XN), y = (int)(col / XN);
        const float px = cx + ((float)x - 0.5f * (XN - 1)) * dx;
        const float py = cy + ((float)y - 0.5f * (YN - 1)) * dx;
        const float pz = cz + ((float)z - 0.5f * (ZN - 1)) * dz;
        float acc = 0.f;
        for (int e = 0; e < n_ell; ++e) {
            const float *E = s_ell + 16 * e;
            const float qx = px - E[1], qy = py - E[2], qz = pz - E[3];
            const float lx = (E[7] * qx + E[8] * qy + E[9] * qz) * E[4];
            const float ly = (E[10] * qx + E[11] * qy + E[12] * qz) * E[5];
            const float lz = (E[13] * qx + E[14] * qy + E[15] * qz) * E[6];
            if (lx * lx + ly * ly + lz * lz <= 1.f) acc += E[0];
        }
        if (clamp_nonneg && acc < 0.f) acc = 0.f;
        vol[i] = acc;
    }
}

} // namespace

cudaError_t launch_sart_proj_weight(float *prj, const float *real, const float *rs, long long n, cudaStream_t s)
{
    sart_proj_weight_kernel<<<grid_for(n), kT, 0, s>>>(prj, real, rs, n);
    return cudaGetLastError();
}
cudaError_t launch_sart_back_weight(float *vol, float *recon, const float *cs, long long n, cudaStream_t s)
{
    sart_back_weight_kernel<<<grid_for(n), kT, 0, s>>>(vol, recon, cs, n);
    return cudaGetLastError();
}
cudaError_t launch_fista_step(const float *las, float *cur, float t1, float t2, long long n, float lo, float hi,
                              cudaStream_t s)
{
    fista_kernel<<<grid_for(n), kT, 0, s>>>(las, cur, t1, t2, n, lo, hi);
    return cudaGetLastError();
}
cudaError_t launch_tv_gradient(const float *f, float *g, int XN, int YN, int ZN, float eps, cudaStream_t s)
{
    const long long n = (long long)XN * YN * ZN;
    tv_gradient_kernel<<<grid_for(n), kT, 0, s>>>(f, g, XN, YN, ZN, eps);
    return cudaGetLastError();
}
cudaError_t launch_fill(float *p, float v, long long n, cudaStream_t s)
{
    fill_kernel<<<grid_for(n), kT, 0, s>>>(p, v, n);
    return cudaGetLastError();
}
cudaError_t launch_mask_fill(float *p, const unsigned char *mask, long long ncols, int ZN, cudaStream_t s)
{
    mask_fill_kernel<<<grid_for(ncols * ZN), kT, 0, s>>>(p, mask, ncols, ZN);
    return cudaGetLastError();
}
cudaError_t launch_tv_step(float *x, const float *z, const float *g, const unsigned char *mask, float lam,
                           long long n, int ZN, cudaStream_t s)
{
    tv_step_kernel<<<grid_for(n), kT, 0, s>>>(x, z, g, mask, lam, n, ZN);
    return cudaGetLastError();
}
cudaError_t launch_add_scaled_div(float *y, const float *q, const float *cs, long long n, cudaStream_t s)
{
    add_scaled_div_kernel<<<grid_for(n), kT, 0, s>>>(y, q, cs, n);
    return cudaGetLastError();
}
cudaError_t launch_gather_views(const float *src, const int *list, int nv, long long per, float *dst,
                                cudaStream_t s)
{
    gather_views_kernel<<<grid_for((long long)nv * per), kT, 0, s>>>(src, list, nv, per, dst);
    return cudaGetLastError();
}
cudaError_t launch_resid2(const float *meas, const float *est, long long n, double *acc, cudaStream_t s)
{
    resid2_kernel<<<grid_for(n), kT, 0, s>>>(meas, est, n, acc);
    return cudaGetLastError();
}
cudaError_t launch_dot(const float *a, const float *b, long long n, double *acc, cudaStream_t s)
{
    dot_kernel<<<grid_for(n), kT, 0, s>>>(a, b, n, acc);
    return cudaGetLastError();
}
cudaError_t launch_axpby(float *y, float alpha, const float *x, float beta, long long n, cudaStream_t s)
{
    axpby_kernel<<<grid_for(n), kT, 0, s>>>(y, alpha, x, beta, n);
    return cudaGetLastError();
}
cudaError_t launch_phantom(float *vol, int XN, int YN, int ZN, float dx, float dz, float cx, float cy, float cz,
                           const float *ell_dev, int n_ell, int clamp_nonneg, cudaStream_t s)
{
    const long long n = (long long)XN * YN * ZN;
    phantom_kernel<<<grid_for(n), kT, sizeof(float) * 16 * (size_t)n_ell, s>>>(vol, XN, YN, ZN, dx, dz, cx, cy, cz,
                                                                              ell_dev, n_ell, clamp_nonneg);
    return cudaGetLastError();
}

} // namespace ctlab
