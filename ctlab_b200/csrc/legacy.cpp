// Host-pointer entry points with the reference's names and argument order
// (DD3Proj_gpu, DD3Back_gpu), plus the elementwise and phantom C ABI.
//
// Each legacy call copies its host inputs to the device, runs the
// device-pointer path on a library-owned stream and copies the result back.
// Geometry plans and device buffers are cached per device (re-created only
// when the geometry changes, buffers only grow), so repeated calls with one
// scan geometry pay no allocation.  Calls on one device are serialised.
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <random>

#include "plan.h"

using namespace ctlab;

namespace {

struct LegacyCtx {
    std::mutex mu;
    ctlab_plan *plan = nullptr;
    unsigned long long key = 0;
    int mode = -1;
    float *d_vol = nullptr;
    size_t vol_cap = 0;
    float *d_prj = nullptr;
    size_t prj_cap = 0;
    unsigned char *d_mask = nullptr;
    size_t mask_cap = 0;
    cudaStream_t stream = nullptr;
};

constexpr int kMaxDevices = 64;
LegacyCtx g_ctx[kMaxDevices];

struct Fnv {
    unsigned long long h = 1469598103934665603ull;
    void add(const void *p, size_t n)
    {
        const unsigned char *b = (const unsigned char *)p;
        for (size_t i = 0; i < n; ++i) {
            h ^= b[i];
            h *= 1099511628211ull;
        }
    }
};

unsigned long long geometry_key(const ctlab_geometry &g)
{
    Fnv f;
    f.add(&g.x0, sizeof(float) * 3);
    f.add(&g.DNU, sizeof(int) * 2);
    f.add(g.xds, sizeof(float) * g.DNU);
    f.add(g.yds, sizeof(float) * g.DNU);
    f.add(g.zds, sizeof(float) * g.DNV);
    f.add(&g.imgXCenter, sizeof(float) * 3);
    f.add(g.hangs, sizeof(float) * g.PN);
    f.add(g.hzPos, sizeof(float) * g.PN);
    int ints[4] = {g.PN, g.XN, g.YN, g.ZN};
    f.add(ints, sizeof ints);
    f.add(&g.dx, sizeof(float) * 2);
    return f.h;
}

template <class T>
int grow(T **p, size_t &cap, size_t n)
{
    if (n <= cap) return CTLAB_OK;
    if (*p) cudaFree(*p);
    *p = nullptr;
    cap = 0;
    cudaError_t e = cudaMalloc((void **)p, n * sizeof(T));
    if (e != cudaSuccess) return cuda_status(e, "legacy device buffer");
    cap = n;
    return CTLAB_OK;
}

// Common prologue: validation, device selection, plan (re)use.
int legacy_prepare(LegacyCtx &c, const ctlab_geometry &g, int gpunum)
{
    if (!g.xds || !g.yds || !g.zds || !g.hangs || !g.hzPos)
        return set_status(CTLAB_ERR_INVALID_ARG, "null geometry array");
    if (g.DNU < 1 || g.DNV < 1 || g.PN < 1 || g.XN < 1 || g.YN < 1 || g.ZN < 1)
        return set_status(CTLAB_ERR_INVALID_ARG, "sizes must be >= 1");
    if (!c.stream) {
        cudaError_t e = cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) return cuda_status(e, "legacy stream");
    }
    // SAT arithmetic of the cached plan: slice-major FP64-accumulated
    // z-prefixes unless CTLAB_LEGACY_SAT selects 0 (2-D FP64 SAT) or 1
    // (compensated FP32 pairs)
    int mode = CTLAB_SAT_ZPREFIX;
    if (const char *env = std::getenv("CTLAB_LEGACY_SAT")) {
        const int m = std::atoi(env);
        if (m == CTLAB_SAT_FP64 || m == CTLAB_SAT_F32PAIR || m == CTLAB_SAT_ZPREFIX) mode = m;
    }
    const unsigned long long key = geometry_key(g);
    if (!c.plan || c.key != key || c.mode != mode) {
        if (c.plan) ctlab_plan_destroy(c.plan);
        c.plan = nullptr;
        int rc = ctlab_plan_create(&g, gpunum, mode, &c.plan);
        if (rc != CTLAB_OK) return rc;
        c.key = key;
        c.mode = mode;
    }
    const size_t nv = (size_t)g.XN * g.YN * g.ZN, np = (size_t)g.PN * g.DNU * g.DNV;
    int rc = grow(&c.d_vol, c.vol_cap, nv);
    if (rc == CTLAB_OK) rc = grow(&c.d_prj, c.prj_cap, np);
    if (rc == CTLAB_OK) rc = grow(&c.d_mask, c.mask_cap, (size_t)g.XN * g.YN);
    return rc;
}

ctlab_geometry make_geom(float x0, float y0, float z0, int DNU, int DNV, float *xds, float *yds, float *zds,
                         float cx, float cy, float cz, float *hangs, float *hzPos, int PN, int XN, int YN,
                         int ZN, float dx, float dz)
{
    ctlab_geometry g;
    g.x0 = x0; g.y0 = y0; g.z0 = z0;
    g.DNU = DNU; g.DNV = DNV;
    g.xds = xds; g.yds = yds; g.zds = zds;
    g.imgXCenter = cx; g.imgYCenter = cy; g.imgZCenter = cz;
    g.hangs = hangs; g.hzPos = hzPos; g.PN = PN;
    g.XN = XN; g.YN = YN; g.ZN = ZN;
    g.dx = dx; g.dz = dz;
    return g;
}

int check_gpu(int gpunum)
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) return set_status(CTLAB_ERR_CUDA, "no CUDA device");
    if (gpunum < 0 || gpunum >= n || gpunum >= kMaxDevices)
        return set_status(CTLAB_ERR_INVALID_ARG, "gpunum out of range");
    return CTLAB_OK;
}

} // namespace

extern "C" {

void DD3Proj_gpu(float x0, float y0, float z0, int DNU, int DNV, float *xds, float *yds, float *zds,
                 float imgXCenter, float imgYCenter, float imgZCenter, float *hangs, float *hzPos, int PN,
                 int XN, int YN, int ZN, float *hvol, float *hprj, float dx, float dz, unsigned char *mask,
                 int gpunum, int prjMode)
{
    if (prjMode != CTLAB_PROJ_BRANCHLESS) {
        set_status(CTLAB_ERR_UNSUPPORTED, "only prjMode 0 (branchless DD) is implemented");
        return;
    }
    if (!hvol || !hprj) {
        set_status(CTLAB_ERR_INVALID_ARG, "null volume or projection");
        return;
    }
    if (check_gpu(gpunum) != CTLAB_OK) return;
    LegacyCtx &c = g_ctx[gpunum];
    std::lock_guard<std::mutex> lk(c.mu);
    DeviceGuard dg(gpunum);
    ctlab_geometry g = make_geom(x0, y0, z0, DNU, DNV, xds, yds, zds, imgXCenter, imgYCenter, imgZCenter, hangs,
                                 hzPos, PN, XN, YN, ZN, dx, dz);
    if (legacy_prepare(c, g, gpunum) != CTLAB_OK) return;
    const size_t nv = (size_t)XN * YN * ZN, np = (size_t)PN * DNU * DNV;
    cudaError_t e = cudaMemcpyAsync(c.d_vol, hvol, nv * sizeof(float), cudaMemcpyHostToDevice, c.stream);
    if (e == cudaSuccess && mask)
        e = cudaMemcpyAsync(c.d_mask, mask, (size_t)XN * YN, cudaMemcpyHostToDevice, c.stream);
    if (e != cudaSuccess) {
        cuda_status(e, "DD3Proj_gpu upload");
        return;
    }
    if (ctlab_proj(c.plan, c.d_vol, mask ? c.d_mask : nullptr, c.d_prj, c.stream) != CTLAB_OK) return;
    e = cudaMemcpyAsync(hprj, c.d_prj, np * sizeof(float), cudaMemcpyDeviceToHost, c.stream);
    if (e != cudaSuccess) {
        cuda_status(e, "DD3Proj_gpu download");
        return;
    }
    if (plan_check_device_error(c.plan, c.stream) != CTLAB_OK) return;
    ok();
}

void DD3Back_gpu(float x0, float y0, float z0, int DNU, int DNV, float *xds, float *yds, float *zds,
                 float imgXCenter, float imgYCenter, float imgZCenter, float *hangs, float *hzPos, int PN,
                 int XN, int YN, int ZN, float *hvol, float *hprj, float dx, float dz, unsigned char *mask,
                 int gpunum, int squared, int prjMode)
{
    (void)squared; // documented by the reference as a fake parameter
    if (prjMode != CTLAB_BACK_BRANCHLESS) {
        set_status(CTLAB_ERR_UNSUPPORTED, "only prjMode 0 (branchless DD) is implemented");
        return;
    }
    if (!hvol || !hprj) {
        set_status(CTLAB_ERR_INVALID_ARG, "null volume or projection");
        return;
    }
    if (check_gpu(gpunum) != CTLAB_OK) return;
    LegacyCtx &c = g_ctx[gpunum];
    std::lock_guard<std::mutex> lk(c.mu);
    DeviceGuard dg(gpunum);
    ctlab_geometry g = make_geom(x0, y0, z0, DNU, DNV, xds, yds, zds, imgXCenter, imgYCenter, imgZCenter, hangs,
                                 hzPos, PN, XN, YN, ZN, dx, dz);
    if (legacy_prepare(c, g, gpunum) != CTLAB_OK) return;
    const size_t nv = (size_t)XN * YN * ZN, np = (size_t)PN * DNU * DNV;
    cudaError_t e = cudaMemcpyAsync(c.d_prj, hprj, np * sizeof(float), cudaMemcpyHostToDevice, c.stream);
    if (e == cudaSuccess && mask)
        e = cudaMemcpyAsync(c.d_mask, mask, (size_t)XN * YN, cudaMemcpyHostToDevice, c.stream);
    if (e != cudaSuccess) {
        cuda_status(e, "DD3Back_gpu upload");
        return;
    }
    if (ctlab_back(c.plan, c.d_prj, mask ? c.d_mask : nullptr, c.d_vol, c.stream) != CTLAB_OK) return;
    e = cudaMemcpyAsync(hvol, c.d_vol, nv * sizeof(float), cudaMemcpyDeviceToHost, c.stream);
    if (e != cudaSuccess) {
        cuda_status(e, "DD3Back_gpu download");
        return;
    }
    if (plan_check_device_error(c.plan, c.stream) != CTLAB_OK) return;
    ok();
}

int ctlab_tv_gradient(const float *d_f, float *d_g, int XN, int YN, int ZN, float eps, void *stream)
{
    if (!d_f || !d_g || XN < 1 || YN < 1 || ZN < 1 || !(eps >= 0))
        return set_status(CTLAB_ERR_INVALID_ARG, "bad TV gradient arguments");
    CTLAB_CUDA_TRY(launch_tv_gradient(d_f, d_g, XN, YN, ZN, eps, (cudaStream_t)stream));
    return ok();
}

int ctlab_fista_step(const float *d_las, float *d_cur, float t1, float t2, long long n, float min_v, float max_v,
                     void *stream)
{
    if (!d_las || !d_cur || n < 0 || t2 == 0.f) return set_status(CTLAB_ERR_INVALID_ARG, "bad FISTA arguments");
    if (n == 0) return ok();
    CTLAB_CUDA_TRY(launch_fista_step(d_las, d_cur, t1, t2, n, min_v, max_v, (cudaStream_t)stream));
    return ok();
}

int ctlab_sart_proj_weight(float *d_prj, const float *d_real, const float *d_row_sum, long long n, void *stream)
{
    if (!d_prj || !d_real || !d_row_sum || n < 0) return set_status(CTLAB_ERR_INVALID_ARG, "bad arguments");
    if (n == 0) return ok();
    CTLAB_CUDA_TRY(launch_sart_proj_weight(d_prj, d_real, d_row_sum, n, (cudaStream_t)stream));
    return ok();
}

int ctlab_sart_back_weight(float *d_vol, float *d_recon, const float *d_col_sum, long long n, void *stream)
{
    if (!d_vol || !d_recon || !d_col_sum || n < 0) return set_status(CTLAB_ERR_INVALID_ARG, "bad arguments");
    if (n == 0) return ok();
    CTLAB_CUDA_TRY(launch_sart_back_weight(d_vol, d_recon, d_col_sum, n, (cudaStream_t)stream));
    return ok();
}

int ctlab_ellipsoid_phantom(float *d_vol, int XN, int YN, int ZN, float dx, float dz, float imgXCenter,
                            float imgYCenter, float imgZCenter, const double *h_ell, int n_ell, int clamp_nonneg,
                            void *stream)
{
    if (!d_vol || XN < 1 || YN < 1 || ZN < 1 || n_ell < 0 || (n_ell > 0 && !h_ell) || n_ell > 512)
        return set_status(CTLAB_ERR_INVALID_ARG, "bad phantom arguments");
    std::vector<float> packed(16 * (size_t)std::max(n_ell, 1), 0.f);
    for (int e = 0; e < n_ell; ++e) {
        const double *E = h_ell + 10 * e;
        if (!(E[4] > 0 && E[5] > 0 && E[6] > 0))
            return set_status(CTLAB_ERR_INVALID_ARG, "ellipsoid semi-axes must be > 0");
        const double cf = std::cos(E[7]), sf = std::sin(E[7]), ct = std::cos(E[8]), st = std::sin(E[8]),
                     cp = std::cos(E[9]), sp = std::sin(E[9]);
        // R = Rz(phi) Rx(theta) Rz(psi); store R^T row-major (= R columns)
        const double R[9] = {cf * cp - sf * ct * sp, -cf * sp - sf * ct * cp, sf * st,
                             sf * cp + cf * ct * sp, -sf * sp + cf * ct * cp, -cf * st,
                             st * sp,                st * cp,                 ct};
        float *P = packed.data() + 16 * e;
        P[0] = (float)E[0];
        P[1] = (float)E[1]; P[2] = (float)E[2]; P[3] = (float)E[3];
        P[4] = (float)(1.0 / E[4]); P[5] = (float)(1.0 / E[5]); P[6] = (float)(1.0 / E[6]);
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) P[7 + 3 * r + c] = (float)R[3 * c + r];
    }
    float *d_ell = nullptr;
    cudaStream_t s = (cudaStream_t)stream;
    CTLAB_CUDA_TRY(cudaMalloc(&d_ell, sizeof(float) * packed.size()));
    cudaError_t e = cudaMemcpyAsync(d_ell, packed.data(), sizeof(float) * packed.size(), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = launch_phantom(d_vol, XN, YN, ZN, dx, dz, imgXCenter, imgYCenter, imgZCenter, d_ell, n_ell,
                           clamp_nonneg, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(d_ell);
    if (e != cudaSuccess) return cuda_status(e, "ellipsoid phantom");
    return ok();
}

int ctlab_random_ellipsoids(unsigned long long seed, int n_min, int n_max, float half_x, float half_y,
                            float half_z, float v_max, double *h_ell, int cap)
{
    if (!h_ell || n_min < 1 || n_max < n_min || cap < 1 || !(half_x > 0) || !(half_y > 0) || !(half_z > 0))
        return -set_status(CTLAB_ERR_INVALID_ARG, "bad random-ellipsoid arguments");
    std::mt19937_64 rng(seed);
    std::uniform_int_distribution<int> count(n_min, n_max);
    std::uniform_real_distribution<double> unit(0.0, 1.0);
    const int n = std::min(count(rng), cap);
    const double hx = half_x, hy = half_y, hz = half_z;
    for (int e = 0; e < n; ++e) {
        double *E = h_ell + 10 * e;
        E[1] = (2.0 * unit(rng) - 1.0) * 0.8 * hx;
        E[2] = (2.0 * unit(rng) - 1.0) * 0.8 * hy;
        E[3] = (2.0 * unit(rng) - 1.0) * 0.8 * hz;
        E[4] = (0.05 + 0.35 * unit(rng)) * hx;
        E[5] = (0.05 + 0.35 * unit(rng)) * hy;
        E[6] = (0.05 + 0.35 * unit(rng)) * hz;
        E[7] = unit(rng) * M_PI;
        E[8] = unit(rng) * M_PI;
        E[9] = unit(rng) * M_PI;
        E[0] = unit(rng) * v_max;
    }
    ok();
    return n;
}

} // extern "C"
