// Host-pointer entry points that split one scan over several GPUs of one
// process, with the reference's names and argument order:
//   DD3Proj_multiGPU (src/DD3_GPU_Proj.h:138-141): GPU i projects the views
//     [startPN[i], startPN[i+1]) of the whole volume (startPN[gpuNum] = PN);
//   DD3Back_multiGPU (src/DD3_GPU_Back.h:138-142): GPU i backprojects the
//     z slab [startVOL[i], startVOL[i+1]) of the volume (startVOL[gpuNum] =
//     ZN) from only the views whose rays can reach the slab -- the role of
//     getPrjIdxPair (src/utilities.cuh:503-532) -- and writes its slab
//     straight into the caller's volume, which is the reference's
//     combineVolume (:538-589) without a host-side copy.
// Projection blocks and volume slabs are disjoint, so no GPU reduces or
// exchanges data with another: each one reads the caller's host arrays and
// writes its own part back.  One host thread per GPU; the parts of one GPU
// run one after another.  The split is exact: a view left out of a slab
// adds exactly zero to it (every voxel boundary of the slab projects outside
// the detector rows and the saturated prefix difference vanishes).
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "plan.h"

using namespace ctlab;

namespace {

constexpr int kMaxDevices = 64;

// Per-device cache of one plan and its device buffers (one for projection,
// one for backprojection), re-created when the part's geometry changes.
struct PartCtx {
    std::mutex mu;
    ctlab_plan *plan = nullptr;
    std::vector<float> key;
    float *d_vol = nullptr;
    size_t vol_cap = 0;
    float *d_prj = nullptr;
    size_t prj_cap = 0;
    unsigned char *d_mask = nullptr;
    size_t mask_cap = 0;
    cudaStream_t stream = nullptr;
};
PartCtx g_proj[kMaxDevices], g_back[kMaxDevices];

template <class T>
int grow(T **p, size_t &cap, size_t n)
{
    if (n <= cap) return CTLAB_OK;
    if (*p) cudaFree(*p);
    *p = nullptr;
    cap = 0;
    cudaError_t e = cudaMalloc((void **)p, std::max<size_t>(n, 1) * sizeof(T));
    if (e != cudaSuccess) return cuda_status(e, "multi-GPU device buffer");
    cap = n;
    return CTLAB_OK;
}

// Every scalar and array of the geometry, as the cache key of a part.
std::vector<float> geometry_key(const ctlab_geometry &g)
{
    std::vector<float> k = {g.x0, g.y0, g.z0, (float)g.DNU, (float)g.DNV, g.imgXCenter, g.imgYCenter, g.imgZCenter,
                            (float)g.PN, (float)g.XN, (float)g.YN, (float)g.ZN, g.dx, g.dz};
    k.insert(k.end(), g.xds, g.xds + g.DNU);
    k.insert(k.end(), g.yds, g.yds + g.DNU);
    k.insert(k.end(), g.zds, g.zds + g.DNV);
    k.insert(k.end(), g.hangs, g.hangs + g.PN);
    k.insert(k.end(), g.hzPos, g.hzPos + g.PN);
    return k;
}

int part_prepare(PartCtx &c, const ctlab_geometry &g, int device, size_t nvol, size_t nprj, size_t nmask)
{
    if (!c.stream) {
        cudaError_t e = cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) return cuda_status(e, "multi-GPU stream");
    }
    std::vector<float> key = geometry_key(g);
    if (!c.plan || key != c.key) {
        if (c.plan) ctlab_plan_destroy(c.plan);
        c.plan = nullptr;
        c.key.clear();
        int rc = ctlab_plan_create(&g, device, CTLAB_SAT_ZPREFIX, &c.plan);
        if (rc != CTLAB_OK) return rc;
        c.key.swap(key);
    }
    int rc = grow(&c.d_vol, c.vol_cap, nvol);
    if (rc == CTLAB_OK) rc = grow(&c.d_prj, c.prj_cap, nprj);
    if (rc == CTLAB_OK) rc = grow(&c.d_mask, c.mask_cap, nmask);
    return rc;
}

// Logical GPU i -> CUDA device i.  With CTLAB_MULTIGPU_WRAP=1 the parts of a
// split larger than the machine wrap around the devices (i mod count) and
// run one after another, which checks the partition on fewer GPUs.
int resolve_devices(int gpuNum, std::vector<int> &dev)
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) return set_status(CTLAB_ERR_CUDA, "no CUDA device");
    if (gpuNum < 1 || gpuNum > kMaxDevices) return set_status(CTLAB_ERR_INVALID_ARG, "gpuNum must be in [1, 64]");
    const char *w = std::getenv("CTLAB_MULTIGPU_WRAP");
    const bool wrap = w && std::atoi(w) != 0;
    if (gpuNum > n && !wrap) {
        return set_status(CTLAB_ERR_INVALID_ARG, "gpuNum (" + std::to_string(gpuNum) + ") exceeds the " +
                                                     std::to_string(n) + " visible CUDA devices");
    }
    dev.resize(gpuNum);
    for (int i = 0; i < gpuNum; ++i) dev[i] = i % n;
    return CTLAB_OK;
}

// start[0..parts-1] -> [lo, hi) per part; start[0] == 0, non-decreasing,
// every start <= total; the last part ends at total.
int parse_starts(const int *start, int parts, int total, const char *what, std::vector<int> &lo, std::vector<int> &hi)
{
    if (!start) return set_status(CTLAB_ERR_INVALID_ARG, std::string("null ") + what);
    lo.resize(parts);
    hi.resize(parts);
    for (int i = 0; i < parts; ++i) {
        const int a = start[i], b = i + 1 < parts ? start[i + 1] : total;
        if ((i == 0 && a != 0) || a < 0 || b < a || b > total)
            return set_status(CTLAB_ERR_INVALID_ARG, std::string(what) +
                                                         " must start at 0, never decrease and stay within the "
                                                         "scan (entry " + std::to_string(i) + ")");
        lo[i] = a;
        hi[i] = b;
    }
    return CTLAB_OK;
}

// Runs fn(part) for every part, one host thread per distinct device (parts
// of one device in order); returns the first failure with its message.
template <class Fn>
int run_parts(const std::vector<int> &dev, Fn fn)
{
    const int parts = (int)dev.size();
    std::vector<int> rc(parts, CTLAB_OK);
    std::vector<std::string> msg(parts);
    std::vector<int> devices(dev);
    std::sort(devices.begin(), devices.end());
    devices.erase(std::unique(devices.begin(), devices.end()), devices.end());
    std::vector<std::thread> workers;
    for (int d : devices) {
        workers.emplace_back([&, d]() {
            for (int i = 0; i < parts; ++i) {
                if (dev[i] != d) continue;
                rc[i] = fn(i);
                if (rc[i] != CTLAB_OK) {
                    msg[i] = ctlab_last_error();
                    break;
                }
            }
        });
    }
    for (auto &t : workers) t.join();
    for (int i = 0; i < parts; ++i)
        if (rc[i] != CTLAB_OK) return set_status(rc[i], "part " + std::to_string(i) + ": " + msg[i]);
    return ok();
}

ctlab_geometry make_geom(float x0, float y0, float z0, int DNU, int DNV, float *xds, float *yds, float *zds, float cx,
                         float cy, float cz, float *hangs, float *hzPos, int PN, int XN, int YN, int ZN, float dx,
                         float dz)
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

int check_scan(const ctlab_geometry &g, const float *hvol, const float *hprj)
{
    if (!hvol || !hprj) return set_status(CTLAB_ERR_INVALID_ARG, "null volume or projection");
    if (!g.xds || !g.yds || !g.zds || !g.hangs || !g.hzPos)
        return set_status(CTLAB_ERR_INVALID_ARG, "null geometry array");
    if (g.DNU < 1 || g.DNV < 1 || g.PN < 1 || g.XN < 1 || g.YN < 1 || g.ZN < 1)
        return set_status(CTLAB_ERR_INVALID_ARG, "sizes must be >= 1");
    return CTLAB_OK;
}

} // namespace

extern "C" {

int ctlab_slab_views(const ctlab_geometry *g, int z0, int z1, int *h_views, int cap)
{
    if (!g || !g->zds || !g->hzPos || g->DNV < 1 || g->PN < 0 || g->ZN < 1 || !(g->dz > 0))
        return -set_status(CTLAB_ERR_INVALID_ARG, "bad geometry");
    if (z0 < 0 || z1 < z0 || z1 > g->ZN) return -set_status(CTLAB_ERR_INVALID_ARG, "slab outside the volume");
    if (cap < 0 || (cap > 0 && !h_views)) return -set_status(CTLAB_ERR_INVALID_ARG, "bad output list");
    // z extent of the detector cells (local, before the view's shift):
    // the cell centres widened by a full row pitch each way
    double zmin = g->zds[0], zmax = g->zds[0], pitch = 0.5;
    for (int v = 0; v < g->DNV; ++v) {
        zmin = std::min(zmin, (double)g->zds[v]);
        zmax = std::max(zmax, (double)g->zds[v]);
        if (v > 0) pitch = std::max(pitch, std::fabs((double)g->zds[v] - g->zds[v - 1]));
    }
    zmin -= pitch;
    zmax += pitch;
    // the slab's z range, widened by one voxel
    const double zlo_vol = (double)g->imgZCenter - 0.5 * g->ZN * g->dz;
    const double slo = zlo_vol + (z0 - 1) * (double)g->dz, shi = zlo_vol + (z1 + 1) * (double)g->dz;
    int n = 0;
    for (int p = 0; p < g->PN && z1 > z0; ++p) {
        // every ray of view p runs between the source and a detector cell
        const double zp = g->hzPos[p];
        const double lo = std::min((double)g->z0, zmin) + zp, hi = std::max((double)g->z0, zmax) + zp;
        if (hi < slo || lo > shi) continue;
        if (n < cap) h_views[n] = p;
        ++n;
    }
    ok();
    return n;
}

int ctlab_proj_multi(const ctlab_geometry *geom, const float *hvol, float *hprj, const unsigned char *mask,
                     const int *startPN, int gpuNum)
{
    if (!geom) return set_status(CTLAB_ERR_INVALID_ARG, "null geometry");
    const ctlab_geometry &g = *geom;
    int rc = check_scan(g, hvol, hprj);
    std::vector<int> dev, lo, hi;
    if (rc == CTLAB_OK) rc = resolve_devices(gpuNum, dev);
    if (rc == CTLAB_OK) rc = parse_starts(startPN, gpuNum, g.PN, "startPN", lo, hi);
    if (rc != CTLAB_OK) return rc;
    const size_t nv = (size_t)g.XN * g.YN * g.ZN, bin = (size_t)g.DNU * g.DNV;
    return run_parts(dev, [&](int i) -> int {
        const int n = hi[i] - lo[i];
        if (n == 0) return CTLAB_OK;
        PartCtx &c = g_proj[dev[i]];
        std::lock_guard<std::mutex> lk(c.mu);
        DeviceGuard dg(dev[i]);
        ctlab_geometry pg = g;
        pg.hangs = g.hangs + lo[i];
        pg.hzPos = g.hzPos + lo[i];
        pg.PN = n;
        int r = part_prepare(c, pg, dev[i], nv, bin * n, (size_t)g.XN * g.YN);
        if (r != CTLAB_OK) return r;
        cudaError_t e = cudaMemcpyAsync(c.d_vol, hvol, nv * sizeof(float), cudaMemcpyHostToDevice, c.stream);
        if (e == cudaSuccess && mask)
            e = cudaMemcpyAsync(c.d_mask, mask, (size_t)g.XN * g.YN, cudaMemcpyHostToDevice, c.stream);
        if (e != cudaSuccess) return cuda_status(e, "DD3Proj_multiGPU upload");
        r = ctlab_proj(c.plan, c.d_vol, mask ? c.d_mask : nullptr, c.d_prj, c.stream);
        if (r != CTLAB_OK) return r;
        e = cudaMemcpyAsync(hprj + bin * lo[i], c.d_prj, bin * n * sizeof(float), cudaMemcpyDeviceToHost, c.stream);
        if (e != cudaSuccess) return cuda_status(e, "DD3Proj_multiGPU download");
        return plan_check_device_error(c.plan, c.stream);
    });
}

int ctlab_back_multi(const ctlab_geometry *geom, const float *hprj, float *hvol, const unsigned char *mask,
                     const int *startVOL, int gpuNum)
{
    if (!geom) return set_status(CTLAB_ERR_INVALID_ARG, "null geometry");
    const ctlab_geometry &g = *geom;
    int rc = check_scan(g, hvol, hprj);
    std::vector<int> dev, lo, hi;
    if (rc == CTLAB_OK) rc = resolve_devices(gpuNum, dev);
    if (rc == CTLAB_OK) rc = parse_starts(startVOL, gpuNum, g.ZN, "startVOL", lo, hi);
    if (rc != CTLAB_OK) return rc;
    const size_t cols = (size_t)g.XN * g.YN, bin = (size_t)g.DNU * g.DNV;
    return run_parts(dev, [&](int i) -> int {
        const int szn = hi[i] - lo[i];
        if (szn == 0) return CTLAB_OK;
        std::vector<int> views(g.PN);
        const int n = ctlab_slab_views(&g, lo[i], hi[i], views.data(), g.PN);
        if (n < 0) return -n;
        views.resize(n);
        // the slab's voxels as a volume of their own: the same columns, SZN
        // slices centred where the slab's slices sit in the whole volume
        std::vector<float> ang(std::max(n, 1)), zpos(std::max(n, 1));
        for (int k = 0; k < n; ++k) {
            ang[k] = g.hangs[views[k]];
            zpos[k] = g.hzPos[views[k]];
        }
        ctlab_geometry sg = g;
        sg.ZN = szn;
        sg.imgZCenter = (float)((double)g.imgZCenter + (lo[i] + 0.5 * szn - 0.5 * g.ZN) * (double)g.dz);
        sg.hangs = ang.data();
        sg.hzPos = zpos.data();
        sg.PN = std::max(n, 1);
        if (n == 0) {
            // no view reaches the slab: its backprojection is zero
            for (size_t col = 0; col < cols; ++col) std::fill(hvol + col * g.ZN + lo[i], hvol + col * g.ZN + hi[i], 0.f);
            return CTLAB_OK;
        }
        PartCtx &c = g_back[dev[i]];
        std::lock_guard<std::mutex> lk(c.mu);
        DeviceGuard dg(dev[i]);
        cudaError_t e = cudaSuccess;
        int r = part_prepare(c, sg, dev[i], cols * szn, bin * n, cols);
        if (r != CTLAB_OK) return r;
        // the slab's views: one copy per run of consecutive views
        for (int k = 0; k < n && e == cudaSuccess;) {
            int k1 = k + 1;
            while (k1 < n && views[k1] == views[k1 - 1] + 1) ++k1;
            e = cudaMemcpyAsync(c.d_prj + bin * k, hprj + bin * views[k], bin * (k1 - k) * sizeof(float),
                                cudaMemcpyHostToDevice, c.stream);
            k = k1;
        }
        if (e == cudaSuccess && mask) e = cudaMemcpyAsync(c.d_mask, mask, cols, cudaMemcpyHostToDevice, c.stream);
        if (e != cudaSuccess) return cuda_status(e, "DD3Back_multiGPU upload");
        r = ctlab_back(c.plan, c.d_prj, mask ? c.d_mask : nullptr, c.d_vol, c.stream);
        if (r != CTLAB_OK) return r;
        // slab [YN*XN][SZN] -> columns of the caller's (Z,X,Y) volume
        e = cudaMemcpy2DAsync(hvol + lo[i], sizeof(float) * g.ZN, c.d_vol, sizeof(float) * szn, sizeof(float) * szn,
                              cols, cudaMemcpyDeviceToHost, c.stream);
        if (e != cudaSuccess) return cuda_status(e, "DD3Back_multiGPU download");
        return plan_check_device_error(c.plan, c.stream);
    });
}

void DD3Proj_multiGPU(float x0, float y0, float z0, int DNU, int DNV, float *xds, float *yds, float *zds,
                      float imgXCenter, float imgYCenter, float imgZCenter, float *hangs, float *hzPos, int PN, int XN,
                      int YN, int ZN, float *hvol, float *hprj, float dx, float dz, unsigned char *mask, int prjMode,
                      int *startPN, int gpuNum)
{
    if (prjMode != CTLAB_PROJ_BRANCHLESS) {
        set_status(CTLAB_ERR_UNSUPPORTED, "only prjMode 0 (branchless DD) is implemented");
        return;
    }
    ctlab_geometry g = make_geom(x0, y0, z0, DNU, DNV, xds, yds, zds, imgXCenter, imgYCenter, imgZCenter, hangs,
                                 hzPos, PN, XN, YN, ZN, dx, dz);
    ctlab_proj_multi(&g, hvol, hprj, mask, startPN, gpuNum);
}

void DD3Back_multiGPU(float x0, float y0, float z0, int DNU, int DNV, float *xds, float *yds, float *zds,
                      float imgXCenter, float imgYCenter, float imgZCenter, float *hangs, float *hzPos, int PN, int XN,
                      int YN, int ZN, float *hvol, float *hprj, float dx, float dz, unsigned char *mask, int methodId,
                      int *startVOL, int gpuNum)
{
    if (methodId != CTLAB_BACK_BRANCHLESS) {
        set_status(CTLAB_ERR_UNSUPPORTED, "only methodId 0 (branchless DD) is implemented");
        return;
    }
    ctlab_geometry g = make_geom(x0, y0, z0, DNU, DNV, xds, yds, zds, imgXCenter, imgYCenter, imgZCenter, hangs,
                                 hzPos, PN, XN, YN, ZN, dx, dz);
    ctlab_back_multi(&g, hprj, hvol, mask, startVOL, gpuNum);
}

} // extern "C"
