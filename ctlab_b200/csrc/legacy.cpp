// Host-pointer entry points with the reference's names and argument order
// (DD3Proj_gpu, DD3Back_gpu), plus the elementwise and phantom C ABI.
//
// Each legacy call copies its host inputs to the device, runs the
// device-pointer path on a library-owned stream and copies the result back.
// Geometry plans and device buffers are cached per device (re-created only
// when the geometry changes, buffers only grow), so repeated calls with one
// scan geometry pay no allocation.  Calls on one device are serialised.
//
// The copies run on a second stream and overlap the compute chunk by chunk
// (z-prefix plans): the volume goes up in y slabs, each slab's column
// z-prefixes built as it lands; projections come back in blocks of view
// groups as they are finished; the projections of a backprojection go up in
// view blocks, each block's v-prefixes built as it lands, and the volume
// comes back in y slabs of bricks as they are finished.  Every chunk runs the
// same per-output arithmetic as the one-launch path, so the results are the
// same bit for bit.  Pageable host buffers are staged through a pinned ring
// (transfer.h).
#include <climits>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <random>

#include "plan.h"
#include "transfer.h"

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
    Stager stager;
    std::vector<cudaEvent_t> ev; // chunk completion events (compute and copy streams)
    // projection chunks of the cached plan: consecutive view groups whose
    // views are the list positions [cut[k], cut[k+1])
    const ctlab_plan *chunk_plan = nullptr;
    std::vector<int> cut;
    std::vector<GroupTab> chunk_groups;
    int *d_chunk_groups = nullptr;
};

constexpr int kChunks = 4;

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
    if (int rc = c.stager.init(); rc != CTLAB_OK) return rc;
    while (c.ev.size() < 2 * kChunks) {
        cudaEvent_t e = nullptr;
        cudaError_t ce = cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
        if (ce != cudaSuccess) return cuda_status(ce, "legacy event");
        c.ev.push_back(e);
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
        c.chunk_plan = nullptr; // a new plan may reuse the old one's address
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

// Splits the plan's projector view groups (over the whole view list) into
// about kChunks runs of consecutive groups whose views are contiguous list
// positions, and uploads each run's group table; one run when the groups do
// not line up that way.  Cached per plan.
int plan_chunks(LegacyCtx &c)
{
    ctlab_plan *p = c.plan;
    if (c.chunk_plan == p) return CTLAB_OK;
    c.chunk_plan = nullptr;
    c.cut.clear();
    c.chunk_groups.clear();
    const HostGeometry &g = p->g;
    std::vector<int> all(g.PN);
    for (int i = 0; i < g.PN; ++i) all[i] = i;
    ProjGroups pg = p->sat_mode == CTLAB_SAT_ZPREFIX ? proj_t_make_groups(g, all, p->tst)
                                                     : proj_make_groups(g, all, p->proj_cmax);
    const int G = pg.G, ng = pg.ngroups;
    // each group's views are consecutive list positions; ordered by their
    // first position the groups tile the list, and runs of them make chunks
    std::vector<std::pair<int, int>> order; // (first position, group)
    bool tiles = G >= 1 && ng >= 1;
    for (int k = 0; k < ng && tiles; ++k) {
        int lo = INT_MAX, hi = -1, cnt = 0;
        for (int q = 0; q < G; ++q) {
            const int v = pg.table[(size_t)k * G + q];
            if (v < 0) continue;
            lo = std::min(lo, v);
            hi = std::max(hi, v);
            ++cnt;
        }
        if (cnt == 0 || hi - lo + 1 != cnt) tiles = false;
        order.push_back({lo, k});
    }
    std::vector<int> table; // the groups in position order
    std::vector<int> gcut = {0}, pcut = {0};
    if (tiles) {
        std::sort(order.begin(), order.end());
        int seen = 0;
        for (int i = 0; i < ng && tiles; ++i) {
            const int k = order[i].second;
            if (order[i].first != seen) tiles = false;
            int cnt = 0;
            for (int q = 0; q < G; ++q) {
                table.push_back(pg.table[(size_t)k * G + q]);
                cnt += pg.table[(size_t)k * G + q] >= 0;
            }
            seen += cnt;
            const int want = (int)pcut.size() * g.PN / kChunks;
            if (tiles && seen >= want && i + 1 < ng && (int)pcut.size() < kChunks) {
                gcut.push_back(i + 1);
                pcut.push_back(seen);
            }
        }
        if (seen != g.PN) tiles = false;
    }
    if (!tiles) { // one chunk: the table as planned
        table = pg.table;
        gcut = {0};
        pcut = {0};
    }
    gcut.push_back(ng);
    pcut.push_back(g.PN);
    pg.table = table;
    if (c.d_chunk_groups) cudaFree(c.d_chunk_groups);
    c.d_chunk_groups = nullptr;
    cudaError_t ce = cudaMalloc(&c.d_chunk_groups, sizeof(int) * std::max<size_t>(pg.table.size(), 1));
    if (ce != cudaSuccess) return cuda_status(ce, "legacy chunk groups");
    // positions in a run's table are relative to the run's first view
    std::vector<int> tab(pg.table.size());
    for (size_t k = 0; k + 1 < gcut.size(); ++k)
        for (int i = gcut[k] * G; i < gcut[k + 1] * G; ++i)
            tab[i] = pg.table[i] < 0 ? -1 : pg.table[i] - pcut[k];
    if (!tab.empty())
        CTLAB_CUDA_TRY(cudaMemcpy(c.d_chunk_groups, tab.data(), sizeof(int) * tab.size(), cudaMemcpyHostToDevice));
    for (size_t k = 0; k + 1 < gcut.size(); ++k) {
        GroupTab t;
        t.d = c.d_chunk_groups + (size_t)gcut[k] * G;
        t.ngroups = gcut[k + 1] - gcut[k];
        t.G = G;
        c.chunk_groups.push_back(t);
    }
    c.cut = pcut;
    c.chunk_plan = p;
    return CTLAB_OK;
}

// y slabs of kChunks parts (boundaries multiples of 32, for the x-slice
// z-prefixes) -- or of 8-voxel brick rows for the backprojector
std::vector<int> y_cuts(int YN, int align)
{
    std::vector<int> cut = {0};
    for (int k = 1; k < kChunks; ++k) {
        const int y = (int)((long long)k * YN / kChunks) / align * align;
        if (y > cut.back() && y < YN) cut.push_back(y);
    }
    cut.push_back(YN);
    return cut;
}

int legacy_proj(LegacyCtx &c, const float *hvol, float *hprj, const unsigned char *mask)
{
    ctlab_plan *p = c.plan;
    const HostGeometry &g = p->g;
    const size_t col = (size_t)g.XN * g.ZN, bin = (size_t)g.DNU * g.DNV;
    cudaStream_t s = c.stream;
    Stager &st = c.stager;
    p->last_launches = 0;
    int rc = plan_chunks(c);
    if (rc != CTLAB_OK) return rc;
    // mask, then the volume in y slabs; z-prefix plans build each slab's
    // column prefixes as it lands
    if (mask) rc = st.h2d(c.d_mask, mask, (size_t)g.XN * g.YN, nullptr);
    const unsigned char *dm = mask ? c.d_mask : nullptr;
    if (p->sat_mode == CTLAB_SAT_ZPREFIX) {
        const std::vector<int> yc = y_cuts(g.YN, 32);
        for (size_t k = 0; k + 1 < yc.size() && rc == CTLAB_OK; ++k) {
            rc = st.h2d(c.d_vol + yc[k] * col, hvol + yc[k] * col, (yc[k + 1] - yc[k]) * col * sizeof(float), nullptr);
            if (rc == CTLAB_OK) CTLAB_CUDA_TRY(cudaEventRecord(c.ev[k], st.stream()));
            if (rc == CTLAB_OK) CTLAB_CUDA_TRY(cudaStreamWaitEvent(s, c.ev[k], 0));
            if (rc == CTLAB_OK) rc = plan_volume_sat_rows(p, c.d_vol, dm, yc[k], yc[k + 1], s);
        }
    } else {
        if (rc == CTLAB_OK) rc = st.h2d(c.d_vol, hvol, g.YN * col * sizeof(float), nullptr);
        if (rc == CTLAB_OK) CTLAB_CUDA_TRY(cudaEventRecord(c.ev[0], st.stream()));
        if (rc == CTLAB_OK) CTLAB_CUDA_TRY(cudaStreamWaitEvent(s, c.ev[0], 0));
        if (rc == CTLAB_OK) rc = plan_volume_sat(p, c.d_vol, dm, s);
    }
    // projection by runs of view groups, each run's views downloaded as soon
    // as it is done
    for (size_t k = 0; k + 1 < c.cut.size() && rc == CTLAB_OK; ++k) {
        const int v0 = c.cut[k], n = c.cut[k + 1] - v0;
        rc = plan_proj_list(p, p->d_all_views + v0, n, c.chunk_groups[k], c.d_prj + bin * v0, s, PROJ_PLAIN, nullptr,
                            nullptr, nullptr);
        if (rc == CTLAB_OK) CTLAB_CUDA_TRY(cudaEventRecord(c.ev[kChunks + k], s));
        if (rc == CTLAB_OK) rc = st.d2h(hprj + bin * v0, c.d_prj + bin * v0, bin * n * sizeof(float), c.ev[kChunks + k]);
    }
    if (rc == CTLAB_OK) rc = st.finish();
    if (rc != CTLAB_OK) {
        st.abandon();
        return rc;
    }
    return plan_check_device_error(p, s);
}

int legacy_back(LegacyCtx &c, const float *hprj, float *hvol, const unsigned char *mask)
{
    ctlab_plan *p = c.plan;
    const HostGeometry &g = p->g;
    if (!g.flat_uniform)
        return set_status(CTLAB_ERR_UNSUPPORTED, "backprojection needs a flat detector with uniform u and v pitch");
    if (p->q_capacity == 0)
        return set_status(CTLAB_ERR_UNSUPPORTED, "DNV beyond the backprojector's shared-memory tiles");
    const size_t col = (size_t)g.XN * g.ZN, bin = (size_t)g.DNU * g.DNV;
    cudaStream_t s = c.stream;
    Stager &st = c.stager;
    p->last_launches = 0;
    int rc = CTLAB_OK;
    if (mask) rc = st.h2d(c.d_mask, mask, (size_t)g.XN * g.YN, nullptr);
    const unsigned char *dm = mask ? c.d_mask : nullptr;
    if (p->sat_mode != CTLAB_SAT_ZPREFIX) {
        if (rc == CTLAB_OK) rc = st.h2d(c.d_prj, hprj, bin * g.PN * sizeof(float), nullptr);
        if (rc == CTLAB_OK) CTLAB_CUDA_TRY(cudaEventRecord(c.ev[0], st.stream()));
        if (rc == CTLAB_OK) CTLAB_CUDA_TRY(cudaStreamWaitEvent(s, c.ev[0], 0));
        if (rc == CTLAB_OK) rc = ctlab_back(p, c.d_prj, dm, c.d_vol, s);
        if (rc == CTLAB_OK) CTLAB_CUDA_TRY(cudaEventRecord(c.ev[kChunks], s));
        if (rc == CTLAB_OK) rc = st.d2h(hvol, c.d_vol, g.YN * col * sizeof(float), c.ev[kChunks]);
    } else {
        // projections in view blocks, each block's v-prefixes built as it lands
        for (int k = 0; k < kChunks && rc == CTLAB_OK; ++k) {
            const int v0 = (int)((long long)k * g.PN / kChunks), v1 = (int)((long long)(k + 1) * g.PN / kChunks);
            if (v1 == v0) continue;
            rc = st.h2d(c.d_prj + bin * v0, hprj + bin * v0, bin * (v1 - v0) * sizeof(float), nullptr);
            if (rc == CTLAB_OK) CTLAB_CUDA_TRY(cudaEventRecord(c.ev[k], st.stream()));
            if (rc == CTLAB_OK) CTLAB_CUDA_TRY(cudaStreamWaitEvent(s, c.ev[k], 0));
            if (rc == CTLAB_OK) rc = plan_proj_sat_range(p, p->d_all_views, v0, v1 - v0, c.d_prj, s);
        }
        // the volume in y slabs of brick rows, each downloaded when done; the
        // slabs end on whole waves of the backprojector's CTAs, so a slab
        // costs no more than the same rows inside one launch
        const int bys = (g.YN + 7) / 8;
        int wave = 0;
        if (rc == CTLAB_OK) rc = plan_back_wave_rows(p, g.PN, &wave);
        std::vector<int> bc = {0};
        for (int k = 1; k < kChunks && wave > 0; ++k) {
            const int r = (int)std::lround((double)k * bys / kChunks / wave) * wave;
            if (r > bc.back() && r < bys) bc.push_back(r);
        }
        bc.push_back(bys);
        for (size_t k = 0; k + 1 < bc.size() && rc == CTLAB_OK; ++k) {
            rc = plan_back_rows(p, p->d_all_views, g.PN, dm, c.d_vol, s, BACK_PLAIN, nullptr, 1.f, 0, 0.f, 0.f,
                                bc[k], bc[k + 1] - bc[k]);
            if (rc == CTLAB_OK) CTLAB_CUDA_TRY(cudaEventRecord(c.ev[kChunks + k], s));
            const size_t y0 = (size_t)bc[k] * 8, y1 = std::min<size_t>((size_t)bc[k + 1] * 8, g.YN);
            if (rc == CTLAB_OK)
                rc = st.d2h(hvol + y0 * col, c.d_vol + y0 * col, (y1 - y0) * col * sizeof(float), c.ev[kChunks + k]);
        }
    }
    if (rc == CTLAB_OK) rc = st.finish();
    if (rc != CTLAB_OK) {
        st.abandon();
        return rc;
    }
    return plan_check_device_error(p, s);
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
    if (legacy_proj(c, hvol, hprj, mask) != CTLAB_OK) return;
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
    if (legacy_back(c, hprj, hvol, mask) != CTLAB_OK) return;
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
