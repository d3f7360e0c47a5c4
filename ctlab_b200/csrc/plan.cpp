// Plans and the device-pointer C ABI: geometry upload, SAT workspaces,
// stream-ordered projection / backprojection.
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <new>

#include "plan.h"

using namespace ctlab;

namespace ctlab {

namespace {

constexpr int kVolChunk = 32;  // rows per CTA of the volume SAT scans
constexpr int kPrjChunk = 32;  // rows per CTA of the projection SAT scans

int round_up(int v, int m) { return (v + m - 1) / m * m; }

template <class T>
cudaError_t dmalloc(T **p, size_t n, long long &bytes)
{
    *p = nullptr;
    if (n == 0) return cudaSuccess;
    cudaError_t e = cudaMalloc((void **)p, n * sizeof(T));
    if (e == cudaSuccess) bytes += (long long)(n * sizeof(T));
    return e;
}

// cuTensorMapEncodeTiled from the driver, looked up once through the runtime
// (no link-time dependency on libcuda).
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

// TMA map of a slice-major z-prefix pair array [na][ZN+1][rs] (nb valid
// columns; each element an 8-byte (P, f) pair, moved as one 64-bit word):
// boxes of CB columns x KB rows x 1 slice, zero fill outside.
int encode_zt_map(CUtensorMap *m, float2 *base, int nb, int ZN, int na, int rs, int CB, int KB)
{
    PFN_cuTensorMapEncodeTiled_v12000 fn = tensor_map_encoder();
    if (!fn) return set_status(CTLAB_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
    const cuuint64_t dims[3] = {(cuuint64_t)nb, (cuuint64_t)ZN + 1, (cuuint64_t)na};
    const cuuint64_t strides[2] = {(cuuint64_t)rs * 8, (cuuint64_t)(ZN + 1) * rs * 8};
    const cuuint32_t box[3] = {(cuuint32_t)CB, (cuuint32_t)KB, 1};
    const cuuint32_t es[3] = {1, 1, 1};
    const CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_UINT64, 3, base, dims, strides, box, es,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return set_status(CTLAB_ERR_CUDA, "cuTensorMapEncodeTiled failed for a z-prefix array");
    return CTLAB_OK;
}

} // namespace

int encode_tiled_map(CUtensorMap *m, CUtensorMapDataType dtype, int rank, void *base, const cuuint64_t *dims,
                     const cuuint64_t *strides, const cuuint32_t *box, CUtensorMapSwizzle swizzle, const char *what)
{
    PFN_cuTensorMapEncodeTiled_v12000 fn = tensor_map_encoder();
    if (!fn) return set_status(CTLAB_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
    const cuuint32_t es[5] = {1, 1, 1, 1, 1};
    const CUresult r = fn(m, dtype, (cuuint32_t)rank, base, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                          swizzle, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return set_status(CTLAB_ERR_CUDA, std::string("cuTensorMapEncodeTiled failed for ") + what);
    return CTLAB_OK;
}

void plan_free(ctlab_plan *p)
{
    if (!p) return;
    DeviceGuard g(p->device);
    void *bufs[] = {p->d_views, p->d_det, p->d_all_views, p->d_list, p->d_sat_y, p->d_sat_x, p->d_zt_y, p->d_zt_x, p->d_pv,
                    p->d_q, p->d_ticket, p->d_flags, p->d_agg, p->d_pref, p->d_err,
                    p->d_groups_all, p->d_groups_scratch, p->d_zrange};
    for (void *b : bufs)
        if (b) cudaFree(b);
    for (auto &e : p->ev)
        if (e) cudaEventDestroy(e);
    solver_work_free(p->sart);
    solver_work_free(p->fista);
    solver_work_free(p->cg);
    delete p;
}

int plan_volume_sat(ctlab_plan *p, const float *d_vol, const unsigned char *d_mask, cudaStream_t s)
{
    const HostGeometry &g = p->g;
    if (p->sat_mode == CTLAB_SAT_ZPREFIX) {
        if (p->need_y) {
            cudaError_t e = launch_zt(d_vol, d_mask, g.XN, g.YN, g.ZN, 0, p->d_zt_y, p->zt_rs_y, s);
            if (e != cudaSuccess) return cuda_status(e, "z-prefixes (y slices)");
            ++p->last_launches;
        }
        if (p->need_x) {
            cudaError_t e = launch_zt(d_vol, d_mask, g.XN, g.YN, g.ZN, 1, p->d_zt_x, p->zt_rs_x, s);
            if (e != cudaSuccess) return cuda_status(e, "z-prefixes (x slices)");
            ++p->last_launches;
        }
        return CTLAB_OK;
    }
    ScanState st{p->d_ticket, p->d_flags, p->d_agg, p->d_pref, p->d_err};
    if (p->need_y) {
        cudaError_t e = launch_volume_sat(d_vol, d_mask, g.XN, g.YN, g.ZN, 0, p->d_sat_y, p->zp, p->sat_mode,
                                          st, kVolChunk, s);
        if (e != cudaSuccess) return cuda_status(e, "volume SAT (y slices)");
        ++p->last_launches;
    }
    if (p->need_x) {
        cudaError_t e = launch_volume_sat(d_vol, d_mask, g.XN, g.YN, g.ZN, 1, p->d_sat_x, p->zp, p->sat_mode,
                                          st, kVolChunk, s);
        if (e != cudaSuccess) return cuda_status(e, "volume SAT (x slices)");
        ++p->last_launches;
    }
    return CTLAB_OK;
}

int plan_groups(ctlab_plan *p, const std::vector<int> &host_list, int *d_dst, int cap, GroupTab &out,
                cudaStream_t s)
{
    std::vector<int> ids(host_list.size());
    for (size_t i = 0; i < host_list.size(); ++i) ids[i] = host_list[i];
    ProjGroups pg = p->sat_mode == CTLAB_SAT_ZPREFIX ? proj_t_make_groups(p->g, ids, p->tst)
                                                     : proj_make_groups(p->g, ids, p->proj_cmax);
    if ((int)pg.table.size() > cap) return set_status(CTLAB_ERR_INTERNAL, "group table capacity exceeded");
    if (!pg.table.empty()) {
        CTLAB_CUDA_TRY(cudaMemcpyAsync(d_dst, pg.table.data(), sizeof(int) * pg.table.size(), cudaMemcpyHostToDevice, s));
        CTLAB_CUDA_TRY(cudaStreamSynchronize(s));
    }
    out.d = d_dst;
    out.ngroups = pg.ngroups;
    out.G = pg.G;
    return CTLAB_OK;
}

int plan_proj_list(ctlab_plan *p, const int *d_list, int n, const GroupTab &gt, float *d_prj, cudaStream_t s,
                   int epilogue, const float *meas, const float *row_sum, double *resid2)
{
    const HostGeometry &g = p->g;
    ProjArgs a;
    std::memset(&a, 0, sizeof a);
    a.sat_y = p->d_sat_y;
    a.sat_x = p->d_sat_x;
    a.zp = p->zp;
    a.XN = g.XN; a.YN = g.YN; a.ZN = g.ZN;
    a.dx = g.dx; a.dz = g.dz; a.z_lo = g.z_lo;
    a.views = p->d_views;
    a.view_list = d_list;
    a.n = n;
    a.det = p->d_det;
    a.DNU = g.DNU; a.DNV = g.DNV;
    a.out = d_prj;
    a.f32pair = p->sat_mode == CTLAB_SAT_F32PAIR;
    a.epilogue = epilogue;
    a.meas = meas;
    a.row_sum = row_sum;
    a.resid2 = resid2;
    a.cmax = p->proj_cmax;
    a.nbuf = p->proj_nbuf;
    a.err = p->d_err;
    a.groups = gt.d;
    a.ngroups = gt.ngroups;
    a.G = gt.G;
    if (p->sat_mode == CTLAB_SAT_ZPREFIX) {
        // view lists that group one view per CTA (ordered subsets of spread
        // views) run with the staging planned for single views
        const bool single = gt.G == 1 && p->tst1.ok && p->tst.G > 1;
        const ProjTStaging &st = single ? p->tst1 : p->tst;
        a.zt_y = p->d_zt_y;
        a.zt_x = p->d_zt_x;
        a.zt_rs_y = p->zt_rs_y;
        a.zt_rs_x = p->zt_rs_x;
        a.t_cb = st.CB;
        a.t_kb = st.KB;
        a.t_kr = st.KR;
        a.t_nstage = st.nstage;
        int nr, rb;
        proj_t_split(st, gt.G, nr, rb);
        a.t_rb = rb;
        a.t_nr = nr;
        a.t_zs = st.ZS;
        a.t_ep = st.EP;
        a.t_gtab = st.G;
        cudaError_t e = single ? launch_proj_t(a, st, p->tm1_y, p->tm1_x, s, &p->last_launches)
                               : launch_proj_t(a, st, p->tm_y, p->tm_x, s, &p->last_launches);
        if (e != cudaSuccess) return cuda_status(e, "DD3 projection kernel (z-prefix)");
        return CTLAB_OK;
    }
    cudaError_t e = launch_proj(a, s, &p->last_launches);
    if (e != cudaSuccess) return cuda_status(e, "DD3 projection kernel");
    return CTLAB_OK;
}

int plan_volume_sat_rows(ctlab_plan *p, const float *d_vol, const unsigned char *d_mask, int y0, int y1,
                         cudaStream_t s)
{
    const HostGeometry &g = p->g;
    if (p->sat_mode != CTLAB_SAT_ZPREFIX) return set_status(CTLAB_ERR_INTERNAL, "row-range SAT needs z-prefix mode");
    if (p->need_y) {
        cudaError_t e = launch_zt_rows(d_vol, d_mask, g.XN, g.YN, g.ZN, 0, p->d_zt_y, p->zt_rs_y, y0, y1, s);
        if (e != cudaSuccess) return cuda_status(e, "z-prefixes (y slices, row range)");
        ++p->last_launches;
    }
    if (p->need_x) {
        cudaError_t e = launch_zt_rows(d_vol, d_mask, g.XN, g.YN, g.ZN, 1, p->d_zt_x, p->zt_rs_x, y0, y1, s);
        if (e != cudaSuccess) return cuda_status(e, "z-prefixes (x slices, row range)");
        ++p->last_launches;
    }
    return CTLAB_OK;
}

int plan_proj_sat_range(ctlab_plan *p, const int *d_list, int first, int n, const float *d_prj, cudaStream_t s)
{
    const HostGeometry &g = p->g;
    if (p->sat_mode != CTLAB_SAT_ZPREFIX) return set_status(CTLAB_ERR_INTERNAL, "view-range prefixes need z-prefix mode");
    if (first < 0 || n < 0 || first + n > p->q_capacity)
        return set_status(CTLAB_ERR_INTERNAL, "projection prefix capacity exceeded");
    if (n == 0) return CTLAB_OK;
    ProjSatArgs a;
    a.prj = d_prj + (size_t)first * g.DNU * g.DNV;
    a.views = p->d_views;
    a.view_list = d_list + first;
    a.n = n;
    a.det = p->d_det;
    a.DNU = g.DNU; a.DNV = g.DNV;
    a.dx = g.dx;
    a.out = p->d_q;
    a.vp = p->vp;
    a.f32pair = 0;
    cudaError_t e = launch_pv(a, p->d_pv + (size_t)first * g.DNU * p->vp, p->vp, s);
    if (e != cudaSuccess) return cuda_status(e, "projection v-prefixes (view range)");
    ++p->last_launches;
    return CTLAB_OK;
}

int plan_proj_sat(ctlab_plan *p, const int *d_list, int n, const float *d_prj, cudaStream_t s)
{
    const HostGeometry &g = p->g;
    if (n > p->q_capacity) return set_status(CTLAB_ERR_INTERNAL, "projection SAT capacity exceeded");
    ProjSatArgs a;
    a.prj = d_prj;
    a.views = p->d_views;
    a.view_list = d_list;
    a.n = n;
    a.det = p->d_det;
    a.DNU = g.DNU; a.DNV = g.DNV;
    a.dx = g.dx;
    a.out = p->d_q;
    a.vp = p->vp;
    a.f32pair = p->sat_mode == CTLAB_SAT_F32PAIR;
    if (p->sat_mode == CTLAB_SAT_ZPREFIX) {
        cudaError_t e = launch_pv(a, p->d_pv, p->vp, s);
        if (e != cudaSuccess) return cuda_status(e, "projection v-prefixes");
        ++p->last_launches;
        return CTLAB_OK;
    }
    ScanState st{p->d_ticket, p->d_flags, p->d_agg, p->d_pref, p->d_err};
    cudaError_t e = launch_proj_sat(a, st, kPrjChunk, s);
    if (e != cudaSuccess) return cuda_status(e, "projection SAT");
    ++p->last_launches;
    return CTLAB_OK;
}

int plan_back_list(ctlab_plan *p, const int *d_list, int n, const unsigned char *d_mask, float *d_vol,
                   cudaStream_t s, int epilogue, const float *col_sum, float lambda, int clamp, float min_v,
                   float max_v)
{
    return plan_back_rows(p, d_list, n, d_mask, d_vol, s, epilogue, col_sum, lambda, clamp, min_v, max_v, 0, 0);
}

static BackArgs back_args(ctlab_plan *p, const int *d_list, int n, const unsigned char *d_mask, float *d_vol,
                          int epilogue, const float *col_sum, float lambda, int clamp, float min_v, float max_v,
                          int by_off, int by_count)
{
    const HostGeometry &g = p->g;
    BackArgs a;
    std::memset(&a, 0, sizeof a);
    a.q = p->d_q;
    a.vp = p->vp;
    a.views = p->d_views;
    a.view_list = d_list;
    a.n = n;
    a.det = p->d_det;
    a.DNU = g.DNU; a.DNV = g.DNV;
    a.dzb = g.dzb;
    a.XN = g.XN; a.YN = g.YN; a.ZN = g.ZN;
    a.dx = g.dx; a.dz = g.dz;
    a.x_c0 = g.cx - 0.5 * (g.XN - 1) * g.dx;
    a.y_c0 = g.cy - 0.5 * (g.YN - 1) * g.dx;
    a.z_lo = g.z_lo;
    a.mask = d_mask;
    a.out = d_vol;
    a.f32pair = p->sat_mode == CTLAB_SAT_F32PAIR;
    a.epilogue = epilogue;
    a.col_sum = col_sum;
    a.lambda = lambda;
    a.clamp = clamp;
    a.min_v = min_v;
    a.max_v = max_v;
    a.rmax = p->back_rmax;
    a.err = p->d_err;
    a.pv = p->d_pv;
    a.zrange = p->d_zrange;
    a.by_off = by_off;
    a.by_count = by_count;
    for (const DevView &V : g.views)
        if (V.zP != g.views[0].zP) a.zskip = 1; // a helical scan
    return a;
}

int plan_back_wave_rows(ctlab_plan *p, int n, int *rows)
{
    *rows = 0;
    if (p->sat_mode != CTLAB_SAT_ZPREFIX || n <= 0) return CTLAB_OK;
    const BackArgs a = back_args(p, p->d_all_views, n, nullptr, nullptr, BACK_PLAIN, nullptr, 1.f, 0, 0.f, 0.f, 0, 0);
    int resident = 0, per_row = 0;
    cudaError_t e = back_t_query(a, &resident, &per_row);
    if (e != cudaSuccess) return cuda_status(e, "backprojector occupancy");
    if (resident <= 0 || per_row <= 0) return CTLAB_OK;
    // the fewest brick rows whose CTAs fill whole waves: lcm(per_row, resident) / per_row
    long long a0 = per_row, b0 = resident;
    while (b0) {
        const long long t = a0 % b0;
        a0 = b0;
        b0 = t;
    }
    *rows = (int)(resident / a0);
    return CTLAB_OK;
}

int plan_back_rows(ctlab_plan *p, const int *d_list, int n, const unsigned char *d_mask, float *d_vol,
                   cudaStream_t s, int epilogue, const float *col_sum, float lambda, int clamp, float min_v,
                   float max_v, int by_off, int by_count)
{
    if ((by_off != 0 || by_count != 0) && (p->sat_mode != CTLAB_SAT_ZPREFIX || n == 0))
        return set_status(CTLAB_ERR_INTERNAL, "brick-row ranges need z-prefix mode and views");
    const HostGeometry &g = p->g;
    const BackArgs a = back_args(p, d_list, n, d_mask, d_vol, epilogue, col_sum, lambda, clamp, min_v, max_v, by_off,
                                 by_count);
    if (n == 0 && epilogue == BACK_PLAIN) {
        CTLAB_CUDA_TRY(cudaMemsetAsync(d_vol, 0, sizeof(float) * (size_t)g.XN * g.YN * g.ZN, s));
        return CTLAB_OK;
    }
    cudaError_t e = p->sat_mode == CTLAB_SAT_ZPREFIX ? launch_back_t(a, s, &p->last_launches)
                                                     : launch_back(a, s, &p->last_launches);
    if (e != cudaSuccess) return cuda_status(e, "DD3 backprojection kernel");
    return CTLAB_OK;
}

int plan_upload_list(ctlab_plan *p, const int *h_views, int n, cudaStream_t s)
{
    if (n < 0 || n > p->g.PN) return set_status(CTLAB_ERR_INVALID_ARG, "view count out of range");
    for (int i = 0; i < n; ++i)
        if (h_views[i] < 0 || h_views[i] >= p->g.PN)
            return set_status(CTLAB_ERR_INVALID_ARG, "view index out of range");
    if (n == 0) return CTLAB_OK;
    // The list buffer is re-used by the next call on the same stream only
    // after this call's kernels, because the copy is stream-ordered; the
    // host array is staged so the caller may free it at once.
    p->h_list.assign(h_views, h_views + n);
    CTLAB_CUDA_TRY(cudaMemcpyAsync(p->d_list, p->h_list.data(), sizeof(int) * (size_t)n, cudaMemcpyHostToDevice, s));
    CTLAB_CUDA_TRY(cudaStreamSynchronize(s));
    return CTLAB_OK;
}

int plan_check_device_error(ctlab_plan *p, cudaStream_t s)
{
    int err = 0;
    CTLAB_CUDA_TRY(cudaMemcpyAsync(&err, p->d_err, sizeof(int), cudaMemcpyDeviceToHost, s));
    CTLAB_CUDA_TRY(cudaStreamSynchronize(s));
    if (err != 0) {
        cudaMemsetAsync(p->d_err, 0, sizeof(int), s);
        cudaStreamSynchronize(s);
        return set_status(CTLAB_ERR_TIMEOUT, "a bounded wait in a SAT scan timed out; results are invalid");
    }
    return CTLAB_OK;
}

int plan_encode_zt(ctlab_plan *p, int orientation, const ProjTStaging &st, CUtensorMap *out)
{
    const HostGeometry &g = p->g;
    return orientation == 0 ? encode_zt_map(out, p->d_zt_y, g.XN, g.ZN, g.YN, p->zt_rs_y, st.CB, st.KB)
                            : encode_zt_map(out, p->d_zt_x, g.YN, g.ZN, g.XN, p->zt_rs_x, st.CB, st.KB);
}

void timing_mark(ctlab_plan *p, int which, cudaStream_t s)
{
    if (p->timing) cudaEventRecord(p->ev[which], s);
}

} // namespace ctlab

extern "C" {

int ctlab_plan_create(const ctlab_geometry *geom, int device, int sat_mode, ctlab_plan **out)
{
    if (!geom || !out) return set_status(CTLAB_ERR_INVALID_ARG, "null geometry or output pointer");
    *out = nullptr;
    if (sat_mode != CTLAB_SAT_FP64 && sat_mode != CTLAB_SAT_F32PAIR && sat_mode != CTLAB_SAT_ZPREFIX)
        return set_status(CTLAB_ERR_INVALID_ARG,
                          "sat_mode must be CTLAB_SAT_FP64, CTLAB_SAT_F32PAIR or CTLAB_SAT_ZPREFIX");
    ctlab_plan *p = new (std::nothrow) ctlab_plan();
    if (!p) return set_status(CTLAB_ERR_OOM, "host allocation failed");
    int rc = build_geometry(*geom, p->g);
    if (rc != CTLAB_OK) {
        delete p;
        return rc;
    }
    const HostGeometry &g = p->g;
    // the FP64 / float-pair projector stages whole SAT columns; the z-prefix
    // projector stages z ranges and splits detector rows over CTAs
    if (sat_mode != CTLAB_SAT_ZPREFIX && !proj_supported(g.ZN, g.DNV)) {
        delete p;
        return set_status(CTLAB_ERR_UNSUPPORTED, "ZN or DNV beyond the projector's shared-memory tiles");
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
        delete p;
        return set_status(CTLAB_ERR_INVALID_ARG, "no such CUDA device");
    }
    p->device = device;
    p->sat_mode = sat_mode;
    DeviceGuard dg(device);
    if (!dg.ok) {
        delete p;
        return set_status(CTLAB_ERR_CUDA, "cudaSetDevice failed");
    }
    for (const auto &v : g.views) (v.xdrv ? p->need_x : p->need_y) = true;
    const bool zpre = sat_mode == CTLAB_SAT_ZPREFIX;
    p->zp = round_up(g.ZN + 1, 2);
    p->vp = zpre ? back_t_pitch(g.DNV) : round_up(g.DNV + 1, 2);
    p->q_capacity = g.PN;
    if (zpre) {
        p->tst = proj_t_staging(g);
        p->tst1 = proj_t_staging(g, 1);
        if (!p->tst.ok) {
            delete p;
            return set_status(CTLAB_ERR_UNSUPPORTED, "DNV beyond the z-prefix projector's tiles");
        }
        p->zt_rs_y = round_up(g.XN, 4);
        p->zt_rs_x = round_up(g.YN, 4);
    } else {
        const ProjStaging st = proj_staging(g, p->zp, 8);
        p->proj_cmax = st.cmax;
        p->proj_nbuf = st.nbuf;
    }
    if (g.flat_uniform) p->back_rmax = zpre ? back_t_staging_rows(g) : back_staging_rows(g, p->vp);

    long long &bytes = p->bytes;
    cudaError_t e = cudaSuccess;
    auto chk = [&](cudaError_t r) {
        if (e == cudaSuccess) e = r;
    };
    chk(dmalloc(&p->d_views, g.views.size(), bytes));
    std::vector<double> det = det_table_host(g);
    chk(dmalloc(&p->d_det, det.size(), bytes));
    chk(dmalloc(&p->d_all_views, (size_t)g.PN, bytes));
    chk(dmalloc(&p->d_list, (size_t)g.PN, bytes));
    const size_t esz = 8; // double or float pair
    if (zpre) {
        if (p->need_y) chk(dmalloc(&p->d_zt_y, (size_t)g.YN * (g.ZN + 1) * p->zt_rs_y, bytes));
        if (p->need_x) chk(dmalloc(&p->d_zt_x, (size_t)g.XN * (g.ZN + 1) * p->zt_rs_x, bytes));
    } else {
        if (p->need_y) chk(dmalloc((char **)&p->d_sat_y, esz * (size_t)g.YN * (g.XN + 1) * p->zp, bytes));
        if (p->need_x) chk(dmalloc((char **)&p->d_sat_x, esz * (size_t)g.XN * (g.YN + 1) * p->zp, bytes));
    }
    if (zpre && back_t_supported(g.DNV) && g.flat_uniform)
        chk(dmalloc(&p->d_pv, (size_t)g.PN * g.DNU * p->vp, bytes));
    else if (!zpre && back_supported(g.DNV) && g.flat_uniform)
        chk(dmalloc((char **)&p->d_q, esz * (size_t)g.PN * (g.DNU + 1) * p->vp, bytes));
    else
        p->q_capacity = 0;
    if (zpre) chk(dmalloc(&p->d_zrange, (size_t)g.ZN / 32 + 2, bytes)); // z blocks of >= 32 voxels
    // lookback state sized for the largest scan
    size_t tiles = 0, state = 0;
    auto need = [&](int planes, int ns, int nk, int chunk) {
        const int c = scan_chunks(ns, nk, chunk, sat_mode);
        tiles = std::max(tiles, (size_t)planes * c);
        state = std::max(state, scan_state_doubles(planes, c, nk));
    };
    if (p->need_y && !zpre) need(g.YN, g.XN, g.ZN, kVolChunk);
    if (p->need_x && !zpre) need(g.XN, g.YN, g.ZN, kVolChunk);
    if (p->q_capacity && !zpre) need(g.PN, g.DNU, g.DNV, kPrjChunk);
    chk(dmalloc(&p->d_ticket, 1, bytes));
    chk(dmalloc(&p->d_flags, tiles, bytes));
    chk(dmalloc(&p->d_agg, state, bytes));
    chk(dmalloc(&p->d_pref, state, bytes));
    chk(dmalloc(&p->d_err, 1, bytes));
    // a view group table holds every run of views padded to whole groups:
    // at most (views per group) entries per view
    p->groups_cap = 16 * g.PN + 16;
    chk(dmalloc(&p->d_groups_all, (size_t)p->groups_cap, bytes));
    chk(dmalloc(&p->d_groups_scratch, (size_t)p->groups_cap, bytes));
    if (e != cudaSuccess) {
        plan_free(p);
        return cuda_status(e, "plan workspace allocation");
    }
    if (zpre && p->tst.CB > 0) {
        int rc2 = CTLAB_OK;
        if (p->need_y) rc2 = encode_zt_map(&p->tm_y, p->d_zt_y, g.XN, g.ZN, g.YN, p->zt_rs_y, p->tst.CB, p->tst.KB);
        if (rc2 == CTLAB_OK && p->need_x)
            rc2 = encode_zt_map(&p->tm_x, p->d_zt_x, g.YN, g.ZN, g.XN, p->zt_rs_x, p->tst.CB, p->tst.KB);
        if (rc2 == CTLAB_OK && p->tst1.ok && p->tst1.CB > 0) {
            if (p->need_y) rc2 = encode_zt_map(&p->tm1_y, p->d_zt_y, g.XN, g.ZN, g.YN, p->zt_rs_y, p->tst1.CB, p->tst1.KB);
            if (rc2 == CTLAB_OK && p->need_x)
                rc2 = encode_zt_map(&p->tm1_x, p->d_zt_x, g.YN, g.ZN, g.XN, p->zt_rs_x, p->tst1.CB, p->tst1.KB);
        } else {
            p->tst1.ok = false;
        }
        if (rc2 != CTLAB_OK) {
            plan_free(p);
            return rc2;
        }
    }
    std::vector<int> all(g.PN);
    for (int i = 0; i < g.PN; ++i) all[i] = i;
    chk(cudaMemcpy(p->d_views, g.views.data(), sizeof(DevView) * g.views.size(), cudaMemcpyHostToDevice));
    chk(cudaMemcpy(p->d_det, det.data(), sizeof(double) * det.size(), cudaMemcpyHostToDevice));
    chk(cudaMemcpy(p->d_all_views, all.data(), sizeof(int) * all.size(), cudaMemcpyHostToDevice));
    chk(cudaMemset(p->d_err, 0, sizeof(int)));
    for (auto &ev : p->ev) chk(cudaEventCreate(&ev));
    if (e != cudaSuccess) {
        plan_free(p);
        return cuda_status(e, "plan upload");
    }
    {
        GroupTab gt;
        int grc = plan_groups(p, all, p->d_groups_all, p->groups_cap, gt, 0);
        if (grc != CTLAB_OK) {
            plan_free(p);
            return grc;
        }
        p->groups_all_n = gt.ngroups;
        p->groups_all_G = gt.G;
    }
    *out = p;
    return ok();
}

int ctlab_plan_destroy(ctlab_plan *plan)
{
    plan_free(plan);
    return ok();
}

long long ctlab_plan_workspace_bytes(const ctlab_plan *plan) { return plan ? plan->bytes : 0; }

int ctlab_plan_set_timing(ctlab_plan *plan, int enable)
{
    if (!plan) return set_status(CTLAB_ERR_INVALID_ARG, "null plan");
    plan->timing = enable != 0;
    return ok();
}

int ctlab_plan_last_times(ctlab_plan *plan, float *sat_ms, float *gather_ms)
{
    if (!plan || !sat_ms || !gather_ms) return set_status(CTLAB_ERR_INVALID_ARG, "null argument");
    if (!plan->timing) return set_status(CTLAB_ERR_INVALID_ARG, "timing is not enabled on this plan");
    DeviceGuard dg(plan->device);
    CTLAB_CUDA_TRY(cudaEventSynchronize(plan->ev[2]));
    CTLAB_CUDA_TRY(cudaEventElapsedTime(sat_ms, plan->ev[0], plan->ev[1]));
    CTLAB_CUDA_TRY(cudaEventElapsedTime(gather_ms, plan->ev[1], plan->ev[2]));
    return ok();
}

int ctlab_plan_last_launches(const ctlab_plan *plan) { return plan ? plan->last_launches : -1; }

int ctlab_plan_sat_layout(const ctlab_plan *plan, int orientation, int *planes, int *rows, int *zp)
{
    if (!plan || !planes || !rows || !zp) return set_status(CTLAB_ERR_INVALID_ARG, "null argument");
    const HostGeometry &g = plan->g;
    if (plan->sat_mode == CTLAB_SAT_ZPREFIX) {
        if (orientation == 0 && plan->need_y) {
            *planes = g.YN; *rows = g.ZN + 1; *zp = plan->zt_rs_y;
        } else if (orientation == 1 && plan->need_x) {
            *planes = g.XN; *rows = g.ZN + 1; *zp = plan->zt_rs_x;
        } else {
            return set_status(CTLAB_ERR_INVALID_ARG, "orientation not used by this plan's views");
        }
        return ok();
    } else if (orientation == 0 && plan->need_y) {
        *planes = g.YN; *rows = g.XN + 1;
    } else if (orientation == 1 && plan->need_x) {
        *planes = g.XN; *rows = g.YN + 1;
    } else {
        return set_status(CTLAB_ERR_INVALID_ARG, "orientation not used by this plan's views");
    }
    *zp = plan->zp;
    return ok();
}

int ctlab_copy_volume_sat(ctlab_plan *plan, int orientation, void *d_out, void *stream)
{
    int planes, rows, zp;
    int rc = ctlab_plan_sat_layout(plan, orientation, &planes, &rows, &zp);
    if (rc != CTLAB_OK) return rc;
    if (!d_out) return set_status(CTLAB_ERR_INVALID_ARG, "null output");
    DeviceGuard dg(plan->device);
    const bool zpre = plan->sat_mode == CTLAB_SAT_ZPREFIX;
    const void *src = zpre ? (const void *)(orientation == 0 ? plan->d_zt_y : plan->d_zt_x)
                           : (orientation == 0 ? plan->d_sat_y : plan->d_sat_x);
    if (zpre) {
        // the prefixes Z = P + k f of the (P, f) pairs
        CTLAB_CUDA_TRY(launch_zt_unpack((const float2 *)src, (float *)d_out, planes, rows, zp, (cudaStream_t)stream));
    } else {
        CTLAB_CUDA_TRY(cudaMemcpyAsync(d_out, src, 8 * (size_t)planes * rows * zp, cudaMemcpyDeviceToDevice,
                                       (cudaStream_t)stream));
    }
    return ok();
}

int ctlab_volume_sat(ctlab_plan *plan, const float *d_vol, const unsigned char *d_mask, void *stream)
{
    if (!plan || !d_vol) return set_status(CTLAB_ERR_INVALID_ARG, "null plan or volume");
    DeviceGuard dg(plan->device);
    plan->last_launches = 0;
    int rc = plan_volume_sat(plan, d_vol, d_mask, (cudaStream_t)stream);
    return rc == CTLAB_OK ? ok() : rc;
}

int ctlab_proj(ctlab_plan *plan, const float *d_vol, const unsigned char *d_mask, float *d_prj, void *stream)
{
    if (!plan || !d_vol || !d_prj) return set_status(CTLAB_ERR_INVALID_ARG, "null plan, volume or projection");
    std::lock_guard<std::mutex> lk(plan->mu);
    DeviceGuard dg(plan->device);
    cudaStream_t s = (cudaStream_t)stream;
    plan->last_launches = 0;
    timing_mark(plan, 0, s);
    int rc = plan_volume_sat(plan, d_vol, d_mask, s);
    if (rc != CTLAB_OK) return rc;
    timing_mark(plan, 1, s);
    rc = plan_proj_list(plan, plan->d_all_views, plan->g.PN, plan_all_groups(plan), d_prj, s, PROJ_PLAIN, nullptr,
                        nullptr, nullptr);
    if (rc != CTLAB_OK) return rc;
    timing_mark(plan, 2, s);
    return ok();
}

int ctlab_proj_views(ctlab_plan *plan, const int *h_views, int n, const float *d_vol,
                     const unsigned char *d_mask, float *d_prj, void *stream)
{
    if (!plan || !h_views || !d_vol || !d_prj) return set_status(CTLAB_ERR_INVALID_ARG, "null argument");
    std::lock_guard<std::mutex> lk(plan->mu);
    DeviceGuard dg(plan->device);
    cudaStream_t s = (cudaStream_t)stream;
    plan->last_launches = 0;
    int rc = plan_upload_list(plan, h_views, n, s);
    if (rc != CTLAB_OK) return rc;
    if (n == 0) return ok();
    std::vector<int> positions(n);
    for (int i = 0; i < n; ++i) positions[i] = h_views[i];
    GroupTab gt;
    rc = plan_groups(plan, positions, plan->d_groups_scratch, plan->groups_cap, gt, s);
    if (rc != CTLAB_OK) return rc;
    timing_mark(plan, 0, s);
    rc = plan_volume_sat(plan, d_vol, d_mask, s);
    if (rc != CTLAB_OK) return rc;
    timing_mark(plan, 1, s);
    rc = plan_proj_list(plan, plan->d_list, n, gt, d_prj, s, PROJ_PLAIN, nullptr, nullptr, nullptr);
    if (rc != CTLAB_OK) return rc;
    timing_mark(plan, 2, s);
    return ok();
}

static int back_common(ctlab_plan *plan, const int *d_list, int n, const float *d_prj,
                       const unsigned char *d_mask, float *d_vol, cudaStream_t s)
{
    if (!plan->g.flat_uniform)
        return set_status(CTLAB_ERR_UNSUPPORTED,
                          "backprojection needs a flat detector with uniform u and v pitch");
    if (plan->q_capacity == 0)
        return set_status(CTLAB_ERR_UNSUPPORTED, "DNV beyond the backprojector's shared-memory tiles");
    timing_mark(plan, 0, s);
    int rc = CTLAB_OK;
    if (n > 0) rc = plan_proj_sat(plan, d_list, n, d_prj, s);
    if (rc != CTLAB_OK) return rc;
    timing_mark(plan, 1, s);
    rc = plan_back_list(plan, d_list, n, d_mask, d_vol, s, BACK_PLAIN, nullptr, 1.f, 0, 0.f, 0.f);
    if (rc != CTLAB_OK) return rc;
    timing_mark(plan, 2, s);
    return ok();
}

int ctlab_back(ctlab_plan *plan, const float *d_prj, const unsigned char *d_mask, float *d_vol, void *stream)
{
    if (!plan || !d_prj || !d_vol) return set_status(CTLAB_ERR_INVALID_ARG, "null plan, projection or volume");
    std::lock_guard<std::mutex> lk(plan->mu);
    DeviceGuard dg(plan->device);
    plan->last_launches = 0;
    return back_common(plan, plan->d_all_views, plan->g.PN, d_prj, d_mask, d_vol, (cudaStream_t)stream);
}

int ctlab_back_views(ctlab_plan *plan, const int *h_views, int n, const float *d_prj,
                     const unsigned char *d_mask, float *d_vol, void *stream)
{
    if (!plan || !h_views || !d_prj || !d_vol) return set_status(CTLAB_ERR_INVALID_ARG, "null argument");
    std::lock_guard<std::mutex> lk(plan->mu);
    DeviceGuard dg(plan->device);
    cudaStream_t s = (cudaStream_t)stream;
    plan->last_launches = 0;
    int rc = plan_upload_list(plan, h_views, n, s);
    if (rc != CTLAB_OK) return rc;
    return back_common(plan, plan->d_list, n, d_prj, d_mask, d_vol, s);
}

} // extern "C"

extern "C" int ctlab_debug_scan_stall(int device, unsigned spin_limit)
{
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev)
        return set_status(CTLAB_ERR_INVALID_ARG, "no such CUDA device");
    if (spin_limit < 1 || spin_limit > (1u << 24))
        return set_status(CTLAB_ERR_INVALID_ARG, "spin_limit must be in [1, 2^24]");
    DeviceGuard dg(device);
    const int rows = 2, nk = 8;
    float *vol = nullptr;
    double *out = nullptr, *agg = nullptr, *pref = nullptr;
    int *ticket = nullptr, *flags = nullptr, *err = nullptr;
    cudaError_t e = cudaMalloc(&vol, sizeof(float) * rows * nk);
    if (e == cudaSuccess) e = cudaMalloc(&out, sizeof(double) * (rows + 1) * (nk + 1));
    if (e == cudaSuccess) e = cudaMalloc(&agg, sizeof(double) * rows * nk);
    if (e == cudaSuccess) e = cudaMalloc(&pref, sizeof(double) * rows * nk);
    if (e == cudaSuccess) e = cudaMalloc(&ticket, sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&flags, sizeof(int) * rows);
    if (e == cudaSuccess) e = cudaMalloc(&err, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(vol, 0, sizeof(float) * rows * nk);
    if (e == cudaSuccess) e = cudaMemset(err, 0, sizeof(int));
    int h_err = 0;
    if (e == cudaSuccess) {
        ScanState st{ticket, flags, agg, pref, err};
        e = launch_scan_stall(vol, rows, nk, out, st, 1, spin_limit, 0);
    }
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(&h_err, err, sizeof(int), cudaMemcpyDeviceToHost);
    void *bufs[] = {vol, out, agg, pref, ticket, flags, err};
    for (void *b : bufs)
        if (b) cudaFree(b);
    if (e != cudaSuccess) return cuda_status(e, "scan stall diagnostic");
    if (h_err == CTLAB_ERR_TIMEOUT)
        return set_status(CTLAB_ERR_TIMEOUT, "bounded wait ran out as intended; the launch terminated");
    return set_status(CTLAB_ERR_INTERNAL, "the stalled scan did not report a timeout");
}
