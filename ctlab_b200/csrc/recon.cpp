// Device-resident OS-SART and FISTA-TV drivers.
//
// Everything stays on the device for the whole solve; per subset step the
// library launches: volume SAT(s) of x, the projector with the SART
// residual weighting fused into its epilogue, the projection SAT of the
// weighted residual, and the backprojector with the OS-SART voxel update
// fused into its epilogue.
#include <cmath>
#include <cstring>
#include <initializer_list>
#include <new>
#include <utility>
#include <vector>

#include "plan.h"

using namespace ctlab;

namespace {

// ||b - A x|| / ||b|| for the current x over the views of d_order (all PN).
int exact_residual(ctlab_plan *p, const float *d_x, const unsigned char *d_mask, const int *d_order,
                   const GroupTab &gt, const float *d_bsub, float *d_est, double *d_acc, cudaStream_t s, float *out)
{
    const HostGeometry &g = p->g;
    const long long nd = (long long)g.DNU * g.DNV;
    int rc = plan_volume_sat(p, d_x, d_mask, s);
    if (rc != CTLAB_OK) return rc;
    rc = plan_proj_list(p, d_order, g.PN, gt, d_est, s, PROJ_PLAIN, nullptr, nullptr, nullptr);
    if (rc != CTLAB_OK) return rc;
    CTLAB_CUDA_TRY(cudaMemsetAsync(d_acc, 0, 2 * sizeof(double), s));
    CTLAB_CUDA_TRY(launch_resid2(d_bsub, d_est, nd * g.PN, d_acc, s));
    double h[2];
    CTLAB_CUDA_TRY(cudaMemcpyAsync(h, d_acc, sizeof h, cudaMemcpyDeviceToHost, s));
    CTLAB_CUDA_TRY(cudaStreamSynchronize(s));
    *out = (float)(h[1] > 0 ? std::sqrt(h[0] / h[1]) : 0.0);
    return CTLAB_OK;
}

} // namespace

namespace ctlab {

// Solver state kept on a plan between calls of one solver (OS-SART,
// FISTA-TV or CG): the buffers, so that repeated solves allocate nothing, and
// for the SART-weighted solvers the view order, group tables and SART
// weights (rowSum = A 1, colSum_s = B_s 1) of the last subsets and mask used,
// identified by a hash of the subset count, the order and the mask bytes.
struct SolverWork {
    unsigned long long key = 0;
    bool weights = false; // rows / cols hold the weights of `key`
    std::vector<GroupTab> gtab;
    struct Buf {
        void *p = nullptr;
        size_t cap = 0;
    } order, groups, bsub, rows, cols, r, ones, acc, est, vol[5];
    ~SolverWork()
    {
        for (Buf *b : {&order, &groups, &bsub, &rows, &cols, &r, &ones, &acc, &est})
            if (b->p) cudaFree(b->p);
        for (Buf &b : vol)
            if (b.p) cudaFree(b.p);
    }
};

void solver_work_free(SolverWork *w) { delete w; }

} // namespace ctlab

namespace {

// Grows b to at least `bytes`; reports whether it was reallocated.
int reserve(SolverWork::Buf &b, size_t bytes, bool *moved)
{
    if (bytes <= b.cap && b.p) return CTLAB_OK;
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.cap = 0;
    cudaError_t e = cudaMalloc(&b.p, bytes ? bytes : 1);
    if (e != cudaSuccess) return cuda_status(e, "reconstruction workspace");
    b.cap = bytes;
    if (moved) *moved = true;
    return CTLAB_OK;
}

unsigned long long sart_key(const ctlab_plan *p, int os_num, const std::vector<int> &order,
                            const std::vector<unsigned char> &mask, bool has_mask)
{
    unsigned long long h = 1469598103934665603ull;
    auto add = [&](const void *q, size_t n) {
        const unsigned char *b = (const unsigned char *)q;
        for (size_t i = 0; i < n; ++i) {
            h ^= b[i];
            h *= 1099511628211ull;
        }
    };
    add(&os_num, sizeof os_num);
    // the projector staging the group tables were planned with (the autotuner may change it)
    for (const ProjTStaging *st : {&p->tst, &p->tst1}) {
        const int f[8] = {st->G, st->NR, st->RB, st->ZS, st->CB, st->KB, st->nstage, (int)st->ok};
        add(f, sizeof f);
    }
    add(order.data(), sizeof(int) * order.size());
    const unsigned char m = has_mask;
    add(&m, 1);
    add(mask.data(), mask.size());
    return h;
}

// The plan's workspace slot *slot, created on first use.
int solver_work(SolverWork **slot, SolverWork **out)
{
    if (!*slot) {
        *slot = new (std::nothrow) SolverWork();
        if (!*slot) return set_status(CTLAB_ERR_OOM, "host allocation failed");
    }
    *out = *slot;
    return CTLAB_OK;
}

// The in-plane mask's bytes (empty without a mask); synchronous.
int mask_bytes(const ctlab_plan *p, const unsigned char *d_mask, cudaStream_t s, std::vector<unsigned char> &out)
{
    out.clear();
    if (!d_mask) return CTLAB_OK;
    out.resize((size_t)p->g.XN * p->g.YN);
    CTLAB_CUDA_TRY(cudaMemcpyAsync(out.data(), d_mask, out.size(), cudaMemcpyDeviceToHost, s));
    CTLAB_CUDA_TRY(cudaStreamSynchronize(s));
    return CTLAB_OK;
}

} // namespace

extern "C" {

int ctlab_os_sart(ctlab_plan *plan, float *d_x, const float *d_meas, const unsigned char *d_mask, int os_num,
                  int iter_num, float lambda, const int *h_order, int clamp, float min_v, float max_v,
                  float *h_resid, void *stream)
{
    if (!plan || !d_x || !d_meas) return set_status(CTLAB_ERR_INVALID_ARG, "null plan, image or projection");
    if (os_num < 1 || iter_num < 0) return set_status(CTLAB_ERR_INVALID_ARG, "os_num must be >= 1, iter_num >= 0");
    const HostGeometry &g = plan->g;
    if (os_num > g.PN) return set_status(CTLAB_ERR_INVALID_ARG, "more subsets than views");
    if (!g.flat_uniform || plan->q_capacity == 0)
        return set_status(CTLAB_ERR_UNSUPPORTED, "OS-SART needs a flat detector with uniform u and v pitch");
    std::lock_guard<std::mutex> lk(plan->mu);
    DeviceGuard dg(plan->device);
    cudaStream_t s = (cudaStream_t)stream;
    plan->last_launches = 0;

    // subset-major view order and subset extents
    std::vector<int> order(g.PN), off(os_num + 1, 0);
    if (h_order) {
        std::vector<char> seen(g.PN, 0);
        for (int i = 0; i < g.PN; ++i) {
            const int v = h_order[i];
            if (v < 0 || v >= g.PN || seen[v])
                return set_status(CTLAB_ERR_INVALID_ARG, "h_order is not a permutation of 0..PN-1");
            seen[v] = 1;
            order[i] = v;
        }
        const int per = (g.PN + os_num - 1) / os_num;
        for (int k = 0; k <= os_num; ++k) off[k] = std::min(g.PN, k * per);
    } else {
        int pos = 0;
        for (int k = 0; k < os_num; ++k) {
            off[k] = pos;
            for (int v = k; v < g.PN; v += os_num) order[pos++] = v;
        }
        off[os_num] = pos;
    }
    int nmax = 0;
    for (int k = 0; k < os_num; ++k) nmax = std::max(nmax, off[k + 1] - off[k]);

    const long long nd = (long long)g.DNU * g.DNV;
    const long long nv = (long long)g.XN * g.YN * g.ZN;
    const int gcap = plan->groups_cap;
    // the mask's bytes identify the weights (a caller may rewrite a mask in place)
    std::vector<unsigned char> hmask;
    SolverWork *wp = nullptr;
    int rc = mask_bytes(plan, d_mask, s, hmask);
    if (rc == CTLAB_OK) rc = solver_work(&plan->sart, &wp);
    if (rc != CTLAB_OK) return rc;
    const unsigned long long key = sart_key(plan, os_num, order, hmask, d_mask != nullptr);
    SolverWork &W = *wp;
    bool moved = false;
    rc = reserve(W.order, sizeof(int) * g.PN, &moved);
    if (rc == CTLAB_OK) rc = reserve(W.groups, sizeof(int) * (size_t)gcap * (os_num + 1), &moved);
    if (rc == CTLAB_OK) rc = reserve(W.rows, sizeof(float) * nd * g.PN, &moved);
    if (rc == CTLAB_OK) rc = reserve(W.cols, sizeof(float) * nv * os_num, &moved);
    if (rc == CTLAB_OK) rc = reserve(W.bsub, sizeof(float) * nd * g.PN, nullptr);
    if (rc == CTLAB_OK) rc = reserve(W.r, sizeof(float) * nd * nmax, nullptr);
    if (rc == CTLAB_OK) rc = reserve(W.ones, sizeof(float) * std::max(nd * nmax, nv), nullptr);
    if (rc == CTLAB_OK) rc = reserve(W.acc, sizeof(double) * 2, nullptr);
    if (rc == CTLAB_OK && h_resid) rc = reserve(W.est, sizeof(float) * nd * g.PN, nullptr);
    if (rc != CTLAB_OK) {
        W.weights = false;
        return rc;
    }
    int *d_order = (int *)W.order.p, *d_groups = (int *)W.groups.p;
    float *d_bsub = (float *)W.bsub.p, *d_rows = (float *)W.rows.p, *d_cols = (float *)W.cols.p;
    float *d_r = (float *)W.r.p, *d_ones = (float *)W.ones.p, *d_est = (float *)W.est.p;
    double *d_acc = (double *)W.acc.p;
    std::vector<GroupTab> &gtab = W.gtab;
    if (moved || !W.weights || W.key != key) {
        W.weights = false;
        CTLAB_CUDA_TRY(cudaMemcpyAsync(d_order, order.data(), sizeof(int) * g.PN, cudaMemcpyHostToDevice, s));
        // projector view groups: the whole order, then each subset
        gtab.assign(os_num + 1, GroupTab());
        rc = plan_groups(plan, order, d_groups + (size_t)gcap * os_num, gcap, gtab[os_num], s);
        for (int k = 0; k < os_num && rc == CTLAB_OK; ++k) {
            std::vector<int> sub(order.begin() + off[k], order.begin() + off[k + 1]);
            rc = plan_groups(plan, sub, d_groups + (size_t)gcap * k, gcap, gtab[k], s);
        }
        if (rc != CTLAB_OK) return rc;
        // rowSum = A 1 (masked volume of ones), colSum_s = B_s 1
        CTLAB_CUDA_TRY(launch_fill(d_ones, 1.f, std::max(nd * nmax, nv), s));
        rc = plan_volume_sat(plan, d_ones, d_mask, s);
        if (rc == CTLAB_OK)
            rc = plan_proj_list(plan, d_order, g.PN, gtab[os_num], d_rows, s, PROJ_PLAIN, nullptr, nullptr, nullptr);
        for (int k = 0; k < os_num && rc == CTLAB_OK; ++k) {
            const int n = off[k + 1] - off[k];
            const int *lst = d_order + off[k];
            rc = plan_proj_sat(plan, lst, n, d_ones, s);
            if (rc == CTLAB_OK)
                rc = plan_back_list(plan, lst, n, d_mask, d_cols + nv * k, s, BACK_PLAIN, nullptr, 1.f, 0, 0.f, 0.f);
        }
        // a scan that timed out while the weights were built leaves them
        // invalid: they are kept only once the device error word is clear
        if (rc == CTLAB_OK) rc = plan_check_device_error(plan, s);
        if (rc != CTLAB_OK) return rc;
        W.key = key;
        W.weights = true;
    }
    CTLAB_CUDA_TRY(launch_gather_views(d_meas, d_order, g.PN, nd, d_bsub, s));

    for (int it = 0; it < iter_num; ++it) {
        for (int k = 0; k < os_num; ++k) {
            const int n = off[k + 1] - off[k];
            if (n == 0) continue;
            const int *lst = d_order + off[k];
            rc = plan_volume_sat(plan, d_x, d_mask, s);
            if (rc == CTLAB_OK)
                rc = plan_proj_list(plan, lst, n, gtab[k], d_r, s, PROJ_SART_RESIDUAL,
                                    d_bsub + nd * off[k], d_rows + nd * off[k], nullptr);
            if (rc == CTLAB_OK) rc = plan_proj_sat(plan, lst, n, d_r, s);
            if (rc == CTLAB_OK)
                rc = plan_back_list(plan, lst, n, d_mask, d_x, s, BACK_SART_UPDATE, d_cols + nv * k,
                                    lambda, clamp, min_v, max_v);
            if (rc != CTLAB_OK) return rc;
        }
        if (h_resid) {
            rc = exact_residual(plan, d_x, d_mask, d_order, gtab[os_num], d_bsub,
                                d_est, d_acc, s, h_resid + it);
            if (rc != CTLAB_OK) return rc;
        }
    }
    rc = plan_check_device_error(plan, s);
    return rc == CTLAB_OK ? ok() : rc;
}

int ctlab_fista_tv(ctlab_plan *plan, float *d_x, const float *d_meas, const unsigned char *d_mask, int iter_num,
                   float tv_lambda, float tv_eps, float min_v, float max_v, float *h_resid, void *stream)
{
    if (!plan || !d_x || !d_meas) return set_status(CTLAB_ERR_INVALID_ARG, "null plan, image or projection");
    if (iter_num < 0 || !(tv_eps >= 0)) return set_status(CTLAB_ERR_INVALID_ARG, "bad FISTA-TV arguments");
    const HostGeometry &g = plan->g;
    if (!g.flat_uniform || plan->q_capacity == 0)
        return set_status(CTLAB_ERR_UNSUPPORTED, "FISTA-TV needs a flat detector with uniform u and v pitch");
    std::lock_guard<std::mutex> lk(plan->mu);
    DeviceGuard dg(plan->device);
    cudaStream_t s = (cudaStream_t)stream;
    plan->last_launches = 0;
    const long long nd = (long long)g.DNU * g.DNV * g.PN;
    const long long nv = (long long)g.XN * g.YN * g.ZN;
    const int *all = plan->d_all_views;

    // workspace and SART weights (rowSum = A 1, colSum = B 1 over all views)
    // kept on the plan, the weights identified by the mask's bytes
    std::vector<unsigned char> hmask;
    SolverWork *wp = nullptr;
    int rc = mask_bytes(plan, d_mask, s, hmask);
    if (rc == CTLAB_OK) rc = solver_work(&plan->fista, &wp);
    if (rc != CTLAB_OK) return rc;
    SolverWork &W = *wp;
    const unsigned long long key = sart_key(plan, 1, std::vector<int>(), hmask, d_mask != nullptr);
    bool moved = false;
    rc = reserve(W.rows, sizeof(float) * nd, &moved);
    if (rc == CTLAB_OK) rc = reserve(W.cols, sizeof(float) * nv, &moved);
    if (rc == CTLAB_OK) rc = reserve(W.r, sizeof(float) * nd, nullptr);
    if (rc == CTLAB_OK) rc = reserve(W.ones, sizeof(float) * std::max(nd, nv), nullptr);
    for (int k = 0; k < 4 && rc == CTLAB_OK; ++k) rc = reserve(W.vol[k], sizeof(float) * nv, nullptr);
    if (rc == CTLAB_OK) rc = reserve(W.acc, sizeof(double) * 2, nullptr);
    if (rc == CTLAB_OK && h_resid) rc = reserve(W.est, sizeof(float) * nd, nullptr);
    if (rc != CTLAB_OK) {
        W.weights = false;
        return rc;
    }
    float *d_rows = (float *)W.rows.p, *d_cols = (float *)W.cols.p, *d_r = (float *)W.r.p;
    float *d_ones = (float *)W.ones.p, *d_g = (float *)W.vol[3].p, *d_est = (float *)W.est.p;
    double *d_acc = (double *)W.acc.p;

    if (moved || !W.weights || W.key != key) {
        W.weights = false;
        CTLAB_CUDA_TRY(launch_fill(d_ones, 1.f, std::max(nd, nv), s));
        rc = plan_volume_sat(plan, d_ones, d_mask, s);
        if (rc == CTLAB_OK)
            rc = plan_proj_list(plan, all, g.PN, plan_all_groups(plan), d_rows, s, PROJ_PLAIN, nullptr, nullptr,
                                nullptr);
        if (rc == CTLAB_OK) rc = plan_proj_sat(plan, all, g.PN, d_ones, s);
        if (rc == CTLAB_OK)
            rc = plan_back_list(plan, all, g.PN, d_mask, d_cols, s, BACK_PLAIN, nullptr, 1.f, 0, 0.f, 0.f);
        // kept only once the device error word is clear
        if (rc == CTLAB_OK) rc = plan_check_device_error(plan, s);
        if (rc != CTLAB_OK) return rc;
        W.key = key;
        W.weights = true;
    }
    float *xk = (float *)W.vol[0].p, *xp = (float *)W.vol[1].p, *y = (float *)W.vol[2].p;
    CTLAB_CUDA_TRY(cudaMemcpyAsync(y, d_x, sizeof(float) * nv, cudaMemcpyDeviceToDevice, s));
    CTLAB_CUDA_TRY(cudaMemcpyAsync(xp, d_x, sizeof(float) * nv, cudaMemcpyDeviceToDevice, s));

    float t = 1.f;
    for (int it = 0; it < iter_num; ++it) {
        rc = plan_volume_sat(plan, y, d_mask, s);
        if (rc == CTLAB_OK)
            rc = plan_proj_list(plan, all, g.PN, plan_all_groups(plan), d_r, s, PROJ_SART_RESIDUAL, d_meas, d_rows,
                                nullptr);
        if (rc == CTLAB_OK) rc = plan_proj_sat(plan, all, g.PN, d_r, s);
        // z = (y + B r / colSum) * mask, in place in y
        if (rc == CTLAB_OK)
            rc = plan_back_list(plan, all, g.PN, d_mask, y, s, BACK_SART_UPDATE, d_cols, 1.f, 0, 0.f, 0.f);
        if (rc != CTLAB_OK) return rc;
        CTLAB_CUDA_TRY(launch_tv_gradient(y, d_g, g.XN, g.YN, g.ZN, tv_eps, s));
        CTLAB_CUDA_TRY(launch_tv_step(xk, y, d_g, d_mask, tv_lambda, nv, g.ZN, s));
        const float tn = 0.5f * (1.f + std::sqrt(1.f + 4.f * t * t));
        CTLAB_CUDA_TRY(cudaMemcpyAsync(y, xk, sizeof(float) * nv, cudaMemcpyDeviceToDevice, s));
        CTLAB_CUDA_TRY(launch_fista_step(xp, y, t, tn, nv, min_v, max_v, s));
        plan->last_launches += 3;
        std::swap(xk, xp); // xp now holds x_k
        t = tn;
        if (h_resid) {
            rc = exact_residual(plan, xp, d_mask, all, plan_all_groups(plan), d_meas, d_est, d_acc, s, h_resid + it);
            if (rc != CTLAB_OK) return rc;
        }
    }
    CTLAB_CUDA_TRY(cudaMemcpyAsync(d_x, xp, sizeof(float) * nv, cudaMemcpyDeviceToDevice, s));
    rc = plan_check_device_error(plan, s);
    return rc == CTLAB_OK ? ok() : rc;
}

int ctlab_cg(ctlab_plan *plan, float *d_x, const float *d_meas, const unsigned char *d_mask, int iter_num, int method,
             float *h_resid, void *stream)
{
    if (!plan || !d_x || !d_meas) return set_status(CTLAB_ERR_INVALID_ARG, "null plan, image or projection");
    if (iter_num < 0) return set_status(CTLAB_ERR_INVALID_ARG, "iter_num must be >= 0");
    if (method < CTLAB_CG_FR || method > CTLAB_CG_DY) return set_status(CTLAB_ERR_INVALID_ARG, "unknown CG beta method");
    const HostGeometry &g = plan->g;
    if (!g.flat_uniform || plan->q_capacity == 0)
        return set_status(CTLAB_ERR_UNSUPPORTED, "CG needs a flat detector with uniform u and v pitch");
    std::lock_guard<std::mutex> lk(plan->mu);
    DeviceGuard dg(plan->device);
    cudaStream_t s = (cudaStream_t)stream;
    plan->last_launches = 0;
    const long long nd = (long long)g.DNU * g.DNV * g.PN;
    const long long nv = (long long)g.XN * g.YN * g.ZN;
    const int *all = plan->d_all_views;

    // workspace kept on the plan (repeated solves allocate nothing)
    SolverWork *wp = nullptr;
    int rc = solver_work(&plan->cg, &wp);
    if (rc != CTLAB_OK) return rc;
    SolverWork &W = *wp;
    rc = reserve(W.r, sizeof(float) * nd, nullptr);
    if (rc == CTLAB_OK) rc = reserve(W.est, sizeof(float) * nd, nullptr);
    for (int k = 0; k < 3 && rc == CTLAB_OK; ++k) rc = reserve(W.vol[k], sizeof(float) * nv, nullptr);
    if (rc == CTLAB_OK) rc = reserve(W.acc, sizeof(double) * 4, nullptr);
    if (rc != CTLAB_OK) return rc;
    float *r = (float *)W.r.p, *q = (float *)W.est.p, *gk = (float *)W.vol[0].p, *gn = (float *)W.vol[1].p,
          *dk = (float *)W.vol[2].p;
    double *acc = (double *)W.acc.p;

    // A v (masked volume) and A^T p (masked), over all views
    auto proj = [&](const float *vol, float *out) {
        int e = plan_volume_sat(plan, vol, d_mask, s);
        if (e == CTLAB_OK)
            e = plan_proj_list(plan, all, g.PN, plan_all_groups(plan), out, s, PROJ_PLAIN, nullptr, nullptr, nullptr);
        return e;
    };
    auto back = [&](const float *prj, float *out) {
        int e = plan_proj_sat(plan, all, g.PN, prj, s);
        if (e == CTLAB_OK) e = plan_back_list(plan, all, g.PN, d_mask, out, s, BACK_PLAIN, nullptr, 1.f, 0, 0.f, 0.f);
        return e;
    };
    // FP64 dot products of up to 4 (a, b, n) terms, read back
    struct Dot {
        const float *a, *b;
        long long n;
    };
    auto dots = [&](std::initializer_list<Dot> terms, double *out) {
        CTLAB_CUDA_TRY(cudaMemsetAsync(acc, 0, sizeof(double) * 4, s));
        int k = 0;
        for (const Dot &t : terms) CTLAB_CUDA_TRY(launch_dot(t.a, t.b, t.n, acc + k++, s));
        CTLAB_CUDA_TRY(cudaMemcpyAsync(out, acc, sizeof(double) * k, cudaMemcpyDeviceToHost, s));
        CTLAB_CUDA_TRY(cudaStreamSynchronize(s));
        return (int)CTLAB_OK;
    };

    double bb = 0.0;
    rc = dots({{d_meas, d_meas, nd}}, &bb);
    // r = A x - b, g = A^T r, d = -g
    if (rc == CTLAB_OK) rc = proj(d_x, r);
    if (rc == CTLAB_OK) rc = launch_axpby(r, -1.f, d_meas, 1.f, nd, s) == cudaSuccess ? CTLAB_OK : CTLAB_ERR_CUDA;
    if (rc == CTLAB_OK) rc = back(r, gk);
    if (rc == CTLAB_OK) rc = launch_axpby(dk, -1.f, gk, 0.f, nv, s) == cudaSuccess ? CTLAB_OK : CTLAB_ERR_CUDA;
    double gg = 0.0;
    if (rc == CTLAB_OK) rc = dots({{gk, gk, nv}}, &gg);
    if (rc != CTLAB_OK) return rc;
    for (int it = 0; it < iter_num; ++it) {
        // exact line search along d for 1/2 ||A x - b||^2
        rc = proj(dk, q);
        double h[4];
        if (rc == CTLAB_OK) rc = dots({{q, q, nd}, {gk, dk, nv}}, h);
        if (rc != CTLAB_OK) return rc;
        const double qq = h[0], gd = h[1];
        if (!(qq > 0.0) || !(gg > 0.0)) {
            for (int k = it; k < iter_num && h_resid; ++k) h_resid[k] = k > 0 ? h_resid[k - 1] : 0.f;
            break;
        }
        const float alpha = (float)(-gd / qq);
        CTLAB_CUDA_TRY(launch_axpby(d_x, alpha, dk, 1.f, nv, s));
        CTLAB_CUDA_TRY(launch_axpby(r, alpha, q, 1.f, nd, s));
        rc = back(r, gn);
        double gng = 0.0, gng_old = 0.0, dgn = 0.0, rr = 0.0;
        if (rc == CTLAB_OK) rc = dots({{gn, gn, nv}, {gn, gk, nv}, {dk, gn, nv}, {r, r, nd}}, h);
        if (rc != CTLAB_OK) return rc;
        rr = h[3];
        gng = h[0];
        gng_old = h[1];
        dgn = h[2];
        // beta of the chosen update (Fletcher-Reeves, Polak-Ribiere-Polyak,
        // Crowder-Wolfe / Hestenes-Stiefel, Dixon, Dai-Yuan)
        const double y_d = dgn - gd; // d^T (g_new - g)
        double beta = 0.0;
        switch (method) {
        case CTLAB_CG_FR: beta = gng / gg; break;
        case CTLAB_CG_PRP: beta = (gng - gng_old) / gg; break;
        case CTLAB_CG_CW: beta = y_d != 0.0 ? (gng - gng_old) / y_d : 0.0; break;
        case CTLAB_CG_DI: beta = gd != 0.0 ? -gng / gd : 0.0; break;
        case CTLAB_CG_DY: beta = y_d != 0.0 ? gng / y_d : 0.0; break;
        }
        if (!std::isfinite(beta)) beta = 0.0;
        CTLAB_CUDA_TRY(launch_axpby(dk, -1.f, gn, (float)beta, nv, s));
        std::swap(gk, gn);
        gg = gng;
        plan->last_launches += 4;
        if (h_resid) h_resid[it] = (float)(bb > 0 ? std::sqrt(rr / bb) : 0.0);
    }
    rc = plan_check_device_error(plan, s);
    return rc == CTLAB_OK ? ok() : rc;
}

} // extern "C"
