// Batched projection of many scans (sat mode ZPREFIX) and the projector
// autotuner.
//
// A batch holds plans of different geometries.  One run builds every
// case's slice-major z-prefixes, then projects all cases with ONE
// persistent launch: CTAs take (case, detector tile, view group, row block)
// work items from a queue sorted longest first, so cases of uneven size
// share the GPU instead of running one after another.  With use_graph the
// whole run is captured once into a CUDA graph and replayed.
//
// The autotuner times the projector of a plan under each candidate staging
// (views per CTA, stage depth), keeps the fastest and records it in a JSON
// cache keyed by the scan geometry, so later plans of the same scan skip
// the timing.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <mutex>
#include <new>
#include <sstream>
#include <string>
#include <vector>

#include "plan.h"

using namespace ctlab;

struct ctlab_batch {
    int device = 0;
    std::vector<ctlab_plan *> plans;
    ProjBatchCase *h_cases = nullptr; // pinned: graph replays copy from it
    ProjBatchCase *d_cases = nullptr;
    int4 *d_items = nullptr;
    int nitems = 0;
    int *d_counter = nullptr;
    size_t smem = 0;
    int grid = 0;
    cudaGraphExec_t gexec = nullptr;
    std::vector<const void *> graph_ptrs; // buffers the graph was captured with
    long long voxel_views = 0;
};

namespace {

// Fills a case's projector arguments for all views of its plan (the
// projection goes to d_prj); mirrors plan_proj_list's ZPREFIX branch.
void fill_case(ctlab_plan *p, float *d_prj, ProjBatchCase &c)
{
    const HostGeometry &g = p->g;
    ProjArgs &a = c.a;
    std::memset(&a, 0, sizeof a);
    a.zp = p->zp;
    a.XN = g.XN; a.YN = g.YN; a.ZN = g.ZN;
    a.dx = g.dx; a.dz = g.dz; a.z_lo = g.z_lo;
    a.views = p->d_views;
    a.view_list = p->d_all_views;
    a.n = g.PN;
    a.det = p->d_det;
    a.DNU = g.DNU; a.DNV = g.DNV;
    a.out = d_prj;
    a.epilogue = PROJ_PLAIN;
    a.err = p->d_err;
    a.groups = p->d_groups_all;
    a.ngroups = p->groups_all_n;
    a.G = p->groups_all_G;
    const ProjTStaging &st = p->tst;
    a.zt_y = p->d_zt_y; a.zt_x = p->d_zt_x;
    a.zt_rs_y = p->zt_rs_y; a.zt_rs_x = p->zt_rs_x;
    a.t_cb = st.CB; a.t_kb = st.KB; a.t_kr = st.KR;
    a.t_nstage = st.nstage; a.t_ep = st.EP; a.t_gtab = st.G;
    int nr = st.NR, rb = st.RB;
    while (a.G * rb * 2 <= 16 && nr >= 16) {
        nr /= 2;
        rb *= 2;
    }
    a.t_rb = rb; a.t_nr = nr; a.t_zs = st.ZS;
    c.tm_y = p->tm_y;
    c.tm_x = p->tm_x;
}

unsigned long long scan_key(const HostGeometry &g)
{
    unsigned long long h = 1469598103934665603ull;
    auto add = [&](const void *q, size_t n) {
        const unsigned char *b = (const unsigned char *)q;
        for (size_t i = 0; i < n; ++i) {
            h ^= b[i];
            h *= 1099511628211ull;
        }
    };
    const int ints[6] = {g.DNU, g.DNV, g.PN, g.XN, g.YN, g.ZN};
    add(ints, sizeof ints);
    const double dbl[5] = {g.dx, g.dz, g.x_lo, g.y_lo, g.z_lo};
    add(dbl, sizeof dbl);
    add(g.bx.data(), sizeof(double) * g.bx.size());
    add(g.by.data(), sizeof(double) * g.by.size());
    add(g.bz.data(), sizeof(double) * g.bz.size());
    for (const DevView &v : g.views) add(&v, sizeof v);
    return h;
}

std::mutex g_cache_mu;

bool cache_lookup(const char *path, unsigned long long key, int &gcap, int &nstage)
{
    if (!path) return false;
    std::lock_guard<std::mutex> lk(g_cache_mu);
    std::ifstream f(path);
    std::string line;
    char want[32];
    std::snprintf(want, sizeof want, "\"%016llx\"", key);
    while (std::getline(f, line)) {
        if (line.find(want) == std::string::npos) continue;
        int a = 0, b = 0;
        const size_t pa = line.find("\"gcap\":"), pb = line.find("\"nstage\":");
        if (pa == std::string::npos || pb == std::string::npos) continue;
        if (std::sscanf(line.c_str() + pa + 7, "%d", &a) == 1 && std::sscanf(line.c_str() + pb + 9, "%d", &b) == 1) {
            gcap = a;
            nstage = b;
            return true;
        }
    }
    return false;
}

void cache_store(const char *path, unsigned long long key, int gcap, int nstage, float ms)
{
    if (!path) return;
    std::lock_guard<std::mutex> lk(g_cache_mu);
    std::ofstream f(path, std::ios::app);
    char buf[160];
    std::snprintf(buf, sizeof buf, "{\"scan\": \"%016llx\", \"gcap\": %d, \"nstage\": %d, \"ms\": %.4f}\n", key, gcap,
                  nstage, ms);
    f << buf;
}

// Installs a projector staging on a plan: the staging, TMA maps of its box,
// and the view grouping of the full view list.
int apply_staging(ctlab_plan *p, const ProjTStaging &st)
{
    const HostGeometry &g = p->g;
    if (!st.ok) return set_status(CTLAB_ERR_INTERNAL, "invalid projector staging");
    p->tst = st;
    if (st.CB > 0) {
        int rc = CTLAB_OK;
        if (p->need_y) rc = plan_encode_zt(p, 0, st, &p->tm_y);
        if (rc == CTLAB_OK && p->need_x) rc = plan_encode_zt(p, 1, st, &p->tm_x);
        if (rc != CTLAB_OK) return rc;
    }
    std::vector<int> all(g.PN);
    for (int i = 0; i < g.PN; ++i) all[i] = i;
    GroupTab gt;
    int rc = plan_groups(p, all, p->d_groups_all, p->groups_cap, gt, 0);
    if (rc != CTLAB_OK) return rc;
    p->groups_all_n = gt.ngroups;
    p->groups_all_G = gt.G;
    return CTLAB_OK;
}

} // namespace

extern "C" {

int ctlab_plan_autotune(ctlab_plan *plan, const float *d_vol, float *d_prj, const char *cache_path, float *best_ms)
{
    if (!plan || !d_vol || !d_prj) return set_status(CTLAB_ERR_INVALID_ARG, "null plan, volume or projection");
    if (plan->sat_mode != CTLAB_SAT_ZPREFIX)
        return set_status(CTLAB_ERR_UNSUPPORTED, "the autotuner tunes the z-prefix projector (sat mode ZPREFIX)");
    DeviceGuard dg(plan->device);
    const HostGeometry &g = plan->g;
    const unsigned long long key = scan_key(g);
    int gcap = 0, ns = 0;
    if (cache_lookup(cache_path, key, gcap, ns)) {
        ProjTStaging st = proj_t_staging(g, gcap, ns);
        if (st.ok) {
            int rc = apply_staging(plan, st);
            if (rc != CTLAB_OK) return rc;
            if (best_ms) *best_ms = -1.f;
            return set_status(CTLAB_OK, "");
        }
    }
    cudaEvent_t e0, e1;
    CTLAB_CUDA_TRY(cudaEventCreate(&e0));
    CTLAB_CUDA_TRY(cudaEventCreate(&e1));
    float best = 1e30f;
    ProjTStaging best_st = plan->tst;
    int best_g = 16, best_n = 0;
    std::vector<std::pair<int, int>> seen;
    for (int gc : {16, 8, 4, 2}) {
        for (int n : {2, 3, 4}) {
            ProjTStaging st = proj_t_staging(g, gc, n);
            if (!st.ok || st.nstage != n) continue;
            const std::pair<int, int> sig{st.G * 10 + st.nstage, st.ZS * 1000 + st.CB};
            if (std::find(seen.begin(), seen.end(), sig) != seen.end()) continue;
            seen.push_back(sig);
            int rc = apply_staging(plan, st);
            if (rc == CTLAB_OK) rc = ctlab_proj(plan, d_vol, nullptr, d_prj, nullptr); // warm-up
            if (rc != CTLAB_OK) {
                cudaEventDestroy(e0);
                cudaEventDestroy(e1);
                return rc;
            }
            cudaEventRecord(e0, 0);
            rc = ctlab_proj(plan, d_vol, nullptr, d_prj, nullptr);
            cudaEventRecord(e1, 0);
            float ms = 0.f;
            if (rc == CTLAB_OK && cudaEventSynchronize(e1) == cudaSuccess && cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess &&
                ms < best) {
                best = ms;
                best_st = st;
                best_g = gc;
                best_n = n;
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    int rc = apply_staging(plan, best_st);
    if (rc != CTLAB_OK) return rc;
    cache_store(cache_path, key, best_g, best_n, best);
    if (best_ms) *best_ms = best;
    return set_status(CTLAB_OK, "");
}

int ctlab_batch_create(ctlab_plan *const *plans, int n, ctlab_batch **out)
{
    if (!plans || n < 1 || !out) return set_status(CTLAB_ERR_INVALID_ARG, "need at least one plan");
    *out = nullptr;
    const int dev = plans[0]->device;
    for (int i = 0; i < n; ++i) {
        if (!plans[i] || plans[i]->sat_mode != CTLAB_SAT_ZPREFIX)
            return set_status(CTLAB_ERR_UNSUPPORTED, "batched projection needs z-prefix plans (sat mode ZPREFIX)");
        if (plans[i]->device != dev) return set_status(CTLAB_ERR_INVALID_ARG, "the plans of a batch share one device");
    }
    ctlab_batch *b = new (std::nothrow) ctlab_batch();
    if (!b) return set_status(CTLAB_ERR_OOM, "host allocation failed");
    b->device = dev;
    b->plans.assign(plans, plans + n);
    DeviceGuard dg(dev);
    // work items, longest first: per item the slices of the driving axis times
    // the views of its group times the detector rows of its block
    struct Item {
        int4 w;
        double cost;
    };
    std::vector<Item> items;
    for (int i = 0; i < n; ++i) {
        ctlab_plan *p = plans[i];
        ProjBatchCase c;
        fill_case(p, nullptr, c);
        b->smem = std::max(b->smem, proj_t_smem_bytes(p->tst));
        const int tiles = (p->g.DNU + 31) / 32;
        const int rows = c.a.t_nr * c.a.t_rb;
        for (int gy = 0; gy < c.a.ngroups; ++gy)
            for (int bx = 0; bx < tiles; ++bx)
                for (int bz = 0; bz < c.a.t_zs; ++bz) {
                    const int na = std::max(p->g.XN, p->g.YN);
                    items.push_back({make_int4(i, bx, gy, bz), (double)na * c.a.G * std::min(rows, p->g.DNV - bz * rows)});
                }
        b->voxel_views += (long long)p->g.XN * p->g.YN * p->g.ZN * p->g.PN;
    }
    std::stable_sort(items.begin(), items.end(), [](const Item &x, const Item &y) { return x.cost > y.cost; });
    std::vector<int4> w(items.size());
    for (size_t k = 0; k < items.size(); ++k) w[k] = items[k].w;
    b->nitems = (int)w.size();
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    b->grid = sms;
    cudaError_t e = cudaMalloc(&b->d_cases, sizeof(ProjBatchCase) * n);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_items, sizeof(int4) * w.size());
    if (e == cudaSuccess) e = cudaMalloc(&b->d_counter, sizeof(int));
    if (e == cudaSuccess) e = cudaMallocHost(&b->h_cases, sizeof(ProjBatchCase) * n);
    if (e == cudaSuccess) e = cudaMemcpy(b->d_items, w.data(), sizeof(int4) * w.size(), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        ctlab_batch_destroy(b);
        return cuda_status(e, "batch buffers");
    }
    *out = b;
    return set_status(CTLAB_OK, "");
}

int ctlab_batch_destroy(ctlab_batch *b)
{
    if (!b) return set_status(CTLAB_OK, "");
    DeviceGuard dg(b->device);
    if (b->gexec) cudaGraphExecDestroy(b->gexec);
    if (b->d_cases) cudaFree(b->d_cases);
    if (b->d_items) cudaFree(b->d_items);
    if (b->d_counter) cudaFree(b->d_counter);
    if (b->h_cases) cudaFreeHost(b->h_cases);
    delete b;
    return set_status(CTLAB_OK, "");
}

long long ctlab_batch_voxel_views(const ctlab_batch *b) { return b ? b->voxel_views : 0; }

// The launches of one batched run, in stream order.
static int batch_enqueue(ctlab_batch *b, const float *const *d_vols, const unsigned char *const *d_masks,
                         cudaStream_t s)
{
    const int n = (int)b->plans.size();
    for (int i = 0; i < n; ++i) {
        ctlab_plan *p = b->plans[i];
        int rc = plan_volume_sat(p, d_vols[i], d_masks ? d_masks[i] : nullptr, s);
        if (rc != CTLAB_OK) return rc;
    }
    CTLAB_CUDA_TRY(cudaMemcpyAsync(b->d_cases, b->h_cases, sizeof(ProjBatchCase) * n, cudaMemcpyHostToDevice, s));
    CTLAB_CUDA_TRY(cudaMemsetAsync(b->d_counter, 0, sizeof(int), s));
    CTLAB_CUDA_TRY(launch_proj_t_batch(b->d_cases, b->d_items, b->nitems, b->d_counter, b->smem, b->grid, s));
    return CTLAB_OK;
}

int ctlab_batch_proj(ctlab_batch *b, const float *const *d_vols, const unsigned char *const *d_masks,
                     float *const *d_prjs, int use_graph, void *stream)
{
    if (!b || !d_vols || !d_prjs) return set_status(CTLAB_ERR_INVALID_ARG, "null batch or buffer list");
    const int n = (int)b->plans.size();
    for (int i = 0; i < n; ++i)
        if (!d_vols[i] || !d_prjs[i]) return set_status(CTLAB_ERR_INVALID_ARG, "null volume or projection buffer");
    DeviceGuard dg(b->device);
    cudaStream_t s = (cudaStream_t)stream;
    // the pinned case table is read by the copy at replay time: wait for the
    // previous run before rewriting it
    CTLAB_CUDA_TRY(cudaStreamSynchronize(s));
    for (int i = 0; i < n; ++i) fill_case(b->plans[i], d_prjs[i], b->h_cases[i]);
    if (!use_graph) {
        int rc = batch_enqueue(b, d_vols, d_masks, s);
        return rc == CTLAB_OK ? set_status(CTLAB_OK, "") : rc;
    }
    std::vector<const void *> ptrs;
    for (int i = 0; i < n; ++i) {
        ptrs.push_back(d_vols[i]);
        ptrs.push_back(d_masks ? d_masks[i] : nullptr);
    }
    if (!b->gexec || ptrs != b->graph_ptrs) {
        if (b->gexec) {
            cudaGraphExecDestroy(b->gexec);
            b->gexec = nullptr;
        }
        if (s == 0) return set_status(CTLAB_ERR_INVALID_ARG, "graph capture needs a non-default stream");
        cudaGraph_t graph;
        CTLAB_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        const int rc = batch_enqueue(b, d_vols, d_masks, s);
        cudaError_t e = cudaStreamEndCapture(s, &graph);
        if (rc != CTLAB_OK) return rc;
        if (e != cudaSuccess) return cuda_status(e, "batch graph capture");
        e = cudaGraphInstantiate(&b->gexec, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) return cuda_status(e, "batch graph instantiation");
        b->graph_ptrs = ptrs;
    }
    CTLAB_CUDA_TRY(cudaGraphLaunch(b->gexec, s));
    return set_status(CTLAB_OK, "");
}

} // extern "C"
