// Batched projection of many scans (sat mode ZPREFIX) and the projector
// autotuner.
//
// A batch holds plans of different geometries.  One run builds every
// case's slice-major z-prefixes, then projects all cases with persistent
// launches: CTAs take (case, detector tile, view group, row block) work
// items from a queue sorted longest first, so cases of uneven size share the
// GPU instead of running one after another.  Cases whose projector has the
// same rows per consumer warp share one launch (its kernel is compiled for
// that row count; the cases' arguments and TMA maps travel as its kernel
// parameters); launches of different row counts run on forked streams, each
// filling the SMs the others free.  With use_graph the whole run is captured
// once into a CUDA graph and replayed.
//
// The autotuner times the projector of a plan under each candidate staging
// (views per CTA, detector-row split, stage depth), keeps the fastest and
// records it in a JSON cache keyed by the scan geometry, so later plans of
// the same scan skip the timing.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <memory>
#include <mutex>
#include <new>
#include <sstream>
#include <string>
#include <vector>

#include "plan.h"

using namespace ctlab;

// Cases whose launches share the rows per consumer warp run in one
// persistent launch (up to kProjBatchMaxCases cases each, their arguments in
// the kernel parameters); launches of different row counts run side by side.
struct BatchLaunch {
    int nr = 0;             // detector rows per consumer warp
    int threads = 0;        // CTA size: 512, or 256 for stagings of 8-warp CTAs (two per SM)
    std::vector<int> cases; // plan indices; work items name positions here
    int first = 0;          // first work item (d_items)
    int count = 0;          // work items
    size_t smem = 0;
    double cost = 0.0;
    std::unique_ptr<ProjBatchParams> params;
};

struct ctlab_batch {
    int device = 0;
    std::vector<ctlab_plan *> plans;
    int4 *d_items = nullptr;
    int nitems = 0;
    int *d_counter = nullptr; // one queue counter per launch
    std::vector<BatchLaunch> launches;
    std::vector<cudaStream_t> side; // launches after the first
    cudaEvent_t fork = nullptr;
    std::vector<cudaEvent_t> join;
    int grid = 0;
    cudaGraphExec_t gexec = nullptr;
    std::vector<const void *> graph_ptrs; // buffers the graph was captured with
    long long voxel_views = 0;
    std::vector<std::vector<int>> staging; // each plan's projector staging when the items were made
};

namespace {

// The fields of a plan's projector staging and view grouping that the work
// items and launch row counts were derived from.
std::vector<int> staging_sig(const ctlab_plan *p)
{
    const ProjTStaging &st = p->tst;
    return {st.G, st.NR, st.RB, st.ZS, st.CB, st.KB, st.KR, st.nstage, p->groups_all_n, p->groups_all_G};
}

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
    int nr, rb;
    proj_t_split(st, a.G, nr, rb);
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

bool cache_lookup(const char *path, unsigned long long key, int &gcap, int &nstage, int &zs, int &warps)
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
            zs = 0;
            const size_t pz = line.find("\"zs\":");
            if (pz != std::string::npos && std::sscanf(line.c_str() + pz + 5, "%d", &a) == 1) zs = a;
            warps = 15;
            const size_t pw = line.find("\"warps\":");
            if (pw != std::string::npos && std::sscanf(line.c_str() + pw + 8, "%d", &a) == 1) warps = a;
            return true;
        }
    }
    return false;
}

void cache_store(const char *path, unsigned long long key, int gcap, int nstage, int zs, int warps, float ms)
{
    if (!path) return;
    std::lock_guard<std::mutex> lk(g_cache_mu);
    std::ofstream f(path, std::ios::app);
    char buf[224];
    std::snprintf(buf, sizeof buf,
                  "{\"scan\": \"%016llx\", \"gcap\": %d, \"nstage\": %d, \"zs\": %d, \"warps\": %d, \"ms\": %.4f}\n",
                  key, gcap, nstage, zs, warps, ms);
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
    int gcap = 0, ns = 0, zs = 0, ws = 15;
    if (cache_lookup(cache_path, key, gcap, ns, zs, ws)) {
        ProjTStaging st = proj_t_staging(g, gcap, ns, zs, ws);
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
    int best_g = 16, best_n = 0, best_z = 0, best_w = 15;
    std::vector<std::vector<int>> seen;
    // candidates: CTAs of 16 warps (one per SM) or of 8 warps (two per SM),
    // views per CTA capped at 16 / 8 / 4 / 2, detector rows split over 1 / 2 /
    // 4 CTAs (the deepest stage ring that fits); each distinct staging timed once
    for (int w : {15, 7})
    for (int gc : {16, 8, 4, 2})
        for (int z : {1, 2, 4}) {
            ProjTStaging st = proj_t_staging(g, gc, 0, z, w);
            const int n = st.nstage;
            if (!st.ok) continue;
            const std::vector<int> sig{st.G, st.NR, st.RB, st.ZS, st.CB, st.KB, st.nstage, st.W};
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
                best_z = z;
                best_w = w;
            }
        }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    int rc = apply_staging(plan, best_st);
    if (rc != CTLAB_OK) return rc;
    cache_store(cache_path, key, best_g, best_n, best_z, best_w, best);
    if (best_ms) *best_ms = best;
    return set_status(CTLAB_OK, "");
}

int ctlab_plan_proj_tiles(const ctlab_plan *plan, int *tiles)
{
    if (!plan || !tiles) return set_status(CTLAB_ERR_INVALID_ARG, "null plan or output");
    if (plan->sat_mode != CTLAB_SAT_ZPREFIX)
        return set_status(CTLAB_ERR_UNSUPPORTED, "projector tiles are defined for sat mode ZPREFIX");
    const ProjTStaging &st = plan->tst;
    tiles[0] = st.G;
    tiles[1] = st.NR;
    tiles[2] = st.RB;
    tiles[3] = st.ZS;
    tiles[4] = st.CB;
    tiles[5] = st.KB;
    tiles[6] = st.nstage;
    tiles[7] = (plan->g.DNU + 31) / 32 * plan->groups_all_n * st.ZS;
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
    // work items: per item the slices of the driving axis times the views of
    // its group times the detector rows of its block.  Cases go to launches
    // by rows per warp and CTA size (in chunks of kProjBatchMaxCases): a case
    // whose staging plans 8-warp CTAs runs two per SM, as its own launches
    // do, not one 16-warp CTA per SM with half the warps idle; items longest first
    // within a launch, the launch with the most work first.
    std::vector<std::vector<int4>> case_items(n);
    std::vector<std::vector<double>> case_cost(n);
    for (int i = 0; i < n; ++i) {
        ctlab_plan *p = plans[i];
        ProjBatchCase c;
        fill_case(p, nullptr, c);
        const int tiles = (p->g.DNU + 31) / 32;
        const int rows = c.a.t_nr * c.a.t_rb;
        const int na = std::max(p->g.XN, p->g.YN);
        for (int gy = 0; gy < c.a.ngroups; ++gy)
            for (int bx = 0; bx < tiles; ++bx)
                for (int bz = 0; bz < c.a.t_zs; ++bz) {
                    case_items[i].push_back(make_int4(0, bx, gy, bz));
                    case_cost[i].push_back((double)na * c.a.G * std::min(rows, p->g.DNV - bz * rows));
                }
        const int threads = p->tst.W <= 7 ? 256 : 512;
        BatchLaunch *L = nullptr;
        for (BatchLaunch &l : b->launches)
            if (l.nr == c.a.t_nr && l.threads == threads && (int)l.cases.size() < kProjBatchMaxCases) L = &l;
        if (!L) {
            b->launches.emplace_back();
            L = &b->launches.back();
            L->nr = c.a.t_nr;
            L->threads = threads;
        }
        L->cases.push_back(i);
        L->smem = std::max(L->smem, proj_t_smem_bytes(p->tst));
        for (double x : case_cost[i]) L->cost += x;
        b->voxel_views += (long long)p->g.XN * p->g.YN * p->g.ZN * p->g.PN;
        b->staging.push_back(staging_sig(p));
    }
    std::stable_sort(b->launches.begin(), b->launches.end(),
                     [](const BatchLaunch &x, const BatchLaunch &y) { return x.cost > y.cost; });
    std::vector<int4> w;
    for (BatchLaunch &l : b->launches) {
        std::vector<std::pair<double, int4>> mine;
        for (int k = 0; k < (int)l.cases.size(); ++k) {
            const int i = l.cases[k];
            for (size_t q = 0; q < case_items[i].size(); ++q) {
                int4 it = case_items[i][q];
                it.x = k;
                mine.push_back({case_cost[i][q], it});
            }
        }
        std::stable_sort(mine.begin(), mine.end(),
                         [](const std::pair<double, int4> &x, const std::pair<double, int4> &y) { return x.first > y.first; });
        l.first = (int)w.size();
        l.count = (int)mine.size();
        for (const auto &m : mine) w.push_back(m.second);
        l.params.reset(new (std::nothrow) ProjBatchParams());
        if (!l.params) {
            ctlab_batch_destroy(b);
            return set_status(CTLAB_ERR_OOM, "host allocation failed");
        }
    }
    b->nitems = (int)w.size();
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    b->grid = sms;
    const int nl = (int)b->launches.size();
    cudaError_t e = cudaMalloc(&b->d_items, sizeof(int4) * w.size());
    if (e == cudaSuccess) e = cudaMalloc(&b->d_counter, sizeof(int) * nl);
    if (e == cudaSuccess) e = cudaMemcpy(b->d_items, w.data(), sizeof(int4) * w.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && nl > 1) e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
    for (int k = 1; k < nl && e == cudaSuccess; ++k) {
        cudaStream_t st = nullptr;
        cudaEvent_t ev = nullptr;
        e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
        if (e == cudaSuccess) b->side.push_back(st);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
        if (e == cudaSuccess) b->join.push_back(ev);
    }
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
    if (b->d_items) cudaFree(b->d_items);
    if (b->d_counter) cudaFree(b->d_counter);
    for (cudaStream_t st : b->side) cudaStreamDestroy(st);
    for (cudaEvent_t ev : b->join) cudaEventDestroy(ev);
    if (b->fork) cudaEventDestroy(b->fork);
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
    const int nl = (int)b->launches.size();
    CTLAB_CUDA_TRY(cudaMemsetAsync(b->d_counter, 0, sizeof(int) * nl, s));
    // the launch with the most work first; the others wait for SMs it frees
    if (nl > 1) CTLAB_CUDA_TRY(cudaEventRecord(b->fork, s));
    for (int k = 0; k < nl; ++k) {
        const BatchLaunch &l = b->launches[k];
        cudaStream_t sk = k == 0 ? s : b->side[k - 1];
        if (k > 0) CTLAB_CUDA_TRY(cudaStreamWaitEvent(sk, b->fork, 0));
        CTLAB_CUDA_TRY(launch_proj_t_batch(l.nr, l.threads, *l.params, b->d_items + l.first, l.count,
                                           b->d_counter + k, l.smem, b->grid * (l.threads == 256 ? 2 : 1), sk));
        if (k > 0) CTLAB_CUDA_TRY(cudaEventRecord(b->join[k - 1], sk));
    }
    for (int k = 1; k < nl; ++k) CTLAB_CUDA_TRY(cudaStreamWaitEvent(s, b->join[k - 1], 0));
    return CTLAB_OK;
}

int ctlab_batch_proj(ctlab_batch *b, const float *const *d_vols, const unsigned char *const *d_masks,
                     float *const *d_prjs, int use_graph, void *stream)
{
    if (!b || !d_vols || !d_prjs) return set_status(CTLAB_ERR_INVALID_ARG, "null batch or buffer list");
    const int n = (int)b->plans.size();
    for (int i = 0; i < n; ++i)
        if (!d_vols[i] || !d_prjs[i]) return set_status(CTLAB_ERR_INVALID_ARG, "null volume or projection buffer");
    for (int i = 0; i < n; ++i)
        if (staging_sig(b->plans[i]) != b->staging[i])
            return set_status(CTLAB_ERR_INVALID_ARG,
                              "a plan's projector staging changed (autotuned?) after the batch was created; "
                              "create the batch again");
    DeviceGuard dg(b->device);
    cudaStream_t s = (cudaStream_t)stream;
    // launch parameters: every case's arguments with its output buffer
    for (BatchLaunch &l : b->launches)
        for (size_t k = 0; k < l.cases.size(); ++k)
            fill_case(b->plans[l.cases[k]], d_prjs[l.cases[k]], l.params->c[k]);
    if (!use_graph) {
        int rc = batch_enqueue(b, d_vols, d_masks, s);
        return rc == CTLAB_OK ? set_status(CTLAB_OK, "") : rc;
    }
    // a graph replays the buffers it was captured with
    std::vector<const void *> ptrs;
    for (int i = 0; i < n; ++i) {
        ptrs.push_back(d_vols[i]);
        ptrs.push_back(d_masks ? d_masks[i] : nullptr);
        ptrs.push_back(d_prjs[i]);
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
