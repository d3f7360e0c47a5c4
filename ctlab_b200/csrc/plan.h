// The plan object behind the C ABI's ctlab_plan handle.
#pragma once

#include <mutex>
#include <vector>

#include "internal.h"

namespace ctlab {
struct SolverWork; // solver workspace and weights kept between calls (recon.cpp)
}

struct ctlab_plan {
    int device = 0;
    int sat_mode = CTLAB_SAT_FP64;
    ctlab::HostGeometry g;
    ctlab::DevView *d_views = nullptr;
    double *d_det = nullptr;
    int *d_all_views = nullptr; // 0..PN-1
    int *d_list = nullptr;      // staged view list [PN]
    std::vector<int> h_list;
    bool need_y = false, need_x = false;
    void *d_sat_y = nullptr, *d_sat_x = nullptr;
    float2 *d_zt_y = nullptr, *d_zt_x = nullptr; // slice-major (P, f) z-prefix pairs (sat mode ZPREFIX)
    int zt_rs_y = 0, zt_rs_x = 0;               // their row strides (floats)
    CUtensorMap tm_y, tm_x;                     // TMA maps of the z-prefix arrays
    ctlab::ProjTStaging tst;                    // z-prefix projector staging
    CUtensorMap tm1_y, tm1_x;                   // the same for launches of single-view groups
    ctlab::ProjTStaging tst1;
    int zp = 0;                 // z stride of the volume SATs
    void *d_q = nullptr; // projection SATs [q_capacity][DNU+1][vp]
    float *d_pv = nullptr; // projection v-prefixes [q_capacity][DNU][vp] (sat mode ZPREFIX)
    int2 *d_zrange = nullptr; // backprojector view range per z block (sat mode ZPREFIX)
    int vp = 0;
    int q_capacity = 0;
    int proj_cmax = 2;  // projector staging columns
    int proj_nbuf = 2;  // projector staging depth
    int *d_groups_all = nullptr;     // projector view groups of the full view list
    int groups_all_n = 0, groups_all_G = 1;
    int *d_groups_scratch = nullptr; // groups of a caller's view list
    int groups_cap = 0;
    int back_rmax = 2;  // backprojector staging rows
    int *d_ticket = nullptr, *d_flags = nullptr, *d_err = nullptr;
    double *d_agg = nullptr, *d_pref = nullptr;
    bool timing = false;
    cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
    int last_launches = 0;
    long long bytes = 0;
    ctlab::SolverWork *sart = nullptr, *fista = nullptr, *cg = nullptr; // per solver
    std::mutex mu;
};

namespace ctlab {

// Device table of projector view groups (see proj_make_groups).
struct GroupTab {
    const int *d = nullptr;
    int ngroups = 0, G = 1;
};

void plan_free(ctlab_plan *p);
void solver_work_free(SolverWork *w);
// Groups the host list (positions into a device view list) and uploads the
// table to d_dst (capacity cap ints); synchronous.
int plan_groups(ctlab_plan *p, const std::vector<int> &host_list, int *d_dst, int cap, GroupTab &out,
                cudaStream_t s);
inline GroupTab plan_all_groups(const ctlab_plan *p) { return {p->d_groups_all, p->groups_all_n, p->groups_all_G}; }
int plan_volume_sat(ctlab_plan *p, const float *d_vol, const unsigned char *d_mask, cudaStream_t s);
int plan_proj_list(ctlab_plan *p, const int *d_list, int n, const GroupTab &gt, float *d_prj, cudaStream_t s,
                   int epilogue, const float *meas, const float *row_sum, double *resid2);
int plan_proj_sat(ctlab_plan *p, const int *d_list, int n, const float *d_prj, cudaStream_t s);
int plan_back_list(ctlab_plan *p, const int *d_list, int n, const unsigned char *d_mask, float *d_vol,
                   cudaStream_t s, int epilogue, const float *col_sum, float lambda, int clamp, float min_v,
                   float max_v);
int plan_upload_list(ctlab_plan *p, const int *h_views, int n, cudaStream_t s);
// z-prefix plans only, for copies overlapped with compute: the volume's
// z-prefixes of the voxel columns with y in [y0, y1) (y0 a multiple of 32);
// the projection v-prefixes of list positions [first, first + n); the
// backprojection of brick rows [by_off, by_off + by_count) (8 voxel rows each).
int plan_volume_sat_rows(ctlab_plan *p, const float *d_vol, const unsigned char *d_mask, int y0, int y1,
                         cudaStream_t s);
int plan_proj_sat_range(ctlab_plan *p, const int *d_list, int first, int n, const float *d_prj, cudaStream_t s);
// The fewest brick rows whose backprojector CTAs (a launch of n views) fill
// whole waves of the device, or 0 when unknown (not a z-prefix plan).
int plan_back_wave_rows(ctlab_plan *p, int n, int *rows);
int plan_back_rows(ctlab_plan *p, const int *d_list, int n, const unsigned char *d_mask, float *d_vol,
                   cudaStream_t s, int epilogue, const float *col_sum, float lambda, int clamp, float min_v,
                   float max_v, int by_off, int by_count);
int plan_check_device_error(ctlab_plan *p, cudaStream_t s);
void timing_mark(ctlab_plan *p, int which, cudaStream_t s);
// TMA map of the plan's z-prefix array of one orientation for a staging.
int plan_encode_zt(ctlab_plan *p, int orientation, const ProjTStaging &st, CUtensorMap *out);

} // namespace ctlab
