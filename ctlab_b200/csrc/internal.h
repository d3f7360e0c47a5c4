// Internal declarations shared by the libctlab_b200 translation units.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/ctlab_b200.h"

namespace ctlab {

// ----------------------------------------------------------------------
// status handling: every C entry point funnels through these
// ----------------------------------------------------------------------
int set_status(int code, const std::string &msg);
inline int ok() { return set_status(CTLAB_OK, ""); }
int cuda_status(cudaError_t e, const char *what);

#define CTLAB_CUDA_TRY(expr)                                                   \
    do {                                                                       \
        cudaError_t _e = (expr);                                               \
        if (_e != cudaSuccess) return ::ctlab::cuda_status(_e, #expr);         \
    } while (0)

// Restores the caller's current device on scope exit.
struct DeviceGuard {
    int prev = -1;
    bool ok = false;
    explicit DeviceGuard(int dev);
    ~DeviceGuard();
};

// ----------------------------------------------------------------------
// geometry
// ----------------------------------------------------------------------

// Per-view constants computed on the host in FP64.  (a, b) are the
// driving axis and the other in-plane axis of the view: a = y, b = x for
// y-driven views (slices y = const, SAT_y), a = x, b = y for x-driven.
struct DevView {
    double c, s;       // cos / sin of the regularised angle
    double Sx, Sy, Sz; // source, world
    double Sa, Sb;     // source along a and b
    double a0;         // a coordinate of slice 0's centre
    double b_lo;       // b coordinate of in-plane boundary 0
    double zP;         // z shift of the view
    double B0x, B0y;   // detector u-boundary 0, world (flat detectors)
    double Ex, Ey;     // detector u pitch vector, world (flat detectors)
    int xdrv;          // 1: x-driven
    int na, nb;        // slices along a, voxels along b
    int pad;
};

// Host-side description of a validated scan.
struct HostGeometry {
    double x0, y0, z0;
    int DNU, DNV, PN, XN, YN, ZN;
    double cx, cy, cz, dx, dz;
    double x_lo, y_lo, z_lo; // voxel boundary 0 along x, y, z
    std::vector<double> bx, by, bz; // local detector boundaries (DNU+1, DNU+1, DNV+1)
    std::vector<double> ux, uy, vz; // local detector centres (DNU, DNU, DNV)
    std::vector<DevView> views;
    std::vector<double> angle; // view angles as given (unwrapped: helical turns stay apart)
    bool flat_uniform = false; // flat detector with uniform u and v pitch
    double dzb = 0;            // v pitch (flat_uniform)
};

// Validates and converts the ctlab_geometry; returns CTLAB_OK or an error
// code with the message recorded.
int build_geometry(const ctlab_geometry &g, HostGeometry &out);

// Detector table on the device, doubles:
//   [0, DNU+1)         bx      local u-boundaries x
//   [DNU+1, 2(DNU+1))  by      local u-boundaries y
//   next DNU           ux      local centres x
//   next DNU           uy      local centres y
//   next DNV+1         bz      local z boundaries
//   next DNV           vz      local z centres
struct DetTable {
    int off_bx, off_by, off_ux, off_uy, off_bz, off_vz, total;
};
__host__ __device__ inline DetTable det_table_layout(int DNU, int DNV)
{
    DetTable t;
    t.off_bx = 0;
    t.off_by = t.off_bx + DNU + 1;
    t.off_ux = t.off_by + DNU + 1;
    t.off_uy = t.off_ux + DNU;
    t.off_bz = t.off_uy + DNU;
    t.off_vz = t.off_bz + DNV + 1;
    t.total = t.off_vz + DNV;
    return t;
}
std::vector<double> det_table_host(const HostGeometry &g);

// Positions of `list` (view indices) split by driving axis into runs of
// angularly adjacent views, each run sorted by angle.
std::vector<std::vector<int>> view_runs(const HostGeometry &g, const std::vector<int> &list);

// ----------------------------------------------------------------------
// kernels (launchers return cudaError_t from the launch)
// ----------------------------------------------------------------------

// Lookback state for the chunked SAT scans: per (plane, chunk) a status flag,
// an aggregate vector and an inclusive-prefix vector.
struct ScanState {
    int *ticket;    // one counter per launch, zeroed before the launch
    int *flags;     // [planes * chunks]
    double *agg;    // [planes * chunks * nk]
    double *pref;   // [planes * chunks * nk]
    int *err;       // device error word (timeouts)
};

size_t scan_state_doubles(int planes, int chunks, int nk);
// Number of chunks the scan of ns rows of nk elements uses for a requested chunk.
int scan_chunks(int ns, int nk, int chunk, int f32pair);

// Volume SAT of one orientation (0: y-slices over (x,z) planes -> SAT_y,
// 1: x-slices over (y,z) planes -> SAT_x), FP64 or float-pair output.
cudaError_t launch_volume_sat(const float *vol, const unsigned char *mask, int XN, int YN, int ZN,
                              int orientation, void *out, int zp, int f32pair, ScanState st,
                              int chunk, cudaStream_t s);

// Slice-major column z-prefixes of the masked volume for one driving axis,
// as affine pieces: out[j][k][c] = (P, f) with f = f(column c of slice j, k)
// (0 for k = ZN) and P = Z - k f, Z = sum_{z<k} f(column c of slice j, z)
// (FP64, P rounded to FP32 once), k in [0, ZN]; row stride rs >= nb pairs
// (pad columns zero).  P + kz f is the exact prefix at kz in [k, k+1].
// orientation 0: slices y, columns x (Z_y); 1: slices x, columns y (Z_x).
cudaError_t launch_zt(const float *vol, const unsigned char *mask, int XN, int YN, int ZN, int orientation,
                      float2 *out, int rs, cudaStream_t s);
// The same for the voxel columns with y in [y0, y1) only (y0 a multiple of
// 32), so a volume uploaded in y slabs can be prefixed slab by slab.
cudaError_t launch_zt_rows(const float *vol, const unsigned char *mask, int XN, int YN, int ZN, int orientation,
                           float2 *out, int rs, int y0, int y1, cudaStream_t s);
// The prefixes Z[k] = P + k f of a pair array [planes][rows][rs] into out.
cudaError_t launch_zt_unpack(const float2 *in, float *out, int planes, int rows, int rs, cudaStream_t s);

// A tiled TMA map (no interleave, zero fill outside the tensor): rank <= 5,
// dims[0] contiguous, strides in bytes of dims 1 .. rank-1 (multiples of
// 16), box extents per dim, the given shared-memory swizzle.  Returns a
// status.
int encode_tiled_map(CUtensorMap *m, CUtensorMapDataType dtype, int rank, void *base, const cuuint64_t *dims,
                     const cuuint64_t *strides, const cuuint32_t *box, CUtensorMapSwizzle swizzle, const char *what);

// Projection SAT: Q[p][u'][v'] of W = prj * L (L = slab path weight of the
// view's driving axis) for n views of the list.
// Projection rows weighted by the slab path length L of the view's driving
// axis: W = prj * dx * |C - S| / |C_a - S_a| with C the cell centre.
struct PrjIn {
    const float *prj;
    const DevView *views;
    const int *list;
    const double *det;
    DetTable t;
    int DNU, DNV;
    double dx;
    __device__ __forceinline__ float operator()(int plane, int u, int v) const
    {
        const DevView &V = views[list[plane]];
        const double lx = det[t.off_ux + u], ly = det[t.off_uy + u];
        const double cx = lx * V.c - ly * V.s, cy = lx * V.s + ly * V.c;
        const float ex = (float)(cx - V.Sx), ey = (float)(cy - V.Sy);
        const float ez = (float)(det[t.off_vz + v] + V.zP - V.Sz);
        const float ea = V.xdrv ? ex : ey;
        const float L = (float)dx * sqrtf(ex * ex + ey * ey + ez * ez) / fabsf(ea);
        return __ldg(prj + ((long long)plane * DNU + u) * DNV + v) * L;
    }
};

struct ProjSatArgs {
    const float *prj;     // [n][DNU][DNV]
    const DevView *views; // plan views
    const int *view_list; // [n] (device)
    int n;
    const double *det;    // detector table
    int DNU, DNV;
    double dx;
    void *out;            // [n][DNU+1][vp]
    int vp;
    int f32pair;
};
cudaError_t launch_proj_sat(const ProjSatArgs &a, ScanState st, int chunk, cudaStream_t s);
// Projection v-prefixes (sat mode ZPREFIX): out[l][u][v'] = sum_{v<v'} W(l, u, v),
// v' in [0, DNV] (entries up to the pitch vp repeat v' = DNV), FP64 sums in FP32.
cudaError_t launch_pv(const ProjSatArgs &a, float *out, int vp, cudaStream_t s);
// Diagnostics: a scan whose first chunk never publishes (see ctlab_debug_scan_stall).
cudaError_t launch_scan_stall(const float *vol, int rows, int nk, void *out, ScanState st, int chunk,
                              unsigned spin_limit, cudaStream_t s);

enum ProjEpilogue { PROJ_PLAIN = 0, PROJ_SART_RESIDUAL = 1 };

struct ProjArgs {
    const void *sat_y; // [YN][XN+1][zp]
    const void *sat_x; // [XN][YN+1][zp]
    int zp;
    int XN, YN, ZN;
    double dx, dz, z_lo;
    const DevView *views;
    const int *view_list; // [n] (device)
    int n;
    const double *det;
    int DNU, DNV;
    float *out;           // [n][DNU][DNV]
    int f32pair;
    int epilogue;
    const float *meas;    // [n][DNU][DNV]  (SART residual)
    const float *row_sum; // [n][DNU][DNV]
    double *resid2;       // accumulates sum (meas - Ax)^2
    int cmax;             // staging-buffer columns (proj_staging_columns)
    int *err;             // device error word (bounded waits)
    const int *groups;    // [ngroups][G] list positions sharing a CTA (-1: empty)
    int ngroups, G;
    int nbuf;             // staging depth (proj_staging)
    // slice-major z-prefix projector (sat mode ZPREFIX)
    const float2 *zt_y, *zt_x; // (P, f) pairs [YN][ZN+1][zt_rs_y], [XN][ZN+1][zt_rs_x]
    int zt_rs_y, zt_rs_x;
    int t_cb, t_kb, t_kr;      // stage: [t_kr][t_cb] pairs, TMA boxes of t_kb rows
    int t_nstage, t_rb, t_ep, t_gtab; // stages, consumer warps per view, z-boundary pitch, table views
    int t_zs;                         // detector rows split over t_zs CTAs
    int t_nr;                         // detector rows per consumer warp (t_nr * t_rb rows per CTA)
};

// Views of one launch grouped by driving axis and angle, G per CTA.
struct ProjGroups {
    std::vector<int> table; // [ngroups][G] list positions, -1 pads a partial group
    int ngroups = 0, G = 1;
};
ProjGroups proj_make_groups(const HostGeometry &g, const std::vector<int> &list, int cmax);
cudaError_t launch_proj(const ProjArgs &a, cudaStream_t s, int *launches);
bool proj_supported(int ZN, int DNV);
struct ProjStaging {
    int cmax = 2; // staged columns per buffer
    int nbuf = 2; // slices in flight
};
ProjStaging proj_staging(const HostGeometry &g, int zp, int elem_bytes);

// Staging of the slice-major z-prefix projector: up to G views per CTA, the
// detector rows split over ZS CTAs, RB consumer warps of NR detector rows
// per view, stages of KR rows x CB
// columns (TMA boxes of KB rows), nstage stages, EP floats per view of
// detector z boundaries.
struct ProjTStaging {
    int G = 1, NR = 4, RB = 1, ZS = 1, CB = 0, KB = 0, KR = 0, nstage = 2, EP = 8;
    int W = 15; // consumer warps per CTA at most (7: two CTAs share an SM)
    size_t smem = 0;
    bool ok = false;
};
// gcap limits the views per CTA (launches whose views group one by one use
// a staging planned with gcap = 1); nstage > 0 fixes the stage depth, zs > 0
// the split of the detector rows over CTAs (1, 2 or 4); wcap the consumer
// warps per CTA (15: one CTA of 16 warps per SM; 7: CTAs of 8 warps and at
// most half the SM's shared memory, two per SM).
ProjTStaging proj_t_staging(const HostGeometry &g, int gcap = 16, int nstage = 0, int zs = 0, int wcap = 0);
size_t proj_t_smem_bytes(const ProjTStaging &st);

// One scan of a batched (persistent) projector launch: its arguments and TMA
// maps, in device memory.
struct __align__(64) ProjBatchCase {
    CUtensorMap tm_y, tm_x;
    ProjArgs a;
};
// The cases of one persistent launch, passed as a kernel parameter (so the
// arguments and TMA maps sit in the constant bank like a single launch's).
constexpr int kProjBatchMaxCases = 31000 / (int)sizeof(ProjBatchCase);
struct ProjBatchParams {
    ProjBatchCase c[kProjBatchMaxCases];
};
// Detector rows per consumer warp (nr) and warps per view (rb) of a launch
// whose view groups hold G views under staging st.
void proj_t_split(const ProjTStaging &st, int G, int &nr, int &rb);
// Runs work items (case, detector tile, view group, row block) of up to
// kProjBatchMaxCases cases whose launches have nr rows per consumer warp, on
// a persistent grid of CTAs of `threads` threads (512, or 256 for cases
// staged for 8-warp CTAs, two per SM); *d_counter must be 0 (stream-ordered).
cudaError_t launch_proj_t_batch(int nr, int threads, const ProjBatchParams &cases, const int4 *d_items, int nitems,
                                int *d_counter, size_t smem, int grid, cudaStream_t s);
ProjGroups proj_t_make_groups(const HostGeometry &g, const std::vector<int> &list, const ProjTStaging &st);
cudaError_t launch_proj_t(const ProjArgs &a, const ProjTStaging &st, const CUtensorMap &tmy, const CUtensorMap &tmx,
                          cudaStream_t s, int *launches);

enum BackEpilogue { BACK_PLAIN = 0, BACK_SART_UPDATE = 1 };

struct BackArgs {
    const void *q;        // [n][DNU+1][vp] projection SATs
    int vp;
    const DevView *views;
    const int *view_list;
    int n;
    const double *det;
    int DNU, DNV;
    double dzb;           // detector v pitch
    int XN, YN, ZN;
    double dx, dz, x_c0, y_c0, z_lo;  // centres of voxel 0 along x, y; z boundary 0
    const unsigned char *mask;
    float *out;           // volume
    int f32pair;
    int epilogue;
    const float *col_sum; // SART update
    float lambda;
    int clamp;
    float min_v, max_v;
    int rmax;             // staging-buffer SAT rows (back_staging_rows)
    int *err;             // device error word (bounded waits)
    const float *pv;      // projection v-prefixes [n][DNU][vp] (sat mode ZPREFIX)
    int zskip;            // a helical scan: views may miss a CTA's z range (tested, then skipped)
    int2 *zrange;         // device scratch, one per z block: list positions [x, y) that can meet it
    int by_off, by_count; // z-prefix mode: brick rows [by_off, by_off + by_count) only (by_count 0: all)
};
cudaError_t launch_back(const BackArgs &a, cudaStream_t s, int *launches);
// Backprojector on projection v-prefixes (sat mode ZPREFIX).
cudaError_t launch_back_t(const BackArgs &a, cudaStream_t s, int *launches);
// Without launching: the CTAs the backprojector launch for `a` keeps resident
// on the device (one wave) and its CTAs per brick row.
cudaError_t back_t_query(const BackArgs &a, int *resident, int *ctas_per_row);
bool back_t_supported(int DNV);
int back_t_pitch(int DNV);
int back_t_staging_rows(const HostGeometry &g);
bool back_supported(int DNV);
int back_staging_rows(const HostGeometry &g, int vp);

// elementwise
cudaError_t launch_sart_proj_weight(float *prj, const float *real, const float *row_sum, long long n,
                                    cudaStream_t s);
cudaError_t launch_sart_back_weight(float *vol, float *recon, const float *col_sum, long long n,
                                    cudaStream_t s);
cudaError_t launch_fista_step(const float *las, float *cur, float t1, float t2, long long n,
                              float min_v, float max_v, cudaStream_t s);
cudaError_t launch_tv_gradient(const float *f, float *g, int XN, int YN, int ZN, float eps,
                               cudaStream_t s);
cudaError_t launch_fill(float *p, float v, long long n, cudaStream_t s);
cudaError_t launch_mask_fill(float *p, const unsigned char *mask, long long ncols, int ZN, cudaStream_t s);
// x = (z - lam * g) * mask ; and the SART-preconditioned step y += q/colSum
cudaError_t launch_tv_step(float *x, const float *z, const float *g, const unsigned char *mask, float lam,
                           long long n, int ZN, cudaStream_t s);
cudaError_t launch_add_scaled_div(float *y, const float *q, const float *col_sum, long long n, cudaStream_t s);
// gathers b[list[i]] views into out (subset-major copy)
cudaError_t launch_gather_views(const float *src, const int *list, int n, long long view_elems, float *dst,
                                cudaStream_t s);
// sum of squares of (a - b) and of a (double accumulators)
cudaError_t launch_resid2(const float *meas, const float *est, long long n, double *acc, cudaStream_t s);

// acc += sum a*b (FP64); y = alpha x + beta y
cudaError_t launch_dot(const float *a, const float *b, long long n, double *acc, cudaStream_t s);
cudaError_t launch_axpby(float *y, float alpha, const float *x, float beta, long long n, cudaStream_t s);

cudaError_t launch_phantom(float *vol, int XN, int YN, int ZN, float dx, float dz, float cx, float cy,
                           float cz, const float *ell_dev, int n_ell, int clamp_nonneg, cudaStream_t s);

} // namespace ctlab
