// Branchless DD cone-beam forward projection on slice-major column
// z-prefixes (sat mode CTLAB_SAT_ZPREFIX).
//
// Volume data, one array per driving axis: planes j (the slices along the
// axis) of ZN+1 rows k by nb columns c, c fastest, of pairs (P, f) with
//     Z[j][k][c] = sum_{z<k} f(column c of slice j, z)   (FP64 sums),
//     f = f(column c of slice j, k),  P = Z - k f   (FP64, stored FP32),
// i.e. for y-driven views planes y, columns x, and for x-driven ones planes
// x, columns y.  For piecewise-constant voxels P + kz f is the exact
// integral of the column up to kz on [k, k+1], so the integral over an
// axis-aligned rectangle of a slice is a weighted sum of column prefixes,
// each one 64-bit load and one FMA -- the difference-of-SAT of the
// branchless DD method with the FP64 in-plane prefix replaced by its exact
// column differences (which the 2-D FP64 SAT path also rounds to FP32).
//
// One CTA owns 32 detector columns (one per lane) of a group of G views of
// one driving axis with adjacent angles and sweeps the slices.
//   producer warp  per slice j, one lane per view maps the tile's two outer
//                  boundary rays onto slice j (FP64) and bounds the
//                  magnification over the tile's columns; a warp reduction
//                  gives the columns and z rows the group touches, and 3-D
//                  TMA tile loads (one per <= 256 rows) bring that
//                  [rows][columns] block into a ring of stages, completed on
//                  a "full" mbarrier;
//   consumer warps one warp per (view, block of NR detector rows), lanes =
//                  detector columns.  Per slice each lane maps its column's
//                  two boundary rays onto the slice (FP64, while the copy is
//                  in flight): SAT columns and fractions -> strip weights,
//                  the central-ray magnification T and 1/(W T) (W the strip
//                  width in columns).  For each of the NR+1 z boundaries e_w,
//                      kz = Z0 + T e_w,
//                      F(kz) = wa Za(kz) + wb Zb(kz) [+ whole columns between],
//                  Zc(kz) = P + kz f of column c's pair at row k, and
//                      acc[v] += (F(kz_{v+1}) - F(kz_v)) / (W T).
//                  Lanes read neighbouring columns of nearly the same rows,
//                  so the shared-memory loads are free of bank conflicts.
//                  Each warp hands the stage back on an "empty" mbarrier.
// floor(kz) comes from the round-toward-zero add of 2^23 and the biased
// result feeds the shared-memory address directly, so the inner loop issues
// no float/int conversions.  Slices whose block exceeds a stage read the
// z-prefixes from global memory instead.  Epilogue: central-ray slab length
// L = dx |C - S| / |C_a - S_a|, 1/(e_{v+1} - e_v), and optionally the SART
// residual (b - Ax)/rowSum with a residual reduction.
#include <cuda.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdlib>

#include "internal.h"
#include "tma.cuh"

namespace ctlab {

namespace {

constexpr int kTU = 32;           // detector columns per CTA (one per lane)
constexpr int kTMaxStage = 4;
constexpr int kTMaxCWarps = 15;   // consumer warps (16 warps with the producer: 128 registers a thread)
constexpr int kTMaxG = 16;        // views per CTA
constexpr int kTMaxThreads = (kTMaxCWarps + 1) * 32;
constexpr size_t kTSmemLimit = 227 * 1024;
constexpr size_t kTStatic = 14 * 1024; // static shared arrays, rounded up

struct TEntry {
    float T, scale, wa, wb;
};
struct TSlice {
    int c_lo, k_lo, fits, nbox;
    float kz_lo, kz_hi;
    float inv_span; // 1 / (kz_hi - kz_lo)
    int pad1;
};

__device__ __forceinline__ float2 lds_f32x2(uint32_t addr)
{
    float2 v;
    asm("ld.shared.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "r"(addr));
    return v;
}
template <int OFF>
__device__ __forceinline__ float2 lds_f32x2_at(uint32_t addr)
{
    float2 v;
    asm("ld.shared.v2.f32 {%0, %1}, [%2+%3];" : "=f"(v.x), "=f"(v.y) : "r"(addr), "n"(OFF));
    return v;
}
__device__ __forceinline__ float4 lds_f32x4(uint32_t addr)
{
    float4 v;
    asm("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];" : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "r"(addr));
    return v;
}

// column prefix at kz from the (P, f) pair at pa
__device__ __forceinline__ float zinterp(uint32_t pa, float kz)
{
    const float2 pf = lds_f32x2(pa);
    return fmaf(kz, pf.y, pf.x);
}

// Staged slice address of the z-prefix pair of the row holding kz, and kz,
// both clamped to the box [kz_lo, kz_hi].  The caller passes kz normalised
// to the box, vn = (kz - kz_lo) / span with span = kz_hi - kz_lo, as
// vn = Tn e + z0n: one saturating FMA clamps, the round-toward-zero FMA
// adding 2^23 leaves floor(vn span) -- the row past kz_lo -- in the mantissa
// bits, and one FMA gives kz; base folds in the box origin and the 2^23
// exponent bits (RS: bytes per staged row).
__device__ __forceinline__ uint32_t zrow_addr(float Tn, float e, float z0n, float span, float kz_lo, uint32_t RS,
                                              uint32_t base, float &kz)
{
    const float vn = __saturatef(fmaf(Tn, e, z0n));
    const float rr = __fmaf_rz(vn, span, 8388608.f);
    kz = fmaf(vn, span, kz_lo);
    return __float_as_uint(rr) * RS + base;
}

// Rows of one detector column on one slice when every strip of the warp
// spans at most two voxel columns: the lower one lo (base) and lo + 1 (the
// next pair, an immediate offset; weight 0 when the strip lies in one
// column).  F(row boundary) = wlo Z(lo) + whi Z(lo + 1); acc[r] += (F(r + 1)
// - F(r)) scale.
template <int NR>
__device__ __forceinline__ void rows_narrow(float (&acc)[NR], float wlo, float whi, float scale, uint32_t e_addr,
                                            uint32_t base, uint32_t RS, float Tn, float z0n, float span, float kz_lo)
{
    float prev = 0.f;
#pragma unroll
    for (int r4 = 0; r4 <= NR; r4 += 4) {
        const float4 e4 = lds_f32x4(e_addr + 4u * r4);
        const float ev[4] = {e4.x, e4.y, e4.z, e4.w};
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int r = r4 + q;
            if (r > NR) break;
            float kz;
            const uint32_t pa = zrow_addr(Tn, ev[q], z0n, span, kz_lo, RS, base, kz);
            const float2 za = lds_f32x2(pa), zb = lds_f32x2_at<8>(pa);
            const float F = fmaf(whi, fmaf(kz, zb.y, zb.x), wlo * fmaf(kz, za.y, za.x));
            if (r > 0) acc[r - 1] = fmaf(F - prev, scale, acc[r - 1]);
            prev = F;
        }
    }
}

// Weight of column a + i sgn(dc) in a strip from column a to column a + dc:
// wa at a, wb at the far column, +-1 for the whole columns between, 0 past
// the strip (those lanes read column a + dc again).
__device__ __forceinline__ float strip_weight(const TEntry &te, int i, int dc, int adc)
{
    return i == 0 ? te.wa : (i < adc ? (dc > 0 ? 1.f : -1.f) : (i == adc ? te.wb : 0.f));
}

// Rows of one detector column when the warp's widest strip spans M + 1
// voxel columns: one pass over the columns a .. a + M sgn(dc) per row.
template <int NR, int M>
__device__ __forceinline__ void rows_wide(float (&acc)[NR], const TEntry &te, int dc, uint32_t e_addr, uint32_t base,
                                          uint32_t RS, float Tn, float z0n, float span, float kz_lo)
{
    const int adc = dc < 0 ? -dc : dc;
    const int step8 = dc < 0 ? -8 : 8;
    float w[M + 1];
    uint32_t off[M + 1];
#pragma unroll
    for (int i = 0; i <= M; ++i) {
        w[i] = strip_weight(te, i, dc, adc);
        off[i] = (uint32_t)(min(i, adc) * step8);
    }
    float prev = 0.f;
#pragma unroll
    for (int r4 = 0; r4 <= NR; r4 += 4) {
        const float4 e4 = lds_f32x4(e_addr + 4u * r4);
        const float ev[4] = {e4.x, e4.y, e4.z, e4.w};
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int r = r4 + q;
            if (r > NR) break;
            float kz;
            const uint32_t pa = zrow_addr(Tn, ev[q], z0n, span, kz_lo, RS, base, kz);
            float F = w[0] * zinterp(pa, kz);
#pragma unroll
            for (int i = 1; i <= M; ++i) F = fmaf(w[i], zinterp(pa + off[i], kz), F);
            if (r > 0) acc[r - 1] = fmaf(F - prev, te.scale, acc[r - 1]);
            prev = F;
        }
    }
}

// Shared state of one projector tile besides the stage ring.
struct ProjTShm {
    uint64_t full[kTMaxStage], empty[kTMaxStage];
    TSlice info[kTMaxStage];
    double c0[kTMaxG][kTU + 1], m[kTMaxG][kTU + 1], r[kTMaxG][kTU];
    double ga0[kTMaxG], rmin[kTMaxG], rmax[kTMaxG];
    float Z0[kTMaxG], emin[kTMaxG], emax[kTMaxG];
    int pos_list[kTMaxG];
    int abort;
    double red[kTMaxCWarps + 1];
};

// One CTA's work: detector tile bx (32 columns), view group by, row block bz
// of the launch described by a.  smem: the 128-byte aligned dynamic shared
// memory (stages and z-boundary tables).
template <int NR, bool kBatch>
__device__ __forceinline__ void proj_t_tile(const ProjArgs &a, const CUtensorMap *tm_y_p, const CUtensorMap *tm_x_p,
                                            int bx, int by, int bz, unsigned char *smem, ProjTShm &sh,
                                            const int4 *s_w)
{
    const int G = a.G, RB = a.t_rb, NWC = G * RB;
    const int vbase = bz * RB * NR; // first detector row of this CTA (rows split over CTAs)
    const int nstage = a.t_nstage;
    const int CB = a.t_cb, KB = a.t_kb, KR = a.t_kr, EP = a.t_ep, GT = a.t_gtab;
    const int stage_elems = KR * CB;
    float2 *stage0 = reinterpret_cast<float2 *>(smem);                        // [nstage][KR][CB] (P, f)
    float *s_e = reinterpret_cast<float *>(smem + 8 * stage_elems * nstage); // [GT][EP]
    auto &s_full = sh.full;
    auto &s_empty = sh.empty;
    auto &s_info = sh.info;
    auto &s_c0 = sh.c0;
    auto &s_m = sh.m;
    auto &s_r = sh.r;
    auto &s_ga0 = sh.ga0;
    auto &s_rmin = sh.rmin;
    auto &s_rmax = sh.rmax;
    auto &s_Z0 = sh.Z0;
    auto &s_emin = sh.emin;
    auto &s_emax = sh.emax;
    auto &s_pos_list = sh.pos_list;
    auto &s_abort = sh.abort;
    auto &s_red = sh.red;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid < G) s_pos_list[tid] = a.groups[by * G + tid];
    if (tid == 0) s_abort = 0;
    const int u0 = bx * kTU;
    const int nu = min(kTU, a.DNU - u0);
    const DetTable t = det_table_layout(a.DNU, a.DNV);
    const double *det = a.det;
    const int ZN = a.ZN, DNV = a.DNV;
    const double dx = a.dx;
    __syncthreads();
    const DevView &V0 = a.views[a.view_list[s_pos_list[0]]]; // all views of the group share the axis
    const int na = V0.na, nb = V0.nb, xdrv = V0.xdrv;
    auto view_of = [&](int g) -> const DevView & {
        const int ps = s_pos_list[g] >= 0 ? s_pos_list[g] : s_pos_list[0];
        return a.views[a.view_list[ps]];
    };

    if (tid == 0) {
        int nact = 0;
        for (int g = 0; g < G; ++g) nact += s_pos_list[g] >= 0;
        for (int i = 0; i < nstage; ++i) {
            mbar_init(&s_full[i], 32);
            mbar_init(&s_empty[i], nact * RB); // one arrival per working consumer warp
        }
        mbar_fence_init();
    }
    const int nthreads = blockDim.x;
    // boundary rays of the tile (boundaries past the tile repeat the last)
    for (int it = tid; it < G * (kTU + 1); it += nthreads) {
        const int g = it / (kTU + 1), q0 = it - g * (kTU + 1);
        const DevView &V = view_of(g);
        const int q = u0 + min(q0, nu);
        const double lx = det[t.off_bx + q], ly = det[t.off_by + q];
        const double wx = lx * V.c - ly * V.s, wy = lx * V.s + ly * V.c;
        const double wa = V.xdrv ? wx : wy, wb = V.xdrv ? wy : wx;
        const double m = (wb - V.Sb) / (wa - V.Sa);
        s_m[g][q0] = m;
        s_c0[g][q0] = (V.Sb - V.b_lo) / dx + m * (V.a0 - V.Sa) / dx;
    }
    // central rays: 1 / (C_a - S_a)
    for (int it = tid; it < G * kTU; it += nthreads) {
        const int g = it / kTU, uq = it - g * kTU;
        const DevView &V = view_of(g);
        const int u = u0 + min(uq, nu - 1);
        const double lx = det[t.off_ux + u], ly = det[t.off_uy + u];
        const double ca = V.xdrv ? (lx * V.c - ly * V.s) : (lx * V.s + ly * V.c);
        s_r[g][uq] = 1.0 / (ca - V.Sa);
    }
    // detector z boundaries of this CTA's rows in SAT-row units, relative to
    // the source; rows past DNV repeat the last boundary (never stored)
    const int nw_local = min(RB * NR, DNV - vbase); // rows of this CTA
    for (int it = tid; it < G * EP; it += nthreads) {
        const int g = it / EP, w = min(vbase + it - g * EP, DNV);
        const DevView &V = view_of(g);
        s_e[it] = (float)((det[t.off_bz + w] + V.zP - V.Sz) / a.dz);
    }
    if (tid < G) {
        const DevView &V = view_of(tid);
        s_ga0[tid] = V.a0 - V.Sa;
        s_Z0[tid] = (float)((V.Sz - a.z_lo) / a.dz);
    }
    __syncthreads();
    if (tid < G) {
        float lo = 1e30f, hi = -1e30f;
        for (int w = 0; w <= nw_local; ++w) {
            lo = fminf(lo, s_e[tid * EP + w]);
            hi = fmaxf(hi, s_e[tid * EP + w]);
        }
        s_emin[tid] = lo;
        s_emax[tid] = hi;
        double rlo = 1e300, rhi = -1e300; // 1/(C_a - S_a) over the tile's columns
        for (int uq = 0; uq < nu; ++uq) {
            rlo = fmin(rlo, s_r[tid][uq]);
            rhi = fmax(rhi, s_r[tid][uq]);
        }
        s_rmin[tid] = rlo;
        s_rmax[tid] = rhi;
    }
    __syncthreads();

    double r2 = 0.0;
    if (warp == NWC) {
        // ------------------------------ producer ------------------------------
        const CUtensorMap *tm = xdrv ? tm_x_p : tm_y_p;
        const int uq = min(lane, nu - 1);
        int issued = 0;
        for (int j = 0; j < na; ++j) {
            const int b = j % nstage;
            if (*(volatile int *)&s_abort) break;
            // slice j's box first (it needs no buffer), then the wait for the
            // stage: only the copy's issue follows the consumers' release
            const double jd = (double)j;
            int cmin = INT_MAX, cmax = INT_MIN;
            float kmin = 1e30f, kmax = -1e30f;
            for (int g = lane; g < G; g += 32) {
                // the outer boundary rays bound the tile's columns (boundary
                // positions are monotone along the detector); one column of
                // margin for rounding between them and the interior rays
                const double x0 = fma(s_m[g][0], jd, s_c0[g][0]), x1 = fma(s_m[g][nu], jd, s_c0[g][nu]);
                const int i0 = min((int)fmin(fmax(x0, 0.0), (double)nb), nb - 1);
                const int i1 = min((int)fmin(fmax(x1, 0.0), (double)nb), nb - 1);
                cmin = min(cmin, max(min(i0, i1) - 1, 0));
                cmax = max(cmax, min(max(i0, i1) + 1, nb - 1));
                // the consumers' kz = fma((float)(t r_u), e, Z0) is monotone in
                // r_u and in e, so the extremes of both bound it exactly
                const double tj = s_ga0[g] + jd * dx;
                const float Ta = (float)(tj * s_rmin[g]), Tb = (float)(tj * s_rmax[g]);
                const float z0 = s_Z0[g], e0 = s_emin[g], e1 = s_emax[g];
                const float c0 = fmaf(Ta, e0, z0), c1 = fmaf(Ta, e1, z0), c2 = fmaf(Tb, e0, z0), c3 = fmaf(Tb, e1, z0);
                const float lo = fminf(fmaxf(fminf(fminf(c0, c1), fminf(c2, c3)), 0.f), (float)ZN);
                const float hi = fminf(fmaxf(fmaxf(fmaxf(c0, c1), fmaxf(c2, c3)), 0.f), (float)ZN);
                kmin = fminf(kmin, lo);
                kmax = fmaxf(kmax, hi);
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                cmin = min(cmin, __shfl_xor_sync(0xffffffffu, cmin, o));
                cmax = max(cmax, __shfl_xor_sync(0xffffffffu, cmax, o));
                kmin = fminf(kmin, __shfl_xor_sync(0xffffffffu, kmin, o));
                kmax = fmaxf(kmax, __shfl_xor_sync(0xffffffffu, kmax, o));
            }
            // TMA: the innermost (column) coordinate must be a multiple of 2
            // pairs (16 bytes); rows need no alignment
            const int c_lo = cmin & ~1;
            const int k_lo = max((int)kmin - 1, 0);
            const int k_top = min((int)kmax + 2, ZN + 1); // row of the last kz's upper neighbour
            const int nk = k_top - k_lo + 1;
            // (one column past cmax: the narrow path reads the pair right of
            // a strip's lower column, with weight 0 where the strip ends there)
            const bool fits = CB > 0 && (cmax - c_lo + 2 <= CB) && (nk <= KR);
            const int nbox = fits ? (nk + KB - 1) / KB : 0;
            if (j >= nstage) {
                bool ok = true;
                if (lane == 0) ok = mbar_wait(&s_empty[b], (uint32_t)(((j / nstage) - 1) & 1));
                ok = __shfl_sync(0xffffffffu, ok, 0);
                if (!ok) {
                    if (lane == 0) {
                        s_abort = 1;
                        if (a.err) atomicExch(a.err, CTLAB_ERR_TIMEOUT);
                    }
                    break;
                }
            }
            if (lane == 0) {
                TSlice in;
                in.c_lo = c_lo;
                in.k_lo = fits ? k_lo : 0;
                in.fits = fits;
                in.nbox = nbox;
                in.kz_lo = fits ? (float)k_lo : 0.f;
                in.kz_hi = fits ? (float)min(ZN, k_lo + KR - 2) : (float)ZN;
                in.inv_span = in.kz_hi > in.kz_lo ? 1.f / (in.kz_hi - in.kz_lo) : 0.f;
                in.pad1 = 0;
                s_info[b] = in;
                mbar_arrive_expect_tx(&s_full[b], (uint32_t)(nbox * KB * CB * 8));
            }
            __syncwarp();
            if (lane < nbox)
                tma_load_3d(stage0 + b * stage_elems + lane * KB * CB, tm, c_lo, k_lo + lane * KB, j, &s_full[b]);
            if (lane != 0) mbar_arrive(&s_full[b]);
            issued = j + 1;
        }
        // copies still in flight land before the CTA may exit
        if (lane == 0)
            for (int j = max(issued - nstage, 0); j < issued; ++j)
                if (!mbar_wait(&s_full[j % nstage], (uint32_t)((j / nstage) & 1)) && a.err)
                    atomicExch(a.err, CTLAB_ERR_TIMEOUT);
    } else if (warp < NWC && s_pos_list[warp / RB] >= 0) {
        // ------------------------------ consumers -----------------------------
        const int g = warp / RB, v0l = (warp - g * RB) * NR;
        const float2 *zt = xdrv ? a.zt_x : a.zt_y;
        const int zrs = xdrv ? a.zt_rs_x : a.zt_rs_y;
        const float z0 = s_Z0[g];
        const uint32_t e_addr = smem_addr(s_e + g * EP + v0l); // 16-byte aligned (EP, v0l multiples of 4)
        const uint32_t stage_addr = smem_addr(stage0);
        const uint32_t RS = 8u * (uint32_t)CB; // bytes per staged row
        // this lane's boundary rays x(q, j) = c0 + m j and 1/(C_a - S_a)
        const double ma = s_m[g][lane], ca0 = s_c0[g][lane], mb = s_m[g][lane + 1], cb0 = s_c0[g][lane + 1];
        const double ru = s_r[g][min(lane, nu - 1)], ga0 = s_ga0[g];
        const double nbd = (double)nb;
        float acc[NR];
#pragma unroll
        for (int r = 0; r < NR; ++r) acc[r] = 0.f;

        for (int j = 0; j < na; ++j) {
            const int b = j % nstage;
            // this column's strip on slice j (FP64 positions, FP32 weights)
            const double jd = (double)j;
            const double xa = fma(ma, jd, ca0), xb = fma(mb, jd, cb0);
            const double xac = fmin(fmax(xa, 0.0), nbd), xbc = fmin(fmax(xb, 0.0), nbd);
            const int ia = min((int)xac, nb - 1), ib = min((int)xbc, nb - 1);
            const float fa = (float)(xac - (double)ia), fb = (float)(xbc - (double)ib);
            TEntry te;
            te.T = (float)((ga0 + jd * dx) * ru);
            const float den = (float)(xb - xa) * te.T;
            te.scale = (den != 0.f) ? __frcp_rn(den) : 0.f;
            const int dc = ib - ia; // column b = column a + dc
            if (dc == 0) {
                te.wa = fb - fa;
                te.wb = 0.f;
            } else if (dc > 0) {
                te.wa = 1.f - fa;
                te.wb = fb;
            } else {
                te.wa = -fa;
                te.wb = fb - 1.f;
            }
            if (!mbar_wait(&s_full[b], (uint32_t)((j / nstage) & 1))) {
                if (lane == 0) {
                    s_abort = 1;
                    if (a.err) atomicExch(a.err, CTLAB_ERR_TIMEOUT);
                }
                break;
            }
            const TSlice in = s_info[b];
            // widest strip of the warp, in columns past column a (warp-uniform);
            // strips of more than four columns (very coarse cells) read the
            // column prefixes from global memory
            const int adc = dc < 0 ? -dc : dc;
            const int m = (int)__reduce_max_sync(0xffffffffu, (unsigned)adc);
            const bool wide = m > 1;
            const bool staged = in.fits && m <= 3;
            // the narrow path addresses the strip's lower column
            const int lo = (m <= 1 && dc < 0) ? ib : ia;
            const int2 cd = make_int2(staged ? lo - in.c_lo : ia, dc);
            if (staged) {
                // address of row k_lo + i, column a = bits(i + 2^23) * RS + base (mod 2^32)
                const uint32_t base = stage_addr + (uint32_t)b * 8u * (uint32_t)stage_elems + 8u * (uint32_t)cd.x -
                                      0x4B000000u * RS;
                // kz normalised to the box: (T e + z0 - kz_lo) / span
                const float span = in.kz_hi - in.kz_lo;
                const float Tn = te.T * in.inv_span, z0n = (z0 - in.kz_lo) * in.inv_span;
                if (m <= 1)
                    rows_narrow<NR>(acc, dc < 0 ? te.wb : te.wa, dc < 0 ? te.wa : te.wb, te.scale, e_addr, base, RS,
                                    Tn, z0n, span, in.kz_lo);
                else if (m == 2)
                    rows_wide<NR, 2>(acc, te, dc, e_addr, base, RS, Tn, z0n, span, in.kz_lo);
                else
                    rows_wide<NR, 3>(acc, te, dc, e_addr, base, RS, Tn, z0n, span, in.kz_lo);
            } else {
                // block wider than a stage, or strips wider than four columns:
                // the column prefixes from global memory
                const float2 *S = zt + (long long)j * (ZN + 1) * zrs;
                float prev = 0.f;
#pragma unroll
                for (int r = 0; r <= NR; ++r) {
                    float kz = fmaf(te.T, s_e[g * EP + v0l + r], z0);
                    kz = fminf(fmaxf(kz, 0.f), (float)ZN);
                    const int k0 = min((int)kz, ZN - 1);
                    const int ia = cd.x + k0 * zrs;
                    auto zc = [&](int i) {
                        const float2 pf = __ldg(S + i);
                        return fmaf(kz, pf.y, pf.x);
                    };
                    float F = te.wa * zc(ia) + te.wb * zc(ia + dc);
                    if (wide) {
                        const int n = dc > 1 ? dc - 1 : (dc < -1 ? -dc - 1 : 0);
                        const int step = dc > 0 ? 1 : -1;
                        float sum = 0.f;
                        for (int i = 1; i <= n; ++i) sum += zc(ia + i * step);
                        F += dc > 0 ? sum : -sum;
                    }
                    if (r > 0) acc[r - 1] = fmaf(F - prev, te.scale, acc[r - 1]);
                    prev = F;
                }
            }
            // every shared-memory read of this stage is consumed before the
            // stage is handed back
#pragma unroll
            for (int r = 0; r < NR; ++r) asm volatile("" ::"f"(acc[r]));
            __syncwarp();
            if (lane == 0) mbar_arrive(&s_empty[b]);
        }

        // epilogue: NR consecutive detector rows of column u per thread.  A
        // persistent (batch) CTA re-reads its arguments and work item here
        // instead of holding them in registers across the slice loop.
        const ProjArgs *ap = &a;
        int ebx = bx, ebz = bz;
        if (kBatch) {
            asm volatile("" : "+l"(ap));
            ebx = *reinterpret_cast<const volatile int *>(&s_w->y);
            ebz = *reinterpret_cast<const volatile int *>(&s_w->w);
        }
        const ProjArgs &ae = *ap;
        const int eu0 = ebx * kTU, enu = min(kTU, ae.DNU - eu0);
        const int eDNV = ae.DNV, ev0 = ebz * ae.t_rb * NR + v0l;
        const DetTable et = det_table_layout(ae.DNU, eDNV);
        const double *edet = ae.det;
        const int li = s_pos_list[g];
        if (lane < enu) {
            const int ps = li >= 0 ? li : s_pos_list[0];
            const DevView &V = ae.views[ae.view_list[ps]];
            const int u = eu0 + lane;
            const double lx = edet[et.off_ux + u], ly = edet[et.off_uy + u];
            const double cx = lx * V.c - ly * V.s, cy = lx * V.s + ly * V.c;
            const double ex = cx - V.Sx, ey = cy - V.Sy;
            const double ea = V.xdrv ? ex : ey;
            const double e2 = ex * ex + ey * ey;
#pragma unroll
            for (int r = 0; r < NR; ++r) {
                const int v = ev0 + r;
                if (v < eDNV) {
                    const double ez = edet[et.off_vz + v] + V.zP - V.Sz;
                    const double L = ae.dx * sqrt(e2 + ez * ez) / fabs(ea);
                    const double de = (edet[et.off_bz + v + 1] - edet[et.off_bz + v]) / ae.dz;
                    const float val = (float)((double)acc[r] * (L / de));
                    const long long idx = ((long long)li * ae.DNU + u) * eDNV + v;
                    if (ae.epilogue == PROJ_SART_RESIDUAL) {
                        const float mv = ae.meas[idx], rsum = ae.row_sum[idx];
                        const float res = mv - val;
                        r2 += (double)res * (double)res;
                        ae.out[idx] = (rsum > 1.0e-7f) ? res / rsum : 0.f;
                    } else {
                        ae.out[idx] = val;
                    }
                }
            }
        }
    }
    if (a.epilogue == PROJ_SART_RESIDUAL && a.resid2) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) r2 += __shfl_down_sync(0xffffffffu, r2, o);
        if (lane == 0) s_red[warp] = r2;
        __syncthreads();
        if (tid == 0) {
            double sum = 0.0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) sum += s_red[w];
            atomicAdd(a.resid2, sum);
        }
    }
}

__device__ __forceinline__ unsigned char *align128(unsigned char *p)
{
    return p + ((128 - (smem_addr(p) & 127)) & 127);
}

template <int NR>
__global__ void __launch_bounds__(kTMaxThreads, 1)
    dd3_proj_t_kernel(ProjArgs a, const __grid_constant__ CUtensorMap tm_y, const __grid_constant__ CUtensorMap tm_x)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ ProjTShm sh;
    // TMA destinations need 128-byte alignment (the launch adds 128 bytes)
    proj_t_tile<NR, false>(a, &tm_y, &tm_x, blockIdx.x, blockIdx.y, blockIdx.z, align128(smem_raw), sh, nullptr);
}

// Persistent projector over many scans: CTAs take (case, tile, group, row
// block) work items from a queue (items sorted longest first) and run them
// with each case's arguments and TMA maps from the kernel parameters.  Every
// case of one launch has NR detector rows per consumer warp.
template <int NR>
__global__ void __launch_bounds__(kTMaxThreads, 1)
    dd3_proj_t_batch_kernel(const __grid_constant__ ProjBatchParams cases, const int4 *__restrict__ items, int nitems,
                            int *counter)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ ProjTShm sh;
    __shared__ int4 s_w;
    unsigned char *smem = align128(smem_raw);
    const int tid = threadIdx.x;
    for (;;) {
        if (tid == 0) {
            const int it = atomicAdd(counter, 1);
            s_w = it < nitems ? items[it] : make_int4(-1, 0, 0, 0);
        }
        __syncthreads();
        const int4 w = s_w;
        if (w.x < 0) break;
        const ProjBatchCase &c = cases.c[w.x];
        proj_t_tile<NR, true>(c.a, &c.tm_y, &c.tm_x, w.y, w.z, w.w, smem, sh, &s_w);
        // every warp is done with this item's barriers and buffers
        __syncthreads();
        if (tid < kTMaxStage) {
            asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_addr(&sh.full[tid])) : "memory");
            asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_addr(&sh.empty[tid])) : "memory");
        }
        __syncthreads();
    }
}

size_t smem_bytes(const ProjTStaging &st)
{
    return 128 + sizeof(float2) * (size_t)st.KR * st.CB * st.nstage + sizeof(float) * (size_t)st.G * st.EP;
}

template <int NR>
cudaError_t launch_t_nr(const ProjArgs &a, const CUtensorMap &tmy, const CUtensorMap &tmx, size_t sm, cudaStream_t s)
{
    auto kern = dd3_proj_t_kernel<NR>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    dim3 grid((a.DNU + kTU - 1) / kTU, a.ngroups, a.t_zs);
    kern<<<grid, (a.G * a.t_rb + 1) * 32, sm, s>>>(a, tmy, tmx);
    return cudaGetLastError();
}

// b-index span (in columns, margins included) of the union of the rays of
// views `vs` (one driving axis) through the tile [u0, u0+nu) on slice j.
int t_span(const HostGeometry &g, const std::vector<const DevView *> &vs, int u0, int nu, int j)
{
    double lo = 1e300, hi = -1e300;
    for (const DevView *V : vs) {
        for (int e = 0; e < 2; ++e) {
            const int q = u0 + (e ? nu : 0);
            const double wx = g.bx[q] * V->c - g.by[q] * V->s, wy = g.bx[q] * V->s + g.by[q] * V->c;
            const double wa = V->xdrv ? wx : wy, wb = V->xdrv ? wy : wx;
            const double m = (wb - V->Sb) / (wa - V->Sa);
            const double x = (V->Sb - V->b_lo) / g.dx + m * (V->a0 - V->Sa) / g.dx + m * j;
            lo = std::min(lo, x);
            hi = std::max(hi, x);
        }
    }
    const int nb = vs[0]->nb;
    lo = std::min(std::max(lo, 0.0), (double)nb);
    hi = std::min(std::max(hi, 0.0), (double)nb);
    // floor(lo) rounded down to 2 (TMA alignment of 8-byte pairs) and one
    // column of margin each side for rounding between host and device
    const int c_lo = std::max((int)lo - 1, 0) & ~1;
    // (+1: the kernel reads the pair right of a strip's lower column)
    const int c_hi = std::min((int)hi + 1, nb - 1) + 1;
    return c_hi - c_lo + 1;
}

// Largest column span of any group (view indices) over all tiles and
// slices; the span is convex in the slice index, so the end slices bound it.
int t_need(const HostGeometry &g, const std::vector<std::vector<int>> &groups)
{
    int need = 4;
    for (const auto &grp : groups) {
        std::vector<const DevView *> vs;
        for (int v : grp) vs.push_back(&g.views[v]);
        const int na = vs[0]->na;
        for (int u0 = 0; u0 < g.DNU; u0 += kTU) {
            const int nu = std::min(kTU, g.DNU - u0);
            need = std::max(need, std::max(t_span(g, vs, u0, nu, 0), t_span(g, vs, u0, nu, na - 1)));
        }
    }
    return need;
}

// Views of `list` (view indices) grouped G at a time within runs of
// angularly adjacent views of one driving axis; returns list positions.
std::vector<std::vector<int>> t_groups(const HostGeometry &g, const std::vector<int> &list, int G)
{
    std::vector<std::vector<int>> out;
    for (const std::vector<int> &run : view_runs(g, list))
        for (size_t i0 = 0; i0 < run.size(); i0 += G) {
            std::vector<int> grp;
            for (size_t k = i0; k < std::min(run.size(), i0 + G); ++k) grp.push_back(run[k]);
            out.push_back(grp);
        }
    return out;
}

std::vector<std::vector<int>> as_views(std::vector<std::vector<int>> groups, const std::vector<int> &list)
{
    for (auto &grp : groups)
        for (int &p : grp) p = list[p];
    return groups;
}

// Rows of z-prefix a CTA stages for one slice (+3: the margins and the
// interpolation neighbour of the kernel's range), the largest over groups,
// tiles, row blocks of `rows` detector rows and (sampled) slices.  kz is
// affine in the magnification T for a fixed boundary, so the columns at the
// ends and the middle of a tile bound it for flat and curved detectors.
int t_zrows(const HostGeometry &g, const std::vector<std::vector<int>> &groups, int rows, int zs)
{
    int need = 4;
    std::vector<double> emins, emaxs; // per (row block, view of the group)
    for (const auto &grp : groups) {
        const DevView &V0 = g.views[grp[0]];
        const int jstep = std::max(1, V0.na / 64);
        // z-boundary extremes of each row block per view (independent of tile and slice)
        emins.assign((size_t)zs * grp.size(), 1e300);
        emaxs.assign((size_t)zs * grp.size(), -1e300);
        for (int zb = 0; zb < zs; ++zb) {
            const int w0 = zb * rows, w1 = std::min(g.DNV, w0 + rows);
            for (size_t q = 0; q < grp.size(); ++q) {
                const DevView &V = g.views[grp[q]];
                double &mn = emins[zb * grp.size() + q], &mx = emaxs[zb * grp.size() + q];
                for (int w = w0; w <= w1; ++w) {
                    const double e = (g.bz[w] + V.zP - V.Sz) / g.dz;
                    mn = std::min(mn, e);
                    mx = std::max(mx, e);
                }
            }
        }
        for (int u0 = 0; u0 < g.DNU; u0 += kTU) {
            const int nu = std::min(kTU, g.DNU - u0);
            const int us[3] = {u0, u0 + nu / 2, u0 + nu - 1};
            for (int zb = 0; zb < zs; ++zb) {
                for (int j = 0; j < V0.na; j += (j + jstep < V0.na || j == V0.na - 1) ? jstep : V0.na - 1 - j) {
                    double lo = 1e300, hi = -1e300;
                    for (size_t q = 0; q < grp.size(); ++q) {
                        const DevView &V = g.views[grp[q]];
                        const double z0 = (V.Sz - g.z_lo) / g.dz;
                        const double emin = emins[zb * grp.size() + q], emax = emaxs[zb * grp.size() + q];
                        for (int u : us) {
                            const double ca = V.xdrv ? (g.ux[u] * V.c - g.uy[u] * V.s) : (g.ux[u] * V.s + g.uy[u] * V.c);
                            const double T = (V.a0 - V.Sa + j * g.dx) / (ca - V.Sa);
                            for (double e : {emin, emax}) {
                                const double kz = std::min(std::max(z0 + T * e, 0.0), (double)g.ZN);
                                lo = std::min(lo, kz);
                                hi = std::max(hi, kz);
                            }
                        }
                    }
                    need = std::max(need, (int)hi - std::max((int)lo - 1, 0) + 3);
                    if (j == V0.na - 1) break;
                }
            }
        }
    }
    return std::min(need, g.ZN + 2);
}

int env_int(const char *name, int dflt)
{
    const char *s = std::getenv(name);
    return s ? std::atoi(s) : dflt;
}

} // namespace

size_t proj_t_smem_bytes(const ProjTStaging &st) { return smem_bytes(st); }

template <int NR>
cudaError_t launch_batch_nr(const ProjBatchParams &cases, const int4 *d_items, int nitems, int *d_counter, size_t smem,
                            int grid, int threads, cudaStream_t s)
{
    auto kern = dd3_proj_t_batch_kernel<NR>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    kern<<<grid, threads, smem, s>>>(cases, d_items, nitems, d_counter);
    return cudaGetLastError();
}

cudaError_t launch_proj_t_batch(int nr, int threads, const ProjBatchParams &cases, const int4 *d_items, int nitems,
                                int *d_counter, size_t smem, int grid, cudaStream_t s)
{
    if (nitems <= 0) return cudaSuccess;
    if (threads != kTMaxThreads && threads != kTMaxThreads / 2) return cudaErrorInvalidValue;
    switch (nr) {
    case 4: return launch_batch_nr<4>(cases, d_items, nitems, d_counter, smem, grid, threads, s);
    case 8: return launch_batch_nr<8>(cases, d_items, nitems, d_counter, smem, grid, threads, s);
    case 12: return launch_batch_nr<12>(cases, d_items, nitems, d_counter, smem, grid, threads, s);
    case 16: return launch_batch_nr<16>(cases, d_items, nitems, d_counter, smem, grid, threads, s);
    case 20: return launch_batch_nr<20>(cases, d_items, nitems, d_counter, smem, grid, threads, s);
    case 24: return launch_batch_nr<24>(cases, d_items, nitems, d_counter, smem, grid, threads, s);
    case 28: return launch_batch_nr<28>(cases, d_items, nitems, d_counter, smem, grid, threads, s);
    case 32: return launch_batch_nr<32>(cases, d_items, nitems, d_counter, smem, grid, threads, s);
    default: return cudaErrorInvalidValue;
    }
}

ProjTStaging proj_t_staging(const HostGeometry &g, int gcap, int nstage_fix, int zs_fix, int wcap)
{
    ProjTStaging st;
    st.ok = false;
    // consumer warps per CTA: 15 (one CTA per SM) or 7 (two CTAs per SM, each
    // within half the shared memory); CTLAB_PROJT_WARPS picks the default
    const int W = (wcap > 0 ? wcap : env_int("CTLAB_PROJT_WARPS", kTMaxCWarps)) <= 7 ? 7 : kTMaxCWarps;
    const size_t smem_cap = W == kTMaxCWarps ? kTSmemLimit : kTSmemLimit / 2 - 1024;
    // CTLAB_PROJT_GMAX caps the views per CTA (1..15), CTLAB_PROJT_ZS fixes
    // the row split (1, 2, 4), CTLAB_PROJT_NSTAGE the stage depth (2..4),
    // CTLAB_PROJT_CBMAX caps the staged columns
    const int gmax = std::max(1, std::min(std::min(env_int("CTLAB_PROJT_GMAX", W), kTMaxG), std::min(gcap, W)));
    const int want_zs = zs_fix > 0 ? zs_fix : env_int("CTLAB_PROJT_ZS", 0);
    const int want_stage = nstage_fix > 0 ? nstage_fix : env_int("CTLAB_PROJT_NSTAGE", 0);
    const int cbmax = std::min(env_int("CTLAB_PROJT_CBMAX", 256), 256);
    std::vector<int> all(g.PN);
    for (int i = 0; i < g.PN; ++i) all[i] = i;
    // candidates (views per CTA, row split): prefer >= 12 consumer warps, then
    // more views per CTA, then fewer row splits
    ProjTStaging best;
    int best_key = -1;
    for (int G = gmax; G >= 1; --G) {
        int CB = (t_need(g, as_views(t_groups(g, all, G), all)) + 1) & ~1;
        // a row stride of a multiple of 16 pairs (128 bytes) puts every
        // column on the same banks in every row, so lanes reading distinct
        // columns never conflict whatever rows they read; take it when it
        // costs little
        const int cb16 = (CB + 15) & ~15;
        if (cb16 - CB <= 8) CB = cb16;
        if (CB > cbmax) {
            if (G > 1) continue;
            CB = cbmax & ~1; // G = 1: wider slices read global memory
        }
        for (int ZS : {1, 2, 4}) {
            if (want_zs && ZS != want_zs) continue;
            if (!want_zs && ZS > 1 && g.DNV < 16 * ZS) continue;
            const int rows = (g.DNV + ZS - 1) / ZS; // detector rows per CTA
            // warps per view: as many as the consumer warps allow while each
            // keeps >= 8 rows, at least enough for <= 32 rows per warp; rows
            // per warp: the rows split evenly, rounded up to 4
            const int rb_min = (rows + 31) / 32;
            const int RB = std::max(rb_min, std::min(W / G, (rows + 7) / 8));
            if (RB * G > W) continue;
            const int NR = std::min(32, ((rows + RB - 1) / RB + 3) & ~3);
            const int key = (RB * G >= (W == kTMaxCWarps ? 12 : 6) ? 1000 : 0) + G * 10 + (4 - ZS);
            if (key <= best_key) continue;
            const int zs = (g.DNV + RB * NR - 1) / (RB * NR); // CTAs over the rows (no empty one)
            // z rows a CTA stages per slice: the clamped kz range of its
            // detector rows over the group's views and the tile's columns
            const int zrows = t_zrows(g, as_views(t_groups(g, all, G), all), RB * NR, zs);
            const int nbox = (zrows + 255) / 256;
            int KB = (zrows + nbox - 1) / nbox;
            // 128-byte aligned TMA destinations: KB * CB * 8 a multiple of 128
            while ((KB * CB) % 16) ++KB;
            if (KB > 256) continue;
            for (int ns = kTMaxStage; ns >= 2; --ns) {
                if (want_stage >= 2 && want_stage <= kTMaxStage && ns != want_stage) continue;
                ProjTStaging c;
                c.G = G;
                c.NR = NR;
                c.RB = RB;
                c.ZS = zs;
                c.CB = CB;
                c.KB = KB;
                c.KR = nbox * KB;
                c.nstage = ns;
                c.EP = RB * NR + 4;
                c.W = W;
                c.smem = smem_bytes(c);
                if (c.smem + kTStatic > smem_cap) continue;
                c.ok = true;
                best = c;
                best_key = key;
                break;
            }
        }
        // a candidate with enough warps beats every smaller group size
        if (best_key >= 1000) break;
    }
    if (best.ok) return best;
    // nothing stages: every slice reads global memory
    st.G = 1;
    st.ZS = 1;
    const int splits = (g.DNV + kTMaxCWarps * 32 - 1) / (kTMaxCWarps * 32);
    const int per = (g.DNV + splits - 1) / splits; // rows per CTA
    st.RB = std::min(kTMaxCWarps, std::max((per + 31) / 32, (per + 7) / 8));
    st.NR = std::min(32, ((per + st.RB - 1) / st.RB + 3) & ~3);
    st.RB = (per + st.NR - 1) / st.NR;
    st.ZS = (g.DNV + st.RB * st.NR - 1) / (st.RB * st.NR);
    st.CB = 0;
    st.KB = 0;
    st.KR = 0;
    st.nstage = 2;
    st.EP = st.RB * st.NR + 4;
    st.smem = smem_bytes(st);
    st.ok = true;
    return st;
}

ProjGroups proj_t_make_groups(const HostGeometry &g, const std::vector<int> &list, const ProjTStaging &st)
{
    ProjGroups out;
    for (int G = st.G; G >= 1; G /= 2) {
        std::vector<std::vector<int>> groups = t_groups(g, list, G);
        if (G > 1 && t_need(g, as_views(groups, list)) > st.CB) continue;
        out.G = G;
        out.table.clear();
        for (auto &grp : groups)
            for (int k = 0; k < G; ++k) out.table.push_back(k < (int)grp.size() ? grp[k] : -1);
        out.ngroups = (int)groups.size();
        return out;
    }
    return out;
}

void proj_t_split(const ProjTStaging &st, int G, int &nr, int &rb)
{
    // launches whose groups hold fewer views than planned keep the rows per
    // CTA and split them over more warps (rows per warp >= 8, a multiple of 4)
    nr = st.NR;
    rb = st.RB;
    while (G * rb * 2 <= st.W && nr >= 16 && nr % 8 == 0) {
        nr /= 2;
        rb *= 2;
    }
}

cudaError_t launch_proj_t(const ProjArgs &a, const ProjTStaging &st, const CUtensorMap &tmy, const CUtensorMap &tmx,
                          cudaStream_t s, int *launches)
{
    if (a.n <= 0 || a.ngroups <= 0) return cudaSuccess;
    if (a.ngroups > 65535 || a.G > st.G || a.G * a.t_rb > kTMaxCWarps) return cudaErrorInvalidConfiguration;
    if (launches) ++*launches;
    const size_t sm = smem_bytes(st);
    if (a.t_nr * a.t_rb != st.NR * st.RB) return cudaErrorInvalidConfiguration;
    switch (a.t_nr) {
    case 4: return launch_t_nr<4>(a, tmy, tmx, sm, s);
    case 8: return launch_t_nr<8>(a, tmy, tmx, sm, s);
    case 12: return launch_t_nr<12>(a, tmy, tmx, sm, s);
    case 16: return launch_t_nr<16>(a, tmy, tmx, sm, s);
    case 20: return launch_t_nr<20>(a, tmy, tmx, sm, s);
    case 24: return launch_t_nr<24>(a, tmy, tmx, sm, s);
    case 28: return launch_t_nr<28>(a, tmy, tmx, sm, s);
    case 32: return launch_t_nr<32>(a, tmy, tmx, sm, s);
    default: return cudaErrorInvalidValue;
    }
}

} // namespace ctlab
