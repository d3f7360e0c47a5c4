// Branchless DD cone-beam backprojection on projection v-prefixes (sat mode
// CTLAB_SAT_ZPREFIX): the voxel-driven gather of back.cu with the 2-D FP64
// projection SAT replaced by per-detector-column prefixes along v,
//     P[l][u][v'] = sum_{v<v'} W(l, u, v),  W = prj * slab length,
// accumulated in FP64 and stored in FP32 (the column differences of the 2-D
// SAT, which the FP64 path also rounds to FP32 before use).
//
// One CTA owns an 8 x 8 brick of voxel columns and a z range of ZS*KSEG
// voxels (ZS z segments per column, one thread each: 256 threads by default,
// two CTAs per SM) and loops over the views.  Per view:
//   geometry   the brick's voxel boundaries across the view's driving axis
//              (8 rows of 9 points) mapped through the source onto the flat
//              detector, and each column's centre ray giving the affine
//              z -> v map (kept normalised by DNV): FP32 on offsets from the
//              brick centre, whose projective map (an anchor) is computed in
//              FP64 for 32 views at a time;
//   staging    the rows [u_lo, u_hi] of the view's P that the brick's
//              footprint covers: one 1-D bulk copy (TMA), double buffered
//              two views ahead and completed on an mbarrier;
//   phase A    per column and detector row boundary v', the strip integral
//              between the column's two u boundaries,
//                 E_c(v') = sg * [ sum of P over whole cells + f_b P_b - f_a P_a ],
//              sg orienting it like the voxel's z axis (FP32), stored per row
//              i as the affine form of its linear piece in vn = v / DNV,
//                 (E_c(i) - i dE_i, DNV dE_i),  dE_i = E_c(i+1) - E_c(i),
//              so that E_c(v) = first + vn * second on [i, i+1]; ZS
//              threads per column each run a contiguous stretch of rows with
//              a warp-uniform trip count, from a strip set-up computed two
//              views ahead;
//   phase B    each voxel boundary k samples E_c linearly at
//              v = DNV * sat(V0 + V1 k) with one 64-bit shared load and the
//              voxel accumulates E_c(v_{k+1}) - E_c(v_k): one saturating FMA
//              clamps, the round-toward-zero FMA with 2^23 gives floor(v)
//              biased for the shared-memory address -- no float/int
//              conversions -- and one FMA evaluates the piece (7
//              instructions per boundary).
// In the 512- and 1024-thread shapes E is double buffered, so one barrier per
// view separates A(l) from B(l) and the issue of view l+2's copy; the
// 256-thread shape keeps one E table and a second barrier after B(l), the
// other CTA on the SM filling the gaps.  Views whose footprint exceeds a
// stage read P from global memory.  Epilogue: in-plane mask and optionally the OS-SART
// update x = (x + lambda * acc/colSum) * mask.
#include <algorithm>
#include <climits>
#include <cstdlib>
#include <cmath>
#include <type_traits>
#include <utility>

#include "internal.h"
#include "tma.cuh"

namespace ctlab {

namespace {

constexpr int kB = 8;                 // brick edge (voxel columns)
constexpr int kCols = kB * kB;        // 64 columns per CTA
// z segments per column ZS (template parameter): 4 (256 threads, KSEG up to
// 64 accumulators a thread, single-buffered E, two CTAs per SM; the default),
// 8 (512 threads, KSEG up to 32) or 16 (1024 threads, at most 64 registers a
// thread)
constexpr size_t kSmemPerCta = 200 * 1024; // one CTA per SM
constexpr size_t kStaticSmem = 20 * 1024;
constexpr int kGeo = 4;               // geometry slots (views l .. l+3)

// Column slot of column (cx, cy) in a row of the piece table: a permutation
// of the 64 columns whose value mod 16 (the bank pair of an 8-byte entry)
// differs within every 8 x 2 block {cx} x {2h, 2h+1} -- the 16 columns of a
// half-warp of phase B -- and within every 4 x 4 quadrant -- the 16 columns
// of a half-warp of phase A.
__host__ __device__ constexpr int e_slot(int cx, int cy)
{
    return 16 * (cy >> 1) + ((cx ^ (4 * ((cy >> 1) & 1))) + 8 * (cy & 1));
}

__device__ __forceinline__ float lds_f32(uint32_t addr)
{
    float v;
    asm("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"(addr));
    return v;
}

__device__ __forceinline__ float2 lds_f32x2(uint32_t addr)
{
    float2 v;
    asm("ld.shared.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "r"(addr));
    return v;
}

template <int OFF>
__device__ __forceinline__ float lds_f32_at(uint32_t addr)
{
    float v;
    asm("ld.shared.f32 %0, [%1+%2];" : "=f"(v) : "r"(addr), "n"(OFF));
    return v;
}
template <int OFF>
__device__ __forceinline__ void sts_f32x2_at(uint32_t addr, float x, float y)
{
    asm volatile("st.shared.v2.f32 [%0+%1], {%2, %3};" ::"r"(addr), "n"(OFF), "f"(x), "f"(y) : "memory");
}
template <int I, int N, class F>
__device__ __forceinline__ void unroll_for(F &&f)
{
    if constexpr (I < N) {
        f(std::integral_constant<int, I>());
        unroll_for<I + 1, N>(f);
    }
}

// The table entry of row i from E(i) and E(i+1): the piece E(i) + (v - i) dE
// as an affine function of vn = v / DNV.
__device__ __forceinline__ float2 affine_piece(float e, float en, float fi, float dnv)
{
    const float d = en - e;
    return make_float2(fmaf(-fi, d, e), dnv * d);
}

// Phase A run of one thread: E at rows i0 .. i0+VPT of one column from the
// staged P rows pa, pb (and NX whole cells pm[] between them), stored as VPT
// affine pieces at eout, kCols entries apart (nfi0 = -i0).  Every address
// carries i0; offsets are immediates.
template <int VPT, int NX>
__device__ __forceinline__ void phase_a_run(uint32_t pa, uint32_t pb, const uint32_t (&pm)[3], const float (&wmv)[3],
                                            float wa, float wb, float nfi0, float dnv, uint32_t eout)
{
    float e_prev = 0.f;
    unroll_for<0, VPT + 1>([&](auto jt) {
        constexpr int j = decltype(jt)::value;
        float e = fmaf(wb, lds_f32_at<4 * j>(pb), wa * lds_f32_at<4 * j>(pa));
        unroll_for<0, NX>([&](auto mt) {
            constexpr int m = decltype(mt)::value;
            e = fmaf(wmv[m], lds_f32_at<4 * j>(pm[m]), e);
        });
        if constexpr (j > 0) {
            // first = E(i) - i d with i = i0 + j - 1
            const float d = e - e_prev;
            float first = fmaf(nfi0, d, e_prev);
            if constexpr (j > 1) first = fmaf(-(float)(j - 1), d, first);
            sts_f32x2_at<8 * kCols * (j - 1)>(eout, first, dnv * d);
        }
        e_prev = e;
    });
}

__device__ __forceinline__ double cross2(double ax, double ay, double bx, double by)
{
    return ax * by - ay * bx;
}

// Phase-A set-up of one column for one view, computed two views ahead by
// 64 threads instead of by each of the column's ZS phase-A threads: byte
// offsets of the strip's staged P rows from the stage origin (a, b and up to
// three whole cells between), the strip weights and the whole-cell count.
struct ASet {
    uint32_t off[5];
    float wa, wb, wm[3];
    int nm, pad;
};

// One view's geometry anchored at the brick centre c (FP64 once, stored
// FP32).  For a point p = c + (ox, oy) dx in the plane, the detector column
// coordinate of the ray through p is
//     u(p) = u0 + (gx ox + gy oy) / (1 + kx ox + ky oy),   u0 = u(c),
// (u = N/D with N, D affine in p: gx, gy = dx (grad N - u0 grad D) / D(c),
// kx, ky = dx grad D / D(c)), and the central-ray magnification of the
// voxel column through p is T0 / (1 + kx ox + ky oy).  The per-view work is
// then FP32 on offsets of a few voxels (u relative to floor(u0)), exact to
// a few 1e-7 of a detector cell.  The z -> v map of a column with
// magnification t is V1 = Cz t, V0 = Az + Bz t (detector rows / DNV).
struct Anchor {
    int iu0;   // floor(u0)
    float fu0; // u0 - floor(u0)
    float gx, gy, kx, ky;
    float T0, Az, Bz, Cz;
    int xdrv;
};
constexpr int kAnc = 32; // anchors per chunk: one warp, one view per lane

template <int ZS, int KSEG, int VPT, bool ZSKIP>
__global__ void __launch_bounds__(kCols * ZS, ZS == 4 ? 2 : 1) dd3_back_t_kernel(BackArgs a, int es2, int rmax)
{
    extern __shared__ __align__(128) unsigned char smem[];
    const int vp = a.vp; // P row pitch (floats, multiple of 4)
    // (E, dE) tables: double buffered (B of a view overlaps A of the next) in
    // the 512- and 1024-thread shapes, single buffered in the 256-thread one,
    // which runs two CTAs per SM and separates B from the next A by a barrier
    constexpr int EB = ZS == 4 ? 1 : 2;
    // the piece tables, row-major: entry i of column c at [i][c], so the 16
    // lanes of a half-warp reading 16 consecutive columns hit distinct banks
    // whatever rows they read
    float2 *E2 = reinterpret_cast<float2 *>(smem);                       // [EB][es2][kCols] pieces
    float *pbuf = reinterpret_cast<float *>(E2 + EB * (size_t)kCols * es2); // [2][rmax][vp]
    __shared__ __align__(8) uint64_t s_bar[2];
    __shared__ int s_ulo[2], s_rows[2];
    __shared__ float s_u[kGeo][kB][kB + 1]; // boundaries on the detector, relative to s_iu0
    __shared__ int s_iu0[kGeo];
    __shared__ Anchor s_anc[2][kAnc];       // chunks of view anchors, double buffered
    __shared__ float s_V0[kGeo][kCols], s_V1[kGeo][kCols];
    __shared__ int s_xdrv[kGeo];
    __shared__ int s_cov[kGeo][2]; // the view's cone meets this CTA's z range (per column half)
    __shared__ __align__(16) ASet s_aset[kGeo][kCols];

    const int tid = threadIdx.x;
    const int bx0 = blockIdx.x * kB, by0 = (blockIdx.y + a.by_off) * kB;
    const int col = tid & (kCols - 1), zs = tid / kCols;
    const int cx = col & (kB - 1), cy = col / kB;
    const int x = bx0 + cx, y = by0 + cy;
    const int k0 = blockIdx.z * (ZS * KSEG) + zs * KSEG;
    const int DNU = a.DNU, DNV = a.DNV, ZN = a.ZN;
    // the list positions this CTA visits: all, or (ZSKIP) the range of views
    // whose cone can meet its z block
    int lb = 0, n = a.n;
    if (ZSKIP && a.zrange) {
        const int2 r = a.zrange[blockIdx.z];
        lb = r.x;
        n = max(r.y - r.x, 0);
    }
    // geometry constants are re-read from the kernel parameters (constant
    // bank) where they are used, so they hold no registers across the loop
    const DetTable t = det_table_layout(DNU, DNV);
    __shared__ double s_zb0; // local z of the detector's first row boundary
    if (tid == 0) s_zb0 = a.det[t.off_bz];
    const bool in_vol = (x < a.XN) && (y < a.YN);
    const float DNVf = (float)DNV;
    // z boundaries this CTA's phase B samples (its segments' k0 .. k0 + KSEG)
    const float kz_lo = (float)(blockIdx.z * (ZS * KSEG)), kz_hi = kz_lo + (float)(ZS * KSEG);

    if (tid == 0) {
        mbar_init(&s_bar[0], 1);
        mbar_init(&s_bar[1], 1);
        mbar_fence_init();
    }

    // FP64 anchors of list entries chunk * kAnc .. + kAnc - 1 into
    // s_anc[chunk & 1] (warp 3, one view per lane)
    auto anchors = [&](int chunk) {
        const int i = tid - 96;
        const int l = chunk * kAnc + i;
        if (i < 0 || i >= kAnc || l >= n) return;
        const DevView &V = a.views[a.view_list[lb + l]];
        const double dpx = a.x_c0 + ((double)bx0 + 3.5) * a.dx - V.Sx;
        const double dpy = a.y_c0 + ((double)by0 + 3.5) * a.dx - V.Sy;
        const double D0 = cross2(V.Ex, V.Ey, dpx, dpy);                     // D(c)
        const double N0 = cross2(V.Sx - V.B0x, V.Sy - V.B0y, dpx, dpy);     // N(c)
        const double rD = 1.0 / D0, u0 = N0 * rD;
        const double dDx = -V.Ey, dDy = V.Ex;                    // grad D
        const double dNx = V.B0y - V.Sy, dNy = V.Sx - V.B0x;     // grad N
        Anchor an;
        const double fl = floor(u0);
        an.iu0 = (int)fl;
        an.fu0 = (float)(u0 - fl);
        an.gx = (float)((dNx - u0 * dDx) * a.dx * rD);
        an.gy = (float)((dNy - u0 * dDy) * a.dx * rD);
        an.kx = (float)(dDx * a.dx * rD);
        an.ky = (float)(dDy * a.dx * rD);
        // central-ray magnification cross2(B0 - S, E) / cross2(c - S, E), the
        // denominator being -D(c); z boundary k' -> detector row v = V0 + V1 k'
        const double zb0 = s_zb0 + V.zP;
        const double inv_n = 1.0 / (a.dzb * a.DNV); // detector rows, normalised by DNV
        an.T0 = (float)(-cross2(V.B0x - V.Sx, V.B0y - V.Sy, V.Ex, V.Ey) * rD);
        an.Az = (float)((V.Sz - zb0) * inv_n);
        an.Bz = (float)((a.z_lo - V.Sz) * inv_n);
        an.Cz = (float)(a.dz * inv_n);
        an.xdrv = V.xdrv;
        s_anc[chunk & 1][i] = an;
    };
    // per-view geometry of view list entry l into slot l % kGeo, from its
    // anchor: the brick's voxel boundaries across the driving axis on the
    // detector (warps 0-2) and each column's z -> v map (warps 4-5)
    auto geometry = [&](int l) {
        if (l >= n) return;
        const Anchor &an = s_anc[(l / kAnc) & 1][l % kAnc];
        const int sl = l % kGeo;
        if (tid < kB * (kB + 1)) {
            // boundary q (voxel q - 1/2) across the driving axis, voxel row r
            // along it, as offsets from the brick centre
            const int r = tid / (kB + 1), q = tid - r * (kB + 1);
            const float oq = (float)q - 4.f, orr = (float)r - 3.5f;
            const float ox = an.xdrv ? orr : oq, oy = an.xdrv ? oq : orr;
            s_u[sl][r][q] = an.fu0 + fmaf(an.gx, ox, an.gy * oy) / fmaf(an.kx, ox, fmaf(an.ky, oy, 1.f));
            if (tid == 0) {
                s_xdrv[sl] = an.xdrv;
                s_iu0[sl] = an.iu0;
            }
        } else if (tid >= 128 && tid < 128 + kCols) {
            const int c = tid - 128;
            const float ox = (float)(c & (kB - 1)) - 3.5f, oy = (float)(c / kB) - 3.5f;
            const float tc = an.T0 / fmaf(an.kx, ox, fmaf(an.ky, oy, 1.f));
            const float V1 = an.Cz * tc, V0 = fmaf(an.Bz, tc, an.Az);
            s_V1[sl][c] = V1;
            s_V0[sl][c] = V0;
            if (ZSKIP) {
                // does this column's z range [kz_lo, kz_hi] reach a detector
                // row?  Outside, every boundary saturates to the same end of
                // the column and the view adds exactly 0 (a helical scan's
                // views far along z)
                const float va = fmaf(V1, kz_lo, V0), vb = fmaf(V1, kz_hi, V0);
                const bool meets = fmaxf(va, vb) > -1e-3f && fminf(va, vb) < 1.f + 1e-3f;
                const unsigned any = __ballot_sync(0xffffffffu, meets);
                if ((tid & 31) == 0) s_cov[sl][(tid - 128) >> 5] = any != 0u;
            }
        }
    };
    // the detector cells [lo, lo + rows) the brick's footprint covers in slot
    // sl (from its corner boundaries; one cell of margin each side)
    auto footprint = [&](int sl, int &lo, int &rows) {
        const float c0 = s_u[sl][0][0], c1 = s_u[sl][0][kB], c2 = s_u[sl][kB - 1][0], c3 = s_u[sl][kB - 1][kB];
        const int iu = s_iu0[sl];
        const int fmin_i = iu + (int)floorf(fminf(fminf(c0, c1), fminf(c2, c3)));
        const int fmax_i = iu + (int)floorf(fmaxf(fmaxf(c0, c1), fmaxf(c2, c3)));
        lo = max(min(max(fmin_i, 0), DNU - 1) - 1, 0);
        rows = min(min(max(fmax_i, 0), DNU - 1) + 2, DNU - 1) - lo + 1;
    };
    // a boundary (relative to iu) clamped to the detector [0, DNU]: its cell
    // and the fraction of the cell below it
    auto cell = [&](float ul, int iu, int &i, float &f) {
        const float uc = fminf(fmaxf(ul, (float)-iu), (float)(DNU - iu));
        i = max(min(iu + (int)floorf(uc), DNU - 1), 0);
        f = uc - (float)(i - iu);
    };
    // staging of list entry l into buffer l & 1 (thread 0): the rows of P the
    // brick's footprint covers, from the corner boundaries of its geometry
    auto issue = [&](int l) {
        if (tid != 0 || l >= n) return;
        const int b = l & 1, sl = l % kGeo;
        // one row of margin each side: interior boundaries may round past
        // the corners' range
        int lo, rows;
        footprint(sl, lo, rows);
        const bool meets = !ZSKIP || s_cov[sl][0] || s_cov[sl][1];
        const bool fits = meets && rows <= rmax;
        s_ulo[b] = lo;
        s_rows[b] = meets ? (fits ? rows : 0) : -1; // -1: the view misses the brick
        mbar_arrive_expect_tx(&s_bar[b], fits ? (uint32_t)(4 * rows * vp) : 0u);
        if (fits)
            bulk_copy_g2s(pbuf + (size_t)b * rmax * vp, a.pv + ((long long)(lb + l) * DNU + lo) * vp,
                          (uint32_t)(4 * rows * vp), &s_bar[b]);
    };

    // phase-A set-up of list entry l into slot l % kGeo (threads 256..319,
    // or 192..255 in the 256-thread shape; one per column): the same staging origin as issue(l), from the same
    // corner boundaries
    auto setup = [&](int l) {
        constexpr int kSet0 = ZS == 4 ? 192 : 256; // a pair of warps the geometry leaves free
        if (l >= n || tid < kSet0 || tid >= kSet0 + kCols) return;
        const int c = tid - kSet0, sl = l % kGeo;
        const int ccx = c & (kB - 1), ccy = c / kB;
        int lo, rows;
        footprint(sl, lo, rows);
        const int xd = s_xdrv[sl], iu = s_iu0[sl];
        const float ua = xd ? s_u[sl][ccx][ccy] : s_u[sl][ccy][ccx];
        const float ub = xd ? s_u[sl][ccx][ccy + 1] : s_u[sl][ccy][ccx + 1];
        int ia, ib;
        float fa, fb;
        cell(ua, iu, ia, fa);
        cell(ub, iu, ib, fb);
        const float sg = ((ub - ua > 0) ? 1.f : -1.f) * ((s_V1[sl][c] > 0.f) ? 1.f : -1.f);
        const int dc = ib - ia;
        float wa, wb;
        if (dc == 0) {
            wa = fb - fa;
            wb = 0.f;
        } else if (dc > 0) {
            wa = 1.f - fa;
            wb = fb;
        } else {
            wa = -fa;
            wb = fb - 1.f;
        }
        const int nm = max(abs(dc) - 1, 0), first = min(ia, ib) + 1;
        const float wm = dc > 0 ? sg : -sg;
        const uint32_t vp4 = 4u * (uint32_t)a.vp;
        auto row = [&](int u) { return (uint32_t)min(max(u - lo, 0), max(rows - 1, 0)) * vp4; };
        ASet st;
        st.off[0] = row(ia);
        st.off[1] = row(ib);
#pragma unroll
        for (int m = 0; m < 3; ++m) {
            st.off[2 + m] = row(min(first + m, max(ia, ib)));
            st.wm[m] = m < nm ? wm : 0.f;
        }
        st.wa = wa * sg;
        st.wb = wb * sg;
        st.nm = nm;
        st.pad = 0;
        s_aset[sl][c] = st;
    };

    __syncthreads(); // s_zb0 visible
    anchors(0);
    __syncthreads(); // the first chunk of anchors visible
    geometry(0);
    geometry(1);
    geometry(2);
    __syncthreads(); // barrier init and geometry visible
    issue(0);
    issue(1);
    setup(0);
    setup(1);
    __syncthreads();

    float acc[KSEG];
#pragma unroll
    for (int r = 0; r < KSEG; ++r) acc[r] = 0.f;
    bool timed_out = false;
    const uint32_t E2_addr = smem_addr(E2);
    // phase A: kAPh threads per column, each a run of vpt consecutive rows.
    // A warp's lanes are 32 columns with the same run, 4 across the view's
    // detector axis x 8 along it, so the P rows its strips read lie within a
    // few cells (distinct banks: the row pitch is 4 mod 8 floats), and its
    // table stores (column slots e_slot) hit distinct banks.  (With 8
    // columns x 4 runs a warp the stores conflicted: 45.4 vs 42.1 ms at
    // 512x512x256 / 984 views.)
    constexpr int kAPh = ZS;
    const int aph = tid / kCols, alane = tid & 31, ahalf = (tid >> 5) & 1;
    const int i0 = aph * VPT; // this thread's entries i0 .. i0+VPT-1 (kAPh*VPT > DNV)
    const float nfi0 = -(float)i0;
    const int eslot_b = e_slot(cx, cy); // phase B's column

    for (int li = 0; li < n; ++li) {
        const int b = li & 1, ls = li % kGeo;
        const int ulo = s_ulo[b], rows = s_rows[b];
        // warp-uniform, so the warp collectives of phase A stay converged
        if (__any_sync(0xffffffffu, !mbar_wait(&s_bar[b], (uint32_t)((li >> 1) & 1)))) timed_out = true;
        const int xdrv = s_xdrv[ls];
        const int eb = EB == 2 ? b : 0;
        float2 *E = E2 + (size_t)eb * kCols * es2; // double buffered: B(li) overlaps A(li+1)
        // this thread's phase-A column: the detector u axis runs along x
        // for y-driven views and along y for x-driven ones
        const int across = (alane & 3) + 4 * ahalf, along = alane >> 2;
        const int acx = xdrv ? along : across, acy = xdrv ? across : along;
        const int ac = acx + kB * acy, eslot_a = e_slot(acx, acy);

        // ---- A: (E_c(i), E_c(i+1) - E_c(i)) for i in [0, DNV], E_c(DNV+1) = E_c(DNV) ----
        // the thread's column strip for this view, recomputed from s_u (the
        // paths the hoisted set-up does not cover)
        struct Strip {
            int ia, ib, nm, first;
            float wa, wb, wm;
        };
        auto strip = [&]() {
            Strip st;
            const float ua = xdrv ? s_u[ls][acx][acy] : s_u[ls][acy][acx];
            const float ub = xdrv ? s_u[ls][acx][acy + 1] : s_u[ls][acy][acx + 1];
            float fa, fb;
            cell(ua, s_iu0[ls], st.ia, fa);
            cell(ub, s_iu0[ls], st.ib, fb);
            const float sgn = ((ub - ua > 0) ? 1.f : -1.f) * ((s_V1[ls][ac] > 0.f) ? 1.f : -1.f);
            const int dc = st.ib - st.ia;
            float wa, wb;
            if (dc == 0) {
                wa = fb - fa;
                wb = 0.f;
            } else if (dc > 0) {
                wa = 1.f - fa;
                wb = fb;
            } else {
                wa = -fa;
                wb = fb - 1.f;
            }
            st.wa = wa * sgn;
            st.wb = wb * sgn;
            // whole cells strictly between a and b
            st.nm = max(abs(dc) - 1, 0);
            st.first = min(st.ia, st.ib) + 1;
            st.wm = dc > 0 ? sgn : -sgn;
            return st;
        };

        if (!timed_out && rows > 0) {
            // staged rows, set-up from s_aset: 32-bit shared addresses, row u at
            // pbase + (u - ulo) * vp4; the pitch covers i0+VPT, and entries past
            // DNV repeat the total
            const uint4 q0 = *reinterpret_cast<const uint4 *>(&s_aset[ls][ac].off[0]);
            const uint4 q1 = *reinterpret_cast<const uint4 *>(&s_aset[ls][ac].off[4]);
            const uint4 q2 = *reinterpret_cast<const uint4 *>(&s_aset[ls][ac].wm[1]);
            const uint32_t pbase = smem_addr(pbuf + (size_t)b * rmax * vp) + 4u * (uint32_t)i0;
            const uint32_t pa = pbase + q0.x, pb = pbase + q0.y;
            const uint32_t pm[3] = {pbase + q0.z, pbase + q0.w, pbase + q1.x};
            const float wa = __uint_as_float(q1.y), wb = __uint_as_float(q1.z);
            const float wmv[3] = {__uint_as_float(q1.w), __uint_as_float(q2.x), __uint_as_float(q2.y)};
            // the warp runs its widest column's whole-cell count, the others with weight 0
            const int nmax = (int)__reduce_max_sync(0xffffffffu, q2.z);
            const uint32_t eout = E2_addr + 8u * (uint32_t)((eb * es2 + i0) * kCols + eslot_a);
            switch (nmax) {
            case 0: phase_a_run<VPT, 0>(pa, pb, pm, wmv, wa, wb, nfi0, DNVf, eout); break;
            case 1: phase_a_run<VPT, 1>(pa, pb, pm, wmv, wa, wb, nfi0, DNVf, eout); break;
            case 2: phase_a_run<VPT, 2>(pa, pb, pm, wmv, wa, wb, nfi0, DNVf, eout); break;
            case 3: phase_a_run<VPT, 3>(pa, pb, pm, wmv, wa, wb, nfi0, DNVf, eout); break;
            default: {
                // cells much wider than voxels: the whole cells by a loop
                const Strip st = strip();
                const uint32_t vp4 = 4u * (uint32_t)vp;
                const uint32_t sbase = smem_addr(pbuf + (size_t)b * rmax * vp) + 4u * (uint32_t)i0;
                auto row = [&](int u) { return sbase + (uint32_t)min(max(u - ulo, 0), rows - 1) * vp4; };
                float2 *Ec = E + eslot_a;
                float e = 0.f;
                for (int j = 0; j <= VPT; ++j) {
                    const uint32_t o = 4u * (uint32_t)j;
                    float en = fmaf(st.wb, lds_f32(row(st.ib) + o), st.wa * lds_f32(row(st.ia) + o));
                    for (int m = 0; m < st.nm; ++m) en = fmaf(st.wm, lds_f32(row(st.first + m) + o), en);
                    if (j > 0) Ec[(i0 + j - 1) * kCols] = affine_piece(e, en, (float)(i0 + j - 1), DNVf);
                    e = en;
                }
            }
            }
        } else if (!timed_out && (!ZSKIP || rows >= 0)) {
            // footprint wider than a stage: P from global memory
            const Strip st = strip();
            const float *Pg = a.pv + (long long)(lb + li) * DNU * vp;
            float2 *Ec = E + eslot_a;
            auto eval = [&](int i) {
                float e = fmaf(st.wb, __ldg(Pg + (size_t)st.ib * vp + i), st.wa * __ldg(Pg + (size_t)st.ia * vp + i));
                for (int m = 0; m < st.nm; ++m) e = fmaf(st.wm, __ldg(Pg + (size_t)(st.first + m) * vp + i), e);
                return e;
            };
            float e = eval(i0);
            for (int j = 0; j < VPT; ++j) {
                const float en = eval(i0 + j + 1);
                Ec[(i0 + j) * kCols] = affine_piece(e, en, (float)(i0 + j), DNVf);
                e = en;
            }
        }
        __syncthreads();

        // ---- stage view li+2 into the buffer just consumed; geometry of li+3 ----
        issue(li + 2);
        // the next chunk of anchors, first read kAnc - 3 views from here
        if (li % kAnc == 0) anchors(li / kAnc + 1);
        geometry(li + 3);
        setup(li + 2);

        // ---- phase B: voxels ----
        if (in_vol && !timed_out && (!ZSKIP || rows >= 0)) {
            const float V0 = s_V0[ls][col], V1 = s_V1[ls][col];
            // address of piece i of this column = bits(i + 2^23) * 8 kCols + base (mod 2^32)
            const uint32_t base = E2_addr + 8u * (uint32_t)(eb * kCols * es2 + eslot_b) - 8u * kCols * 0x4B000000u;
            const float vb0 = fmaf(V1, (float)k0, V0);
            float prev = 0.f;
#pragma unroll
            for (int r = 0; r <= KSEG; ++r) {
                const float vn = __saturatef(fmaf(V1, (float)r, vb0));
                const float rr = __fmaf_rz(vn, DNVf, 8388608.f); // 2^23 + floor(DNV vn)
                const float2 pc = lds_f32x2(__float_as_uint(rr) * (8u * kCols) + base);
                const float ev = fmaf(vn, pc.y, pc.x); // E_c(DNV vn)
                if (r > 0) acc[r - 1] += ev - prev;
                prev = ev;
            }
        }
        if constexpr (EB == 1) __syncthreads(); // the single E table is rewritten by the next A
    }
    if (timed_out && a.err) atomicExch(a.err, CTLAB_ERR_TIMEOUT);

    if (!in_vol) return;
    const long long colidx = (long long)y * a.XN + x;
    const float m = a.mask ? (a.mask[colidx] ? 1.f : 0.f) : 1.f;
    float *o = a.out + colidx * ZN;
    if (a.epilogue == BACK_SART_UPDATE) {
        // x = (x + lambda * acc / colSum) * mask, eight voxels at a time: their
        // loads are issued together (the image and the column sums are read
        // through different pointers, so the compiler would otherwise keep each
        // load behind the previous voxel's store)
        const float *cs_col = a.col_sum + colidx * ZN;
#pragma unroll
        for (int r0 = 0; r0 < KSEG; r0 += 8) {
            float cs[8], xv[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const int k = k0 + r0 + q;
                cs[q] = 0.f;
                xv[q] = 0.f;
                if (r0 + q < KSEG && k < ZN) {
                    cs[q] = __ldg(cs_col + k);
                    xv[q] = o[k];
                }
            }
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const int k = k0 + r0 + q;
                if (r0 + q < KSEG && k < ZN) {
                    const float upd = (cs[q] > 1.0e-7f) ? acc[r0 + q] / cs[q] : 0.f;
                    float v = (xv[q] + a.lambda * upd) * m;
                    if (a.clamp) v = fminf(fmaxf(v, a.min_v), a.max_v);
                    o[k] = v;
                }
            }
        }
    } else {
#pragma unroll
        for (int r = 0; r < KSEG; ++r) {
            const int k = k0 + r;
            if (k < ZN) o[k] = acc[r] * m;
        }
    }
}

// Projection v-prefixes: one warp per detector column (view l, cell u) scans
// the weighted column in FP64 32 rows at a time with shuffles and a carried
// total; out[l][u][v'] for v' in [0, DNV], entries past DNV repeat the total.
__global__ void __launch_bounds__(256) pv_kernel(PrjIn in, long long ncols, int DNU, int DNV, float *__restrict__ out,
                                                 int vp)
{
    const int lane = threadIdx.x & 31;
    const long long cidx = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (cidx >= ncols) return;
    const int l = (int)(cidx / DNU), u = (int)(cidx - (long long)l * DNU);
    float *o = out + cidx * vp;
    double carry = 0.0;
    if (lane == 0) o[0] = 0.f;
    for (int v0 = 0; v0 < DNV; v0 += 32) {
        const int v = v0 + lane;
        double s = v < DNV ? (double)in(l, u, v) : 0.0;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const double y = __shfl_up_sync(0xffffffffu, s, d);
            if (lane >= d) s += y;
        }
        s += carry;
        if (v < DNV) o[v + 1] = (float)s;
        carry = __shfl_sync(0xffffffffu, s, 31);
    }
    for (int v = DNV + 1 + lane; v < vp; v += 32) o[v] = (float)carry;
}

// Rows of E per phase-A thread with ZS threads per column: ZS * VPT > DNV,
// from a few compiled sizes.
int vpt_of(int DNV, int zs)
{
    const int need = (DNV + 1 + zs - 1) / zs;
    for (int v : {2, 5, 9, 17, 33})
        if (v >= need) return v;
    return 0;
}
int e_pitch(int DNV, int zs) { return (zs * vpt_of(DNV, zs)) | 1; }
// the largest (E, dE) pitch over the two block shapes
int e_pitch_max(int DNV) { return std::max(std::max(e_pitch(DNV, 8), e_pitch(DNV, 16)), e_pitch(DNV, 4)); }

// z segments per column forced by CTLAB_BACKT_ZS (4, 8, 16), or 0: chosen
// per launch (launch_shape).  All shapes give the same results.  On the
// B200 at 512x512x256 / 984 views: 42.1 ms with 256 threads (4); with the
// earlier phase-A lane order, 45.4 ms (4) and 52.3 ms (8).  A warp's
// per-view bookkeeping (loop, waits, slot addresses, phase-A
// set-up loads) is spread over the voxels of its threads' segments, 64 / 32
// / 16 of them; the 256-thread shape still runs 16 warps per SM, as two
// independent CTAs whose barriers do not align.
int back_t_zs()
{
    static const int zs = [] {
        const char *e = std::getenv("CTLAB_BACKT_ZS");
        const int v = e ? std::atoi(e) : 0;
        return (v == 4 || v == 8 || v == 16) ? v : 0;
    }();
    return zs;
}
size_t dyn_smem(int rmax, int vp, int es2, int ebuf = 2)
{
    return 4 * 2 * (size_t)rmax * vp + sizeof(float2) * (size_t)ebuf * kCols * es2;
}

// Per z block of zblk voxels (one CTA each): the first and one-past-last list
// positions of the views whose cone can meet the block anywhere over the
// volume's footprint.  A voxel at height z meets the detector when the ray's
// detector z, S_z + t (z - S_z), lies within the rows; t = 1 / w with w the
// point's distance from the source over the detector's, linear in the point,
// so its extremes are at the footprint's corners.  One voxel of margin.
__global__ void __launch_bounds__(256) zrange_kernel(BackArgs a, int zblk, int2 *out)
{
    __shared__ int s_lo[8], s_hi[8];
    const int bz = blockIdx.x;
    const double zb_lo = a.z_lo + (double)bz * zblk * a.dz - a.dz;
    const double zb_hi = a.z_lo + (double)min((bz + 1) * zblk, a.ZN) * a.dz + a.dz;
    const DetTable t = det_table_layout(a.DNU, a.DNV);
    const double d_lo = fmin(a.det[t.off_bz], a.det[t.off_bz + a.DNV]);
    const double d_hi = fmax(a.det[t.off_bz], a.det[t.off_bz + a.DNV]);
    const double x0 = a.x_c0 - 0.5 * a.dx, x1 = x0 + a.XN * a.dx;
    const double y0 = a.y_c0 - 0.5 * a.dx, y1 = y0 + a.YN * a.dx;
    int lo = INT_MAX, hi = -1;
    for (int l = threadIdx.x; l < a.n; l += blockDim.x) {
        const DevView &V = a.views[a.view_list[l]];
        const double den = cross2(V.B0x - V.Sx, V.B0y - V.Sy, V.Ex, V.Ey);
        double wmin = 1e300, wmax = -1e300;
        for (int c = 0; c < 4; ++c) {
            const double px = (c & 1) ? x1 : x0, py = (c & 2) ? y1 : y0;
            const double w = cross2(px - V.Sx, py - V.Sy, V.Ex, V.Ey) / den;
            wmin = fmin(wmin, w);
            wmax = fmax(wmax, w);
        }
        bool meets = true;
        if (wmin > 0.0) {
            const double e0 = d_lo + V.zP - V.Sz, e1 = d_hi + V.zP - V.Sz;
            const double zlo = V.Sz + fmin(fmin(wmin * e0, wmax * e0), fmin(wmin * e1, wmax * e1));
            const double zhi = V.Sz + fmax(fmax(wmin * e0, wmax * e0), fmax(wmin * e1, wmax * e1));
            meets = zhi >= zb_lo && zlo <= zb_hi;
        }
        if (meets) {
            lo = min(lo, l);
            hi = max(hi, l);
        }
    }
    lo = (int)__reduce_min_sync(0xffffffffu, (unsigned)lo);
    hi = __reduce_max_sync(0xffffffffu, hi);
    if ((threadIdx.x & 31) == 0) {
        s_lo[threadIdx.x >> 5] = lo;
        s_hi[threadIdx.x >> 5] = hi;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
            lo = min(lo, s_lo[w]);
            hi = max(hi, s_hi[w]);
        }
        out[bz] = hi >= lo ? make_int2(lo, hi + 1) : make_int2(0, 0);
    }
}

// With q set, a launch is not made: q receives the CTAs one launch of this
// kernel keeps resident on the device and the CTAs of one brick row.
struct BackLaunchQuery {
    int resident = 0, ctas_per_row = 0;
};

template <int ZS, int KSEG, int VPT, bool ZSKIP>
cudaError_t launch_k(const BackArgs &a, cudaStream_t s, BackLaunchQuery *q)
{
    const int es2 = e_pitch(a.DNV, ZS); // pieces per column
    const size_t sm = dyn_smem(a.rmax, a.vp, es2, ZS == 4 ? 1 : 2);
    auto kern = dd3_back_t_kernel<ZS, KSEG, VPT, ZSKIP>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    const int bys = (a.YN + kB - 1) / kB;
    if (a.by_off < 0 || a.by_count < 0 || (a.by_count == 0 && a.by_off != 0) || a.by_off + a.by_count > bys)
        return cudaErrorInvalidValue;
    dim3 grid((a.XN + kB - 1) / kB, a.by_count > 0 ? a.by_count : bys, (a.ZN + ZS * KSEG - 1) / (ZS * KSEG));
    if (q) {
        int dev = 0, sms = 0, per_sm = 0;
        e = cudaGetDevice(&dev);
        if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kCols * ZS, sm);
        q->resident = sms * per_sm;
        q->ctas_per_row = (int)(grid.x * grid.z);
        return e;
    }
    if (ZSKIP && a.zrange) {
        zrange_kernel<<<grid.z, 256, 0, s>>>(a, ZS * KSEG, a.zrange);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    kern<<<grid, kCols * ZS, sm, s>>>(a, es2, a.rmax);
    return cudaGetLastError();
}

// Segment length by ZN (z blocks of 256 voxels at most); volumes of several
// z blocks (and helical scans) test each view against each CTA's z range and
// skip the views whose cone misses it.  256 threads: segments up to 64
// voxels; 512 threads: up to 32; 1024 threads: up to 16.
template <int ZS, int VPT>
cudaError_t launch_z(const BackArgs &a, cudaStream_t s, BackLaunchQuery *q)
{
    constexpr int KMAX = 256 / ZS;
    if (a.ZN <= ZS * 4) return launch_k<ZS, 4, VPT, false>(a, s, q);
    if (a.ZN <= ZS * 8) return launch_k<ZS, 8, VPT, false>(a, s, q);
    if (ZS * 16 < 256 && a.ZN <= ZS * 16) return launch_k<ZS, 16, VPT, false>(a, s, q);
    if (ZS * 32 < 256 && a.ZN <= ZS * 32) return launch_k<ZS, 32, VPT, false>(a, s, q);
    if (a.zskip || a.ZN > 256) return launch_k<ZS, KMAX, VPT, true>(a, s, q);
    return launch_k<ZS, KMAX, VPT, false>(a, s, q);
}

template <int ZS>
cudaError_t launch_vpt(const BackArgs &a, cudaStream_t s, BackLaunchQuery *q)
{
    switch (vpt_of(a.DNV, ZS)) {
    case 2: return launch_z<ZS, 2>(a, s, q);
    case 5: return launch_z<ZS, 5>(a, s, q);
    case 9: return launch_z<ZS, 9>(a, s, q);
    case 17: return launch_z<ZS, 17>(a, s, q);
    case 33: return launch_z<ZS, 33>(a, s, q);
    default: return cudaErrorInvalidValue;
    }
}

// The launch's block shape: CTLAB_BACKT_ZS=4, 8 or 16 forces it; otherwise
// 256 threads (two CTAs per SM), the fastest at every view count measured
// (B200: 24 ... 984 views at 512x512x256 and 256x256x128; OS-SART with 24
// subsets of 30 views at 256x256x128, 40.8 vs 42.4 ms per iteration with
// the fused update on 512 threads).
cudaError_t launch_shape(const BackArgs &a, cudaStream_t s, BackLaunchQuery *q)
{
    int zs = back_t_zs();
    if (zs == 0) zs = 4;
    if (zs == 4 && vpt_of(a.DNV, 4) == 0) zs = 8;
    if (zs == 4) return launch_vpt<4>(a, s, q);
    return zs == 16 ? launch_vpt<16>(a, s, q) : launch_vpt<8>(a, s, q);
}

} // namespace

bool back_t_supported(int DNV)
{
    if (vpt_of(DNV, 8) == 0 || vpt_of(DNV, 16) == 0) return false;
    return dyn_smem(2, back_t_pitch(DNV), e_pitch_max(DNV)) + kStaticSmem <= 227 * 1024;
}

// P row pitch: DNV+1 prefixes, then the total repeated up to the last row a
// phase-A run reads (kAPh * VPT), rounded to 16 bytes
int back_t_pitch(int DNV)
{
    return (std::max(DNV + 2, std::max(std::max(8 * vpt_of(DNV, 8), 16 * vpt_of(DNV, 16)), 4 * vpt_of(DNV, 4)) + 1) +
            3) & ~3;
}

// Staged P rows: the widest u footprint of any brick on the volume's outer
// ring of bricks (nearest the source in some view), +2, capped so two CTAs
// fit an SM (at least 2; wider footprints read global memory).
int back_t_staging_rows(const HostGeometry &g)
{
    const int vp = back_t_pitch(g.DNV);
    const int es2 = e_pitch_max(g.DNV);
    const double x_c0 = g.cx - 0.5 * (g.XN - 1) * g.dx, y_c0 = g.cy - 0.5 * (g.YN - 1) * g.dx;
    const double x_lo = x_c0 - 0.5 * g.dx, y_lo = y_c0 - 0.5 * g.dx;
    const int nbx = (g.XN + kB - 1) / kB, nby = (g.YN + kB - 1) / kB;
    int need = 2;
    auto uof = [](const DevView &V, double px, double py) {
        const double dpx = px - V.Sx, dpy = py - V.Sy;
        const double num = (V.Sx - V.B0x) * dpy - (V.Sy - V.B0y) * dpx;
        return num / (V.Ex * dpy - V.Ey * dpx);
    };
    for (const DevView &V : g.views) {
        for (int by = 0; by < nby; ++by) {
            for (int bx = 0; bx < nbx; ++bx) {
                if (by != 0 && by != nby - 1 && bx != 0 && bx != nbx - 1) continue;
                const int bx0 = bx * kB, by0 = by * kB;
                double px0, px1, py0, py1;
                if (!V.xdrv) {
                    px0 = x_lo + bx0 * g.dx; px1 = x_lo + (bx0 + kB) * g.dx;
                    py0 = y_c0 + by0 * g.dx; py1 = y_c0 + (by0 + kB - 1) * g.dx;
                } else {
                    px0 = x_c0 + bx0 * g.dx; px1 = x_c0 + (bx0 + kB - 1) * g.dx;
                    py0 = y_lo + by0 * g.dx; py1 = y_lo + (by0 + kB) * g.dx;
                }
                const double u0 = uof(V, px0, py0), u1 = uof(V, px1, py0), u2 = uof(V, px0, py1),
                             u3 = uof(V, px1, py1);
                const double umin = std::min(std::max(std::min(std::min(u0, u1), std::min(u2, u3)), 0.0),
                                             (double)(g.DNU - 1));
                const double umax = std::min(std::max(std::max(std::max(u0, u1), std::max(u2, u3)), 0.0),
                                             (double)(g.DNU - 1));
                need = std::max(need, std::min((int)umax + 2, g.DNU - 1) - std::max((int)umin - 1, 0) + 1);
            }
        }
    }
    const size_t fixed = dyn_smem(0, vp, es2) + kStaticSmem;
    const int cap = kSmemPerCta > fixed ? (int)((kSmemPerCta - fixed) / (4 * 2 * (size_t)vp)) : 0;
    return std::max(2, std::min(need, cap));
}

cudaError_t launch_pv(const ProjSatArgs &a, float *out, int vp, cudaStream_t s)
{
    PrjIn in{a.prj, a.views, a.view_list, a.det, det_table_layout(a.DNU, a.DNV), a.DNU, a.DNV, a.dx};
    const long long ncols = (long long)a.n * a.DNU;
    const long long blocks = (ncols * 32 + 255) / 256;
    if (blocks > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
    pv_kernel<<<(unsigned)blocks, 256, 0, s>>>(in, ncols, a.DNU, a.DNV, out, vp);
    return cudaGetLastError();
}

cudaError_t back_t_query(const BackArgs &a, int *resident, int *ctas_per_row)
{
    BackLaunchQuery q;
    cudaError_t e = a.n > 0 ? launch_shape(a, nullptr, &q) : cudaErrorInvalidValue;
    *resident = q.resident;
    *ctas_per_row = q.ctas_per_row;
    return e;
}

cudaError_t launch_back_t(const BackArgs &a, cudaStream_t s, int *launches)
{
    if (launches) ++*launches;
    if (a.n <= 0) return cudaSuccess;
    return launch_shape(a, s, nullptr);
}

} // namespace ctlab
