// Branchless DD cone-beam backprojection (voxel-driven gather over the
// per-view projection SATs).
//
// One CTA (256 threads) owns a brick of 8 x 8 voxel columns (x, y) and a z
// range of 4*KSEG voxels, and loops over the views.  Per view:
//   geometry   the brick's voxel boundaries across the view's driving axis
//              (8 rows of 9 points) are mapped through the source onto the
//              flat detector, u = cross(S-B0, P-S) / cross(E, P-S) (FP64);
//              each column's centre ray gives the affine z -> v map
//              v(k') = V0 + V1 k' over z-boundary indices k';
//   staging    the rows [u_lo, u_hi] of the view's projection SAT that the
//              brick's footprint covers are one contiguous block: a single
//              1-D bulk copy (TMA) brings it into shared memory, double
//              buffered two views ahead and completed on an mbarrier;
//   phase A    for every column c and detector row boundary v', the strip
//              integral of the weighted projection between the column's two
//              u boundaries, E_c(v') = Q(u_{c+1}, v') - Q(u_c, v'), from the
//              staged SAT rows in FP64 (where the large prefix values cancel)
//              and rounded once to FP32;
//   phase B    each voxel samples E_c linearly at its two z boundaries and
//              accumulates the oriented difference in registers (FP32).
// E is double buffered, so one barrier per view separates A(li) from the
// issue of view li+2's copy and B(li).  Views whose
// footprint does not fit the staging buffer read the SAT from global memory
// instead.  The epilogue applies the in-plane mask and optionally fuses the
// OS-SART update
// x = (x + lambda * acc/colSum) * mask.
#include <cmath>

#include "ffloat.cuh"
#include "internal.h"
#include "tma.cuh"

namespace ctlab {

namespace {

constexpr int kB = 8;                 // brick edge (voxel columns)
constexpr int kCols = kB * kB;        // 64 columns per CTA
constexpr int kZS = 4;                // z segments per column
constexpr int kThreads = kCols * kZS; // 256
constexpr size_t kSmemPerCta = 110 * 1024; // two CTAs per SM
constexpr size_t kStaticSmem = 5 * 1024;

__device__ __forceinline__ double q_ld(const double *p) { return *p; }
__device__ __forceinline__ ff2 q_ld(const ff2 *p)
{
    const float2 f = *reinterpret_cast<const float2 *>(p);
    return {f.x, f.y};
}
// Q(u_b) - Q(u_a) with Q(i + f) = Q_i + f (Q_{i+1} - Q_i), in FP64 (or
// float-float), rounded once to FP32.
__device__ __forceinline__ float strip(double a0, double a1, double b0, double b1, double fa, double fb)
{
    return (float)((b0 - a0) + (fb * (b1 - b0) - fa * (a1 - a0)));
}
__device__ __forceinline__ float strip(ff2 a0, ff2 a1, ff2 b0, ff2 b1, double fa, double fb)
{
    const ff2 d = ff_sub(b0, a0);
    const ff2 tb = ff_mul_f(ff_sub(b1, b0), (float)fb);
    const ff2 ta = ff_mul_f(ff_sub(a1, a0), (float)fa);
    return ff_to_float(ff_add(d, ff_sub(tb, ta)));
}

__device__ __forceinline__ float e_sample(const float *col, float v, int dnv)
{
    v = fminf(fmaxf(v, 0.f), (float)dnv);
    int i = (int)v;
    i = min(i, dnv - 1);
    const float f = v - (float)i;
    const float e0 = col[i], e1 = col[i + 1];
    return fmaf(f, e1 - e0, e0);
}

__device__ __forceinline__ double cross2(double ax, double ay, double bx, double by)
{
    return ax * by - ay * bx;
}

__device__ __forceinline__ double u_of(const DevView &V, double px, double py)
{
    const double dpx = px - V.Sx, dpy = py - V.Sy;
    return cross2(V.Sx - V.B0x, V.Sy - V.B0y, dpx, dpy) / cross2(V.Ex, V.Ey, dpx, dpy);
}

template <int KSEG, class T>
__global__ void __launch_bounds__(kThreads, 2) dd3_back_kernel(BackArgs a, int es, int rmax)
{
    extern __shared__ __align__(128) unsigned char smem[];
    T *qbuf = reinterpret_cast<T *>(smem);                                             // [2][rmax][vp]
    float *E2 = reinterpret_cast<float *>(smem + sizeof(T) * 2 * (size_t)rmax * a.vp); // [2][kCols][es]
    __shared__ __align__(8) uint64_t s_bar[2];
    __shared__ int s_ulo[2], s_rows[2];
    __shared__ double s_u[3][kB][kB + 1];
    __shared__ float s_V0[3][kCols], s_V1[3][kCols];

    const int tid = threadIdx.x;
    const int bx0 = blockIdx.x * kB, by0 = blockIdx.y * kB;
    const int col = tid & (kCols - 1), zs = tid / kCols;
    const int cx = col & (kB - 1), cy = col / kB;
    const int x = bx0 + cx, y = by0 + cy;
    const int k0 = blockIdx.z * (kZS * KSEG) + zs * KSEG;
    const int DNU = a.DNU, DNV = a.DNV, vp = a.vp, ZN = a.ZN, n = a.n;
    const double dx = a.dx;
    const double x_lo = a.x_c0 - 0.5 * dx, y_lo = a.y_c0 - 0.5 * dx;
    const DetTable t = det_table_layout(DNU, DNV);
    const double zb0_local = a.det[t.off_bz];
    const bool in_vol = (x < a.XN) && (y < a.YN);
    const T *Qall = reinterpret_cast<const T *>(a.q);
    const long long qstride = (long long)(DNU + 1) * vp;

    if (tid == 0) {
        mbar_init(&s_bar[0], 1);
        mbar_init(&s_bar[1], 1);
        mbar_fence_init();
    }

    // per-view geometry of view list entry l into slot l % 3
    auto geometry = [&](int l) {
        if (l >= n) return;
        const DevView &V = a.views[a.view_list[l]];
        const int sl = l % 3;
        if (tid < kB * (kB + 1)) {
            const int r = tid / (kB + 1), q = tid - r * (kB + 1);
            double px, py;
            if (!V.xdrv) {
                px = x_lo + (double)(bx0 + q) * dx;
                py = a.y_c0 + (double)(by0 + r) * dx;
            } else {
                px = a.x_c0 + (double)(bx0 + r) * dx;
                py = y_lo + (double)(by0 + q) * dx;
            }
            s_u[sl][r][q] = u_of(V, px, py);
        } else if (tid >= 128 && tid < 128 + kCols) {
            const int c = tid - 128;
            const double pcx = a.x_c0 + (double)(bx0 + (c & (kB - 1))) * dx;
            const double pcy = a.y_c0 + (double)(by0 + c / kB) * dx;
            const double tc = cross2(V.B0x - V.Sx, V.B0y - V.Sy, V.Ex, V.Ey) /
                              cross2(pcx - V.Sx, pcy - V.Sy, V.Ex, V.Ey);
            const double zb0 = zb0_local + V.zP;
            s_V1[sl][c] = (float)(tc * a.dz / a.dzb);
            s_V0[sl][c] = (float)((V.Sz + tc * (a.z_lo - V.Sz) - zb0) / a.dzb);
        }
    };
    // staging of list entry l into buffer l & 1 (thread 0)
    auto issue = [&](int l) {
        if (tid != 0 || l >= n) return;
        const DevView &V = a.views[a.view_list[l]];
        const int b = l & 1;
        double px0, px1, py0, py1;
        if (!V.xdrv) {
            px0 = x_lo + bx0 * dx; px1 = x_lo + (bx0 + kB) * dx;
            py0 = a.y_c0 + by0 * dx; py1 = a.y_c0 + (by0 + kB - 1) * dx;
        } else {
            px0 = a.x_c0 + bx0 * dx; px1 = a.x_c0 + (bx0 + kB - 1) * dx;
            py0 = y_lo + by0 * dx; py1 = y_lo + (by0 + kB) * dx;
        }
        const double u0 = u_of(V, px0, py0), u1 = u_of(V, px1, py0), u2 = u_of(V, px0, py1), u3 = u_of(V, px1, py1);
        const double umin = fmin(fmax(fmin(fmin(u0, u1), fmin(u2, u3)), 0.0), (double)(DNU - 1));
        const double umax = fmin(fmax(fmax(fmax(u0, u1), fmax(u2, u3)), 0.0), (double)(DNU - 1));
        // one row of margin each side: interior boundaries may round past
        // the corners' range by an ulp
        const int lo = max((int)umin - 1, 0), rows = min((int)umax + 2, DNU) - lo + 1;
        const bool fits = rows <= rmax;
        s_ulo[b] = lo;
        s_rows[b] = fits ? rows : 0;
        mbar_arrive_expect_tx(&s_bar[b], fits ? (uint32_t)(sizeof(T) * rows * vp) : 0u);
        if (fits)
            bulk_copy_g2s(qbuf + (size_t)b * rmax * vp, Qall + l * qstride + (long long)lo * vp,
                          (uint32_t)(sizeof(T) * rows * vp), &s_bar[b]);
    };

    geometry(0);
    geometry(1);
    __syncthreads(); // barrier init visible before any copy
    issue(0);
    issue(1);
    __syncthreads();

    float acc[KSEG];
#pragma unroll
    for (int r = 0; r < KSEG; ++r) acc[r] = 0.f;
    bool timed_out = false;

    for (int li = 0; li < n; ++li) {
        const int b = li & 1, ls = li % 3;
        const int ulo = s_ulo[b], rows = s_rows[b];
        if (!mbar_wait(&s_bar[b], (uint32_t)((li >> 1) & 1))) timed_out = true;
        const int xdrv = a.views[a.view_list[li]].xdrv;

        const T *Qg = Qall + li * qstride;
        const T *Qs = qbuf + (size_t)b * rmax * vp;
        float *E = E2 + (size_t)b * kCols * es; // double buffered: B(li) overlaps A(li+1)

        // ---- A: strip integrals E_c(v') = Q(u_b, v') - Q(u_a, v'), FP64 -> FP32 ----
        if (!timed_out) {
            const int nit = kCols * (DNV + 1);
            for (int item = tid; item < nit; item += kThreads) {
                const int c = item / (DNV + 1), vv = item - c * (DNV + 1);
                const int ccx = c & (kB - 1), ccy = c / kB;
                const double ua = xdrv ? s_u[ls][ccx][ccy] : s_u[ls][ccy][ccx];
                const double ub = xdrv ? s_u[ls][ccx][ccy + 1] : s_u[ls][ccy][ccx + 1];
                const double uca = fmin(fmax(ua, 0.0), (double)DNU), ucb = fmin(fmax(ub, 0.0), (double)DNU);
                const int ia = min((int)uca, DNU - 1), ib = min((int)ucb, DNU - 1);
                const double fa = uca - ia, fb = ucb - ib;
                const T *pa, *pb;
                if (rows > 0) {
                    pa = Qs + (size_t)min(max(ia - ulo, 0), rows - 2) * vp + vv;
                    pb = Qs + (size_t)min(max(ib - ulo, 0), rows - 2) * vp + vv;
                } else {
                    pa = Qg + (long long)ia * vp + vv;
                    pb = Qg + (long long)ib * vp + vv;
                }
                E[c * es + vv] = strip(q_ld(pa), q_ld(pa + vp), q_ld(pb), q_ld(pb + vp), fa, fb);
            }
        }
        __syncthreads();

        // ---- stage view li+2 into the buffer just consumed; its geometry ----
        issue(li + 2);
        geometry(li + 2);

        // ---- phase B: voxels ----
        if (in_vol) {
            const float V0 = s_V0[ls][col], V1 = s_V1[ls][col];
            const double du = xdrv ? (s_u[ls][cx][cy + 1] - s_u[ls][cx][cy]) : (s_u[ls][cy][cx + 1] - s_u[ls][cy][cx]);
            const float sg = ((du > 0) ? 1.f : -1.f) * ((V1 > 0) ? 1.f : -1.f);
            const float *Ec = E + col * es;
            float lo = e_sample(Ec, fmaf(V1, (float)k0, V0), DNV);
#pragma unroll
            for (int r = 0; r < KSEG; ++r) {
                const float hi = e_sample(Ec, fmaf(V1, (float)(k0 + r + 1), V0), DNV);
                acc[r] = fmaf(hi - lo, sg, acc[r]);
                lo = hi;
            }
        }
    }
    if (timed_out && a.err) atomicExch(a.err, CTLAB_ERR_TIMEOUT);

    if (!in_vol) return;
    const long long colidx = (long long)y * a.XN + x;
    const float m = a.mask ? (a.mask[colidx] ? 1.f : 0.f) : 1.f;
    float *o = a.out + colidx * ZN;
#pragma unroll
    for (int r = 0; r < KSEG; ++r) {
        const int k = k0 + r;
        if (k < ZN) {
            if (a.epilogue == BACK_SART_UPDATE) {
                const float cs = a.col_sum[colidx * ZN + k];
                const float upd = (cs > 1.0e-7f) ? acc[r] / cs : 0.f;
                float v = (o[k] + a.lambda * upd) * m;
                if (a.clamp) v = fminf(fmaxf(v, a.min_v), a.max_v);
                o[k] = v;
            } else {
                o[k] = acc[r] * m;
            }
        }
    }
}

size_t dyn_smem(int rmax, int vp, int es)
{
    return 8 * 2 * (size_t)rmax * vp + sizeof(float) * 2 * (size_t)kCols * es;
}

template <int KSEG, class T>
cudaError_t launch_k(const BackArgs &a, cudaStream_t s)
{
    const int es = (a.DNV + 1) | 1;
    const size_t sm = dyn_smem(a.rmax, a.vp, es);
    auto kern = dd3_back_kernel<KSEG, T>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    dim3 grid((a.XN + kB - 1) / kB, (a.YN + kB - 1) / kB, (a.ZN + kZS * KSEG - 1) / (kZS * KSEG));
    kern<<<grid, kThreads, sm, s>>>(a, es, a.rmax);
    return cudaGetLastError();
}

template <class T>
cudaError_t launch_t(const BackArgs &a, cudaStream_t s)
{
    if (a.ZN <= kZS * 8) return launch_k<8, T>(a, s);
    if (a.ZN <= kZS * 16) return launch_k<16, T>(a, s);
    if (a.ZN <= kZS * 32) return launch_k<32, T>(a, s);
    return launch_k<64, T>(a, s);
}

} // namespace

bool back_supported(int DNV)
{
    const int es = (DNV + 1) | 1;
    const int vp = (DNV + 2) & ~1;
    return dyn_smem(2, vp, es) + kStaticSmem <= 227 * 1024;
}

// Staging rows for the plan: the widest u footprint of any brick on the
// volume's outer ring of bricks (nearest the source in some view), +2,
// capped so two CTAs fit an SM (at least 2; wider footprints read global).
int back_staging_rows(const HostGeometry &g, int vp)
{
    const int es = (g.DNV + 1) | 1;
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
                need = std::max(need, std::min((int)umax + 2, g.DNU) - std::max((int)umin - 1, 0) + 1);
            }
        }
    }
    const size_t fixed = dyn_smem(0, vp, es) + kStaticSmem;
    const int cap = kSmemPerCta > fixed ? (int)((kSmemPerCta - fixed) / (8 * 2 * (size_t)vp)) : 0;
    return std::max(2, std::min(need, cap));
}

cudaError_t launch_back(const BackArgs &a, cudaStream_t s, int *launches)
{
    if (launches) ++*launches;
    if (a.n <= 0) return cudaSuccess;
    return a.f32pair ? launch_t<ff2>(a, s) : launch_t<double>(a, s);
}

} // namespace ctlab
