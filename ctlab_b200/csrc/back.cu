// Branchless DD cone-beam backprojection (voxel-driven gather over the
// per-view projection SATs).
//
// One CTA owns a brick of 8 x 8 voxel columns (x, y) and a z range of
// 4*KSEG voxels, and loops over the views.  Per view:
//   boundaries  the brick's voxel boundaries across the view's driving axis
//               (8 rows of 9 points) are mapped through the source onto the
//               flat detector: u = cross(S-B0, P-S) / cross(E, P-S)   (FP64);
//               each column's centre ray gives the affine z -> v map
//               v(k') = V0 + V1 k' over z-boundary indices k';
//   phase A     for every detector row boundary v', the strip integral of
//               the weighted projection between a column's two u boundaries
//                  E_c(v') = Q(u_{c+1}, v') - Q(u_c, v')
//               from the projection SAT Q interpolated along u (FP64 or
//               float-float), then FP32;
//   phase B     each voxel samples E_c linearly at its two z boundaries
//               (FP32) and accumulates the oriented difference in registers.
// The epilogue applies the in-plane mask and optionally fuses the OS-SART
// update x = (x + lambda * acc/colSum) * mask.
#include "ffloat.cuh"
#include "internal.h"

namespace ctlab {

namespace {

constexpr int kB = 8;                 // brick edge (voxel columns)
constexpr int kCols = kB * kB;        // 64 columns per CTA
constexpr int kZS = 4;                // z segments per column
constexpr int kThreads = kCols * kZS; // 256

__device__ __forceinline__ double q_ld(const double *p) { return __ldg(p); }
__device__ __forceinline__ ff2 q_ld(const ff2 *p)
{
    const float2 f = __ldg(reinterpret_cast<const float2 *>(p));
    return {f.x, f.y};
}
__device__ __forceinline__ double q_lerp(double s0, double s1, double f) { return fma(f, s1 - s0, s0); }
__device__ __forceinline__ ff2 q_lerp(ff2 s0, ff2 s1, double f)
{
    return ff_add(s0, ff_mul_f(ff_sub(s1, s0), (float)f));
}
__device__ __forceinline__ float q_diff(double a, double b) { return (float)(a - b); }
__device__ __forceinline__ float q_diff(ff2 a, ff2 b) { return ff_to_float(ff_sub(a, b)); }

template <class T>
__device__ __forceinline__ T q_sample(const T *Q, int vp, int DNU, double u, int vv)
{
    const double uc = fmin(fmax(u, 0.0), (double)DNU);
    const int iu = min((int)uc, DNU - 1);
    const double fu = uc - (double)iu;
    const T *c0 = Q + (long long)iu * vp + vv;
    return q_lerp(q_ld(c0), q_ld(c0 + vp), fu);
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

template <int KSEG, class T>
__global__ void __launch_bounds__(kThreads, 2) dd3_back_kernel(BackArgs a, int es)
{
    extern __shared__ __align__(16) unsigned char smem[];
    float *E = reinterpret_cast<float *>(smem); // [kCols][es]
    __shared__ double s_u[kB][kB + 1];
    __shared__ float s_V0[kCols], s_V1[kCols], s_sg[kCols];

    const int tid = threadIdx.x;
    const int bx0 = blockIdx.x * kB, by0 = blockIdx.y * kB;
    const int col = tid & (kCols - 1), zs = tid / kCols;
    const int cx = col & (kB - 1), cy = col / kB;
    const int x = bx0 + cx, y = by0 + cy;
    const int k0 = blockIdx.z * (kZS * KSEG) + zs * KSEG;
    const int DNU = a.DNU, DNV = a.DNV, vp = a.vp, ZN = a.ZN;
    const double dx = a.dx;
    const double x_lo = a.x_c0 - 0.5 * dx, y_lo = a.y_c0 - 0.5 * dx;
    const DetTable t = det_table_layout(DNU, DNV);
    const double zb0_local = a.det[t.off_bz];
    const bool in_vol = (x < a.XN) && (y < a.YN);

    float acc[KSEG];
#pragma unroll
    for (int r = 0; r < KSEG; ++r) acc[r] = 0.f;

    const int nitems = kB * (DNV + 1);
    for (int li = 0; li < a.n; ++li) {
        const DevView &V = a.views[a.view_list[li]];
        const double Sx = V.Sx, Sy = V.Sy;
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
            const double dpx = px - Sx, dpy = py - Sy;
            s_u[r][q] = cross2(Sx - V.B0x, Sy - V.B0y, dpx, dpy) / cross2(V.Ex, V.Ey, dpx, dpy);
        } else if (tid >= 128 && tid < 128 + kCols) {
            const int c = tid - 128;
            const double pcx = a.x_c0 + (double)(bx0 + (c & (kB - 1))) * dx;
            const double pcy = a.y_c0 + (double)(by0 + c / kB) * dx;
            const double tc = cross2(V.B0x - Sx, V.B0y - Sy, V.Ex, V.Ey) /
                              cross2(pcx - Sx, pcy - Sy, V.Ex, V.Ey);
            const double zb0 = zb0_local + V.zP;
            s_V1[c] = (float)(tc * a.dz / a.dzb);
            s_V0[c] = (float)((V.Sz + tc * (a.z_lo - V.Sz) - zb0) / a.dzb);
        }
        __syncthreads();
        if (tid < kCols) {
            const int ccx = tid & (kB - 1), ccy = tid / kB;
            const double du = V.xdrv ? (s_u[ccx][ccy + 1] - s_u[ccx][ccy]) : (s_u[ccy][ccx + 1] - s_u[ccy][ccx]);
            s_sg[tid] = ((du > 0) ? 1.f : -1.f) * ((s_V1[tid] > 0) ? 1.f : -1.f);
        }
        const T *Q = reinterpret_cast<const T *>(a.q) + (long long)li * (DNU + 1) * vp;
        for (int item = tid; item < nitems; item += kThreads) {
            const int r = item / (DNV + 1), vv = item - r * (DNV + 1);
            T gp = q_sample(Q, vp, DNU, s_u[r][0], vv);
#pragma unroll
            for (int q = 1; q <= kB; ++q) {
                const T g = q_sample(Q, vp, DNU, s_u[r][q], vv);
                const int c = V.xdrv ? ((q - 1) * kB + r) : (r * kB + q - 1);
                E[c * es + vv] = q_diff(g, gp);
                gp = g;
            }
        }
        __syncthreads();
        if (in_vol) {
            const float V0 = s_V0[col], V1 = s_V1[col], sg = s_sg[col];
            const float *Ec = E + col * es;
            float lo = e_sample(Ec, fmaf(V1, (float)k0, V0), DNV);
#pragma unroll
            for (int r = 0; r < KSEG; ++r) {
                const float hi = e_sample(Ec, fmaf(V1, (float)(k0 + r + 1), V0), DNV);
                acc[r] = fmaf(hi - lo, sg, acc[r]);
                lo = hi;
            }
        }
        __syncthreads();
    }

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

template <int KSEG, class T>
cudaError_t launch_k(const BackArgs &a, cudaStream_t s)
{
    const int es = (a.DNV + 1) | 1;
    const size_t sm = sizeof(float) * (size_t)kCols * es;
    auto kern = dd3_back_kernel<KSEG, T>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    dim3 grid((a.XN + kB - 1) / kB, (a.YN + kB - 1) / kB, (a.ZN + kZS * KSEG - 1) / (kZS * KSEG));
    kern<<<grid, kThreads, sm, s>>>(a, es);
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
    return sizeof(float) * (size_t)kCols * es <= 200 * 1024;
}

cudaError_t launch_back(const BackArgs &a, cudaStream_t s, int *launches)
{
    if (launches) ++*launches;
    if (a.n <= 0) {
        // no views: plain backprojection of nothing is zero; the SART update
        // leaves x unchanged apart from the mask, done by the caller.
        return cudaSuccess;
    }
    return a.f32pair ? launch_t<ff2>(a, s) : launch_t<double>(a, s);
}

} // namespace ctlab
