// Branchless DD cone-beam forward projection (gather over the volume SAT).
//
// One CTA owns one view and a tile of kU detector columns and sweeps every
// slice j of the view's driving axis a.  Per slice:
//   positions  the tile's kU+1 in-plane boundary rays meet the slice plane at
//              b-index  x_q(j) = c0_q + m_q * j   (FP64, affine in j);
//   phase A    for every z boundary row k of the SAT, the strip integral
//              between consecutive boundary rays
//                 D_u(k) = F(x_{u+1}, k) - F(x_u, k)
//              where F(x, k) is the SAT row k interpolated along b in FP64
//              (or float-float), converted to FP32 once the large prefix
//              values have cancelled; coalesced loads along z;
//   phase B    each cell (u, v) maps its two z boundaries along the column's
//              central ray, kz = Z0 + T_u(j) e_w, samples D_u linearly in z
//              (FP32) and accumulates R / (w_x T_u) in registers.
// The epilogue multiplies by the central-ray slab length and 1/(e_{v+1}-e_v)
// and optionally fuses the SART residual weighting (b - Ax)/rowSum.
#include "ffloat.cuh"
#include "internal.h"

namespace ctlab {

namespace {

constexpr int kU = 32;              // detector columns per CTA
constexpr int kVS = 8;              // threads per column in phase B
constexpr int kThreads = kU * kVS;  // 256

__device__ __forceinline__ double sat_ld(const double *p) { return __ldg(p); }
__device__ __forceinline__ ff2 sat_ld(const ff2 *p)
{
    const float2 f = __ldg(reinterpret_cast<const float2 *>(p));
    return {f.x, f.y};
}
__device__ __forceinline__ double sat_lerp(double s0, double s1, double f) { return fma(f, s1 - s0, s0); }
__device__ __forceinline__ ff2 sat_lerp(ff2 s0, ff2 s1, double f)
{
    return ff_add(s0, ff_mul_f(ff_sub(s1, s0), (float)f));
}
__device__ __forceinline__ float sat_diff(double a, double b) { return (float)(a - b); }
__device__ __forceinline__ float sat_diff(ff2 a, ff2 b) { return ff_to_float(ff_sub(a, b)); }

// Linear sample of a D column at z-boundary coordinate kz, clamped to [0, zn].
__device__ __forceinline__ float sample_col(const float *col, float kz, int zn)
{
    kz = fminf(fmaxf(kz, 0.f), (float)zn);
    int i = (int)kz;
    i = min(i, zn - 1);
    const float f = kz - (float)i;
    const float d0 = col[i], d1 = col[i + 1];
    return fmaf(f, d1 - d0, d0);
}

template <int NR, class T>
__global__ void __launch_bounds__(kThreads) dd3_proj_kernel(ProjArgs a, int ds)
{
    extern __shared__ __align__(16) unsigned char smem[];
    float *D = reinterpret_cast<float *>(smem); // [kU][ds]
    float *s_e = D + kU * ds;                   // [DNV+1]
    __shared__ double s_pos[2][kU + 1];
    __shared__ double s_f[2][kU + 1];
    __shared__ int s_i[2][kU + 1];
    __shared__ double s_c0[kU + 1], s_m[kU + 1];
    __shared__ double s_r[kU];

    const int tid = threadIdx.x;
    const int li = blockIdx.y;
    const int p = a.view_list[li];
    const DevView V = a.views[p];
    const int u0 = blockIdx.x * kU;
    const int nu = min(kU, a.DNU - u0);
    const DetTable t = det_table_layout(a.DNU, a.DNV);
    const double *det = a.det;
    const int na = V.na, nb = V.nb, ZN = a.ZN, DNV = a.DNV;
    const double dx = a.dx;

    auto set_pos = [&](int buf, int q, double x) {
        s_pos[buf][q] = x;
        const double xc = fmin(fmax(x, 0.0), (double)nb);
        int i = min((int)xc, nb - 1);
        s_i[buf][q] = i;
        s_f[buf][q] = xc - (double)i;
    };

    if (tid <= nu) {
        const int q = u0 + tid;
        const double lx = det[t.off_bx + q], ly = det[t.off_by + q];
        const double wx = lx * V.c - ly * V.s, wy = lx * V.s + ly * V.c;
        const double wa = V.xdrv ? wx : wy, wb = V.xdrv ? wy : wx;
        const double m = (wb - V.Sb) / (wa - V.Sa);
        const double c0 = (V.Sb - V.b_lo) / dx + m * (V.a0 - V.Sa) / dx;
        s_m[tid] = m;
        s_c0[tid] = c0;
        set_pos(0, tid, c0);
    }
    if (tid < nu) {
        const int u = u0 + tid;
        const double lx = det[t.off_ux + u], ly = det[t.off_uy + u];
        const double ca = V.xdrv ? (lx * V.c - ly * V.s) : (lx * V.s + ly * V.c);
        s_r[tid] = 1.0 / (ca - V.Sa);
    }
    for (int w = tid; w <= DNV; w += kThreads)
        s_e[w] = (float)((det[t.off_bz + w] + V.zP - V.Sz) / a.dz);
    for (int q = tid; q < kU; q += kThreads) D[q * ds] = 0.f;
    const float Z0 = (float)((V.Sz - a.z_lo) / a.dz);
    __syncthreads();

    // phase A thread mapping: k in [1, ZN]; small ZN splits the boundaries
    // of the tile among several groups of threads.
    int groups = 1, g = 0, kstart = tid + 1, kstep = kThreads;
    if (ZN < kThreads) {
        groups = max(1, min(nu, kThreads / ZN));
        g = tid / ZN;
        kstart = tid - g * ZN + 1;
        kstep = ZN;
    }
    const int qper = (nu + groups - 1) / groups;
    const int qa = min(g * qper, nu), qb = min(nu, qa + qper);
    const bool a_active = g < groups && qa < qb;

    const int uu = tid % kU, vs = tid / kU, v0 = vs * NR;
    float acc[NR];
#pragma unroll
    for (int r = 0; r < NR; ++r) acc[r] = 0.f;

    const T *sat = reinterpret_cast<const T *>(V.xdrv ? a.sat_x : a.sat_y);
    const long long pstride = (long long)(nb + 1) * a.zp;
    const double ga0 = V.a0 - V.Sa;

    for (int j = 0; j < na; ++j) {
        const int buf = j & 1;
        const T *S = sat + (long long)j * pstride;
        if (a_active) {
            for (int k = kstart; k <= ZN; k += kstep) {
                T gp = sat_lerp(sat_ld(S + (long long)s_i[buf][qa] * a.zp + k),
                                sat_ld(S + (long long)(s_i[buf][qa] + 1) * a.zp + k), s_f[buf][qa]);
                for (int q = qa + 1; q <= qb; ++q) {
                    const long long base = (long long)s_i[buf][q] * a.zp + k;
                    const T gq = sat_lerp(sat_ld(S + base), sat_ld(S + base + a.zp), s_f[buf][q]);
                    D[(q - 1) * ds + k] = sat_diff(gq, gp);
                    gp = gq;
                }
            }
        }
        __syncthreads();
        if (uu < nu && v0 < DNV) {
            const double ga = ga0 + (double)j * dx;
            const float T_ = (float)(ga * s_r[uu]);
            const float wxu = (float)(s_pos[buf][uu + 1] - s_pos[buf][uu]);
            const float den = wxu * T_;
            const float scale = (den != 0.f) ? 1.f / den : 0.f;
            const float *Du = D + uu * ds;
            float dp = sample_col(Du, fmaf(T_, s_e[v0], Z0), ZN);
#pragma unroll
            for (int r = 0; r < NR; ++r) {
                const int v = v0 + r;
                if (v < DNV) {
                    const float dn = sample_col(Du, fmaf(T_, s_e[v + 1], Z0), ZN);
                    acc[r] = fmaf(dn - dp, scale, acc[r]);
                    dp = dn;
                }
            }
        }
        if (tid <= nu && j + 1 < na) set_pos(buf ^ 1, tid, s_c0[tid] + s_m[tid] * (double)(j + 1));
        __syncthreads();
    }

    // epilogue
    double r2 = 0.0;
    if (uu < nu) {
        const int u = u0 + uu;
        const double lx = det[t.off_ux + u], ly = det[t.off_uy + u];
        const double cx = lx * V.c - ly * V.s, cy = lx * V.s + ly * V.c;
        const double ex = cx - V.Sx, ey = cy - V.Sy;
        const double ea = V.xdrv ? ex : ey;
#pragma unroll
        for (int r = 0; r < NR; ++r) {
            const int v = v0 + r;
            if (v < DNV) {
                const double ez = det[t.off_vz + v] + V.zP - V.Sz;
                const double L = dx * sqrt(ex * ex + ey * ey + ez * ez) / fabs(ea);
                const double de = (det[t.off_bz + v + 1] - det[t.off_bz + v]) / a.dz;
                const float val = (float)((double)acc[r] * (L / de));
                const long long idx = ((long long)li * a.DNU + u) * DNV + v;
                if (a.epilogue == PROJ_SART_RESIDUAL) {
                    const float m = a.meas[idx], rs = a.row_sum[idx];
                    const float res = m - val;
                    r2 += (double)res * (double)res;
                    a.out[idx] = (rs > 1.0e-7f) ? res / rs : 0.f;
                } else {
                    a.out[idx] = val;
                }
            }
        }
    }
    if (a.epilogue == PROJ_SART_RESIDUAL && a.resid2) {
        __shared__ double s_red[kThreads / 32];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) r2 += __shfl_down_sync(0xffffffffu, r2, o);
        if ((tid & 31) == 0) s_red[tid >> 5] = r2;
        __syncthreads();
        if (tid == 0) {
            double sum = 0.0;
            for (int w = 0; w < kThreads / 32; ++w) sum += s_red[w];
            atomicAdd(a.resid2, sum);
        }
    }
}

template <int NR, class T>
cudaError_t launch_nr(const ProjArgs &a, cudaStream_t s)
{
    const int ds = (a.ZN + 1) | 1;
    const size_t sm = sizeof(float) * ((size_t)kU * ds + a.DNV + 1);
    auto kern = dd3_proj_kernel<NR, T>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    dim3 grid((a.DNU + kU - 1) / kU, a.n);
    kern<<<grid, kThreads, sm, s>>>(a, ds);
    return cudaGetLastError();
}

template <class T>
cudaError_t launch_t(const ProjArgs &a, cudaStream_t s)
{
    const int need = (a.DNV + kVS - 1) / kVS;
    if (need <= 1) return launch_nr<1, T>(a, s);
    if (need <= 2) return launch_nr<2, T>(a, s);
    if (need <= 4) return launch_nr<4, T>(a, s);
    if (need <= 8) return launch_nr<8, T>(a, s);
    if (need <= 16) return launch_nr<16, T>(a, s);
    if (need <= 32) return launch_nr<32, T>(a, s);
    return cudaErrorInvalidValue;
}

} // namespace

// Largest supported sizes of the projector (shared-memory bound).
bool proj_supported(int ZN, int DNV)
{
    const int ds = (ZN + 1) | 1;
    const size_t sm = sizeof(float) * ((size_t)kU * ds + DNV + 1);
    return DNV <= 256 && sm <= 200 * 1024;
}

cudaError_t launch_proj(const ProjArgs &a, cudaStream_t s, int *launches)
{
    if (a.n <= 0) return cudaSuccess;
    if (a.n > 65535) return cudaErrorInvalidConfiguration;
    if (launches) ++*launches;
    return a.f32pair ? launch_t<ff2>(a, s) : launch_t<double>(a, s);
}

} // namespace ctlab
