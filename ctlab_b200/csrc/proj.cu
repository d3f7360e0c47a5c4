// Branchless DD cone-beam forward projection (gather over the volume SAT).
//
// One CTA (512 threads) owns a tile of kU = 32 detector columns for a group
// of G views sharing one driving axis (adjacent angles, grouped on the
// host), and sweeps every slice j of that axis.  Per slice:
//   staging    the SAT columns the group's rays cross on slice j -- the
//              union over the G views of the b-index ranges, and of the z
//              ranges -- are copied into shared memory by 1-D bulk copies
//              (TMA, one per column), double buffered two slices ahead and
//              completed on an mbarrier; the G views share the staged data;
//   phase A    (per view) for every SAT row k, the strip integral between
//              consecutive boundary rays of the tile
//                 D_u(k) = F(x_{u+1}, k) - F(x_u, k)
//                        = (S_i' - S_i) + f' C_i'(k) - f C_i(k),
//              F(x, k) the SAT row k interpolated along b (x = i + f) and
//              C_i = S_{i+1} - S_i.  A thread owns two rows and a run of
//              boundaries, walking the staged columns in order with the two
//              current columns in registers: the FP64 difference C_i (where
//              the large prefix values cancel) is formed once per column and
//              rounded to FP32; everything after it is FP32;
//   phase B    (per view) each cell (u, v) maps its two z boundaries along
//              the column's central ray, kz = Z0 + T_u(j) e_w, samples D_u
//              linearly in z and accumulates R / (w_x T_u) in registers.
// D is double buffered across the views of a slice and across slices: one
// barrier per view separates A from B; the copies of slice j+2 are issued
// once the last view's phase A has consumed the staged buffer.  Slices whose column span
// exceeds the staging buffer read the SAT from global memory instead.
// The epilogue multiplies by the central-ray slab length and 1/(e_{v+1}-e_v)
// and optionally fuses the SART residual weighting (b - Ax)/rowSum.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <type_traits>

#include "ffloat.cuh"
#include "internal.h"
#include "tma.cuh"

namespace ctlab {

namespace {

constexpr int kU = 32;                // detector columns per CTA
constexpr int kThreads = 512;         // 16 warps
constexpr int kVS = kThreads / kU;    // threads per column in phase B
constexpr int kGMax = 4;              // views per CTA, at most
constexpr int kMaxBuf = 4;            // staging depth (slices in flight), at most
constexpr size_t kSmemLimit = 227 * 1024;
constexpr size_t kStaticSmem = 12 * 1024; // static shared arrays + alignment slack

struct SliceInfo {
    int i_lo, ncols, k_lo, k_hi, k_lo_a, kcount, fits, pad;
};

__device__ __forceinline__ double sat_ld(const double *p) { return *p; }
__device__ __forceinline__ ff2 sat_ld(const ff2 *p)
{
    const float2 f = *reinterpret_cast<const float2 *>(p);
    return {f.x, f.y};
}
__device__ __forceinline__ float col_diff(double hi, double lo) { return (float)(hi - lo); }
__device__ __forceinline__ float col_diff(ff2 hi, ff2 lo) { return ff_to_float(ff_sub(hi, lo)); }

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

// Phase A for one view: D rows of the tile for SAT rows ks..k_hi.  QPER
// boundaries per thread (compile time, unrolled); 32/QPER groups of threads
// split the tile's boundaries and a warp shares its group.  Every strip is
// computed independently from its two boundaries' SAT columns,
//   D = (S_c' - S_c) + f' C_c' - f C_c,  C_c = S_{c+1} - S_c,
// with the two FP64 differences rounded to FP32, so the loads of all
// boundaries issue back to back.
template <int QPER, class T>
__device__ __forceinline__ void phase_a(const SliceInfo &in, const int2 *cf, float *D, int ds, const T *S, int kstr,
                                        const T *Sg, long long zp, int tid)
{
    constexpr int kGroups = kU / QPER;
    constexpr int mstep = kThreads / kGroups;
    const int ks = max(in.k_lo, 1);
    const int half = (in.k_hi - ks + 2) >> 1;
    const int g = tid / mstep, m0 = tid - g * mstep;
    const int qa = g * QPER;
    if (in.fits) {
        int cq[QPER + 1];
        float fq[QPER + 1];
#pragma unroll
        for (int i = 0; i <= QPER; ++i) {
            const int2 e = cf[qa + i];
            cq[i] = e.x * kstr;
            fq[i] = __int_as_float(e.y);
        }
        for (int m = m0; m < half; m += mstep) {
            const int k = ks + m;
            const int k1 = min(k + half, in.k_hi); // odd count: the last row repeats
#pragma unroll 1
            for (int h = 0; h < 2; ++h) {
                const int kk = h ? k1 : k;
                const T *Sk = S + (kk - in.k_lo_a);
                // every boundary's two SAT columns: independent loads
                T s0[QPER + 1], s1[QPER + 1];
#pragma unroll
                for (int i = 0; i <= QPER; ++i) {
                    s0[i] = Sk[cq[i]];
                    s1[i] = Sk[cq[i] + kstr];
                }
                float Cp = col_diff(s1[0], s0[0]);
#pragma unroll
                for (int i = 1; i <= QPER; ++i) {
                    const float Ci = col_diff(s1[i], s0[i]);
                    const float dS = col_diff(s0[i], s0[i - 1]); // 0 or a few whole columns, FP64 first
                    D[(qa + i - 1) * ds + kk] = dS + (fq[i] * Ci - fq[i - 1] * Cp);
                    Cp = Ci;
                }
            }
        }
    } else {
        // column span wider than the staging buffer: the FP64 strip
        // difference straight from the SAT in global memory
        for (int m = m0; m < half; m += mstep) {
            const int k = ks + m;
            const int k1 = min(k + half, in.k_hi);
            for (int q = qa; q < qa + QPER; ++q) {
                const int2 ea = cf[q], eb = cf[q + 1];
                const float fa = __int_as_float(ea.y), fb = __int_as_float(eb.y);
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int kk = h ? k1 : k;
                    const T a0 = sat_ld(Sg + (long long)ea.x * zp + kk), a1 = sat_ld(Sg + (long long)(ea.x + 1) * zp + kk);
                    const T b0 = sat_ld(Sg + (long long)eb.x * zp + kk), b1 = sat_ld(Sg + (long long)(eb.x + 1) * zp + kk);
                    D[q * ds + kk] = col_diff(b0, a0) + (fb * col_diff(b1, b0) - fa * col_diff(a1, a0));
                }
            }
        }
    }
}

template <int NR, int G, class T>
__global__ void __launch_bounds__(kThreads, 1) dd3_proj_kernel(ProjArgs a, int ds, int cmax, int kstr)
{
    extern __shared__ __align__(128) unsigned char smem[];
    const int nbuf = a.nbuf;                                                            // staging depth
    T *colbuf = reinterpret_cast<T *>(smem);                                            // [nbuf][cmax][kstr]
    float *D2 = reinterpret_cast<float *>(smem + sizeof(T) * nbuf * (size_t)cmax * kstr); // [2][kU][ds]
    float *s_e = D2 + 2 * kU * ds;                                                       // [G][DNV+1]
    __shared__ __align__(8) uint64_t s_bar[kMaxBuf];
    __shared__ SliceInfo s_info[kMaxBuf];
    __shared__ double s_c0[G][kU + 1], s_m[G][kU + 1];
    __shared__ double s_r[G][kU];
    __shared__ double s_pos[kMaxBuf + 1][G][kU + 1];
    __shared__ int2 s_cf[kMaxBuf + 1][G][kU + 1]; // per view and boundary: staged column, fraction bits
    __shared__ int s_pos_list[G];       // list positions of the group's views (-1: empty slot)
    __shared__ double s_ga0[G];         // a0 - Sa per view
    __shared__ float s_Z0[G];           // z offset of the source in SAT-row units

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid < G) s_pos_list[tid] = a.groups[blockIdx.y * G + tid];
    const int u0 = blockIdx.x * kU;
    const int nu = min(kU, a.DNU - u0);
    const DetTable t = det_table_layout(a.DNU, a.DNV);
    const double *det = a.det;
    const int ZN = a.ZN, DNV = a.DNV, zp = a.zp;
    const double dx = a.dx;
    __syncthreads();
    const DevView &V0 = a.views[a.view_list[s_pos_list[0]]]; // all views share the axis
    const int na = V0.na, nb = V0.nb;
    // column (slice j, boundary column c) starts at sat + j*s_slice + c*s_col:
    // 2-D SATs hold nb+1 boundary columns per slice
    constexpr int kAlign = 16 / (int)sizeof(T); // elements per 16 bytes
    const T *sat = reinterpret_cast<const T *>(V0.xdrv ? a.sat_x : a.sat_y);
    const long long s_col = zp;
    const long long s_slice = (long long)(nb + 1) * zp;
    const int ccap = nb; // last column index
    auto view_of = [&](int g) -> const DevView & {
        const int ps = s_pos_list[g] >= 0 ? s_pos_list[g] : s_pos_list[0];
        return a.views[a.view_list[ps]];
    };

    if (tid == 0) {
        for (int i = 0; i < nbuf; ++i) mbar_init(&s_bar[i], 1);
        mbar_fence_init();
    }
    for (int it = tid; it < G * (kU + 1); it += kThreads) {
        const int g = it / (kU + 1), q0 = it - g * (kU + 1);
        const DevView &V = view_of(g);
        const int q = u0 + min(q0, nu); // boundaries past the tile repeat the last one
        const double lx = det[t.off_bx + q], ly = det[t.off_by + q];
        const double wx = lx * V.c - ly * V.s, wy = lx * V.s + ly * V.c;
        const double wa = V.xdrv ? wx : wy, wb = V.xdrv ? wy : wx;
        const double m = (wb - V.Sb) / (wa - V.Sa);
        s_m[g][q0] = m;
        s_c0[g][q0] = (V.Sb - V.b_lo) / dx + m * (V.a0 - V.Sa) / dx;
    }
    for (int it = tid; it < G * kU; it += kThreads) {
        const int g = it / kU, uq = it - g * kU;
        const DevView &V = view_of(g);
        const int u = u0 + min(uq, nu - 1);
        const double lx = det[t.off_ux + u], ly = det[t.off_uy + u];
        const double ca = V.xdrv ? (lx * V.c - ly * V.s) : (lx * V.s + ly * V.c);
        s_r[g][uq] = 1.0 / (ca - V.Sa);
    }
    for (int it = tid; it < G * (DNV + 1); it += kThreads) {
        const int g = it / (DNV + 1), w = it - g * (DNV + 1);
        const DevView &V = view_of(g);
        s_e[it] = (float)((det[t.off_bz + w] + V.zP - V.Sz) / a.dz);
    }
    for (int q = tid; q < 2 * kU; q += kThreads) D2[q * ds] = 0.f; // D(k = 0) = 0: SAT row 0 is zero
    if (tid < G) {
        const DevView &V = view_of(tid);
        s_ga0[tid] = V.a0 - V.Sa;
        s_Z0[tid] = (float)((V.Sz - a.z_lo) / a.dz);
    }
    __syncthreads();

    // union over the group of the staged column range of slice j
    auto col_range = [&](int j, int &i_lo, int &ncols) {
        double xmin = 1e300, xmax = -1e300;
#pragma unroll
        for (int g = 0; g < G; ++g) {
            const double x0 = s_c0[g][0] + s_m[g][0] * (double)j, x1 = s_c0[g][kU] + s_m[g][kU] * (double)j;
            xmin = fmin(xmin, fmin(x0, x1));
            xmax = fmax(xmax, fmax(x0, x1));
        }
        xmin = fmin(fmax(xmin, 0.0), (double)(nb - 1));
        xmax = fmin(fmax(xmax, 0.0), (double)(nb - 1));
        // one column of margin each side: interior boundaries may round past
        // the end boundaries' range by an ulp
        i_lo = max((int)xmin - 1, 0);
        ncols = min((int)xmax + 2, ccap) - i_lo + 1;
    };
    // boundary positions of slice j into slot j % (nbuf+1) (threads 0 .. G*(kU+1)-1)
    auto set_pos = [&](int j) {
        if (tid < G * (kU + 1) && j < na) {
            const int g = tid / (kU + 1), q = tid - g * (kU + 1);
            const int sl = j % (nbuf + 1);
            const double x = s_c0[g][q] + s_m[g][q] * (double)j;
            const double xc = fmin(fmax(x, 0.0), (double)nb);
            const int i = min((int)xc, nb - 1);
            int i_lo, ncols;
            col_range(j, i_lo, ncols);
            const int c = (ncols <= cmax) ? min(max(i - i_lo, 0), ncols - 2) : i;
            s_pos[sl][g][q] = x;
            s_cf[sl][g][q] = make_int2(c, __float_as_int((float)(xc - (double)i)));
        }
    };
    // staging of slice j into buffer j % nbuf (warp 0)
    auto issue = [&](int j) {
        if (warp != 0 || j >= na) return;
        const int b = j % nbuf;
        if (lane == 0) {
            SliceInfo in;
            col_range(j, in.i_lo, in.ncols);
            float zmin = 1e30f, zmax = -1e30f;
#pragma unroll
            for (int g = 0; g < G; ++g) {
                const double ga = s_ga0[g] + (double)j * dx;
                const float Ta = (float)(ga * s_r[g][0]), Tb = (float)(ga * s_r[g][nu - 1]);
                const float e0 = s_e[g * (DNV + 1)], e1 = s_e[g * (DNV + 1) + DNV];
                const float Z0 = s_Z0[g];
                const float c0 = Ta * e0, c1 = Ta * e1, c2 = Tb * e0, c3 = Tb * e1;
                zmin = fminf(zmin, Z0 + fminf(fminf(c0, c1), fminf(c2, c3)));
                zmax = fmaxf(zmax, Z0 + fmaxf(fmaxf(c0, c1), fmaxf(c2, c3)));
            }
            const float zl = fminf(fmaxf(floorf(zmin) - 1.f, 0.f), (float)(ZN - 1));
            in.k_lo = (int)zl;
            const float zh = fminf(fmaxf(floorf(zmax) + 2.f, (float)(in.k_lo + 1)), (float)ZN);
            in.k_hi = (int)zh;
            in.k_lo_a = in.k_lo & ~(kAlign - 1);
            in.kcount = min((in.k_hi + kAlign) & ~(kAlign - 1), zp) - in.k_lo_a;
            in.fits = in.ncols <= cmax;
            in.pad = 0;
            s_info[b] = in;
            mbar_arrive_expect_tx(&s_bar[b], in.fits ? (uint32_t)(sizeof(T) * in.ncols * in.kcount) : 0u);
        }
        __syncwarp();
        const SliceInfo in = s_info[b];
        if (in.fits) {
            const T *src = sat + (long long)j * s_slice + (long long)in.i_lo * s_col + in.k_lo_a;
            T *dst = colbuf + (size_t)b * cmax * kstr;
            for (int c = lane; c < in.ncols; c += 32)
                bulk_copy_g2s(dst + (size_t)c * kstr, src + (long long)c * s_col, (uint32_t)(sizeof(T) * in.kcount),
                              &s_bar[b]);
        }
    };

    for (int i = 0; i < nbuf; ++i) {
        set_pos(i);
        issue(i);
    }
    __syncthreads();

    const int uu = tid % kU, vs = tid / kU, v0 = vs * NR;
    // per view, this thread's column as affine functions of the slice j
    // (evaluated in FP32; relative error ~1e-7): T_u(j) = T0 + j dT,
    // w_x(j) = W0 + j dW, and the z offset Z0
    float cT0[G], cdT[G], cW0[G], cdW[G], cZ0[G];
#pragma unroll
    for (int g = 0; g < G; ++g) {
        const DevView &V = view_of(g);
        const double r = s_r[g][min(uu, nu - 1)];
        cT0[g] = (float)((V.a0 - V.Sa) * r);
        cdT[g] = (float)(dx * r);
        const int q = min(uu, nu - 1);
        cW0[g] = (float)(s_c0[g][q + 1] - s_c0[g][q]);
        cdW[g] = (float)(s_m[g][q + 1] - s_m[g][q]);
        cZ0[g] = (float)((V.Sz - a.z_lo) / a.dz);
    }
    float acc[G][NR];
#pragma unroll
    for (int g = 0; g < G; ++g)
#pragma unroll
        for (int r = 0; r < NR; ++r) acc[g][r] = 0.f;
    bool timed_out = false;
    int dslot = 0;

    for (int j = 0; j < na; ++j) {
        const int b = j % nbuf, js = j % (nbuf + 1);
        const SliceInfo in = s_info[b];
        if (!mbar_wait(&s_bar[b], (uint32_t)((j / nbuf) & 1))) timed_out = true;
        const T *S = colbuf + (size_t)b * cmax * kstr;
        const T *Sg = sat + (long long)j * s_slice;
        const int half = (in.k_hi - max(in.k_lo, 1) + 2) >> 1;
        const float jf = (float)j;
#pragma unroll
        for (int g = 0; g < G; ++g) {
            if (s_pos_list[g] < 0) continue; // uniform: empty slot of a partial group
            float *D = D2 + dslot * kU * ds;
            dslot ^= 1;
            if (!timed_out) {
                // pick the boundaries per thread so that one pass of the
                // thread rows covers the SAT rows (mstep = kThreads*QPER/kU)
                if (half > kThreads / 8) phase_a<8, T>(in, s_cf[js][g], D, ds, S, kstr, Sg, s_col, tid);
                else if (half > kThreads / 16) phase_a<4, T>(in, s_cf[js][g], D, ds, S, kstr, Sg, s_col, tid);
                else phase_a<2, T>(in, s_cf[js][g], D, ds, S, kstr, Sg, s_col, tid);
            }
            __syncthreads();
            if (g == G - 1 || s_pos_list[g + 1] < 0) {
                // the staged slice is consumed: stage slice j+nbuf, its positions
                issue(j + nbuf);
                set_pos(j + nbuf);
            }
            if (uu < nu && v0 < DNV) {
                const float T_ = fmaf(jf, cdT[g], cT0[g]);
                const float den = fmaf(jf, cdW[g], cW0[g]) * T_;
                const float scale = (den != 0.f) ? __frcp_rn(den) : 0.f;
                const float Z0 = cZ0[g];
                const float *Du = D + uu * ds;
                const float *e = s_e + g * (DNV + 1);
                float dp = sample_col(Du, fmaf(T_, e[v0], Z0), ZN);
#pragma unroll
                for (int r = 0; r < NR; ++r) {
                    const int v = v0 + r;
                    if (v < DNV) {
                        const float dn = sample_col(Du, fmaf(T_, e[v + 1], Z0), ZN);
                        acc[g][r] = fmaf(dn - dp, scale, acc[g][r]);
                        dp = dn;
                    }
                }
            }
        }
    }
    if (timed_out && a.err) atomicExch(a.err, CTLAB_ERR_TIMEOUT);

    // epilogue
    double r2 = 0.0;
#pragma unroll
    for (int g = 0; g < G; ++g) {
        const int li = s_pos_list[g];
        if (li < 0 || uu >= nu) continue;
        const DevView &V = view_of(g);
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
                const float val = (float)((double)acc[g][r] * (L / de));
                const long long idx = ((long long)li * a.DNU + u) * DNV + v;
                if (a.epilogue == PROJ_SART_RESIDUAL) {
                    const float mv = a.meas[idx], rs = a.row_sum[idx];
                    const float res = mv - val;
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
        if (lane == 0) s_red[warp] = r2;
        __syncthreads();
        if (tid == 0) {
            double sum = 0.0;
            for (int w = 0; w < kThreads / 32; ++w) sum += s_red[w];
            atomicAdd(a.resid2, sum);
        }
    }
}

size_t dyn_smem(int cmax, int kstr, int ds, int DNV, int G, size_t elem, int nbuf)
{
    return elem * nbuf * (size_t)cmax * kstr + sizeof(float) * (2 * (size_t)kU * ds + (size_t)G * (DNV + 1));
}

template <int NR, int G, class T>
cudaError_t launch_g(const ProjArgs &a, cudaStream_t s)
{
    const int ds = (a.ZN + 1) | 1;
    const size_t sm = dyn_smem(a.cmax, a.zp, ds, a.DNV, G, sizeof(T), a.nbuf);
    auto kern = dd3_proj_kernel<NR, G, T>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    dim3 grid((a.DNU + kU - 1) / kU, a.ngroups);
    kern<<<grid, kThreads, sm, s>>>(a, ds, a.cmax, a.zp);
    return cudaGetLastError();
}

template <int NR, class T>
cudaError_t launch_nr(const ProjArgs &a, cudaStream_t s)
{
    switch (a.G) {
    case 1: return launch_g<NR, 1, T>(a, s);
    case 2: return launch_g<NR, 2, T>(a, s);
    case 4: return launch_g<NR, 4, T>(a, s);
    default: return cudaErrorInvalidValue;
    }
}

template <class T>
cudaError_t launch_t(const ProjArgs &a, cudaStream_t s)
{
    static_assert(sizeof(T) == 8, "SAT element");
    const int need = (a.DNV + kVS - 1) / kVS;
    if (need <= 1) return launch_nr<1, T>(a, s);
    if (need <= 2) return launch_nr<2, T>(a, s);
    if (need <= 4) return launch_nr<4, T>(a, s);
    if (need <= 8) return launch_nr<8, T>(a, s);
    return cudaErrorInvalidValue;
}

// b-index span (in columns, margins included) of the union of the rays of
// views `vs` (one driving axis) through one tile on slice j, affine in j.
int tile_span(const HostGeometry &g, const std::vector<const DevView *> &vs, int u0, int nu, int j)
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
    lo = std::min(std::max(lo, 0.0), (double)(nb - 1));
    hi = std::min(std::max(hi, 0.0), (double)(nb - 1));
    return std::min((int)hi + 2, nb) - std::max((int)lo - 1, 0) + 1;
}

} // namespace

bool proj_supported(int ZN, int DNV)
{
    const int ds = (ZN + 1) | 1;
    const int zp = (ZN + 2) & ~1;
    return DNV <= 8 * kVS && dyn_smem(2, zp, ds, DNV, kGMax, 8, 2) + kStaticSmem <= kSmemLimit;
}

ProjStaging proj_staging(const HostGeometry &g, int zp, int elem_bytes)
{
    // columns the widest tile needs on any slice, one view per CTA and the
    // union of groups of kGMax adjacent views
    int need1 = 2, needg = 2;
    for (size_t p = 0; p < g.views.size(); ++p) {
        const DevView &V = g.views[p];
        std::vector<const DevView *> vs{&V}, vg;
        for (size_t q = p; q < g.views.size() && (int)vg.size() < kGMax; ++q)
            if (g.views[q].xdrv == V.xdrv) vg.push_back(&g.views[q]);
        for (int u0 = 0; u0 < g.DNU; u0 += kU) {
            const int nu = std::min(kU, g.DNU - u0);
            need1 = std::max(need1, std::max(tile_span(g, vs, u0, nu, 0), tile_span(g, vs, u0, nu, V.na - 1)));
            if ((p % kGMax) == 0)
                needg = std::max(needg, std::max(tile_span(g, vg, u0, nu, 0), tile_span(g, vg, u0, nu, V.na - 1)));
        }
    }
    // deepest staging (2..4 slices in flight) whose buffers hold the group
    // span, else the single-view span; CTLAB_PROJ_NBUF overrides the depth
    const int ds = (g.ZN + 1) | 1;
    const size_t fixed = dyn_smem(0, zp, ds, g.DNV, kGMax, elem_bytes, 0) + kStaticSmem;
    auto cap_of = [&](int nbuf) { return (int)((kSmemLimit - fixed) / ((size_t)elem_bytes * nbuf * (size_t)zp)); };
    int want = 0;
    if (const char *env = std::getenv("CTLAB_PROJ_NBUF")) want = std::atoi(env);
    ProjStaging st;
    if (want >= 2 && want <= kMaxBuf) {
        st.nbuf = want;
    } else {
        st.nbuf = 2;
        for (int need : {needg, need1}) {
            bool found = false;
            for (int nbuf = kMaxBuf; nbuf >= 2 && !found; --nbuf)
                if (cap_of(nbuf) >= need) {
                    st.nbuf = nbuf;
                    found = true;
                }
            if (found) break;
        }
    }
    st.cmax = std::max(2, cap_of(st.nbuf));
    return st;
}

ProjGroups proj_make_groups(const HostGeometry &g, const std::vector<int> &list, int cmax)
{
    // positions of the list in runs of angularly adjacent views of one axis
    const std::vector<std::vector<int>> byaxis = view_runs(g, list);
    // CTLAB_PROJ_GMAX (1, 2 or 4) caps the views per CTA; default 4
    int gmax = kGMax;
    if (const char *env = std::getenv("CTLAB_PROJ_GMAX")) {
        const int v = std::atoi(env);
        if (v == 1 || v == 2 || v == 4) gmax = v;
    }
    ProjGroups out;
    for (int G : {4, 2, 1}) {
        if (G > gmax) continue;
        bool ok = true;
        std::vector<int> table;
        for (const auto &v : byaxis) {
            for (size_t i0 = 0; i0 < v.size() && ok; i0 += G) {
                std::vector<const DevView *> vs;
                for (int k = 0; k < G; ++k) {
                    const bool has = i0 + k < v.size();
                    table.push_back(has ? v[i0 + k] : -1);
                    if (has) vs.push_back(&g.views[list[v[i0 + k]]]);
                }
                if (G > 1)
                    for (int u0 = 0; u0 < g.DNU && ok; u0 += kU) {
                        const int nu = std::min(kU, g.DNU - u0);
                        const int na = vs[0]->na;
                        if (tile_span(g, vs, u0, nu, 0) > cmax || tile_span(g, vs, u0, nu, na - 1) > cmax) ok = false;
                    }
            }
        }
        if (ok || G == 1) {
            out.G = G;
            out.table = std::move(table);
            out.ngroups = (int)out.table.size() / G;
            return out;
        }
    }
    return out;
}

cudaError_t launch_proj(const ProjArgs &a, cudaStream_t s, int *launches)
{
    if (a.n <= 0 || a.ngroups <= 0) return cudaSuccess;
    if (a.ngroups > 65535) return cudaErrorInvalidConfiguration;
    if (launches) ++*launches;
    return a.f32pair ? launch_t<ff2>(a, s) : launch_t<double>(a, s);
}

} // namespace ctlab
