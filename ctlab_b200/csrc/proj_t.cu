// Branchless DD cone-beam forward projection on slice-major column
// z-prefixes (sat mode CTLAB_SAT_ZPREFIX).
//
// Volume data, one array per driving axis: planes j (the slices along the
// axis) of ZN+1 rows k by nb columns c, c fastest,
//     Z[j][k][c] = sum_{z<k} f(column c of slice j, z)   (FP64 sums, FP32),
// i.e. Z_y[y][k][x] for y-driven views and Z_x[x][k][y] for x-driven ones.
// For piecewise-constant voxels the z-prefix interpolated linearly in z is
// the exact integral of the column up to kz, so the integral over an
// axis-aligned rectangle of a slice is a weighted sum of interpolated
// column prefixes -- the difference-of-SAT of the branchless DD method with
// the FP64 in-plane prefix replaced by its exact column differences (which
// the 2-D FP64 SAT path also rounds to FP32 before use).
//
// One CTA owns 32 detector columns (one per lane) of a group of G views of
// one driving axis with adjacent angles and sweeps the slices.
//   producer warp  per slice j, every lane maps the two boundary rays of its
//                  detector column onto slice j for every view of the group
//                  in FP64: SAT columns and fractions -> the strip weights,
//                  the central-ray magnification T and 1/(W T) (W the strip
//                  width in columns); a warp reduction gives the columns and
//                  z rows the group touches; one 3-D TMA tile load per 256
//                  rows brings that [rows][columns] block into a ring of
//                  stages, completed on a "full" mbarrier together with the
//                  per-view tables;
//   consumer warps lanes = detector columns, warp w = NR detector rows.  For
//                  each of the NR+1 z boundaries e_w of its rows,
//                      kz = Z0 + T e_w,
//                      F(kz) = wa Za(kz) + wb Zb(kz) [+ whole columns between],
//                  Zc(kz) the column prefix interpolated in z, and
//                      acc[v] += (F(kz_{v+1}) - F(kz_v)) / (W T).
//                  Lanes read neighbouring columns of nearly the same rows,
//                  so the shared-memory loads are free of bank conflicts.
//                  Each warp hands the stage back on an "empty" mbarrier.
// floor(kz) comes from the round-toward-zero add of 2^23, so the inner loop
// issues no float/int conversions.  Slices whose block exceeds a stage read
// the z-prefixes from global memory instead.  Epilogue: central-ray slab
// length L = dx |C - S| / |C_a - S_a|, 1/(e_{v+1} - e_v), and optionally the
// SART residual (b - Ax)/rowSum with a residual reduction.
#include <cuda.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdlib>
#include <type_traits>
#include <utility>

#include "internal.h"
#include "tma.cuh"

namespace ctlab {

namespace {

constexpr int kTU = 32;          // detector columns per CTA (one per lane)
constexpr int kTMaxStage = 4;
constexpr int kTMaxWarps = 8;    // consumer warps
constexpr int kTMaxG = 8;
constexpr size_t kTSmemLimit = 227 * 1024;
constexpr size_t kTStatic = 10 * 1024; // static shared arrays, rounded up

struct __align__(16) TEntry {
    float T, scale, wa, wb;
};
struct TSlice {
    int c_lo, k_lo, fits, nbox;
    float kz_lo, kz_hi;
    int pad0, pad1;
};

// f(integral_constant<int, 0>) ... f(integral_constant<int, N-1>): a loop
// whose index is a compile-time constant in the body (register arrays).
template <class F, int... I>
__device__ __forceinline__ void static_for_impl(F &&f, std::integer_sequence<int, I...>)
{
    (f(std::integral_constant<int, I>()), ...);
}
template <int N, class F>
__device__ __forceinline__ void static_for(F &&f)
{
    static_for_impl(f, std::make_integer_sequence<int, N>());
}

template <int NR, int G>
__global__ void __launch_bounds__((kTMaxWarps + 1) * 32, 1)
    dd3_proj_t_kernel(ProjArgs a, const __grid_constant__ CUtensorMap tm_y, const __grid_constant__ CUtensorMap tm_x)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    // TMA destinations need 128-byte alignment (the launch adds 128 bytes)
    unsigned char *smem = smem_raw + ((128 - (smem_addr(smem_raw) & 127)) & 127);
    const int NW = a.t_nw, nstage = a.t_nstage;
    const int CB = a.t_cb, KB = a.t_kb, KR = a.t_kr, EP = a.t_ep, GT = a.t_gtab;
    const int stage_floats = KR * CB;
    float *stage0 = reinterpret_cast<float *>(smem);                                 // [nstage][KR][CB]
    TEntry *s_tab = reinterpret_cast<TEntry *>(smem + 4 * stage_floats * nstage);    // [nstage][GT][32]
    int2 *s_cd = reinterpret_cast<int2 *>(s_tab + nstage * GT * kTU);                // [nstage][GT][32]
    float *s_e = reinterpret_cast<float *>(s_cd + nstage * GT * kTU);                // [G][EP]
    __shared__ __align__(8) uint64_t s_full[kTMaxStage], s_empty[kTMaxStage];
    __shared__ TSlice s_info[kTMaxStage];
    __shared__ double s_c0[G][kTU + 1], s_m[G][kTU + 1], s_r[G][kTU];
    __shared__ double s_ga0[G];
    __shared__ float s_Z0[G], s_emin[G], s_emax[G];
    __shared__ int s_pos_list[G];
    __shared__ int s_abort;
    __shared__ double s_red[kTMaxWarps + 1];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid < G) s_pos_list[tid] = a.groups[blockIdx.y * G + tid];
    if (tid == 0) s_abort = 0;
    const int u0 = blockIdx.x * kTU;
    const int nu = min(kTU, a.DNU - u0);
    const DetTable t = det_table_layout(a.DNU, a.DNV);
    const double *det = a.det;
    const int ZN = a.ZN, DNV = a.DNV;
    const double dx = a.dx;
    __syncthreads();
    const DevView &V0 = a.views[a.view_list[s_pos_list[0]]]; // all views of the group share the axis
    const int na = V0.na, nb = V0.nb, xdrv = V0.xdrv;
    const float *zt = xdrv ? a.zt_x : a.zt_y;
    const int zrs = xdrv ? a.zt_rs_x : a.zt_rs_y;
    auto view_of = [&](int g) -> const DevView & {
        const int ps = s_pos_list[g] >= 0 ? s_pos_list[g] : s_pos_list[0];
        return a.views[a.view_list[ps]];
    };

    if (tid == 0) {
        for (int i = 0; i < nstage; ++i) {
            mbar_init(&s_full[i], 32);
            mbar_init(&s_empty[i], NW);
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
    // detector z boundaries in SAT-row units, relative to the source; rows
    // past DNV repeat the last boundary (their cells are never stored)
    for (int it = tid; it < G * EP; it += nthreads) {
        const int g = it / EP, w = min(it - g * EP, DNV);
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
        for (int w = 0; w <= DNV; ++w) {
            lo = fminf(lo, s_e[tid * EP + w]);
            hi = fmaxf(hi, s_e[tid * EP + w]);
        }
        s_emin[tid] = lo;
        s_emax[tid] = hi;
    }
    __syncthreads();

    double r2 = 0.0;
    if (warp == NW) {
        // ------------------------------ producer ------------------------------
        const CUtensorMap *tm = xdrv ? &tm_x : &tm_y;
        const int uq = min(lane, nu - 1);
        int issued = 0;
        for (int j = 0; j < na; ++j) {
            const int b = j % nstage;
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
            if (*(volatile int *)&s_abort) break;
            const double jd = (double)j;
            int cmin = INT_MAX, cmax = INT_MIN;
            float kmin = 1e30f, kmax = -1e30f;
            int ia_g[G], dc_g[G];
            TEntry te_g[G];
#pragma unroll
            for (int g = 0; g < G; ++g) {
                const double xa = fma(s_m[g][uq], jd, s_c0[g][uq]);
                const double xb = fma(s_m[g][uq + 1], jd, s_c0[g][uq + 1]);
                const double xac = fmin(fmax(xa, 0.0), (double)nb), xbc = fmin(fmax(xb, 0.0), (double)nb);
                const int ia = min((int)xac, nb - 1), ib = min((int)xbc, nb - 1);
                const float fa = (float)(xac - (double)ia), fb = (float)(xbc - (double)ib);
                const double T = (s_ga0[g] + jd * dx) * s_r[g][uq];
                const double den = (xb - xa) * T;
                const int dc = ib - ia;
                TEntry te;
                te.T = (float)T;
                te.scale = (den != 0.0) ? (float)(1.0 / den) : 0.f;
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
                te_g[g] = te;
                ia_g[g] = ia;
                dc_g[g] = dc;
                cmin = min(cmin, min(ia, ib));
                cmax = max(cmax, max(ia, ib));
                // z rows of the group: the consumers' kz = fma(T, e, Z0) is
                // monotone in e, so the extremes of e bound it exactly
                const float z0 = s_Z0[g];
                float k0 = fmaf(te.T, s_emin[g], z0), k1 = fmaf(te.T, s_emax[g], z0);
                k0 = fminf(fmaxf(k0, 0.f), (float)ZN);
                k1 = fminf(fmaxf(k1, 0.f), (float)ZN);
                kmin = fminf(kmin, fminf(k0, k1));
                kmax = fmaxf(kmax, fmaxf(k0, k1));
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                cmin = min(cmin, __shfl_xor_sync(0xffffffffu, cmin, o));
                cmax = max(cmax, __shfl_xor_sync(0xffffffffu, cmax, o));
                kmin = fminf(kmin, __shfl_xor_sync(0xffffffffu, kmin, o));
                kmax = fmaxf(kmax, __shfl_xor_sync(0xffffffffu, kmax, o));
            }
            // TMA: the innermost (column) coordinate must be a multiple of 4
            // floats (16 bytes); rows need no alignment
            const int c_lo = cmin & ~3;
            const int k_lo = max((int)kmin - 1, 0);
            const int k_top = min((int)kmax + 2, ZN + 1); // row of the last kz's upper neighbour
            const int nk = k_top - k_lo + 1;
            const bool fits = CB > 0 && (cmax - c_lo + 1 <= CB) && (nk <= KR);
            const int nbox = fits ? (nk + KB - 1) / KB : 0;
#pragma unroll
            for (int g = 0; g < G; ++g) {
                s_tab[(b * GT + g) * kTU + lane] = te_g[g];
                s_cd[(b * GT + g) * kTU + lane] = make_int2(fits ? ia_g[g] - c_lo : ia_g[g], dc_g[g]);
            }
            if (lane == 0) {
                TSlice in;
                in.c_lo = c_lo;
                in.k_lo = fits ? k_lo : 0;
                in.fits = fits;
                in.nbox = nbox;
                in.kz_lo = fits ? (float)k_lo : 0.f;
                in.kz_hi = fits ? (float)min(ZN, k_lo + KR - 2) : (float)ZN;
                in.pad0 = in.pad1 = 0;
                s_info[b] = in;
                mbar_arrive_expect_tx(&s_full[b], (uint32_t)(nbox * KB * CB * 4));
            }
            __syncwarp();
            if (lane < nbox)
                tma_load_3d(stage0 + b * stage_floats + lane * KB * CB, tm, c_lo, k_lo + lane * KB, j,
                            &s_full[b]);
            if (lane != 0) mbar_arrive(&s_full[b]);
            issued = j + 1;
        }
        // copies still in flight land before the CTA may exit
        if (lane == 0)
            for (int j = max(issued - nstage, 0); j < issued; ++j)
                if (!mbar_wait(&s_full[j % nstage], (uint32_t)((j / nstage) & 1)) && a.err)
                    atomicExch(a.err, CTLAB_ERR_TIMEOUT);
    } else {
        // ------------------------------ consumers -----------------------------
        const int v0 = warp * NR;
        float acc[G][NR];
#pragma unroll
        for (int g = 0; g < G; ++g)
#pragma unroll
            for (int r = 0; r < NR; ++r) acc[g][r] = 0.f;

        for (int j = 0; j < na; ++j) {
            const int b = j % nstage;
            if (!mbar_wait(&s_full[b], (uint32_t)((j / nstage) & 1))) {
                if (lane == 0) {
                    s_abort = 1;
                    if (a.err) atomicExch(a.err, CTLAB_ERR_TIMEOUT);
                }
                break;
            }
            const TSlice in = s_info[b];
            // one slice of one view g; GLB: the block is read from global memory
            auto slice_view = [&](auto glb_tag, auto g_tag) {
                constexpr bool GLB = decltype(glb_tag)::value;
                constexpr int g = decltype(g_tag)::value;
                const TEntry te = s_tab[(b * GT + g) * kTU + lane];
                const int2 cd = s_cd[(b * GT + g) * kTU + lane];
                const float z0 = s_Z0[g];
                const float *e = s_e + g * EP + v0;
                const float *S;
                int rs;
                if constexpr (GLB) {
                    S = zt + (long long)j * (ZN + 1) * zrs;
                    rs = zrs;
                } else {
                    S = stage0 + b * stage_floats;
                    rs = CB;
                }
                const int dc = cd.y;
                const int dstep = max(-1, min(1, dc)); // column b = a + dstep on the fast path
                const bool wide = __any_sync(0xffffffffu, dc > 1 || dc < -1);
                const float kzlo = in.kz_lo, kzhi = in.kz_hi;
                const int base = cd.x - (GLB ? 0 : in.k_lo) * rs;
                float prev = 0.f;
#pragma unroll
                for (int r = 0; r <= NR; ++r) {
                    float kz = fmaf(te.T, e[r], z0);
                    kz = fminf(fmaxf(kz, kzlo), kzhi);
                    int k0;
                    float fz;
                    if constexpr (GLB) {
                        k0 = min((int)kz, ZN - 1);
                        fz = kz - (float)k0;
                    } else {
                        // 0 <= kz < 2^23: adding 2^23 toward zero leaves floor(kz) in the mantissa
                        const float rr = __fadd_rz(kz, 8388608.f);
                        k0 = __float_as_int(rr) - 0x4B000000;
                        fz = kz - (rr - 8388608.f);
                    }
                    const int ia = base + k0 * rs;
                    const float a0 = S[ia], a1 = S[ia + rs];
                    const float b0 = S[ia + dstep], b1 = S[ia + dstep + rs];
                    const float Za = fmaf(fz, a1 - a0, a0);
                    const float Zb = fmaf(fz, b1 - b0, b0);
                    float F = fmaf(te.wb, Zb, te.wa * Za);
                    if (wide) {
                        // cells wider than a voxel column: whole columns between a and b
                        const int n = dc > 1 ? dc - 1 : (dc < -1 ? -dc - 1 : 0);
                        const int step = dc > 0 ? 1 : -1;
                        float sum = 0.f;
                        for (int i = 1; i <= n; ++i) {
                            const int ic = ia + i * step;
                            const float c0 = S[ic], c1 = S[ic + rs];
                            sum += fmaf(fz, c1 - c0, c0);
                        }
                        F += dc > 0 ? sum : -sum;
                    }
                    if (r > 0) acc[g][r - 1] = fmaf(F - prev, te.scale, acc[g][r - 1]);
                    prev = F;
                }
            };
            static_for<G>([&](auto g_tag) {
                constexpr int g = decltype(g_tag)::value;
                if (s_pos_list[g] < 0) return; // uniform: empty slot of a partial group
                if (in.fits)
                    slice_view(std::integral_constant<bool, false>(), g_tag);
                else
                    slice_view(std::integral_constant<bool, true>(), g_tag);
            });
            __syncwarp();
            if (lane == 0) mbar_arrive(&s_empty[b]);
        }

        // epilogue
        const bool owner = lane < nu;
#pragma unroll
        for (int g = 0; g < G; ++g) {
            const int li = s_pos_list[g];
            if (li < 0 || !owner) continue;
            const DevView &V = view_of(g);
            const int u = u0 + lane;
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
                        const float mv = a.meas[idx], rsum = a.row_sum[idx];
                        const float res = mv - val;
                        r2 += (double)res * (double)res;
                        a.out[idx] = (rsum > 1.0e-7f) ? res / rsum : 0.f;
                    } else {
                        a.out[idx] = val;
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
            for (int w = 0; w <= NW; ++w) sum += s_red[w];
            atomicAdd(a.resid2, sum);
        }
    }
}

size_t smem_bytes(const ProjTStaging &st)
{
    return 128 + 4 * (size_t)st.KR * st.CB * st.nstage + (size_t)st.nstage * st.G * kTU * (sizeof(TEntry) + sizeof(int2)) +
           sizeof(float) * (size_t)st.G * st.EP;
}

template <int NR, int G>
cudaError_t launch_t_g(const ProjArgs &a, const CUtensorMap &tmy, const CUtensorMap &tmx, size_t sm, cudaStream_t s)
{
    auto kern = dd3_proj_t_kernel<NR, G>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    dim3 grid((a.DNU + kTU - 1) / kTU, a.ngroups);
    kern<<<grid, (a.t_nw + 1) * 32, sm, s>>>(a, tmy, tmx);
    return cudaGetLastError();
}

template <int NR>
cudaError_t launch_t_nr(const ProjArgs &a, const CUtensorMap &tmy, const CUtensorMap &tmx, size_t sm,
                        cudaStream_t s)
{
    switch (a.G) {
    case 1: return launch_t_g<NR, 1>(a, tmy, tmx, sm, s);
    case 2: return launch_t_g<NR, 2>(a, tmy, tmx, sm, s);
    case 4: return launch_t_g<NR, 4>(a, tmy, tmx, sm, s);
    case 8:
        if constexpr (NR <= 8) return launch_t_g<NR, 8>(a, tmy, tmx, sm, s);
        return cudaErrorInvalidValue;
    default: return cudaErrorInvalidValue;
    }
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
    // floor(lo) rounded down to 4 (TMA alignment) and one column of margin
    // each side for rounding between host and device
    const int c_lo = std::max((int)lo - 1, 0) & ~3;
    const int c_hi = std::min((int)hi + 1, nb - 1);
    return c_hi - c_lo + 1;
}

// Largest column span of any group of G views (by axis, adjacent angles)
// over all tiles and slices; the span is convex in the slice index, so the
// end slices bound it.
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

// Views of `list` (view indices) grouped G at a time: by driving axis, then
// within runs of angularly adjacent views (a view's axis covers two opposite
// quadrant pairs, so the sorted angles of one axis have gaps); returns list
// positions.
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

int env_int(const char *name, int dflt)
{
    const char *s = std::getenv(name);
    return s ? std::atoi(s) : dflt;
}

} // namespace

ProjTStaging proj_t_staging(const HostGeometry &g)
{
    ProjTStaging st;
    st.ok = false;
    if (g.DNV > kTMaxWarps * 16) return st;
    st.NR = 1;
    while ((g.DNV + st.NR - 1) / st.NR > kTMaxWarps) st.NR *= 2;
    st.NW = (g.DNV + st.NR - 1) / st.NR;
    st.EP = ((st.NW * st.NR + 1) + 3) & ~3;
    const int nbox = (g.ZN + 2 + 255) / 256;
    const int kb0 = (g.ZN + 2 + nbox - 1) / nbox;
    // CTLAB_PROJT_GMAX caps the views per CTA (1, 2, 4, 8), CTLAB_PROJT_NSTAGE
    // fixes the depth (2..4), CTLAB_PROJT_CBMAX caps the staged columns
    const int gmax = std::min(env_int("CTLAB_PROJT_GMAX", kTMaxG), st.NR <= 8 ? 8 : 4);
    const int want_stage = env_int("CTLAB_PROJT_NSTAGE", 0);
    const int cbmax = std::min(env_int("CTLAB_PROJT_CBMAX", 256), 256);
    std::vector<int> all(g.PN);
    for (int i = 0; i < g.PN; ++i) all[i] = i;
    for (int G = 8; G >= 1; G /= 2) {
        if (G > gmax) continue;
        std::vector<std::vector<int>> groups = t_groups(g, all, G);
        for (auto &grp : groups)
            for (int &p : grp) p = all[p];
        int CB = (t_need(g, groups) + 3) & ~3;
        // a row stride of 16 (mod 32) floats keeps lanes that read neighbouring
        // rows off each other's banks; take it when it costs little
        const int cb16 = CB + ((16 - CB % 32) + 32) % 32;
        if (cb16 - CB <= 12) CB = cb16;
        if (CB > cbmax) {
            if (G > 1) continue;
            CB = cbmax & ~3; // G = 1: wider slices read global memory
        }
        // 128-byte aligned TMA destinations: KB * CB * 4 a multiple of 128
        int KB = kb0;
        while ((KB * CB) % 32) ++KB;
        if (KB > 256) continue;
        const int KR = nbox * KB;
        for (int ns = kTMaxStage; ns >= 2; --ns) {
            if (want_stage >= 2 && want_stage <= kTMaxStage && ns != want_stage) continue;
            ProjTStaging c = st;
            c.G = G;
            c.CB = CB;
            c.KB = KB;
            c.KR = KR;
            c.nstage = ns;
            c.smem = smem_bytes(c);
            // prefer two CTAs per SM (depth >= 2 within half the shared memory)
            const bool two = c.smem + kTStatic <= kTSmemLimit / 2;
            if (c.smem + kTStatic > kTSmemLimit) continue;
            if (!two && ns > 2 && want_stage == 0) {
                // a deep stage that forces one CTA per SM: try fewer stages first
                ProjTStaging c2 = c;
                c2.nstage = 2;
                c2.smem = smem_bytes(c2);
                if (c2.smem + kTStatic <= kTSmemLimit / 2) continue;
            }
            c.ok = true;
            return c;
        }
    }
    // nothing stages: every slice reads global memory
    st.G = 1;
    st.CB = 0;
    st.KB = 0;
    st.KR = 0;
    st.nstage = 2;
    st.smem = smem_bytes(st);
    st.ok = true;
    return st;
}

ProjGroups proj_t_make_groups(const HostGeometry &g, const std::vector<int> &list, const ProjTStaging &st)
{
    ProjGroups out;
    for (int G = st.G; G >= 1; G /= 2) {
        std::vector<std::vector<int>> groups = t_groups(g, list, G);
        if (G > 1) {
            std::vector<std::vector<int>> vgroups = groups;
            for (auto &grp : vgroups)
                for (int &p : grp) p = list[p];
            if (t_need(g, vgroups) > st.CB) continue;
        }
        out.G = G;
        out.table.clear();
        for (auto &grp : groups)
            for (int k = 0; k < G; ++k) out.table.push_back(k < (int)grp.size() ? grp[k] : -1);
        out.ngroups = (int)groups.size();
        return out;
    }
    return out;
}

cudaError_t launch_proj_t(const ProjArgs &a, const ProjTStaging &st, const CUtensorMap &tmy, const CUtensorMap &tmx,
                          cudaStream_t s, int *launches)
{
    if (a.n <= 0 || a.ngroups <= 0) return cudaSuccess;
    if (a.ngroups > 65535 || a.G > st.G) return cudaErrorInvalidConfiguration;
    if (launches) ++*launches;
    const size_t sm = smem_bytes(st);
    switch (st.NR) {
    case 1: return launch_t_nr<1>(a, tmy, tmx, sm, s);
    case 2: return launch_t_nr<2>(a, tmy, tmx, sm, s);
    case 4: return launch_t_nr<4>(a, tmy, tmx, sm, s);
    case 8: return launch_t_nr<8>(a, tmy, tmx, sm, s);
    case 16: return launch_t_nr<16>(a, tmy, tmx, sm, s);
    default: return cudaErrorInvalidValue;
    }
}

} // namespace ctlab
