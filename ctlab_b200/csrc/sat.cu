// Summed-area tables: single-pass chunked scans.
//
// A SAT set is a stack of planes; in each plane the contiguous axis k (z for
// volumes, v for projections) is scanned inside a CTA with warp shuffles,
// and the strided axis s (the in-plane axis across the slice, or u for
// projections) is scanned sequentially per thread over a chunk of rows and
// across chunks with a decoupled lookback: each CTA publishes its chunk
// aggregate, then walks back over its predecessors' published aggregates or
// inclusive prefixes.  Chunks are handed out by an atomic ticket so every
// predecessor of a running CTA has already started, and every spin on a
// predecessor's flag is bounded: on timeout the CTA raises the device error
// word and stops looking back, so the launch always terminates.
//
// Output layout: out[plane][s'][k'] for s' in [0, ns], k' in [0, nk] with
// row stride kp (padded), zero first row and column:
//   out[P][s'][k'] = sum_{s < s', k < k'} in(P, s, k)
#include "ffloat.cuh"
#include "internal.h"

namespace ctlab {

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr unsigned kFull = 0xffffffffu;

template <class T> struct Acc;

template <> struct Acc<double> {
    static __device__ __forceinline__ double zero() { return 0.0; }
    static __device__ __forceinline__ double from(float x) { return (double)x; }
    static __device__ __forceinline__ double add(double a, double b) { return a + b; }
    static __device__ __forceinline__ double shfl_up(double v, int d) { return __shfl_up_sync(kFull, v, d); }
};

template <> struct Acc<ff2> {
    static __device__ __forceinline__ ff2 zero() { return {0.f, 0.f}; }
    static __device__ __forceinline__ ff2 from(float x) { return {x, 0.f}; }
    static __device__ __forceinline__ ff2 add(ff2 a, ff2 b) { return ff_add(a, b); }
    static __device__ __forceinline__ ff2 shfl_up(ff2 v, int d)
    {
        return {__shfl_up_sync(kFull, v.hi, d), __shfl_up_sync(kFull, v.lo, d)};
    }
};

// Block-wide exclusive scan of one value per thread.  s_warp is a
// [2][kWarps] buffer used alternately by consecutive calls (parity) so one
// barrier per call suffices between reuse.
template <class T>
__device__ __forceinline__ T block_exclusive_scan(T v, T *s_warp, int parity)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    T x = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        T y = Acc<T>::shfl_up(x, d);
        if (lane >= d) x = Acc<T>::add(y, x);
    }
    T ex_lane = Acc<T>::shfl_up(x, 1);
    if (lane == 0) ex_lane = Acc<T>::zero();
    T *sw = s_warp + parity * kWarps;
    if (lane == 31) sw[wid] = x;
    __syncthreads();
    T wpre = Acc<T>::zero();
    for (int w = 0; w < wid; ++w) wpre = Acc<T>::add(wpre, sw[w]);
    return Acc<T>::add(wpre, ex_lane);
}

// L2 loads of a predecessor's published vector (never served from L1).
__device__ __forceinline__ double ldcg_val(const double *p) { return __ldcg(p); }
__device__ __forceinline__ ff2 ldcg_val(const ff2 *p)
{
    const float2 f = __ldcg(reinterpret_cast<const float2 *>(p));
    return {f.x, f.y};
}

__device__ __forceinline__ int ld_flag(const int *p)
{
    return *(volatile const int *)p;
}

// Bounded wait for a predecessor's status flag; returns the flag, or -1
// after spin_limit polls (and raises the error word).
__device__ int wait_flag(const int *flag, int *err, unsigned spin_limit)
{
    int f = ld_flag(flag);
    unsigned n = 0;
    while (f == 0) {
        if (++n > spin_limit) {
            atomicExch(err, CTLAB_ERR_TIMEOUT);
            return -1;
        }
        __nanosleep(64);
        f = ld_flag(flag);
    }
    __threadfence();
    return f;
}

// Input functors: value of element (plane, s, k).
struct VolInY { // SAT_y: plane = y slice j, s = x index, k = z
    const float *vol;
    const unsigned char *mask;
    int XN, ZN;
    __device__ __forceinline__ float operator()(int plane, int s, int k) const
    {
        const long long col = (long long)plane * XN + s;
        const float m = mask ? (mask[col] ? 1.f : 0.f) : 1.f;
        return __ldg(vol + col * ZN + k) * m;
    }
};

struct VolInX { // SAT_x: plane = x slice i, s = y index, k = z
    const float *vol;
    const unsigned char *mask;
    int XN, ZN;
    __device__ __forceinline__ float operator()(int plane, int s, int k) const
    {
        const long long col = (long long)s * XN + plane;
        const float m = mask ? (mask[col] ? 1.f : 0.f) : 1.f;
        return __ldg(vol + col * ZN + k) * m;
    }
};


template <class In, class T, int KPT>
__global__ void __launch_bounds__(kThreads)
    sat_scan_kernel(In in, T *__restrict__ out, int ns, int nk, int kp, int chunk, int nchunks,
                    int *ticket, int *flags, T *agg, T *pref, int *err, unsigned spin_limit,
                    int stall_tile)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *buf = reinterpret_cast<T *>(smem_raw); // [chunk][kThreads*KPT]
    __shared__ T s_warp[2 * kWarps];
    __shared__ int s_tile, s_flag;

    const int tid = threadIdx.x;
    if (tid == 0) s_tile = atomicAdd(ticket, 1);
    __syncthreads();
    const int tile = s_tile;
    const int plane = tile / nchunks, c = tile - plane * nchunks;
    const int s0 = c * chunk, s1 = min(ns, s0 + chunk);
    const int k0 = tid * KPT;
    const int bw = kThreads * KPT;

    T run[KPT];
#pragma unroll
    for (int r = 0; r < KPT; ++r) run[r] = Acc<T>::zero();

    for (int s = s0; s < s1; ++s) {
        T loc[KPT];
        T tot = Acc<T>::zero();
#pragma unroll
        for (int r = 0; r < KPT; ++r) {
            const int k = k0 + r;
            const float v = (k < nk) ? in(plane, s, k) : 0.f;
            tot = Acc<T>::add(tot, Acc<T>::from(v));
            loc[r] = tot;
        }
        const T ex = block_exclusive_scan(tot, s_warp, s & 1);
#pragma unroll
        for (int r = 0; r < KPT; ++r) {
            run[r] = Acc<T>::add(run[r], Acc<T>::add(ex, loc[r]));
            buf[(s - s0) * bw + k0 + r] = run[r];
        }
    }

    // Publish the chunk aggregate (or, for chunk 0, the inclusive prefix).
    const long long sidx = (long long)plane * nchunks + c;
    T excl[KPT];
#pragma unroll
    for (int r = 0; r < KPT; ++r) excl[r] = Acc<T>::zero();
    const bool publish = (tile != stall_tile); // stall_tile: diagnostics only, never set in normal use
    if (c == 0) {
#pragma unroll
        for (int r = 0; r < KPT; ++r)
            if (k0 + r < nk) pref[sidx * nk + k0 + r] = run[r];
        __threadfence();
        __syncthreads();
        if (tid == 0 && publish) atomicExch(flags + sidx, 2);
    } else {
#pragma unroll
        for (int r = 0; r < KPT; ++r)
            if (k0 + r < nk) agg[sidx * nk + k0 + r] = run[r];
        __threadfence();
        __syncthreads();
        if (tid == 0 && publish) atomicExch(flags + sidx, 1);

        // Decoupled lookback over predecessors of the same plane.
        for (int pred = c - 1; pred >= 0; --pred) {
            const long long pidx = (long long)plane * nchunks + pred;
            if (tid == 0) s_flag = wait_flag(flags + pidx, err, spin_limit);
            __syncthreads();
            const int f = s_flag;
            __syncthreads();
            if (f < 0) break;
            const T *src = (f == 2) ? pref : agg;
#pragma unroll
            for (int r = 0; r < KPT; ++r)
                if (k0 + r < nk) {
                    excl[r] = Acc<T>::add(excl[r], ldcg_val(src + pidx * nk + k0 + r));
                }
            if (f == 2) break;
        }
#pragma unroll
        for (int r = 0; r < KPT; ++r)
            if (k0 + r < nk) pref[sidx * nk + k0 + r] = Acc<T>::add(excl[r], run[r]);
        __threadfence();
        __syncthreads();
        if (tid == 0 && publish) atomicExch(flags + sidx, 2);
    }

    // Write the chunk's rows: out[plane][s+1][k+1] = excl + running sum.
    const long long pstride = (long long)(ns + 1) * kp;
    T *op = out + plane * pstride;
    for (int s = s0; s < s1; ++s) {
        T *row = op + (long long)(s + 1) * kp;
#pragma unroll
        for (int r = 0; r < KPT; ++r) {
            const int k = k0 + r;
            if (k < nk) row[k + 1] = Acc<T>::add(excl[r], buf[(s - s0) * bw + k]);
        }
        if (tid == 0) row[0] = Acc<T>::zero();
    }
    if (c == 0)
        for (int k = tid; k <= nk; k += kThreads) op[k] = Acc<T>::zero();
}

// Default bound on polls of one predecessor flag (each poll sleeps ~64 ns,
// so about a second of waiting before the launch gives up).
constexpr unsigned kSpinLimit = 1u << 24;

template <class In, class T, int K>
cudaError_t launch_scan_k(In in, T *out, int ns, int nk, int kp, int chunk, int nchunks,
                          unsigned tiles, ScanState st, cudaStream_t s, unsigned spin_limit, int stall)
{
    const size_t sm = sizeof(T) * (size_t)chunk * kThreads * K;
    auto kern = sat_scan_kernel<In, T, K>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    kern<<<tiles, kThreads, sm, s>>>(in, out, ns, nk, kp, chunk, nchunks, st.ticket, st.flags,
                                     reinterpret_cast<T *>(st.agg), reinterpret_cast<T *>(st.pref),
                                     st.err, spin_limit, stall);
    return cudaGetLastError();
}

int kpt_for(int nk)
{
    const int need = (nk + kThreads - 1) / kThreads;
    int k = 1;
    while (k < need) k <<= 1;
    return k;
}

// Largest chunk whose row buffer fits in ~96 KB of shared memory.
int clamp_chunk(int chunk, int kpt, size_t elem)
{
    const size_t per_row = elem * (size_t)kThreads * kpt;
    int cmax = (int)((96 * 1024) / per_row);
    if (cmax < 1) cmax = 1;
    return chunk < cmax ? chunk : cmax;
}

template <class In, class T>
cudaError_t launch_scan(In in, T *out, int nplanes, int ns, int nk, int kp, ScanState st, int chunk,
                        cudaStream_t s, unsigned spin_limit, int stall = -1)
{
    if (nplanes <= 0 || ns <= 0 || nk <= 0) return cudaSuccess;
    const int kpt = kpt_for(nk);
    if (kpt > 16) return cudaErrorInvalidValue;
    chunk = clamp_chunk(chunk < 1 ? 1 : chunk, kpt, sizeof(T));
    const int nchunks = (ns + chunk - 1) / chunk;
    const long long tiles = (long long)nplanes * nchunks;
    if (tiles > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
    cudaError_t e = cudaMemsetAsync(st.ticket, 0, sizeof(int), s);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(st.flags, 0, sizeof(int) * (size_t)tiles, s);
    if (e != cudaSuccess) return e;
    switch (kpt) {
    case 1: return launch_scan_k<In, T, 1>(in, out, ns, nk, kp, chunk, nchunks, (unsigned)tiles, st, s, spin_limit, stall);
    case 2: return launch_scan_k<In, T, 2>(in, out, ns, nk, kp, chunk, nchunks, (unsigned)tiles, st, s, spin_limit, stall);
    case 4: return launch_scan_k<In, T, 4>(in, out, ns, nk, kp, chunk, nchunks, (unsigned)tiles, st, s, spin_limit, stall);
    case 8: return launch_scan_k<In, T, 8>(in, out, ns, nk, kp, chunk, nchunks, (unsigned)tiles, st, s, spin_limit, stall);
    default: return launch_scan_k<In, T, 16>(in, out, ns, nk, kp, chunk, nchunks, (unsigned)tiles, st, s, spin_limit, stall);
    }
}

} // namespace

size_t scan_state_doubles(int planes, int chunks, int nk)
{
    return (size_t)planes * (size_t)chunks * (size_t)nk;
}

int scan_chunks(int ns, int nk, int chunk, int f32pair)
{
    (void)f32pair;
    const int c = clamp_chunk(chunk < 1 ? 1 : chunk, kpt_for(nk), 8);
    return (ns + c - 1) / c;
}

cudaError_t launch_volume_sat(const float *vol, const unsigned char *mask, int XN, int YN, int ZN,
                              int orientation, void *out, int zp, int f32pair, ScanState st,
                              int chunk, cudaStream_t s)
{
    if (orientation == 0) {
        VolInY in{vol, mask, XN, ZN};
        return f32pair ? launch_scan(in, (ff2 *)out, YN, XN, ZN, zp, st, chunk, s, kSpinLimit)
                       : launch_scan(in, (double *)out, YN, XN, ZN, zp, st, chunk, s, kSpinLimit);
    }
    VolInX in{vol, mask, XN, ZN};
    return f32pair ? launch_scan(in, (ff2 *)out, XN, YN, ZN, zp, st, chunk, s, kSpinLimit)
                   : launch_scan(in, (double *)out, XN, YN, ZN, zp, st, chunk, s, kSpinLimit);
}

namespace {

// Slice-major z-prefixes: one CTA per 32 columns of one slice.  Each warp
// scans 4 columns 32 rows at a time (coalesced loads along z, FP64 warp
// scan plus a carried FP64 total); row k of a column is the pair (P, f):
// f = f[k], the voxel value and exact slope of the prefix on [k, k+1] (0 at
// k = ZN), and P = Z[k] - k f with Z[k] the FP64 prefix of the voxels below
// k, so that P + kz f is the prefix at kz in [k, k+1] (P rounded to FP32
// once).  The pairs go through a padded shared tile and the CTA writes them
// out as rows of 32 adjacent columns.
__global__ void __launch_bounds__(256) zt_kernel(const float *__restrict__ vol, const unsigned char *mask, int XN,
                                                 int ZN, int nb, int orientation, float2 *__restrict__ out, int rs,
                                                 int j0, int c_off)
{
    __shared__ float2 tile[32][33];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int j = blockIdx.y + j0, c0 = blockIdx.x * 32 + c_off;
    const float *col[4];
    float m[4];
    double carry[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int c = c0 + warp * 4 + i;
        const bool valid = c < nb;
        const int x = orientation ? j : c, y = orientation ? c : j;
        const long long ci = valid ? (long long)y * XN + x : 0;
        col[i] = vol + ci * ZN;
        m[i] = valid ? (mask ? (mask[ci] ? 1.f : 0.f) : 1.f) : 0.f;
        carry[i] = 0.0;
    }
    float2 *plane = out + (long long)j * (ZN + 1) * rs;
    const int cw = c0 + lane;
    for (int z0 = 0; z0 < ZN; z0 += 32) {
        const int z = z0 + lane;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const float f = (z < ZN && m[i] != 0.f) ? __ldg(col[i] + z) * m[i] : 0.f;
            double v = (double)f;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const double y = __shfl_up_sync(kFull, v, d);
                if (lane >= d) v += y;
            }
            v += carry[i];
            // the prefix below row z: the inclusive prefix of the lane below
            const double below = __shfl_up_sync(kFull, v, 1);
            const double zk = lane == 0 ? carry[i] : below;
            tile[lane][warp * 4 + i] = make_float2((float)(zk - (double)z * (double)f), f);
            carry[i] = __shfl_sync(kFull, v, 31);
        }
        __syncthreads();
        for (int rr = warp; rr < 32; rr += 8) {
            const int k = z0 + rr;
            if (k < ZN && cw < rs) plane[(long long)k * rs + cw] = cw < nb ? tile[rr][lane] : make_float2(0.f, 0.f);
        }
        __syncthreads();
    }
    // row ZN: the column total, slope 0
    if (lane == 0) {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int c = c0 + warp * 4 + i;
            if (c < rs) plane[(long long)ZN * rs + c] = make_float2(c < nb ? (float)carry[i] : 0.f, 0.f);
        }
    }
}

// Z[k] = P + k f of every pair of a z-prefix array [planes][rows][rs].
__global__ void __launch_bounds__(256) zt_unpack_kernel(const float2 *__restrict__ in, float *__restrict__ out,
                                                        long long n, int rows, int rs)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int k = (int)((i / rs) % rows);
        const float2 pf = in[i];
        out[i] = fmaf((float)k, pf.y, pf.x);
    }
}

} // namespace

cudaError_t launch_zt_unpack(const float2 *in, float *out, int planes, int rows, int rs, cudaStream_t s)
{
    const long long n = (long long)planes * rows * rs;
    if (n <= 0) return cudaSuccess;
    const int grid = (int)std::min<long long>((n + 255) / 256, 148 * 16);
    zt_unpack_kernel<<<grid, 256, 0, s>>>(in, out, n, rows, rs);
    return cudaGetLastError();
}

cudaError_t launch_zt(const float *vol, const unsigned char *mask, int XN, int YN, int ZN, int orientation,
                      float2 *out, int rs, cudaStream_t s)
{
    return launch_zt_rows(vol, mask, XN, YN, ZN, orientation, out, rs, 0, YN, s);
}

cudaError_t launch_zt_rows(const float *vol, const unsigned char *mask, int XN, int YN, int ZN, int orientation,
                           float2 *out, int rs, int y0, int y1, cudaStream_t s)
{
    const int nb = orientation ? YN : XN, na = orientation ? XN : YN;
    if (rs < nb || na > 65535 || y0 < 0 || y1 > YN || y0 > y1) return cudaErrorInvalidValue;
    if (y1 == y0) return cudaSuccess;
    if (orientation == 0) {
        // slices y0 .. y1-1, every column
        dim3 grid((rs + 31) / 32, y1 - y0);
        zt_kernel<<<grid, 256, 0, s>>>(vol, mask, XN, ZN, nb, 0, out, rs, y0, 0);
    } else {
        // every slice, columns y0 .. y1-1 (y0 a multiple of 32; the range that
        // ends the volume also covers the pad columns up to rs)
        if (y0 % 32) return cudaErrorInvalidValue;
        const int c1 = y1 == YN ? rs : y1;
        dim3 grid((c1 - y0 + 31) / 32, na);
        zt_kernel<<<grid, 256, 0, s>>>(vol, mask, XN, ZN, nb, 1, out, rs, 0, y0);
    }
    return cudaGetLastError();
}

cudaError_t launch_scan_stall(const float *vol, int rows, int nk, void *out, ScanState st, int chunk,
                              unsigned spin_limit, cudaStream_t s)
{
    // One plane whose first chunk never publishes: its successor's bounded
    // wait must run out and raise the error word.
    VolInY in{vol, nullptr, rows, nk};
    return launch_scan(in, (double *)out, 1, rows, nk, nk + 1, st, chunk, s, spin_limit, 0);
}

cudaError_t launch_proj_sat(const ProjSatArgs &a, ScanState st, int chunk, cudaStream_t s)
{
    PrjIn in{a.prj, a.views, a.view_list, a.det, det_table_layout(a.DNU, a.DNV), a.DNU, a.DNV, a.dx};
    return a.f32pair ? launch_scan(in, (ff2 *)a.out, a.n, a.DNU, a.DNV, a.vp, st, chunk, s, kSpinLimit)
                     : launch_scan(in, (double *)a.out, a.n, a.DNU, a.DNV, a.vp, st, chunk, s, kSpinLimit);
}

} // namespace ctlab
