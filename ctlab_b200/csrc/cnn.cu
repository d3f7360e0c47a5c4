// Learned warm start: kernels of a 2.5D residual CNN (3x3 convolutions,
// NHWC BF16 activations and weights, FP32 accumulation on the tensor cores).
//
// Network (one z slice at a time, H x W = YN x XN): 5 input channels (the
// slice and its two neighbours each side of an OS-SART image, scaled),
// conv 5->64 + ReLU, 6 x (conv 64->64 + ReLU), conv 64->1; the output is the
// centre channel plus the last convolution (a residual correction).
// Channels are padded to 16 (input, last output) or 64.
//
//   conv3x3_kernel  implicit GEMM, M = pixels (an 8 x 16 tile per CTA), N =
//                   output channels, K = 9 taps x input channels; the CTA
//                   keeps the layer's weights in shared memory and loops over
//                   tiles; the input halo tile and the weights use a 16-byte
//                   XOR swizzle so ldmatrix reads are bank-conflict free;
//                   mma.sync m16n8k16 BF16 -> FP32.  Epilogues: bias + ReLU
//                   (forward), mask by an activation's sign (backward through
//                   ReLU: the data gradient is the same convolution with the
//                   weights flipped in space and transposed in channels), or
//                   bias + centre channel in FP32 (the output layer).
//   wgrad_kernel    dW[co][tap][ci] = sum_p dPre[p][co] act[p + tap][ci]: per
//                   CTA one tap and a split of the pixels (the K of this GEMM),
//                   A and B fragments by ldmatrix.trans from the NHWC tiles,
//                   FP32 partial sums added atomically at the end.
//   small kernels   input packing, loss gradient, bias gradient, Adam (FP32
//                   master weights -> forward and flipped BF16 copies),
//                   prediction unpacking into the volume.
#include <cuda_bf16.h>

#include <cstdint>

#include "internal.h"

namespace ctlab {

namespace {

typedef __nv_bfloat16 bf16;

constexpr int kTH = 8, kTW = 16;               // output tile of a CTA: 8 rows x 16 columns
constexpr int kHH = kTH + 2, kHW = kTW + 2;    // input halo tile
constexpr int kCT = 128;                       // 4 warps, two tile rows each

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// 16-byte chunk c of row r of a [rows][CH chunks] tile, XOR-swizzled so the
// 8 rows an ldmatrix reads land in different banks.
template <int CH>
__device__ __forceinline__ int swz(int r, int c)
{
    if constexpr (CH >= 8) return c ^ (r & 7);
    else return c ^ ((r >> 2) & (CH - 1));
}

__device__ __forceinline__ void ldsm_x4(uint32_t addr, uint32_t &r0, uint32_t &r1, uint32_t &r2, uint32_t &r3)
{
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0, %1, %2, %3}, [%4];"
                 : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
                 : "r"(addr));
}
__device__ __forceinline__ void ldsm_x4_t(uint32_t addr, uint32_t &r0, uint32_t &r1, uint32_t &r2, uint32_t &r3)
{
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0, %1, %2, %3}, [%4];"
                 : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
                 : "r"(addr));
}
__device__ __forceinline__ void mma_bf16(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, uint32_t b0,
                                         uint32_t b1)
{
    asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
                 "{%0, %1, %2, %3};"
                 : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                 : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

struct ConvArgs {
    const bf16 *in;      // [B][H][W][CI]
    const bf16 *w;       // [CO][9][CI]
    const float *bias;   // [CO] (forward epilogues)
    bf16 *out;           // [B][H][W][CO] (BF16 epilogues)
    const bf16 *mask;    // [B][H][W][CO]: output kept where mask > 0 (CTLAB_CNN_EPI_MASK)
    float *out_f32;      // [B][H][W] (CTLAB_CNN_EPI_RESIDUAL)
    const float *center; // [B][H][W] (CTLAB_CNN_EPI_RESIDUAL)
    int B, H, W, epi;
};

template <int CI, int CO>
__global__ void __launch_bounds__(kCT) conv3x3_kernel(ConvArgs a)
{
    constexpr int NCH = CI / 8;  // 16-byte chunks per input pixel
    constexpr int NT = CO / 8;   // n8 tiles
    extern __shared__ __align__(128) unsigned char smem[];
    bf16 *s_w = reinterpret_cast<bf16 *>(smem);               // [CO][9][CI] swizzled
    bf16 *s_in = s_w + CO * 9 * CI;                           // [kHH*kHW][CI] swizzled
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

    // the layer's weights, once per CTA
    for (int i = tid; i < CO * 9 * NCH; i += kCT) {
        const int c = i % NCH, rt = i / NCH; // rt = co*9 + tap
        const int co = rt / 9;
        const uint4 v = *reinterpret_cast<const uint4 *>(a.w + (size_t)rt * CI + c * 8);
        *reinterpret_cast<uint4 *>(s_w + ((size_t)rt * NCH + swz<NCH>(co, c)) * 8) = v;
    }
    const int tiles_y = (a.H + kTH - 1) / kTH, tiles_x = (a.W + kTW - 1) / kTW;
    const int ntiles = a.B * tiles_y * tiles_x;
    const uint32_t w_base = smem_u32(s_w), in_base = smem_u32(s_in);

    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int b = tile / (tiles_y * tiles_x), tr = tile % (tiles_y * tiles_x);
        const int y0 = (tr / tiles_x) * kTH, x0 = (tr % tiles_x) * kTW;
        __syncthreads(); // previous tile's reads of s_in done (and the weights stored)
        for (int i = tid; i < kHH * kHW * NCH; i += kCT) {
            const int c = i % NCH, q = i / NCH;
            const int y = y0 - 1 + q / kHW, x = x0 - 1 + q % kHW;
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (y >= 0 && y < a.H && x >= 0 && x < a.W)
                v = *reinterpret_cast<const uint4 *>(a.in + (((size_t)b * a.H + y) * a.W + x) * CI + c * 8);
            *reinterpret_cast<uint4 *>(s_in + ((size_t)q * NCH + swz<NCH>(q, c)) * 8) = v;
        }
        __syncthreads();

        float acc[2][NT][4];
#pragma unroll
        for (int m = 0; m < 2; ++m)
#pragma unroll
            for (int n = 0; n < NT; ++n)
#pragma unroll
                for (int e = 0; e < 4; ++e) acc[m][n][e] = 0.f;

        const int mi = lane >> 3, ri = lane & 7;
#pragma unroll 1
        for (int t = 0; t < 9; ++t) {
            const int dy = t / 3, dx = t % 3;
#pragma unroll
            for (int c16 = 0; c16 < CI / 16; ++c16) {
                uint32_t af[2][4];
#pragma unroll
                for (int m = 0; m < 2; ++m) {
                    const int r = warp * 2 + m; // tile row
                    const int px = (mi & 1) * 8 + ri, ch = 2 * c16 + (mi >> 1);
                    const int q = (r + dy) * kHW + px + dx;
                    ldsm_x4(in_base + (uint32_t)((q * NCH + swz<NCH>(q, ch)) * 16), af[m][0], af[m][1], af[m][2],
                            af[m][3]);
                }
#pragma unroll
                for (int n2 = 0; n2 < NT / 2; ++n2) {
                    const int co = n2 * 16 + (mi >> 1) * 8 + ri, ch = 2 * c16 + (mi & 1);
                    uint32_t b0, b1, b2, b3;
                    ldsm_x4(w_base + (uint32_t)(((co * 9 + t) * NCH + swz<NCH>(co, ch)) * 16), b0, b1, b2, b3);
#pragma unroll
                    for (int m = 0; m < 2; ++m) {
                        mma_bf16(acc[m][2 * n2], af[m][0], af[m][1], af[m][2], af[m][3], b0, b1);
                        mma_bf16(acc[m][2 * n2 + 1], af[m][0], af[m][1], af[m][2], af[m][3], b2, b3);
                    }
                }
            }
        }

        // epilogue: fragment (row lane/4 (+8), channels 2*(lane%4) + {0,1})
#pragma unroll
        for (int m = 0; m < 2; ++m) {
            const int y = y0 + warp * 2 + m;
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int x = x0 + (lane >> 2) + 8 * h;
                if (y >= a.H || x >= a.W) continue;
                const size_t pix = ((size_t)b * a.H + y) * a.W + x;
#pragma unroll
                for (int n = 0; n < NT; ++n) {
                    const int co = n * 8 + 2 * (lane & 3);
                    float v0 = acc[m][n][2 * h], v1 = acc[m][n][2 * h + 1];
                    if (a.epi == CTLAB_CNN_EPI_RESIDUAL) {
                        if (co == 0) a.out_f32[pix] = v0 + a.bias[0] + a.center[pix];
                        continue;
                    }
                    if (a.epi == CTLAB_CNN_EPI_RELU) {
                        v0 = fmaxf(v0 + a.bias[co], 0.f);
                        v1 = fmaxf(v1 + a.bias[co + 1], 0.f);
                    } else if (a.epi == CTLAB_CNN_EPI_MASK) {
                        const __nv_bfloat162 mk = *reinterpret_cast<const __nv_bfloat162 *>(a.mask + pix * CO + co);
                        if (!(__bfloat162float(mk.x) > 0.f)) v0 = 0.f;
                        if (!(__bfloat162float(mk.y) > 0.f)) v1 = 0.f;
                    }
                    *reinterpret_cast<__nv_bfloat162 *>(a.out + pix * CO + co) = __floats2bfloat162_rn(v0, v1);
                }
            }
        }
    }
}

// dW[co][tap][ci] += sum over pixels p of dpre[p][co] * act[p shifted by tap][ci].
// Grid (9 taps, splits); each CTA takes a contiguous range of 128-pixel tiles.
template <int CI, int CO>
__global__ void __launch_bounds__(kCT) wgrad_kernel(const bf16 *__restrict__ dpre, const bf16 *__restrict__ act,
                                                    float *__restrict__ dw, int B, int H, int W)
{
    constexpr int NCI = CI / 8, NCO = CO / 8;
    constexpr int MT = CO / 16, NT = CI / 8, WN = NT * MT / 4; // m16 tiles, n8 tiles, n8 tiles per warp
    static_assert(WN >= 1 && (WN % 2) == 0, "warp split");
    __shared__ __align__(128) bf16 s_d[128 * CO];  // [pixel][co] swizzled
    __shared__ __align__(128) bf16 s_a[128 * CI];  // [pixel][ci] swizzled
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int t = blockIdx.x, dy = t / 3 - 1, dx = t % 3 - 1;
    const long long P = (long long)B * H * W;
    const long long ntile = (P + 127) / 128;
    const long long per = (ntile + gridDim.y - 1) / gridDim.y;
    const long long t0 = blockIdx.y * per, t1 = min(ntile, t0 + per);
    const int mtile = warp % MT, nbase = (warp / MT) * WN;
    float acc[WN][4];
#pragma unroll
    for (int n = 0; n < WN; ++n)
#pragma unroll
        for (int e = 0; e < 4; ++e) acc[n][e] = 0.f;
    const uint32_t d_base = smem_u32(s_d), a_base = smem_u32(s_a);
    const int mi = lane >> 3, ri = lane & 7;

    for (long long tl = t0; tl < t1; ++tl) {
        __syncthreads();
        for (int i = tid; i < 128 * NCO; i += kCT) {
            const int c = i % NCO, q = i / NCO;
            const long long p = tl * 128 + q;
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (p < P) v = *reinterpret_cast<const uint4 *>(dpre + p * CO + c * 8);
            *reinterpret_cast<uint4 *>(s_d + ((size_t)q * NCO + swz<NCO>(q, c)) * 8) = v;
        }
        for (int i = tid; i < 128 * NCI; i += kCT) {
            const int c = i % NCI, q = i / NCI;
            const long long p = tl * 128 + q;
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (p < P) {
                const int x = (int)(p % W), y = (int)((p / W) % H);
                const long long b = p / ((long long)W * H);
                const int ys = y + dy, xs = x + dx;
                if (ys >= 0 && ys < H && xs >= 0 && xs < W)
                    v = *reinterpret_cast<const uint4 *>(act + ((b * H + ys) * W + xs) * CI + c * 8);
            }
            *reinterpret_cast<uint4 *>(s_a + ((size_t)q * NCI + swz<NCI>(q, c)) * 8) = v;
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < 8; ++k) { // 16 pixels per step
            // A (co x p) from [p][co]: matrices (co 0-7|8-15) x (p 0-7|8-15)
            uint32_t a0, a1, a2, a3;
            {
                const int q = k * 16 + (mi >> 1) * 8 + ri, ch = mtile * 2 + (mi & 1);
                ldsm_x4_t(d_base + (uint32_t)((q * NCO + swz<NCO>(q, ch)) * 16), a0, a1, a2, a3);
            }
#pragma unroll
            for (int n2 = 0; n2 < WN / 2; ++n2) {
                // B (p x ci) from [p][ci]: two n8 tiles
                const int q = k * 16 + (mi & 1) * 8 + ri, ch = nbase + 2 * n2 + (mi >> 1);
                uint32_t b0, b1, b2, b3;
                ldsm_x4_t(a_base + (uint32_t)((q * NCI + swz<NCI>(q, ch)) * 16), b0, b1, b2, b3);
                mma_bf16(acc[2 * n2], a0, a1, a2, a3, b0, b1);
                mma_bf16(acc[2 * n2 + 1], a0, a1, a2, a3, b2, b3);
            }
        }
    }
    // accumulate: fragment rows = co (lane/4, +8), columns = ci (2*(lane%4) + {0,1})
#pragma unroll
    for (int n = 0; n < WN; ++n) {
        const int ci = (nbase + n) * 8 + 2 * (lane & 3);
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int co = mtile * 16 + (lane >> 2) + 8 * h;
            atomicAdd(dw + ((size_t)co * 9 + t) * CI + ci, acc[n][2 * h]);
            atomicAdd(dw + ((size_t)co * 9 + t) * CI + ci + 1, acc[n][2 * h + 1]);
        }
    }
}

// db[co] += sum over pixels of dpre[p][co]
template <int CO>
__global__ void bias_grad_kernel(const bf16 *__restrict__ dpre, long long P, float *__restrict__ db)
{
    __shared__ float s[CO];
    for (int i = threadIdx.x; i < CO; i += blockDim.x) s[i] = 0.f;
    __syncthreads();
    const int co = threadIdx.x % CO, lanes = blockDim.x / CO;
    float sum = 0.f;
    for (long long p = blockIdx.x * (long long)lanes + threadIdx.x / CO; p < P; p += (long long)gridDim.x * lanes)
        sum += __bfloat162float(dpre[p * CO + co]);
    atomicAdd(&s[co], sum);
    __syncthreads();
    for (int i = threadIdx.x; i < CO; i += blockDim.x) atomicAdd(db + i, s[i]);
}

// Slice z of the volume (Z,X,Y order, [YN][XN][ZN]) -> NHWC input [H=YN][W=XN][16]:
// channels 0..4 = z-2 .. z+2 (clamped to the volume) times scale, 5..15 zero;
// centre[y][x] = vol[y][x][z] * scale.
__global__ void pack_kernel(const float *__restrict__ vol, int XN, int YN, int ZN, const int *__restrict__ zs, int nb,
                            float scale, bf16 *__restrict__ in, float *__restrict__ center)
{
    const long long n = (long long)nb * YN * XN;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int b = (int)(i / ((long long)YN * XN));
        const long long col = i - (long long)b * YN * XN; // y*XN + x
        const int z = min(max(zs[b], 0), ZN - 1);
        const float *c = vol + col * ZN;
        __align__(16) bf16 v[16];
#pragma unroll
        for (int k = 0; k < 16; ++k) v[k] = __float2bfloat16(0.f);
#pragma unroll
        for (int k = 0; k < 5; ++k) v[k] = __float2bfloat16(c[min(max(z + k - 2, 0), ZN - 1)] * scale);
        uint4 *o = reinterpret_cast<uint4 *>(in + i * 16);
        o[0] = *reinterpret_cast<const uint4 *>(v);
        o[1] = *reinterpret_cast<const uint4 *>(v + 8);
        if (center) center[i] = c[z] * scale;
    }
}

// Target slices (scaled) of a volume.
__global__ void slice_kernel(const float *__restrict__ vol, int XN, int YN, int ZN, const int *__restrict__ zs, int nb,
                             float scale, float *__restrict__ out)
{
    const long long n = (long long)nb * YN * XN;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int b = (int)(i / ((long long)YN * XN));
        const long long col = i - (long long)b * YN * XN;
        out[i] = vol[col * ZN + min(max(zs[b], 0), ZN - 1)] * scale;
    }
}

// Predicted slices (scaled) back into the volume: vol[y][x][z_b] = pred / scale.
__global__ void unpack_kernel(const float *__restrict__ pred, int XN, int YN, int ZN, const int *__restrict__ zs,
                              int nb, float inv_scale, float *__restrict__ vol)
{
    const long long n = (long long)nb * YN * XN;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int b = (int)(i / ((long long)YN * XN));
        const long long col = i - (long long)b * YN * XN;
        vol[col * ZN + min(max(zs[b], 0), ZN - 1)] = pred[i] * inv_scale;
    }
}

// MSE loss gradient: g[p][0] = 2 (pred - target) / n as BF16 (channels 1..15
// zero), and acc += sum (pred - target)^2.
__global__ void loss_grad_kernel(const float *__restrict__ pred, const float *__restrict__ target, long long n,
                                 bf16 *__restrict__ g, double *__restrict__ acc)
{
    double s = 0.0;
    const float k = 2.f / (float)n;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float d = pred[i] - target[i];
        s += (double)d * d;
        __align__(16) bf16 v[16];
#pragma unroll
        for (int c = 0; c < 16; ++c) v[c] = __float2bfloat16(0.f);
        v[0] = __float2bfloat16(k * d);
        uint4 *o = reinterpret_cast<uint4 *>(g + i * 16);
        o[0] = *reinterpret_cast<const uint4 *>(v);
        o[1] = *reinterpret_cast<const uint4 *>(v + 8);
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0 && acc) atomicAdd(acc, s);
}

// Adam on FP32 master weights w[CO][9][CI] (+ bias[CO]); writes the BF16
// forward copy and the flipped, channel-transposed copy for the data
// gradient: wt[ci][8 - tap][co] = w[co][tap][ci].  Gradients are cleared.
__global__ void adam_kernel(float *w, float *m, float *v, float *g, int CO, int CI, int n_bias_off, float lr, float b1,
                            float b2, float eps, float c1, float c2, bf16 *wf, bf16 *wt)
{
    const int nw = CO * 9 * CI, n = nw + CO;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float wi = w[i] - lr * (mi * c1) / (sqrtf(vi * c2) + eps);
        w[i] = wi;
        g[i] = 0.f;
        if (i < nw) {
            const int ci = i % CI, t = (i / CI) % 9, co = i / (9 * CI);
            wf[i] = __float2bfloat16(wi);
            if (wt) wt[((size_t)ci * 9 + (8 - t)) * CO + co] = __float2bfloat16(wi);
        }
    }
    (void)n_bias_off;
}

unsigned grid_n(long long n, int bs)
{
    long long g = (n + bs - 1) / bs;
    return (unsigned)std::min<long long>(std::max<long long>(g, 1), 148LL * 16);
}

template <int CI, int CO>
cudaError_t conv_launch(const ConvArgs &a, cudaStream_t s)
{
    const size_t sm = sizeof(bf16) * ((size_t)CO * 9 * CI + (size_t)kHH * kHW * CI);
    auto k = conv3x3_kernel<CI, CO>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    const long long ntiles = (long long)a.B * ((a.H + kTH - 1) / kTH) * ((a.W + kTW - 1) / kTW);
    const unsigned grid = (unsigned)std::min<long long>(ntiles, 148LL * 2 * 4);
    k<<<grid, kCT, sm, s>>>(a);
    return cudaGetLastError();
}

template <int CI, int CO>
cudaError_t wgrad_launch(const bf16 *dpre, const bf16 *act, float *dw, int B, int H, int W, cudaStream_t s)
{
    const long long P = (long long)B * H * W, ntile = (P + 127) / 128;
    const int splits = (int)std::min<long long>(ntile, 64);
    wgrad_kernel<CI, CO><<<dim3(9, splits), kCT, 0, s>>>(dpre, act, dw, B, H, W);
    return cudaGetLastError();
}

} // namespace

} // namespace ctlab

using namespace ctlab;

extern "C" {

int ctlab_cnn_conv(const void *d_in, int ci, const void *d_w, const float *d_bias, int co, int B, int H, int W,
                   int epi, void *d_out, const void *d_mask, float *d_out_f32, const float *d_center, void *stream)
{
    if (!d_in || !d_w || B < 1 || H < 1 || W < 1) return set_status(CTLAB_ERR_INVALID_ARG, "bad convolution arguments");
    if ((epi == CTLAB_CNN_EPI_RELU || epi == CTLAB_CNN_EPI_RESIDUAL) && !d_bias)
        return set_status(CTLAB_ERR_INVALID_ARG, "the bias epilogues need a bias");
    if (epi == CTLAB_CNN_EPI_RESIDUAL ? (!d_out_f32 || !d_center) : !d_out)
        return set_status(CTLAB_ERR_INVALID_ARG, "missing convolution output");
    if (epi == CTLAB_CNN_EPI_MASK && !d_mask) return set_status(CTLAB_ERR_INVALID_ARG, "the mask epilogue needs a mask");
    ConvArgs a{(const bf16 *)d_in, (const bf16 *)d_w, d_bias, (bf16 *)d_out, (const bf16 *)d_mask, d_out_f32,
               d_center, B, H, W, epi};
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e;
    if (ci == 16 && co == 64) e = conv_launch<16, 64>(a, s);
    else if (ci == 64 && co == 64) e = conv_launch<64, 64>(a, s);
    else if (ci == 64 && co == 16) e = conv_launch<64, 16>(a, s);
    else return set_status(CTLAB_ERR_UNSUPPORTED, "convolution channels must be (16,64), (64,64) or (64,16)");
    return e == cudaSuccess ? set_status(CTLAB_OK, "") : cuda_status(e, "convolution");
}

int ctlab_cnn_wgrad(const void *d_dpre, int co, const void *d_act, int ci, int B, int H, int W, float *d_dw,
                    float *d_db, void *stream)
{
    if (!d_dpre || !d_act || !d_dw || B < 1 || H < 1 || W < 1)
        return set_status(CTLAB_ERR_INVALID_ARG, "bad weight-gradient arguments");
    cudaStream_t s = (cudaStream_t)stream;
    const bf16 *dp = (const bf16 *)d_dpre, *ac = (const bf16 *)d_act;
    cudaError_t e;
    if (ci == 16 && co == 64) e = wgrad_launch<16, 64>(dp, ac, d_dw, B, H, W, s);
    else if (ci == 64 && co == 64) e = wgrad_launch<64, 64>(dp, ac, d_dw, B, H, W, s);
    else if (ci == 64 && co == 16) e = wgrad_launch<64, 16>(dp, ac, d_dw, B, H, W, s);
    else return set_status(CTLAB_ERR_UNSUPPORTED, "weight-gradient channels must be (16,64), (64,64) or (64,16)");
    if (e == cudaSuccess && d_db) {
        const long long P = (long long)B * H * W;
        if (co == 64) bias_grad_kernel<64><<<grid_n(P, 256) / 4 + 1, 256, 0, s>>>(dp, P, d_db);
        else bias_grad_kernel<16><<<grid_n(P, 256) / 4 + 1, 256, 0, s>>>(dp, P, d_db);
        e = cudaGetLastError();
    }
    return e == cudaSuccess ? set_status(CTLAB_OK, "") : cuda_status(e, "weight gradient");
}

int ctlab_cnn_pack(const float *d_vol, int XN, int YN, int ZN, const int *d_z, int nb, float scale, void *d_in,
                   float *d_center, float *d_target_of_vol, const float *d_vol_target, void *stream)
{
    if (!d_vol || !d_z || !d_in || nb < 1) return set_status(CTLAB_ERR_INVALID_ARG, "bad pack arguments");
    cudaStream_t s = (cudaStream_t)stream;
    const long long n = (long long)nb * XN * YN;
    pack_kernel<<<grid_n(n, 256), 256, 0, s>>>(d_vol, XN, YN, ZN, d_z, nb, scale, (bf16 *)d_in, d_center);
    if (d_target_of_vol && d_vol_target)
        slice_kernel<<<grid_n(n, 256), 256, 0, s>>>(d_vol_target, XN, YN, ZN, d_z, nb, scale, d_target_of_vol);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? set_status(CTLAB_OK, "") : cuda_status(e, "pack");
}

int ctlab_cnn_unpack(const float *d_pred, int XN, int YN, int ZN, const int *d_z, int nb, float scale, float *d_vol,
                     void *stream)
{
    if (!d_pred || !d_z || !d_vol || nb < 1 || !(scale != 0.f)) return set_status(CTLAB_ERR_INVALID_ARG, "bad unpack");
    const long long n = (long long)nb * XN * YN;
    unpack_kernel<<<grid_n(n, 256), 256, 0, (cudaStream_t)stream>>>(d_pred, XN, YN, ZN, d_z, nb, 1.f / scale, d_vol);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? set_status(CTLAB_OK, "") : cuda_status(e, "unpack");
}

int ctlab_cnn_loss_grad(const float *d_pred, const float *d_target, long long n, void *d_g, double *d_acc,
                        void *stream)
{
    if (!d_pred || !d_target || !d_g || n < 1) return set_status(CTLAB_ERR_INVALID_ARG, "bad loss arguments");
    loss_grad_kernel<<<grid_n(n, 256), 256, 0, (cudaStream_t)stream>>>(d_pred, d_target, n, (bf16 *)d_g, d_acc);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? set_status(CTLAB_OK, "") : cuda_status(e, "loss gradient");
}

int ctlab_cnn_adam(float *d_w, float *d_m, float *d_v, float *d_g, int co, int ci, float lr, float b1, float b2,
                   float eps, int step, void *d_wf, void *d_wt, void *stream)
{
    if (!d_w || !d_m || !d_v || !d_g || !d_wf || step < 1) return set_status(CTLAB_ERR_INVALID_ARG, "bad Adam arguments");
    const float c1 = 1.f / (1.f - powf(b1, (float)step)), c2 = 1.f / (1.f - powf(b2, (float)step));
    const long long n = (long long)co * 9 * ci + co;
    adam_kernel<<<grid_n(n, 256), 256, 0, (cudaStream_t)stream>>>(d_w, d_m, d_v, d_g, co, ci, 0, lr, b1, b2, eps, c1,
                                                                    c2, (bf16 *)d_wf, (bf16 *)d_wt);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? set_status(CTLAB_OK, "") : cuda_status(e, "Adam");
}

} // extern "C"
