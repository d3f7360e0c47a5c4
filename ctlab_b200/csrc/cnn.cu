// Learned warm start: kernels of a 2.5D residual CNN (3x3 convolutions,
// NHWC BF16 activations and weights, FP32 accumulation on the tensor cores).
//
// Network (one z slice at a time, H x W = YN x XN): 5 input channels (the
// slice and its two neighbours each side of an OS-SART image, scaled),
// conv 5->64 + ReLU, 6 x (conv 64->64 + ReLU), conv 64->1; the output is the
// centre channel plus the last convolution (a residual correction).
// Channels are padded to 16 (input, last output) or 64.
//
//   conv3x3_kernel  implicit GEMM on the 5th-generation tensor cores
//                   (tcgen05): M = 128 output pixels (an 8 x 16 tile), N =
//                   output channels, K = 9 taps x input channels, one
//                   M128 x N x K16 MMA per (tap, 16 channels) with both
//                   operands in shared memory and the FP32 accumulator in
//                   tensor memory; the CTA keeps the layer's weights in
//                   shared memory and loops over tiles, halo and
//                   accumulator double buffered (a tile's MMAs overlap the
//                   previous tile's epilogue).  Epilogues: bias +
//                   ReLU, mask by an activation's sign (the data gradient =
//                   the same convolution with the weights flipped in space
//                   and transposed in channels), bias + centre channel in
//                   FP32 (output layer).
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
#include "tma.cuh"

namespace ctlab {

namespace {

typedef __nv_bfloat16 bf16;

constexpr int kTH = 8, kTW = 16;               // output tile of a CTA: 8 rows x 16 columns
constexpr int kHH = kTH + 2;                   // input halo rows
constexpr int kCT = 128;                       // 4 warps, two tile rows each (weight gradient)
constexpr int kCTC = 256;                      // convolution CTA: 8 epilogue warps ...
constexpr int kCTP = kCTC + 32;                // ... and the producer warp

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

// ---- 5th-generation tensor cores (tcgen05): one M = 128 x N = CO x K = 16 MMA
// per (tap, 16 input channels), operands in shared memory, FP32 accumulator
// in tensor memory.  Both operands are K-major.  B (the weights, stored by
// the threads) has no swizzle: 16-byte chunks of 8 channels, the rows of a
// chunk plane 16 bytes apart, groups of 8 rows SBO bytes apart, the two
// 8-channel halves of an MMA's K LBO bytes apart.  A (the input halo, stored
// by TMA) is one pixel per row of CI * 2 bytes in the 128-byte (CI = 64) or
// 32-byte (CI = 16) swizzle, addressed by umma_desc_sw.

constexpr int kTPix = kTH * kTW;       // 128 output pixels: the MMA's M
constexpr int kShift = kHH * kTW;      // 160 pixels of one column-shifted input tile (10 rows x 16)

__device__ __forceinline__ uint64_t umma_desc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
    // start >> 4 in [0, 14), LBO >> 4 in [16, 30), SBO >> 4 in [32, 46),
    // descriptor version 1 in [46, 48), no swizzle
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// The same for a K-major operand stored by TMA with a swizzle: rows of
// `row` bytes (one swizzle atom wide), groups of 8 rows SBO = 8 row bytes
// apart, layout type 2 (128-byte swizzle) or 6 (32-byte swizzle) in bits
// [61, 64), LBO unused (1); the atoms 1024-byte aligned (base offset 0).
__device__ __forceinline__ uint64_t umma_desc_sw(uint32_t addr, uint32_t sbo, uint32_t layout)
{
    return (uint64_t)((addr >> 4) & 0x3FFFu) | (1ull << 16) | ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46) |
           ((uint64_t)layout << 61);
}

// Instruction descriptor, kind::f16: FP32 accumulator (bits 4-5 = 1), A and
// B BF16 (bits 7-9, 10-12 = 1), both K-major, N >> 3 at bit 17, M >> 4 at 24.
template <int N>
constexpr uint32_t umma_idesc_bf16_m128()
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(kTPix >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                          uint32_t accumulate)
{
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t"
        "}\n" ::"r"(tmem_d),
        "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate), "r"(0u));
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16])
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
                 "%13, %14, %15}, [%16];"
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                   "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
                   "=r"(v[15])
                 : "r"(taddr));
}

__device__ int g_cnn_err; // a convolution's MMA wait ran out (read by ctlab_cnn_check)

// 3x3 convolution, implicit GEMM on tcgen05: per tile of 8 x 16 output
// pixels, M = 128 pixels, N = CO, K = 9 taps x CI.  The CTA keeps the layer's
// weights in shared memory as [tap][chunk][co] and, per tile, three copies of
// the input halo shifted by one column each, [dx][10 rows x 16 pixels][CI]
// in swizzled pixel rows, each loaded by one TMA tile load (zero fill outside
// the image): the A operand of tap (dy, dx) is then the 128 consecutive
// pixel rows of copy dx from row dy, one swizzled descriptor.  One producer
// thread (lane 0 of warp 8) requests the halos and issues each tile's
// 9 * CI/16 MMAs, committed to an mbarrier; warps 0 .. 7 run the epilogues
// (warp w reads TMEM lanes 32 (w % 4) .. + 31, one output pixel each, and
// half w / 4 of the output channels).  Halo copies and TMEM accumulators are
// double buffered and the two roles meet only at mbarriers, so the MMAs of
// tile t, the copy of tile t+1's halo and the epilogue of tile t-1 overlap.
template <int CI, int CO>
__global__ void __launch_bounds__(kCTP, 1) conv3x3_kernel(ConvArgs a, const __grid_constant__ CUtensorMap tm_in)
{
    static_assert(CI == 16 || CI == 64, "pixel rows of 32 or 128 bytes (one swizzle atom)");
    constexpr int NCH = CI / 8;                 // 16-byte chunks per input pixel
    constexpr int TCOLS = CO < 32 ? 32 : CO;    // TMEM columns of one accumulator (a power of 2 >= 32)
    constexpr uint32_t kRowB = CI * 2;           // bytes of one pixel: a swizzle atom's row
    constexpr uint32_t kCopyBytes = kHH * kTW * kRowB; // one column-shifted copy, [10 rows x 16][CI]
    constexpr uint32_t kHaloBytes = 3 * kCopyBytes;    // the three shifted copies of one tile
    constexpr uint32_t kSwLayout = CI == 64 ? 2u : 6u; // 128- or 32-byte swizzle
    constexpr uint32_t kIdesc = umma_idesc_bf16_m128<CO>();
    constexpr int kEH = CO >= 32 ? 2 : 1;       // epilogue channel halves (warps 4-7 take the second)
    constexpr int kECH = CO / kEH;              // channels per epilogue thread
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char *s_w = smem;                          // [9][NCH][CO] chunks
    unsigned char *s_a = smem + 9 * NCH * CO * 16;      // [2][3][kShift pixels][CI], swizzled
    __shared__ __align__(8) uint64_t s_bar[2];  // MMAs of the tile in accumulator / halo buffer 0, 1 done
    __shared__ __align__(8) uint64_t s_hbar[2]; // halo buffer 0, 1 landed
    __shared__ __align__(8) uint64_t s_tfree[2]; // accumulator 0, 1 read out (one arrival per epilogue warp)
    __shared__ uint32_t s_tmem;
    __shared__ int s_abort; // a wait ran out: both roles stop
    __shared__ float s_bias[CO];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid < CO) s_bias[tid] = a.bias ? a.bias[tid] : 0.f;
    if (tid == 0) s_abort = 0;

    // the layer's weights, 12 loads in flight per thread
    constexpr int kWChunks = CO * 9 * NCH;
    for (int i0 = 0; tid < kCTC && i0 < kWChunks; i0 += 12 * kCTC) {
        uint4 v[12];
#pragma unroll
        for (int u = 0; u < 12; ++u) {
            const int i = i0 + u * kCTC + tid;
            if (i < kWChunks) v[u] = *reinterpret_cast<const uint4 *>(a.w + (size_t)(i / NCH) * CI + (i % NCH) * 8);
        }
#pragma unroll
        for (int u = 0; u < 12; ++u) {
            const int i = i0 + u * kCTC + tid;
            if (i < kWChunks) {
                const int kc = i % NCH, rt = i / NCH; // rt = co*9 + tap
                const int co = rt / 9, t = rt - co * 9;
                *reinterpret_cast<uint4 *>(s_w + ((size_t)(t * NCH + kc) * CO + co) * 16) = v[u];
            }
        }
    }
    __syncwarp(); // the .sync.aligned tcgen05 instructions need converged warps
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&s_tmem)),
                     "r"(2 * TCOLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    if (tid == 0) {
        mbar_init(&s_bar[0], 1);
        mbar_init(&s_bar[1], 1);
        mbar_init(&s_hbar[0], 1);
        mbar_init(&s_hbar[1], 1);
        mbar_init(&s_tfree[0], kCTC / 32);
        mbar_init(&s_tfree[1], kCTC / 32);
        mbar_fence_init();
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); // weights visible to the tensor cores
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = s_tmem;
    const uint32_t w_addr = smem_addr(s_w), a_addr = smem_addr(s_a);

    const int tiles_y = (a.H + kTH - 1) / kTH, tiles_x = (a.W + kTW - 1) / kTW;
    const int ntiles = a.B * tiles_y * tiles_x;
    // the halo of `tile` into buffer hb (producer): three TMA tile loads of
    // the NHWC input, one per column shift dx, each box 10 rows x 16 columns
    // x CI channels (pixel rows of one swizzle atom), zero outside the image
    auto request_halo = [&](int tile, int hb) {
        const int b = tile / (tiles_y * tiles_x), tr = tile % (tiles_y * tiles_x);
        const int y0 = (tr / tiles_x) * kTH, x0 = (tr % tiles_x) * kTW;
        mbar_arrive_expect_tx(&s_hbar[hb], kHaloBytes);
#pragma unroll
        for (int dx = 0; dx < 3; ++dx)
            tma_load_4d(s_a + (size_t)hb * kHaloBytes + (size_t)dx * kCopyBytes, &tm_in, 0, x0 - 1 + dx, y0 - 1, b,
                        &s_hbar[hb]);
    };
    // tile's MMAs (producer): A from halo buffer hb, accumulator hb, committed to s_bar[hb]
    auto issue_mma = [&](int hb) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t a_hb = a_addr + (uint32_t)hb * kHaloBytes;
#pragma unroll
        for (int t = 0; t < 9; ++t) {
            const int dy = t / 3, dx = t - dy * 3;
#pragma unroll
            for (int kk = 0; kk < CI / 16; ++kk) {
                const uint64_t ad = umma_desc_sw(a_hb + (uint32_t)dx * kCopyBytes + (uint32_t)(dy * kTW) * kRowB +
                                                     (uint32_t)kk * 32u,
                                                 8 * kRowB, kSwLayout);
                const uint64_t bd = umma_desc(w_addr + (uint32_t)((t * NCH + 2 * kk) * CO) * 16, CO * 16, 128);
                umma_bf16(tmem + (uint32_t)(hb * TCOLS), ad, bd, kIdesc, (t | kk) != 0);
            }
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         smem_addr(&s_bar[hb]))
                     : "memory");
    };
    // epilogue of `tile` from accumulator ab: accumulator row m = 32 (warp % 4)
    // + lane is output pixel (m / 16, m % 16); this warp's channel half
    auto epilogue = [&](int tile, int ab) {
        const int half = warp >> 2;
        if (half >= kEH) return; // warp-uniform
        const int b = tile / (tiles_y * tiles_x), tr = tile % (tiles_y * tiles_x);
        const int y0 = (tr / tiles_x) * kTH, x0 = (tr % tiles_x) * kTW;
        uint32_t v[kECH];
#pragma unroll
        for (int j = 0; j < kECH / 16; ++j) {
            uint32_t r16[16];
            tmem_ld16(tmem + ((uint32_t)((warp & 3) * 32) << 16) + (uint32_t)(ab * TCOLS + half * kECH + j * 16), r16);
#pragma unroll
            for (int e = 0; e < 16; ++e) v[j * 16 + e] = r16[e];
        }
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        const int m = (warp & 3) * 32 + lane;
        const int y = y0 + m / kTW, x = x0 + m % kTW;
        if (y >= a.H || x >= a.W) return;
        const size_t pix = ((size_t)b * a.H + y) * a.W + x;
        if (a.epi == CTLAB_CNN_EPI_RESIDUAL) {
            if (half == 0) a.out_f32[pix] = __uint_as_float(v[0]) + s_bias[0] + a.center[pix];
            return;
        }
        const int c0 = half * kECH;
        uint4 mk[kECH / 8];
        if (a.epi == CTLAB_CNN_EPI_MASK) {
#pragma unroll
            for (int c8 = 0; c8 < kECH / 8; ++c8)
                mk[c8] = *reinterpret_cast<const uint4 *>(a.mask + pix * CO + c0 + c8 * 8);
        }
#pragma unroll
        for (int c8 = 0; c8 < kECH / 8; ++c8) {
            float f[8];
#pragma unroll
            for (int e = 0; e < 8; ++e) f[e] = __uint_as_float(v[c8 * 8 + e]);
            if (a.epi == CTLAB_CNN_EPI_RELU) {
#pragma unroll
                for (int e = 0; e < 8; ++e) f[e] = fmaxf(f[e] + s_bias[c0 + c8 * 8 + e], 0.f);
            } else if (a.epi == CTLAB_CNN_EPI_MASK) {
                const __nv_bfloat16 *mb = reinterpret_cast<const __nv_bfloat16 *>(&mk[c8]);
#pragma unroll
                for (int e = 0; e < 8; ++e)
                    if (!(__bfloat162float(mb[e]) > 0.f)) f[e] = 0.f;
            }
            uint4 o;
            __nv_bfloat162 *ob = reinterpret_cast<__nv_bfloat162 *>(&o);
#pragma unroll
            for (int e = 0; e < 4; ++e) ob[e] = __floats2bfloat162_rn(f[2 * e], f[2 * e + 1]);
            *reinterpret_cast<uint4 *>(a.out + pix * CO + c0 + c8 * 8) = o;
        }
    };

    // Iteration it (tile `tile`) uses halo buffer and accumulator it & 1.
    // The producer polls two conditions: the MMAs of it - 1 completed (the
    // last reader of the other buffer), upon which it requests the halo of
    // it + 1 there; and the halo of it landed with the accumulator released
    // by the epilogue of it - 2, upon which it issues the MMAs of it.  The
    // epilogue warps wait for the MMAs of each tile and release its
    // accumulator.  A wait that runs out sets s_abort, which stops both
    // roles; the producer then waits (bounded) for its MMAs and halo copies
    // in flight, so that neither lands after the CTA frees its tensor and
    // shared memory.  The launch's output is invalid once g_cnn_err is set.
    // The swizzled halo copies need 1024-byte aligned buffers: a misaligned
    // one stops the CTA before any copy.
    const volatile int *abort_flag = &s_abort;
    bool ok = (a_addr & 1023u) == 0;
    if (warp == kCTC / 32) {
        if (lane == 0 && ok) {
            int it = 0, issued = 0, landed = 0, requested = 1; // MMA batches, halos seen landed, halos requested
            request_halo(blockIdx.x, 0);
            for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++it) {
                const int hb = it & 1;
                bool need_req = tile + (int)gridDim.x < ntiles, need_mma = true;
                for (uint32_t n = 0; (need_req || need_mma) && n < kMbarTestLimit; ++n) {
                    if (need_req && (it == 0 || mbar_test_wait(&s_bar[hb ^ 1], (uint32_t)(((it - 1) >> 1) & 1)))) {
                        request_halo(tile + gridDim.x, hb ^ 1);
                        requested = it + 2;
                        need_req = false;
                    }
                    if (need_mma && mbar_test_wait(&s_hbar[hb], (uint32_t)((it >> 1) & 1)) &&
                        (it < 2 || mbar_test_wait(&s_tfree[hb], (uint32_t)(((it - 2) >> 1) & 1)))) {
                        landed = it + 1;
                        issue_mma(hb);
                        issued = it + 1;
                        need_mma = false;
                    }
                    if ((n & 1023u) == 1023u && *abort_flag) break;
                }
                if (need_req || need_mma) {
                    ok = false;
                    break;
                }
            }
            // drain: the last MMA commit covers every MMA issued; halos
            // landed .. requested - 1 may still be in flight
            if (issued > 0 && !mbar_wait(&s_bar[(issued - 1) & 1], (uint32_t)(((issued - 1) >> 1) & 1))) ok = false;
            for (int k = landed; k < requested; ++k)
                if (!mbar_wait(&s_hbar[k & 1], (uint32_t)((k >> 1) & 1))) ok = false;
        }
    } else {
        int it = 0;
        for (int tile = blockIdx.x; ok && tile < ntiles; tile += gridDim.x, ++it) {
            const int hb = it & 1;
            bool waited = false;
            for (uint32_t n = 0; !waited && n < kMbarSpinLimit; ++n) {
                waited = mbar_try_wait(&s_bar[hb], (uint32_t)((it >> 1) & 1));
                if (!waited && (n & 255u) == 255u && *abort_flag) break;
            }
            if (!__all_sync(0xffffffffu, waited)) {
                ok = false;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            epilogue(tile, hb);
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(&s_tfree[hb]);
        }
    }
    if (!ok && lane == 0) s_abort = 1;
    __syncwarp();
    __syncthreads();
    if (tid == 0 && s_abort) atomicExch(&g_cnn_err, 1);
    __syncwarp();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * TCOLS));
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
    // weights and two buffers of the three shifted halo copies
    const size_t sm = 16 * ((size_t)9 * (CI / 8) * CO + (size_t)2 * 3 * (CI / 8) * kShift);
    auto k = conv3x3_kernel<CI, CO>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 148, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kCTP, sm);
    if (e != cudaSuccess) return e;
    // resident CTAs each hold two accumulators of max(CO, 32) of the SM's 512 TMEM columns
    per_sm = std::max(1, std::min(per_sm, 512 / (2 * std::max(CO, 32))));
    const long long ntiles = (long long)a.B * ((a.H + kTH - 1) / kTH) * ((a.W + kTW - 1) / kTW);
    const unsigned grid = (unsigned)std::min<long long>(ntiles, (long long)sms * per_sm);
    // the NHWC input, boxes of 10 rows x 16 columns x CI channels, each pixel
    // a swizzle atom's row (128-byte swizzle for 64 channels, 32-byte for 16)
    CUtensorMap tm;
    const cuuint64_t dims[4] = {(cuuint64_t)CI, (cuuint64_t)a.W, (cuuint64_t)a.H, (cuuint64_t)a.B};
    const cuuint64_t strides[3] = {(cuuint64_t)CI * 2, (cuuint64_t)a.W * CI * 2, (cuuint64_t)a.H * a.W * CI * 2};
    const cuuint32_t box[4] = {(cuuint32_t)CI, (cuuint32_t)kTW, (cuuint32_t)kHH, 1};
    if (encode_tiled_map(&tm, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<bf16 *>(a.in), dims, strides, box,
                         CI == 64 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_32B,
                         "a convolution input") != CTLAB_OK)
        return cudaErrorInvalidValue;
    k<<<grid, kCTP, sm, s>>>(a, tm);
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

int ctlab_cnn_check(void *stream)
{
    cudaStream_t s = (cudaStream_t)stream;
    int err = 0;
    CTLAB_CUDA_TRY(cudaMemcpyFromSymbolAsync(&err, g_cnn_err, sizeof(int), 0, cudaMemcpyDeviceToHost, s));
    CTLAB_CUDA_TRY(cudaStreamSynchronize(s));
    if (err) {
        const int zero = 0;
        CTLAB_CUDA_TRY(cudaMemcpyToSymbol(g_cnn_err, &zero, sizeof(int)));
        return set_status(CTLAB_ERR_TIMEOUT, "a convolution's tensor-core wait ran out");
    }
    return set_status(CTLAB_OK, "");
}

} // extern "C"
