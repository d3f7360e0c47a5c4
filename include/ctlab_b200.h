/*
 * ctlab_b200.h -- C ABI of libctlab_b200.so, a B200 (sm_100a) implementation
 * of CTLAB's branchless distance-driven (DD3) cone-beam projector,
 * backprojector and the OS-SART / FISTA-TV loops that drive them.
 *
 * Data conventions (identical for every entry point):
 *   volume   float[XN*YN*ZN] in (Z,X,Y) order, z fastest:
 *              vol[(y*XN + x)*ZN + z]
 *   mask     unsigned char[XN*YN], mask[y*XN + x] != 0 keeps the voxel
 *            column; applied to every z.  NULL means "all ones".
 *   proj     float[PN*DNU*DNV] in [view][u][v] order, v fastest.
 *   geometry the source starts at (x0,y0,z0), detector cell centres at
 *            (xds[u], yds[u], zds[v]); view p rotates both by
 *            theta = hangs[p] (radians, regularised to [0,2pi)) about z and
 *            shifts z by hzPos[p].  Voxel (x,y,z) is centred at
 *            (imgXCenter + (x-(XN-1)/2)*dx, imgYCenter + (y-(YN-1)/2)*dx,
 *             imgZCenter + (z-(ZN-1)/2)*dz).  Lengths in one unit (mm).
 *   backprojection and the reconstruction loops need a flat detector with
 *            uniform pitch in u and in v; projection takes any detector.
 *
 * Errors: every int-returning entry point returns CTLAB_OK (0) or one of the
 * CTLAB_ERR_* codes and records a message readable with ctlab_last_error()
 * on the calling thread.  The void entry points kept from the reference
 * record the status the same way (read it with ctlab_last_status()).  The
 * library never exits the process.
 */
#ifndef CTLAB_B200_H_
#define CTLAB_B200_H_

#ifdef __cplusplus
extern "C" {
#endif

#define CTLAB_OK 0
#define CTLAB_ERR_INVALID_ARG 1
#define CTLAB_ERR_UNSUPPORTED 2
#define CTLAB_ERR_CUDA 3
#define CTLAB_ERR_OOM 4
#define CTLAB_ERR_TIMEOUT 5
#define CTLAB_ERR_INTERNAL 6

/* Projection / backprojection models (ForwardDDMethod / BackwardDDMethod,
 * src/utilities.cuh:853-854; prjMode values of src/DD3_GPU_Proj.h:40 and
 * src/DD3_GPU_Back.h:39).  Only the branchless model (0) is implemented;
 * any other value returns CTLAB_ERR_UNSUPPORTED. */
#define CTLAB_PROJ_BRANCHLESS 0
#define CTLAB_BACK_BRANCHLESS 0

/* Summed-area-table arithmetic of a plan.  FP64: 2-D FP64 prefix sums of the
 * volume slices and projections; F32PAIR: the same as compensated FP32 pairs
 * (hi+lo float-float sums); both 8 bytes per entry.  ZPREFIX (the default of
 * the legacy entry points and of the Python Plan): the projector stages
 * per-column z prefix sums accumulated in FP64, slice-major per driving axis,
 * as affine pieces (P, f) of two FP32 values (the prefix at kz is P + kz f),
 * and forms the in-plane integral from adjacent columns -- the same FP32
 * quantities the 2-D FP64 path forms after its column differences; the
 * backprojector likewise reads per-detector-column v prefix sums of the
 * weighted projections, accumulated in FP64 and stored in FP32. */
#define CTLAB_SAT_FP64 0
#define CTLAB_SAT_F32PAIR 1
#define CTLAB_SAT_ZPREFIX 2

/* ---------------------------------------------------------------------- */
/* Entry points with the reference's names and argument order             */
/* ---------------------------------------------------------------------- */

/* Branchless DD forward projection of the host volume hvol into the host
 * projection hprj on GPU gpunum.  Replaces DD3Proj_gpu,
 * src/DD3_GPU_Proj.h:41-44 (same name, arguments and order). */
void DD3Proj_gpu(float x0, float y0, float z0, int DNU, int DNV, float *xds, float *yds,
                 float *zds, float imgXCenter, float imgYCenter, float imgZCenter,
                 float *hangs, float *hzPos, int PN, int XN, int YN, int ZN, float *hvol,
                 float *hprj, float dx, float dz, unsigned char *mask, int gpunum, int prjMode);

/* Branchless DD backprojection of the host projection hprj into the host
 * volume hvol on GPU gpunum; `squared` is ignored, as documented by the
 * reference.  Replaces DD3Back_gpu, src/DD3_GPU_Back.h:40-44. */
void DD3Back_gpu(float x0, float y0, float z0, int DNU, int DNV, float *xds, float *yds,
                 float *zds, float imgXCenter, float imgYCenter, float imgZCenter,
                 float *hangs, float *hzPos, int PN, int XN, int YN, int ZN, float *hvol,
                 float *hprj, float dx, float dz, unsigned char *mask, int gpunum,
                 int squared, int prjMode);

/* One scan split over gpuNum GPUs of this process (GPU i = CUDA device i):
 * GPU i projects the views [startPN[i], startPN[i+1]) of the whole volume,
 * startPN[gpuNum] taken as PN (startPN[0] == 0, non-decreasing), into its
 * block of hprj.  Replaces DD3Proj_multiGPU, src/DD3_GPU_Proj.h:138-141
 * (same name, arguments and order; prjMode 0 only).  With the environment
 * variable CTLAB_MULTIGPU_WRAP=1 a split larger than the visible devices
 * wraps around them (part i on device i mod count, parts of one device in
 * turn); otherwise gpuNum must not exceed the device count. */
void DD3Proj_multiGPU(float x0, float y0, float z0, int DNU, int DNV, float *xds, float *yds,
                      float *zds, float imgXCenter, float imgYCenter, float imgZCenter,
                      float *hangs, float *hzPos, int PN, int XN, int YN, int ZN, float *hvol,
                      float *hprj, float dx, float dz, unsigned char *mask, int prjMode,
                      int *startPN, int gpuNum);

/* GPU i backprojects the z slab [startVOL[i], startVOL[i+1]) of the volume
 * (startVOL[gpuNum] taken as ZN, startVOL[0] == 0, non-decreasing) from the
 * views whose rays can reach the slab (ctlab_slab_views), and writes the
 * slab's slices of every voxel column of hvol.  Replaces DD3Back_multiGPU,
 * src/DD3_GPU_Back.h:138-142 (methodId 0 only); the per-slab view range
 * plays the part of getPrjIdxPair, src/utilities.cuh:503-532. */
void DD3Back_multiGPU(float x0, float y0, float z0, int DNU, int DNV, float *xds, float *yds,
                      float *zds, float imgXCenter, float imgYCenter, float imgZCenter,
                      float *hangs, float *hzPos, int PN, int XN, int YN, int ZN, float *hvol,
                      float *hprj, float dx, float dz, unsigned char *mask, int methodId,
                      int *startVOL, int gpuNum);

/* Status of the last call on this thread (CTLAB_OK or CTLAB_ERR_*), and its
 * message ("" after success).  New in this library: the reference ignores
 * CUDA errors or exits (src/utilities.cuh:63-76). */
int ctlab_last_status(void);
const char *ctlab_last_error(void);

/* ---------------------------------------------------------------------- */
/* Plans: device-resident geometry, workspaces and stream-ordered calls     */
/* ---------------------------------------------------------------------- */

/* Geometry of one scan.  Pointers are HOST arrays read during
 * ctlab_plan_create only: xds, yds [DNU]; zds [DNV]; hangs, hzPos [PN].
 * Mirrors the scalar and array arguments of DD3Proj_gpu. */
typedef struct ctlab_geometry {
    float x0, y0, z0;
    int DNU, DNV;
    const float *xds;
    const float *yds;
    const float *zds;
    float imgXCenter, imgYCenter, imgZCenter;
    const float *hangs;
    const float *hzPos;
    int PN;
    int XN, YN, ZN;
    float dx, dz;
} ctlab_geometry;

typedef struct ctlab_plan ctlab_plan;

/* Validates the geometry, uploads per-view constants and allocates the SAT
 * workspaces on `device`.  sat_mode is CTLAB_SAT_FP64, CTLAB_SAT_F32PAIR or
 * CTLAB_SAT_ZPREFIX.  The plan is used from one stream at a time.
 * New in this library (the reference recomputes everything per call). */
int ctlab_plan_create(const ctlab_geometry *geom, int device, int sat_mode, ctlab_plan **out);
int ctlab_plan_destroy(ctlab_plan *plan);
/* Device bytes held by the plan. */
long long ctlab_plan_workspace_bytes(const ctlab_plan *plan);

/* Forward projection of the device volume d_vol (masked by d_mask, may be
 * NULL) into d_prj[PN][DNU][DNV], stream-ordered on `stream`
 * (a cudaStream_t; NULL = legacy default stream).  Device pointers are owned
 * by the caller.  The device-pointer form of DD3Proj_gpu. */
int ctlab_proj(ctlab_plan *plan, const float *d_vol, const unsigned char *d_mask, float *d_prj,
               void *stream);

/* Forward projection of the views listed in h_views[n] (host indices into
 * the plan's views) into d_prj[n][DNU][DNV]. */
int ctlab_proj_views(ctlab_plan *plan, const int *h_views, int n, const float *d_vol,
                     const unsigned char *d_mask, float *d_prj, void *stream);

/* Backprojection of d_prj[PN][DNU][DNV] into d_vol (overwritten), masked by
 * d_mask.  The device-pointer form of DD3Back_gpu. */
int ctlab_back(ctlab_plan *plan, const float *d_prj, const unsigned char *d_mask, float *d_vol,
               void *stream);

/* Backprojection of d_prj[n][DNU][DNV] holding the views h_views[n]. */
int ctlab_back_views(ctlab_plan *plan, const int *h_views, int n, const float *d_prj,
                     const unsigned char *d_mask, float *d_vol, void *stream);

/* Builds the two volume SATs of the masked volume into the plan's
 * workspace (the first step of ctlab_proj), for tests and timing. */
int ctlab_volume_sat(ctlab_plan *plan, const float *d_vol, const unsigned char *d_mask,
                     void *stream);

/* Views of the scan whose rays can reach the z slab [z0, z1) of the volume,
 * in increasing order, into h_views (capacity cap); returns how many there
 * are (also when more than cap), or minus a CTLAB_ERR_* code.  A ray of
 * view p runs between the source (z0 + hzPos[p]) and a detector cell
 * (zds + hzPos[p]); a view is kept when that z range, widened by one row
 * pitch, meets the slab widened by one voxel.  The views left out add
 * exactly zero to the slab's backprojection.  Host only.  The counterpart
 * of getPrjIdxPair, src/utilities.cuh:503-532 (which assumes hzPos sorted;
 * this test takes any order). */
int ctlab_slab_views(const ctlab_geometry *geom, int z0, int z1, int *h_views, int cap);

/* The two multi-GPU splits with a plan-style geometry and status return
 * (DD3Proj_multiGPU / DD3Back_multiGPU call these). */
int ctlab_proj_multi(const ctlab_geometry *geom, const float *hvol, float *hprj,
                     const unsigned char *mask, const int *startPN, int gpuNum);
int ctlab_back_multi(const ctlab_geometry *geom, const float *hprj, float *hvol,
                     const unsigned char *mask, const int *startVOL, int gpuNum);

/* Allocation-free form of ctlab_volume_sat, for callers that cannot
 * allocate device memory mid-reconstruction: systems that reserve their
 * whole device-memory budget up front, or that must not let cudaMalloc /
 * cudaFree synchronise the device behind their other streams.  Builds the
 * FP64 volume SAT of one orientation (0: y slices -> [YN][XN+1][zp],
 * 1: x slices -> [XN][YN+1][zp], zp >= ZN+1) of the masked volume into the
 * caller's d_sat, with the scan's lookback scratch in a fixed 32 MiB device
 * array inside the library (held by every GPU that loads the library until
 * exit).  No cudaMalloc, cudaFree or allocating library call is made.
 * Volumes whose scan needs more than 32 MiB of scratch are rejected with
 * CTLAB_ERR_INVALID_ARG (512x512x256 needs about 23 MB).  The first call on
 * a device looks up the array's device address; make that call before any
 * stream capture.  All calls share the array, so calls that overlap on the
 * GPU (other streams, other threads) race; serialise them.  Asynchronous on
 * `stream`: a lookback wait that runs out inside the scan cannot be
 * returned here; it raises the array's error word, which
 * ctlab_noalloc_check reports.  No counterpart in the reference. */
int ctlab_volume_sat_noalloc(const float *d_vol, const unsigned char *d_mask, int XN, int YN, int ZN,
                             int orientation, double *d_sat, int zp, void *stream);

/* Waits for `stream` and reports whether any allocation-free call on the
 * current device since the previous check hit a bounded-wait timeout:
 * CTLAB_ERR_TIMEOUT (the output of that call is invalid) or CTLAB_OK.  The
 * error word is sticky until this call reads it and clears it.  Allocates
 * nothing.  No counterpart in the reference. */
int ctlab_noalloc_check(void *stream);

/* Diagnostics: runs a two-chunk lookback scan on the allocation-free array
 * whose first chunk never publishes, so that the second chunk's bounded
 * wait (spin_limit polls, 1..2^24) runs out and raises the error word that
 * ctlab_noalloc_check reports.  No counterpart in the reference. */
int ctlab_debug_noalloc_stall(unsigned spin_limit, void *stream);

/* Copies the plan's volume SAT of one orientation to d_out (FP64 plans:
 * doubles, [planes][rows][zp] as reported by ctlab_plan_sat_layout;
 * F32PAIR plans: float pairs (hi, lo) with the same indexing; ZPREFIX plans:
 * floats [planes][rows][zp] = slice-major column z-prefixes, [YN][ZN+1][rs]
 * (x fastest) for orientation 0 and [XN][ZN+1][rs] (y fastest) for 1, rs the
 * row stride reported as zp, pad columns zero). */
int ctlab_plan_sat_layout(const ctlab_plan *plan, int orientation, int *planes, int *rows,
                          int *zp);
int ctlab_copy_volume_sat(ctlab_plan *plan, int orientation, void *d_out, void *stream);

/* Elapsed device milliseconds of the last ctlab_proj / ctlab_back call
 * split into SAT build and gather kernels (measured with CUDA events on the
 * launching stream when timing is enabled with ctlab_plan_set_timing). */
int ctlab_plan_set_timing(ctlab_plan *plan, int enable);
int ctlab_plan_last_times(ctlab_plan *plan, float *sat_ms, float *gather_ms);

/* Number of the library's kernels launched by the last ctlab_proj /
 * ctlab_back / reconstruction call on this plan. */
int ctlab_plan_last_launches(const ctlab_plan *plan);

/* ---------------------------------------------------------------------- */
/* Reconstruction                                                          */
/* ---------------------------------------------------------------------- */

/* OS-SART on the device.  d_x holds the initial image and receives the
 * result; d_meas is the measured projection [PN][DNU][DNV].  Views are split
 * into os_num interleaved subsets {s, s+os_num, ...} unless h_order[PN] (a
 * permutation of 0..PN-1, may be NULL) gives the subset-major view order,
 * subset s taking positions [s*ceil(PN/os_num), ...).  Each subset step:
 *   r = (b_s - A_s x)/rowSum_s   (0 where rowSum_s <= 1e-7)
 *   x = (x + lambda * (B_s r)/colSum_s) * mask  (0 where colSum_s <= 1e-7)
 * optionally clamped to [min_v, max_v] when clamp != 0.  If h_resid is not
 * NULL it receives iter_num values ||b - A x_k|| / ||b|| after each
 * iteration.  The plan keeps the call's workspace and SART weights; a later
 * call with the same subsets, order and mask bytes reuses them without
 * allocating (the mask is read back to the host to compare it).  Replaces the
 * GPU body of OS_SART, src/DD3_GPU_recon.h:60-65. */
int ctlab_os_sart(ctlab_plan *plan, float *d_x, const float *d_meas, const unsigned char *d_mask,
                  int os_num, int iter_num, float lambda, const int *h_order, int clamp,
                  float min_v, float max_v, float *h_resid, void *stream);

/* FISTA-TV on the device: SART-preconditioned gradient step over all views,
 * one TV-gradient step of weight tv_lambda (smoothing tv_eps), FISTA
 * momentum clamped to [min_v, max_v] (FISTA_functor,
 * src/FastIterativeShrinkageAlgorithm.h:17-42).  h_resid as for
 * ctlab_os_sart.  The plan keeps the call's workspace and SART weights
 * (rowSum = A 1, colSum = B 1 over all views); a later call with the same
 * mask bytes reuses them without allocating. */
int ctlab_fista_tv(ctlab_plan *plan, float *d_x, const float *d_meas,
                   const unsigned char *d_mask, int iter_num, float tv_lambda, float tv_eps,
                   float min_v, float max_v, float *h_resid, void *stream);

/* Nonlinear conjugate gradient for min 1/2 ||A x - b||^2 over the masked
 * volume, all views, exact line search along each direction; the beta
 * update is CTLAB_CG_FR (Fletcher-Reeves), _PRP (Polak-Ribiere-Polyak), _CW
 * (Crowder-Wolfe, the Hestenes-Stiefel form), _DI (Dixon) or _DY
 * (Dai-Yuan), the members of CGMethod, src/DD3_GPU_recon.h:14-19.  d_x holds
 * the initial image and receives the result; h_resid (may be NULL) receives
 * ||A x_k - b|| / ||b|| after each iteration.  The plan keeps the call's
 * workspace for later calls.  Replaces the GPU body of CG,
 * src/DD3_GPU_recon.h:98-103. */
#define CTLAB_CG_FR 0
#define CTLAB_CG_PRP 1
#define CTLAB_CG_CW 2
#define CTLAB_CG_DI 3
#define CTLAB_CG_DY 4
int ctlab_cg(ctlab_plan *plan, float *d_x, const float *d_meas, const unsigned char *d_mask, int iter_num,
             int method, float *h_resid, void *stream);

/* Smoothed isotropic TV gradient of d_f into d_g (both (Z,X,Y)).  The 3-D
 * form of GradientOfTV_GPU, src/differentialFuncs.hpp:491-501. */
int ctlab_tv_gradient(const float *d_f, float *d_g, int XN, int YN, int ZN, float eps,
                      void *stream);

/* FISTA momentum step on device arrays: cur = clamp(cur + (t1-1)/t2 (cur -
 * las), minV, maxV).  FISTA, src/FastIterativeShrinkageAlgorithm.h:44-48. */
int ctlab_fista_step(const float *d_las, float *d_cur, float t1, float t2, long long n,
                     float min_v, float max_v, void *stream);

/* SART weightings on device arrays, epsilon 1e-7:
 *   prj = rowSum > eps ? (real - prj)/rowSum : 0
 *   vol = colSum > eps ? vol/colSum : 0;  recon += vol
 * SART_Weighting::Proj_ptr / Back_ptr, src/SARTWeighting.h:38-91. */
int ctlab_sart_proj_weight(float *d_prj, const float *d_real, const float *d_row_sum, long long n,
                           void *stream);
int ctlab_sart_back_weight(float *d_vol, float *d_recon, const float *d_col_sum, long long n,
                           void *stream);

/* ---------------------------------------------------------------------- */
/* Batched projection of many scans and the projector autotuner (no       */
/* counterpart in the reference)                                          */
/* ---------------------------------------------------------------------- */

/* Times the z-prefix projector of `plan` under each candidate staging (views
 * per CTA 2..16, stage depth 2..4) on d_vol (d_prj receives projections),
 * keeps the fastest, and appends it to the JSON-lines cache file cache_path
 * (may be NULL) keyed by the scan geometry; a cached scan is not re-timed
 * (*best_ms = -1).  Synchronous. */
int ctlab_plan_autotune(ctlab_plan *plan, const float *d_vol, float *d_prj, const char *cache_path,
                        float *best_ms);

/* The projector staging of a z-prefix plan: tiles[0..7] = views per CTA,
 * detector rows per consumer warp, consumer warps per view, z splits, staged
 * columns per box, staged z-prefix rows per box, stage depth, and the CTAs of
 * a projection of all views. */
int ctlab_plan_proj_tiles(const ctlab_plan *plan, int *tiles);

/* A batch projects the scans of n z-prefix plans (one device) together.  The
 * plans must outlive the batch; tune them (ctlab_plan_autotune) before
 * creating it: a batch whose plans were re-staged afterwards refuses to run
 * (CTLAB_ERR_INVALID_ARG). */
typedef struct ctlab_batch ctlab_batch;
int ctlab_batch_create(ctlab_plan *const *plans, int n, ctlab_batch **out);
int ctlab_batch_destroy(ctlab_batch *batch);
/* Sum over the cases of XN*YN*ZN*PN. */
long long ctlab_batch_voxel_views(const ctlab_batch *batch);
/* Projects d_vols[i] (masks d_masks[i], d_masks may be NULL) into d_prjs[i]
 * for every case: each case's z-prefixes, then one persistent projector
 * launch over the work items of all cases (sorted longest first).  With
 * use_graph the sequence is captured into a CUDA graph on the first call
 * (stream must not be the legacy default stream) and replayed while the
 * volume, mask and projection pointers stay the same. */
int ctlab_batch_proj(ctlab_batch *batch, const float *const *d_vols, const unsigned char *const *d_masks,
                     float *const *d_prjs, int use_graph, void *stream);

/* ---------------------------------------------------------------------- */
/* Learned warm start: 2.5D residual CNN kernels (no counterpart in the   */
/* reference; the network that warm-starts OS-SART)                       */
/* ---------------------------------------------------------------------- */

/* Convolution epilogues. */
#define CTLAB_CNN_EPI_RELU 0     /* out = bf16(relu(conv + bias)) */
#define CTLAB_CNN_EPI_MASK 1     /* out = bf16(conv) where mask > 0, else 0 (backward through ReLU) */
#define CTLAB_CNN_EPI_RESIDUAL 2 /* out_f32 = conv[channel 0] + bias[0] + center (output layer) */

/* 3x3 convolution, stride 1, zero padding, on NHWC BF16 tensors
 * d_in [B][H][W][ci] with weights d_w [co][9][ci] (tap = 3*dy + dx), FP32
 * accumulation on the 5th-generation tensor cores (tcgen05, TMEM
 * accumulator).  (ci, co) is (16, 64), (64, 64) or
 * (64, 16).  The data gradient of a layer is this convolution with the
 * flipped, channel-transposed weights (ctlab_cnn_adam writes them) and the
 * MASK epilogue. */
int ctlab_cnn_conv(const void *d_in, int ci, const void *d_w, const float *d_bias, int co, int B, int H, int W,
                   int epi, void *d_out, const void *d_mask, float *d_out_f32, const float *d_center,
                   void *stream);

/* Synchronises the stream and reports whether a convolution since the last
 * check gave up waiting for its tensor-core MMAs (CTLAB_ERR_TIMEOUT; its
 * outputs are then invalid).  Clears the flag. */
int ctlab_cnn_check(void *stream);

/* Weight (and, with d_db, bias) gradients of a convolution, accumulated:
 * d_dw [co][9][ci] += sum_p dpre[p][co] * act[p + tap][ci]. */
int ctlab_cnn_wgrad(const void *d_dpre, int co, const void *d_act, int ci, int B, int H, int W, float *d_dw,
                    float *d_db, void *stream);

/* Network inputs for the z slices d_z[nb] of a (Z,X,Y) volume: NHWC BF16
 * [nb][YN][XN][16] holding slices z-2..z+2 (clamped) times scale, the FP32
 * centre slices (may be NULL), and optionally the same slices of a target
 * volume (scaled, FP32). */
int ctlab_cnn_pack(const float *d_vol, int XN, int YN, int ZN, const int *d_z, int nb, float scale, void *d_in,
                   float *d_center, float *d_target_of_vol, const float *d_vol_target, void *stream);

/* Writes predicted slices (scaled) back into the volume: vol[y][x][z_b] = pred / scale. */
int ctlab_cnn_unpack(const float *d_pred, int XN, int YN, int ZN, const int *d_z, int nb, float scale,
                     float *d_vol, void *stream);

/* MSE gradient 2 (pred - target) / n into channel 0 of a BF16 [n][16]
 * tensor; d_acc (may be NULL) += sum of squared differences. */
int ctlab_cnn_loss_grad(const float *d_pred, const float *d_target, long long n, void *d_g, double *d_acc,
                        void *stream);

/* Adam step (bias-corrected, step >= 1) on FP32 master parameters laid out
 * as [co][9][ci] weights followed by co biases (d_w, moments d_m / d_v,
 * gradient d_g, cleared afterwards); writes the BF16 weights d_wf
 * [co][9][ci] and, if d_wt is not NULL, the flipped transposed copy
 * d_wt [ci][9][co] (wt[ci][8 - tap][co] = w[co][tap][ci]). */
int ctlab_cnn_adam(float *d_w, float *d_m, float *d_v, float *d_g, int co, int ci, float lr, float b1, float b2,
                   float eps, int step, void *d_wf, void *d_wt, void *stream);

/* ---------------------------------------------------------------------- */
/* Phantoms (test and benchmark inputs)                                    */
/* ---------------------------------------------------------------------- */

/* Point-sampled sum of rotated ellipsoids at voxel centres into d_vol.
 * h_ell holds n_ell records of 10 floats: value, cx, cy, cz, ax, ay, az
 * (semi-axes), phi, theta, psi (R = Rz(phi) Rx(theta) Rz(psi)). */
int ctlab_ellipsoid_phantom(float *d_vol, int XN, int YN, int ZN, float dx, float dz,
                            float imgXCenter, float imgYCenter, float imgZCenter,
                            const double *h_ell, int n_ell, int clamp_nonneg, void *stream);

/* Random-ellipsoid parameters drawn with std::mt19937_64(seed): count
 * uniform in [n_min, n_max], centres uniform in 0.8 x the half extents,
 * semi-axes U(0.05,0.4) x half extent per axis, Euler angles U(0,pi),
 * values U(0, v_max).  Writes up to cap records into h_ell, returns the
 * count (or a negative CTLAB_ERR_* value). */
int ctlab_random_ellipsoids(unsigned long long seed, int n_min, int n_max, float half_x,
                            float half_y, float half_z, float v_max, double *h_ell, int cap);

/* ---------------------------------------------------------------------- */
/* Diagnostics                                                             */
/* ---------------------------------------------------------------------- */

/* Runs a two-chunk SAT scan on `device` whose first chunk never publishes
 * its result, so the second chunk's bounded wait (spin_limit polls of about
 * 64 ns) runs out.  Returns CTLAB_ERR_TIMEOUT when the timeout was detected
 * and reported through the device error word as designed (the launch
 * terminates and the context stays usable), CTLAB_ERR_INTERNAL otherwise.
 * No counterpart in the reference, which has no device-side waits. */
int ctlab_debug_scan_stall(int device, unsigned spin_limit);

#ifdef __cplusplus
}
#endif

#endif /* CTLAB_B200_H_ */
