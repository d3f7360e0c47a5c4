/* C++ entry points of libctlab_b200 with the reference's C++ signatures
 * (thrust::host_vector arguments, C++ linkage): include this header instead
 * of the reference's DD3_GPU_recon.h.  The enumerations keep the reference's
 * names and values (src/utilities.cuh:853-854, src/DD3_GPU_recon.h:14-19) so
 * the mangled names of the functions are the ones an application already
 * calls.  Errors are recorded like the C entry points: read them with
 * ctlab_last_status() / ctlab_last_error() (ctlab_b200.h). */
#pragma once

#include <string>

#include <thrust/host_vector.h>

#include "ctlab_b200.h"

typedef unsigned char byte;

/* Projection / backprojection models; only the branchless ones are built. */
enum ForwardDDMethod { PROJ_BRANCHLESS = 0, PROJ_PSEUDODISTANCE = 2 };
enum BackwardDDMethod { BACK_BRANCHLESS = 0, BACK_PSEUDODISTANCE = 2, BACK_ZLINEBRANCHLESS = 3 };

/* Beta update of the conjugate gradient method (ctlab_cg's CTLAB_CG_*). */
enum CGMethod { CG_FR, CG_PRP, CG_CW, CG_DI, CG_DY };

/* Projects (forwardProjection) or backprojects an all-ones input over the
 * built-in 128x128x64 / 360-view / 256x64 scan (0.5 mm voxels, SOD 541 mm,
 * SDD 949 mm, 1 mm cells) on the current device and prints the output's
 * minimum, maximum, sum and device time: the row / column sums A 1 and B 1
 * of the SART weighting.  Replaces evalProjBack, src/DD3_GPU_recon.h:25-28
 * (whose scan is not published). */
void evalProjBack(bool forwardProjection, ForwardDDMethod forwardMethod, BackwardDDMethod backwardMethod);

/* OS-SART on the current device.  The scan is the reference's flat
 * equal-distance detector: source (0, sid, 0), detector plane y = sid - sdd,
 * cells ((u - (DNU-1)/2 - col_offset) col_size, (v - (DNV-1)/2 - row_offset)
 * row_size); views hangs[PN], z shifts hzPos[PN].  initImg / reconImg are
 * (Z,X,Y) [YN][XN][ZN] volumes, hprj [PN][DNU][DNV], mask [YN][XN] (empty:
 * all ones).  osNum interleaved subsets, iterNum iterations, relaxation 1.
 * A non-empty VolumeName receives the result as raw float32 in the same
 * order; with outputMedRes each iteration's image is also written to
 * VolumeName + "_iter<k>" (k from 1).  Replaces OS_SART,
 * src/DD3_GPU_recon.h:60-65. */
void OS_SART(thrust::host_vector<float> &reconImg, thrust::host_vector<float> &initImg,
             thrust::host_vector<float> &hprj, thrust::host_vector<float> &hangs,
             thrust::host_vector<float> &hzPos, thrust::host_vector<byte> &mask, const std::string &VolumeName,
             const int osNum, const int iterNum, const bool outputMedRes, const float sid, const float sdd,
             const int DNU, const int DNV, const int PN, const float imgXCenter, const float imgYCenter,
             const float imgZCenter, const int XN, const int YN, const int ZN, const float dx, const float dz,
             const float col_size, const float row_size, const float col_offset, const float row_offset,
             const ForwardDDMethod forwardMethod, const BackwardDDMethod backwardMethod);

/* Conjugate gradient (ctlab_cg) over the same scan description as OS_SART;
 * all views per iteration (osNum is accepted for signature compatibility
 * and not used).  Replaces CG, src/DD3_GPU_recon.h:98-103. */
void CG(thrust::host_vector<float> &reconImg, thrust::host_vector<float> &initImg, thrust::host_vector<float> &hprj,
        thrust::host_vector<float> &hangs, thrust::host_vector<float> &hzPos, thrust::host_vector<byte> &mask,
        const std::string &VolumeName, const int osNum, const int iterNum, const bool outputMedRes, const float sid,
        const float sdd, const int DNU, const int DNV, const int PN, const float imgXCenter, const float imgYCenter,
        const float imgZCenter, const int XN, const int YN, const int ZN, const float dx, const float dz,
        const float col_size, const float row_size, const float col_offset, const float row_offset,
        const ForwardDDMethod forwardMethod, const BackwardDDMethod backwardMethod, const CGMethod cgm);
