// TEST INFRASTRUCTURE ONLY.  Compiles the reference's own header-inline
// helpers, where they lie in the reference tree (utilities.cuh,
// SARTWeighting.h, FastIterativeShrinkageAlgorithm.h), into oracle/_ref/ so
// the CPU restatement in dd3_oracle.c can be checked against them.  Only the
// golden-vector generator under tests/golden/ and CPU tests load the result.
#include "utilities.cuh"
#include "SARTWeighting.h"
#include "FastIterativeShrinkageAlgorithm.h"

extern "C" {

// DD3Boundaries, src/utilities.cuh:413-433
void ref_dd3_boundaries_f(int nb, const float *c, float *b)
{
    DD3Boundaries<float>(nb, const_cast<float *>(c), b);
}
void ref_dd3_boundaries_d(int nb, const double *c, double *b)
{
    DD3Boundaries<double>(nb, const_cast<double *>(c), b);
}

// regularizeAngle, src/utilities.cuh:279-286
float ref_regularize_angle_f(float a) { return regularizeAngle<float>(a); }
double ref_regularize_angle_d(double a) { return regularizeAngle<double>(a); }

// invRotVox, src/utilities.cuh:289-298
void ref_inv_rot_vox(const float *in3, float *out3, float c, float s, float zP)
{
    float3 a = make_float3(in3[0], in3[1], in3[2]);
    float3 o;
    invRotVox(a, o, make_float2(c, s), zP);
    out3[0] = o.x; out3[1] = o.y; out3[2] = o.z;
}

// SART_Weighting<float>::Proj_ptr / Back_ptr, src/SARTWeighting.h:38-91
void ref_sart_proj_ptr(float *prj, const float *real, const float *row_sum, int n)
{
    SART_Weighting<float>::Proj_ptr(prj, real, row_sum, n);
}
void ref_sart_back_ptr(float *vol, float *recon, const float *col_sum, int n)
{
    SART_Weighting<float>::Back_ptr(vol, recon, col_sum, n);
}

// FISTA, src/FastIterativeShrinkageAlgorithm.h:44-48
void ref_fista(float *las, float *cur, float t1, float t2, int n, float minV, float maxV)
{
    FISTA<float>(las, cur, t1, t2, n, minV, maxV);
}

}
