// TEST INFRASTRUCTURE ONLY.  Compiles the reference's utilities.hpp, where it
// lies in the reference tree, to expose its host-callable SART / update
// helpers for golden-vector generation (see ref_helpers_cuh.cu).
#include "utilities.hpp"

extern "C" {

// _Update, src/utilities.hpp:1062-1094
void ref_update(float *img, const float *cor, const float *weg, const float *msk, int n,
                float lambda, int keep, float minV, float maxV)
{
    _Update<float> f(lambda, keep != 0, minV, maxV);
    for (int i = 0; i < n; ++i) img[i] = f(thrust::make_tuple(img[i], cor[i], weg[i], msk[i]));
}

// prjWeight / bakWeight (OpenMP, epsilon _EPSILON), src/utilities.hpp:4304-4405
void ref_prj_weight(float *prj, float *real, float *row_sum, int n)
{
    prjWeight<float>(prj, real, row_sum, n);
}
void ref_bak_weight(float *vol, float *recon, float *col_sum, int n)
{
    bakWeight<float>(vol, recon, col_sum, n);
}

}
