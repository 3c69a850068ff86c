// mset_rotate.cuh -- Fourier-shear rotation of volumes (mset_rotate.cu)
#pragma once
#include <cuda_runtime.h>
#include <vector>

namespace mset {

struct RotPlan {
    bool active;   // false when all angles are within 0.5 degrees (no rotation)
    int num_step;  // sub-rotations of <= 11 degrees
    int dim[4];    // shear axis (1, 2, 3 = MATLAB dims) of the four shears of a sub-step
    double a[4], b[4];
};

// plan of Func_rot_3Dvol_FourierShear (inverse = false) or
// Func_inv_rot_3Dvol_FourierShear (inverse = true); returns plan->active
bool rot_plan(const double *v1, const double *v2, const double *v3, double phi, double theta, double psi, bool inverse,
              RotPlan *plan);
bool rot_supported(int n);
int rot_twiddles(int n, std::vector<float2> &h);
// out = rotation of vol (device, [n][n][n]); S: n^3 complex work buffer
int rot_apply(const RotPlan &pl, int n, const float *vol, float *out, float2 *S, const float2 *twn, int sms,
              cudaStream_t st);
// any shape [n3][n2][n1] (every side a supported line length): each shear as
// batched 1D transforms; S: n1 n2 n3 complex work buffer
bool rot_line_supported(int n);
int rot_apply3(const RotPlan &pl, int n1, int n2, int n3, const float *vol, float *out, float2 *S, int sms,
               cudaStream_t st);

}  // namespace mset
