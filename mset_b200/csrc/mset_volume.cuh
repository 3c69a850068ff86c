// mset_volume.cuh -- volume kernels of the reconstruction update (mset_volume.cu)
#pragma once
#include <cuda_runtime.h>

namespace mset {

struct TvArgs {
    const float *in;  // [n3][n2][n1] input
    float *out;       // output, distinct from in
    float *P, *Y;     // [3][V] dual variables (work)
    float *D;         // [V] work
    int n1, n2, n3;
    double lambda;
    int niter;
    int fista;               // 1: TV_FISTA_method, 0: TV_method
    double *err;             // optional device accumulator: += lambda * TV_error(output)
};

int tv_prox(const TvArgs &a, cudaStream_t st);
int vol_max(const float *v, long n, unsigned *bits, float *mx, cudaStream_t st);
int vol_scale(const float *v, float *out, long n, const float *div, cudaStream_t st);
int vol_mul(const float *v, float *out, long n, const float *mul, cudaStream_t st);
int vol_positivity(float *v, long n, cudaStream_t st);
// [n3][n2][n1] volume <-> [n3][n][n] window (laterally centred)
int vol_pad(const float *src, float *V, int n1, int n2, int n3, int n, cudaStream_t st);
int vol_slab_to_volume(const double *G, float *out, int n1, int n2, int n3, int n, int b, cudaStream_t st);
int vol_accumulate(const float *g, double *acc, long n, bool zero, cudaStream_t st);
int vol_update(float *rec, const double *acc, long n, float step0, cudaStream_t st);

}  // namespace mset
