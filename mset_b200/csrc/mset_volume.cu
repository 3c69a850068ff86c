// mset_volume.cu -- volume kernels of the reconstruction update:
// TV / TV-FISTA proximal operator (func_lib/TV_method.m:5-28 and helpers
// :32-83, func_lib/TV_FISTA_method.m:5-38), positivity
// (Run_MSET_recon.m:183-185), max-normalisation (Run_MSET_recon.m:268-270),
// and the glue between beam-frame slab gradients and the lab-frame volume.
//
// All stencils are periodic (MATLAB circshift).  Volumes are C order
// [n3][n2][n1] = MATLAB (n1, n2, n3); MATLAB dim 1 is the fastest axis.
// HBM/L2-bound elementwise work: grid-stride loops over 148 x 8 CTAs (the
// TV stencils: over rows, one CTA per row).
#include <algorithm>
#include <cmath>

#include "mset_volume.cuh"

namespace mset {

namespace {
constexpr int kThreads = 256;

inline int grid_for(long total) {
    long g = (total + kThreads - 1) / kThreads;
    return (int)std::min<long>(std::max<long>(g, 1), 148L * 8);
}

__device__ __forceinline__ long wrap(long i, long n) { return i < 0 ? i + n : (i >= n ? i - n : i); }

// The TV stencils run one CTA per row (i2, i3) of the volume in a
// grid-stride loop over rows, threads over i1: the periodic neighbours' rows
// are found once per row (one 32-bit division) instead of three 64-bit
// divisions per element, which made these kernels integer-bound.
struct Rows {
    int n1, n2, n3;
    long V;
    // first element of row (i2, i3); neighbour rows with periodic wrap
    __device__ __forceinline__ long at(int i2, int i3) const { return ((long)i3 * n2 + i2) * n1; }
};

// D = TV_div(Y) - in / lambda   (the argument of TV_del in TV_method.m:21)
__global__ void k_tv_d(const float *Y, const float *in, float *D, Rows g, float inv_lam) {
    const long V = g.V;
    for (int row = blockIdx.x; row < g.n2 * g.n3; row += gridDim.x) {
        const int i2 = row % g.n2, i3 = row / g.n2;
        const long b = g.at(i2, i3), b2 = g.at(i2 == 0 ? g.n2 - 1 : i2 - 1, i3),
                   b3 = g.at(i2, i3 == 0 ? g.n3 - 1 : i3 - 1);
        for (int i1 = threadIdx.x; i1 < g.n1; i1 += blockDim.x) {
            const long r = b + i1;
            const int i1m = i1 == 0 ? g.n1 - 1 : i1 - 1;
            const float d = Y[r] + Y[V + r] + Y[2 * V + r] - Y[b + i1m] - Y[V + b2 + i1] - Y[2 * V + b3 + i1];
            D[r] = d - in[r] * inv_lam;
        }
    }
}

// P <- TV_project(src + tau TV_del(D)); FISTA: Y <- P + m (P - P_old) in FP64
__global__ void k_tv_step(float *P, float *Y, const float *D, Rows g, float tau, double m, int fista) {
    const long V = g.V;
    for (int row = blockIdx.x; row < g.n2 * g.n3; row += gridDim.x) {
        const int i2 = row % g.n2, i3 = row / g.n2;
        const long b = g.at(i2, i3), b2 = g.at(i2 == g.n2 - 1 ? 0 : i2 + 1, i3),
                   b3 = g.at(i2, i3 == g.n3 - 1 ? 0 : i3 + 1);
        for (int i1 = threadIdx.x; i1 < g.n1; i1 += blockDim.x) {
            const long r = b + i1;
            const int i1p = i1 == g.n1 - 1 ? 0 : i1 + 1;
            const float d0 = D[r];
            const float t1 = tau * (D[b + i1p] - d0);
            const float t2 = tau * (D[b2 + i1] - d0);
            const float t3 = tau * (D[b3 + i1] - d0);
            const float *src = fista ? Y : P;
            const float q1 = src[r] + t1, q2 = src[V + r] + t2, q3 = src[2 * V + r] + t3;
            const float nrm = sqrtf(fmaxf(1.0f, q1 * q1 + q2 * q2 + q3 * q3));
            const float p1 = q1 / nrm, p2 = q2 / nrm, p3 = q3 / nrm;
            if (fista) {
                const double o1 = P[r], o2 = P[V + r], o3 = P[2 * V + r];
                Y[r] = (float)(p1 + m * (p1 - o1));
                Y[V + r] = (float)(p2 + m * (p2 - o2));
                Y[2 * V + r] = (float)(p3 + m * (p3 - o3));
            }
            P[r] = p1;
            P[V + r] = p2;
            P[2 * V + r] = p3;
        }
    }
}

// out = in - lambda TV_div(P)   (TV_method.m:26)
__global__ void k_tv_out(const float *P, const float *in, float *out, Rows g, float lam) {
    const long V = g.V;
    for (int row = blockIdx.x; row < g.n2 * g.n3; row += gridDim.x) {
        const int i2 = row % g.n2, i3 = row / g.n2;
        const long b = g.at(i2, i3), b2 = g.at(i2 == 0 ? g.n2 - 1 : i2 - 1, i3),
                   b3 = g.at(i2, i3 == 0 ? g.n3 - 1 : i3 - 1);
        for (int i1 = threadIdx.x; i1 < g.n1; i1 += blockDim.x) {
            const long r = b + i1;
            const int i1m = i1 == 0 ? g.n1 - 1 : i1 - 1;
            const float dv = P[r] + P[V + r] + P[2 * V + r] - P[b + i1m] - P[V + b2 + i1] - P[2 * V + b3 + i1];
            out[r] = in[r] - lam * dv;
        }
    }
}

// err += lambda sum |TV_del(u)|   (TV_method.m:27, 71-83), FP64 accumulation
__global__ void k_tv_err(const float *u, Rows g, double lam, double *err) {
    double acc = 0.0;
    for (int row = blockIdx.x; row < g.n2 * g.n3; row += gridDim.x) {
        const int i2 = row % g.n2, i3 = row / g.n2;
        const long b = g.at(i2, i3), b2 = g.at(i2 == g.n2 - 1 ? 0 : i2 + 1, i3),
                   b3 = g.at(i2, i3 == g.n3 - 1 ? 0 : i3 + 1);
        for (int i1 = threadIdx.x; i1 < g.n1; i1 += blockDim.x) {
            const long r = b + i1;
            const int i1p = i1 == g.n1 - 1 ? 0 : i1 + 1;
            const float u0 = u[r];
            const float d1 = u[b + i1p] - u0;
            const float d2 = u[b2 + i1] - u0;
            const float d3 = u[b3 + i1] - u0;
            acc += sqrt((double)d1 * d1 + (double)d2 * d2 + (double)d3 * d3);
        }
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(err, lam * acc);
}

// The same three stencils with four consecutive voxels per thread (n1 a
// multiple of 4): 16-byte loads and stores of every array, the one periodic
// neighbour along i1 outside the thread's four voxels read as a 4-byte load
// (an L1 hit: the neighbouring thread loads its line).  Fewer, wider requests
// keep more bytes in flight per SM; same arithmetic per voxel.
__device__ __forceinline__ float4 ld4(const float *p) { return *reinterpret_cast<const float4 *>(p); }
__device__ __forceinline__ void st4(float *p, float4 v) { *reinterpret_cast<float4 *>(p) = v; }

__global__ void k_tv_d4(const float *Y, const float *in, float *D, Rows g, float inv_lam) {
    const long V = g.V;
    const int q1 = g.n1 / 4;
    for (int row = blockIdx.x; row < g.n2 * g.n3; row += gridDim.x) {
        const int i2 = row % g.n2, i3 = row / g.n2;
        const long b = g.at(i2, i3), b2 = g.at(i2 == 0 ? g.n2 - 1 : i2 - 1, i3),
                   b3 = g.at(i2, i3 == 0 ? g.n3 - 1 : i3 - 1);
        for (int k = threadIdx.x; k < q1; k += blockDim.x) {
            const int i1 = 4 * k;
            const long r = b + i1;
            const float4 y1 = ld4(Y + r), y2 = ld4(Y + V + r), y3 = ld4(Y + 2 * V + r);
            const float4 m2 = ld4(Y + V + b2 + i1), m3 = ld4(Y + 2 * V + b3 + i1), u = ld4(in + r);
            const float y1m = Y[b + (i1 == 0 ? g.n1 - 1 : i1 - 1)];
            float4 d;
            d.x = (y1.x + y2.x + y3.x - y1m - m2.x - m3.x) - u.x * inv_lam;
            d.y = (y1.y + y2.y + y3.y - y1.x - m2.y - m3.y) - u.y * inv_lam;
            d.z = (y1.z + y2.z + y3.z - y1.y - m2.z - m3.z) - u.z * inv_lam;
            d.w = (y1.w + y2.w + y3.w - y1.z - m2.w - m3.w) - u.w * inv_lam;
            st4(D + r, d);
        }
    }
}

__device__ __forceinline__ void tv_project(float q1, float q2, float q3, float &p1, float &p2, float &p3) {
    const float nrm = sqrtf(fmaxf(1.0f, q1 * q1 + q2 * q2 + q3 * q3));
    p1 = q1 / nrm;
    p2 = q2 / nrm;
    p3 = q3 / nrm;
}

__global__ void k_tv_step4(float *P, float *Y, const float *D, Rows g, float tau, double m, int fista) {
    const long V = g.V;
    const int q1 = g.n1 / 4;
    for (int row = blockIdx.x; row < g.n2 * g.n3; row += gridDim.x) {
        const int i2 = row % g.n2, i3 = row / g.n2;
        const long b = g.at(i2, i3), b2 = g.at(i2 == g.n2 - 1 ? 0 : i2 + 1, i3),
                   b3 = g.at(i2, i3 == g.n3 - 1 ? 0 : i3 + 1);
        for (int k = threadIdx.x; k < q1; k += blockDim.x) {
            const int i1 = 4 * k;
            const long r = b + i1;
            const float4 d0 = ld4(D + r), dn2 = ld4(D + b2 + i1), dn3 = ld4(D + b3 + i1);
            const float dp = D[b + (i1 + 4 == g.n1 ? 0 : i1 + 4)];
            const float *src = fista ? Y : P;
            const float4 s1 = ld4(src + r), s2 = ld4(src + V + r), s3 = ld4(src + 2 * V + r);
            const float d[5] = {d0.x, d0.y, d0.z, d0.w, dp};
            const float e2[4] = {dn2.x, dn2.y, dn2.z, dn2.w}, e3[4] = {dn3.x, dn3.y, dn3.z, dn3.w};
            const float a1[4] = {s1.x, s1.y, s1.z, s1.w}, a2[4] = {s2.x, s2.y, s2.z, s2.w},
                        a3[4] = {s3.x, s3.y, s3.z, s3.w};
            float o1[4], o2[4], o3[4];
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const float t1 = tau * (d[e + 1] - d[e]);
                const float t2 = tau * (e2[e] - d[e]);
                const float t3 = tau * (e3[e] - d[e]);
                tv_project(a1[e] + t1, a2[e] + t2, a3[e] + t3, o1[e], o2[e], o3[e]);
            }
            if (fista) {
                const float4 p1 = ld4(P + r), p2 = ld4(P + V + r), p3 = ld4(P + 2 * V + r);
                const float b1[4] = {p1.x, p1.y, p1.z, p1.w}, b2v[4] = {p2.x, p2.y, p2.z, p2.w},
                            b3v[4] = {p3.x, p3.y, p3.z, p3.w};
                float y1[4], y2[4], y3[4];
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    y1[e] = (float)(o1[e] + m * (o1[e] - (double)b1[e]));
                    y2[e] = (float)(o2[e] + m * (o2[e] - (double)b2v[e]));
                    y3[e] = (float)(o3[e] + m * (o3[e] - (double)b3v[e]));
                }
                st4(Y + r, make_float4(y1[0], y1[1], y1[2], y1[3]));
                st4(Y + V + r, make_float4(y2[0], y2[1], y2[2], y2[3]));
                st4(Y + 2 * V + r, make_float4(y3[0], y3[1], y3[2], y3[3]));
            }
            st4(P + r, make_float4(o1[0], o1[1], o1[2], o1[3]));
            st4(P + V + r, make_float4(o2[0], o2[1], o2[2], o2[3]));
            st4(P + 2 * V + r, make_float4(o3[0], o3[1], o3[2], o3[3]));
        }
    }
}

__global__ void k_tv_out4(const float *P, const float *in, float *out, Rows g, float lam) {
    const long V = g.V;
    const int q1 = g.n1 / 4;
    for (int row = blockIdx.x; row < g.n2 * g.n3; row += gridDim.x) {
        const int i2 = row % g.n2, i3 = row / g.n2;
        const long b = g.at(i2, i3), b2 = g.at(i2 == 0 ? g.n2 - 1 : i2 - 1, i3),
                   b3 = g.at(i2, i3 == 0 ? g.n3 - 1 : i3 - 1);
        for (int k = threadIdx.x; k < q1; k += blockDim.x) {
            const int i1 = 4 * k;
            const long r = b + i1;
            const float4 p1 = ld4(P + r), p2 = ld4(P + V + r), p3 = ld4(P + 2 * V + r);
            const float4 m2 = ld4(P + V + b2 + i1), m3 = ld4(P + 2 * V + b3 + i1), u = ld4(in + r);
            const float p1m = P[b + (i1 == 0 ? g.n1 - 1 : i1 - 1)];
            float4 o;
            o.x = u.x - lam * (p1.x + p2.x + p3.x - p1m - m2.x - m3.x);
            o.y = u.y - lam * (p1.y + p2.y + p3.y - p1.x - m2.y - m3.y);
            o.z = u.z - lam * (p1.z + p2.z + p3.z - p1.y - m2.z - m3.z);
            o.w = u.w - lam * (p1.w + p2.w + p3.w - p1.z - m2.w - m3.w);
            st4(out + r, o);
        }
    }
}

// in = vol / max(vol) with max from *mx; the max itself by k_max
__global__ void k_max(const float *v, long n, unsigned *mx_bits) {
    float m = -INFINITY;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        m = fmaxf(m, v[i]);
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    // order-preserving integer image of the float
    if ((threadIdx.x & 31) == 0) {
        unsigned b = __float_as_uint(m);
        b = (b & 0x80000000u) ? ~b : (b | 0x80000000u);
        atomicMax(mx_bits, b);
    }
}

__global__ void k_bits_to_float(const unsigned *mx_bits, float *mx) {
    unsigned b = *mx_bits;
    b = (b & 0x80000000u) ? (b & 0x7fffffffu) : ~b;
    *mx = __uint_as_float(b);
}

__global__ void k_scale(const float *v, float *out, long n, const float *div) {
    const float d = *div;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        out[i] = v[i] / d;
}

__global__ void k_mul(const float *v, float *out, long n, const float *mul) {
    const float m = *mul;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        out[i] = v[i] * m;
}

__global__ void k_positivity(float *v, long n) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        if (v[i] < 0.f) v[i] = 0.f;
}

// beam-frame volume of a tilt: V[z][y][x] (n x n window) = centred copy of
// the rotated nv^3 volume (zero elsewhere): the volume zero-padded laterally
// to the probe window (exact under the periodic multislice: V = 0 gives T = 1)
// beam-frame volume [n3][n2][n1] centred in the n x n window: V [n3][n][n]
__global__ void k_pad(const float *src, float *V, int n1, int n2, int n3, int n) {
    const long nn = (long)n * n, total = nn * n3;
    const int o1 = (n - n1) / 2, o2 = (n - n2) / 2;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
        const int z = (int)(i / nn), y = (int)((i / n) % n), x = (int)(i % n);
        const int yy = y - o2, xx = x - o1;
        V[i] = (yy >= 0 && yy < n2 && xx >= 0 && xx < n1) ? src[((long)z * n2 + yy) * n1 + xx] : 0.f;
    }
}

// lab-frame gradient contribution of a tilt: slab gradient G[s] (n x n,
// FP64) replicated over the slab's voxels and cropped to the [n3][n2][n1] volume
__global__ void k_slab_to_volume(const double *G, float *out, int n1, int n2, int n3, int n, int b) {
    const long total = (long)n1 * n2 * n3;
    const int o1 = (n - n1) / 2, o2 = (n - n2) / 2;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
        const int z = (int)(i / ((long)n1 * n2)), y = (int)((i / n1) % n2), x = (int)(i % n1);
        out[i] = (float)G[(long)(z / b) * n * n + (long)(y + o2) * n + (x + o1)];
    }
}

__global__ void k_accumulate(const float *g, double *acc, long n, int zero) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        acc[i] = (zero ? 0.0 : acc[i]) + (double)g[i];
}

// rec += step0 * acc
__global__ void k_update(float *rec, const double *acc, long n, float step0) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        rec[i] += step0 * (float)acc[i];
}
}  // namespace

int tv_prox(const TvArgs &a, cudaStream_t st) {
    const long V = (long)a.n1 * a.n2 * a.n3;
    const Rows rows{a.n1, a.n2, a.n3, V};
    // threads over i1 (whole warps, at most 256), CTAs over rows: up to 16
    // CTAs of 128 threads per SM
    const int bt = std::min(256, (a.n1 + 31) / 32 * 32);
    const int g = (int)std::min<long>((long)a.n2 * a.n3, 148L * (2048 / bt));
    // four voxels per thread where rows split into 16-byte groups (every
    // array is 16-byte aligned and n1 a multiple of 4)
    const bool vec = a.n1 % 4 == 0;
    const int bt4 = std::min(256, (a.n1 / 4 + 31) / 32 * 32);
    const int g4 = (int)std::min<long>((long)a.n2 * a.n3, 148L * std::min(32, 2048 / bt4));
    cudaError_t e;
    if ((e = cudaMemsetAsync(a.P, 0, sizeof(float) * 3 * V, st)) != cudaSuccess) return (int)e;
    if ((e = cudaMemsetAsync(a.Y, 0, sizeof(float) * 3 * V, st)) != cudaSuccess) return (int)e;
    const float tau = 1.0f / 12.0f;  // 3D (TV_method.m:13-16)
    double t = 1.0;
    for (int it = 0; it < a.niter; ++it) {
        const double t0 = t;
        t = (1.0 + std::sqrt(1.0 + 4.0 * t0 * t0)) / 2.0;  // TV_FISTA_method.m:31
        const double m = (t0 - 1.0) / t;
        if (vec) {
            k_tv_d4<<<g4, bt4, 0, st>>>(a.fista ? a.Y : a.P, a.in, a.D, rows, (float)(1.0 / a.lambda));
            k_tv_step4<<<g4, bt4, 0, st>>>(a.P, a.Y, a.D, rows, tau, m, a.fista);
        } else {
            k_tv_d<<<g, bt, 0, st>>>(a.fista ? a.Y : a.P, a.in, a.D, rows, (float)(1.0 / a.lambda));
            k_tv_step<<<g, bt, 0, st>>>(a.P, a.Y, a.D, rows, tau, m, a.fista);
        }
    }
    if (vec) k_tv_out4<<<g4, bt4, 0, st>>>(a.P, a.in, a.out, rows, (float)a.lambda);
    else k_tv_out<<<g, bt, 0, st>>>(a.P, a.in, a.out, rows, (float)a.lambda);
    if (a.err) k_tv_err<<<g, bt, 0, st>>>(a.out, rows, a.lambda, a.err);
    return (int)cudaGetLastError();
}

int vol_max(const float *v, long n, unsigned *bits, float *mx, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(bits, 0, sizeof(unsigned), st);
    if (e != cudaSuccess) return (int)e;
    k_max<<<grid_for(n), kThreads, 0, st>>>(v, n, bits);
    k_bits_to_float<<<1, 1, 0, st>>>(bits, mx);
    return (int)cudaGetLastError();
}

int vol_scale(const float *v, float *out, long n, const float *div, cudaStream_t st) {
    k_scale<<<grid_for(n), kThreads, 0, st>>>(v, out, n, div);
    return (int)cudaGetLastError();
}

int vol_mul(const float *v, float *out, long n, const float *mul, cudaStream_t st) {
    k_mul<<<grid_for(n), kThreads, 0, st>>>(v, out, n, mul);
    return (int)cudaGetLastError();
}

int vol_positivity(float *v, long n, cudaStream_t st) {
    k_positivity<<<grid_for(n), kThreads, 0, st>>>(v, n);
    return (int)cudaGetLastError();
}

int vol_pad(const float *src, float *V, int n1, int n2, int n3, int n, cudaStream_t st) {
    k_pad<<<grid_for((long)n * n * n3), kThreads, 0, st>>>(src, V, n1, n2, n3, n);
    return (int)cudaGetLastError();
}

int vol_slab_to_volume(const double *G, float *out, int n1, int n2, int n3, int n, int b, cudaStream_t st) {
    k_slab_to_volume<<<grid_for((long)n1 * n2 * n3), kThreads, 0, st>>>(G, out, n1, n2, n3, n, b);
    return (int)cudaGetLastError();
}

int vol_accumulate(const float *g, double *acc, long n, bool zero, cudaStream_t st) {
    k_accumulate<<<grid_for(n), kThreads, 0, st>>>(g, acc, n, zero ? 1 : 0);
    return (int)cudaGetLastError();
}

int vol_update(float *rec, const double *acc, long n, float step0, cudaStream_t st) {
    k_update<<<grid_for(n), kThreads, 0, st>>>(rec, acc, n, step0);
    return (int)cudaGetLastError();
}

}  // namespace mset
