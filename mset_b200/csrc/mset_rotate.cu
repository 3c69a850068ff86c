// mset_rotate.cu -- Fourier-shear 3D rotation of cubic volumes on the GPU
// (the reference's Func_rot_3Dvol_FourierShear / Func_inv_rot_3Dvol_FourierShear,
// func_lib/Func_rotate_3Dvol_ROTmat_FourierShear.m:14-134).
//
// A rotation is split into numStep sub-rotations of at most 11 degrees, each
// a product of four shears (Welling et al., Graphical Models 68 (2006)
// 356-370).  A shear along axis d is, for every plane at a fixed coordinate
// along d, a 2D Fourier shift: FFT over the plane, a linear phase, inverse
// FFT (SheerTransforms_for3Drot.m:29-49).  One CTA transforms one plane in
// shared memory with the same radix passes as the multislice kernel; the
// phase is the separable product ex(kx) ey(ky) computed in double per plane,
// except where the reference's grid is zeroed (any Nyquist index), where it
// is 1.  The complex volume stays L2-resident (16 MB at 128^3).
#include <cmath>
#include <vector>

#include "fft_core.cuh"
#include "mset_rotate.cuh"

namespace mset {

// ifftshift(k - round((n+1)/2)) grid with the Nyquist index zeroed
// (Func_rotate_3Dvol_ROTmat_FourierShear.m:70-90)
__host__ __device__ inline int rot_grid_val(int i, int n, bool *nyq) {
    const int h = (n + 1) / 2;
    int k = (i - h) % n;
    if (k < 0) k += n;
    const int c = (n + 2) / 2;  // round((n+1)/2) for n >= 1
    *nyq = (n % 2 == 0) && (i == c - 1);
    return *nyq ? 0 : (k + 1 - c);
}

template <int N>
struct RotSmem {
    static constexpr int EX = 0;  // float2 offsets after the field + twiddles
};

// complex S = ifftshift(real vol)
__global__ void k_rot_pre(const float *vol, float2 *S, int n) {
    const long nn = (long)n * n, total = nn * n;
    const int h = (n + 1) / 2;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
        const int i3 = (int)(i / nn), i2 = (int)((i / n) % n), i1 = (int)(i % n);
        const long o = (long)((i3 + h) % n) * nn + (long)((i2 + h) % n) * n + (i1 + h) % n;
        S[o] = make_float2(vol[i], 0.f);
    }
}

// out = fftshift(real(S)); out[(i + floor(n/2)) mod n] = S[i]
__global__ void k_rot_post(const float2 *S, float *out, int n) {
    const long nn = (long)n * n, total = nn * n;
    const int h = n / 2;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
        const int i3 = (int)(i / nn), i2 = (int)((i / n) % n), i1 = (int)(i % n);
        const long o = (long)((i3 + h) % n) * nn + (long)((i2 + h) % n) * n + (i1 + h) % n;
        out[o] = S[i].x;
    }
}

// One shear along MATLAB dimension `dim` (1: x fastest, 2: y, 3: z) with
// coefficients (ca, cb) for every plane; REAL keeps only the real part
// (the fourth shear of a sub-step, Func_rotate_3Dvol_ROTmat_FourierShear.m:121, 126).
template <class G, bool REAL>
__global__ void __launch_bounds__(G::NT, 1) k_shear(float2 *S, const float2 *twn, int dim, double ca, double cb) {
    constexpr int N = G::N, R1 = G::R1, R2 = G::R2;
    extern __shared__ __align__(16) float2 sm[];
    float2 *buf = sm;
    float2 *tw = buf + G::FIELD;
    float2 *ex = tw + N;
    float2 *ey = ex + N;
    __shared__ int nyx[N], nyy[N];
    for (int i = threadIdx.x; i < N; i += G::NT) tw[i] = twn[i];
    const long nn = (long)N * N;
    // plane axes: x' (fast, shared-memory rows) and y' (slow)
    long sx, sy, sc;
    if (dim == 1) {
        sx = N; sy = nn; sc = 1;      // plane (i2, i3) at fixed i1
    } else if (dim == 2) {
        sx = 1; sy = nn; sc = N;      // plane (i1, i3) at fixed i2
    } else {
        sx = 1; sy = N; sc = nn;      // plane (i1, i2) at fixed i3
    }
    const float inv = 1.0f / (float)(N * N);
    // one plane per CTA, or per cluster when the plane is split by rows
    const int yb = G::ybase();
    sync_all<G>();  // (cluster) every CTA has started before any remote access
    for (int c = blockIdx.x / G::CL; c < N; c += gridDim.x / G::CL) {
        bool qc;
        const int gc = rot_grid_val(c, N, &qc);
        if (qc) {
            // the reference's grids are zero on this plane: no shift; only the
            // fourth shear's real() acts
            if (REAL) {
                for (int i = threadIdx.x; i < G::ROWS * N; i += G::NT) {
                    float2 *p = S + (long)c * sc + (long)G::gy(yb, i / N) * sy + (long)(i % N) * sx;
                    p->y = 0.f;
                }
            }
            sync_all<G>();
            continue;
        }
        // per-plane phase factors (double): phase = 2 pi gc (cx gx(kx) + cy gy(ky)) / N
        double cx, cy;
        if (dim == 1) {
            cx = ca; cy = cb;  // a with n2 (x'), b with n3 (y')
        } else if (dim == 2) {
            cx = cb; cy = ca;  // b with n1 (x'), a with n3 (y')
        } else {
            cx = ca; cy = cb;  // a with n1 (x'), b with n2 (y')
        }
        for (int L = threadIdx.x; L < N; L += G::NT) {
            const int k = G::scr(L);
            bool q;
            const int g = rot_grid_val(k, N, &q);
            double s, co;
            sincospi(2.0 * (double)gc * cx * (double)g / (double)N, &s, &co);
            ex[L] = make_float2((float)co, (float)s);
            nyx[L] = q;
            sincospi(2.0 * (double)gc * cy * (double)g / (double)N, &s, &co);
            ey[L] = make_float2((float)co, (float)s);
            nyy[L] = q;
        }
        for (int i = threadIdx.x; i < G::ROWS * N; i += G::NT) {
            const int yy = i / N, xx = i % N;
            buf[G::at(yy, xx)] = S[(long)c * sc + (long)G::gy(yb, yy) * sy + (long)xx * sx];
        }
        __syncthreads();
        row_passA<G, 0, -1>(buf, tw, NoOp{});
        sync_rows();
        row_passB<G, -1>(buf);
        sync_rowcol();
        col_passA<G, -1, true>(buf, tw);
        sync_cols<G>();
        col_passB<G, -1, +1>(buf, [&](int y0, int x, float2 *v) {
            const float2 e = ex[x];
            const bool qx = nyx[x];
#pragma unroll
            for (int j = 0; j < R1; ++j) {
                const float2 f = (qx || nyy[y0 + j]) ? make_float2(inv, 0.f) : cscale(cmul(e, ey[y0 + j]), inv);
                v[j] = cmul(v[j], f);
            }
        });
        sync_cols<G>();
        col_passA<G, +1, false>(buf, tw);
        sync_rowcol();
        row_passB<G, +1>(buf);
        sync_rows();
        row_passA<G, +1, 0>(buf, tw, NoOp{});
        __syncthreads();
        for (int i = threadIdx.x; i < G::ROWS * N; i += G::NT) {
            const int yy = i / N, xx = i % N;
            float2 v = buf[G::at(yy, xx)];
            if (REAL) v.y = 0.f;
            S[(long)c * sc + (long)G::gy(yb, yy) * sy + (long)xx * sx] = v;
        }
        sync_all<G>();
        (void)R2;
    }
}

template <class G>
static size_t shear_smem() {
    return sizeof(float2) * ((size_t)G::FIELD + 3 * G::N);
}

template <class G, bool REAL>
static int launch_shear_k(float2 *S, const float2 *twn, int dim, double a, double b, int grid, cudaStream_t st) {
    auto k = k_shear<G, REAL>;
    const size_t sm = shear_smem<G>();
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return (int)e;
    if constexpr (G::CL > 1) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(grid);
        cfg.blockDim = dim3(G::NT);
        cfg.dynamicSmemBytes = sm;
        cfg.stream = st;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = G::CL;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        return (int)cudaLaunchKernelEx(&cfg, k, S, twn, dim, a, b);
    } else {
        k<<<grid, G::NT, sm, st>>>(S, twn, dim, a, b);
        return (int)cudaGetLastError();
    }
}

template <class G>
static int launch_shear(float2 *S, const float2 *twn, int dim, double a, double b, bool real, int sms,
                        cudaStream_t st) {
    // planes in flight: one per CTA, or one per cluster of CL CTAs
    const int grid = std::min(G::N, sms / G::CL) * G::CL;
    return real ? launch_shear_k<G, true>(S, twn, dim, a, b, grid, st)
                : launch_shear_k<G, false>(S, twn, dim, a, b, grid, st);
}

#define MSET_ROT_GEOS(X) X(24, 8, 64) X(32, 8, 128) X(48, 16, 192) X(64, 8, 256) X(96, 16, 384) X(128, 16, 512) X(160, 16, 640)
// 256^2 planes do not fit one SM: split by rows over a 4-CTA cluster
using RotGeo256 = GeoCl<256, 16, 512, 4>;

bool rot_supported(int n) {
#define X(N_, R1_, NT_) \
    if (n == N_) return true;
    MSET_ROT_GEOS(X)
#undef X
    return n == 256;
}

int rot_r1(int n) {
#define X(N_, R1_, NT_) \
    if (n == N_) return R1_;
    MSET_ROT_GEOS(X)
#undef X
    return n == 256 ? RotGeo256::R1 : 0;
}

static int shear(int n, float2 *S, const float2 *twn, int dim, double a, double b, bool real, int sms,
                 cudaStream_t st) {
#define X(N_, R1_, NT_) \
    if (n == N_) return launch_shear<Geo<N_, R1_, NT_>>(S, twn, dim, a, b, real, sms, st);
    MSET_ROT_GEOS(X)
#undef X
    if (n == 256) return launch_shear<RotGeo256>(S, twn, dim, a, b, real, sms, st);
    return (int)cudaErrorInvalidValue;
}

// ---------------------------------------------------------------------------
// volumes of any shape n1 x n2 x n3: every shear as batched 1D transforms
// ---------------------------------------------------------------------------
// A shear along axis d multiplies the 2D spectrum of each plane (axes a, b)
// by exp(i 2 pi g_d (c_a g_a + c_b g_b) / n_d), or by 1 where any of the
// three grids is at its Nyquist index (SheerTransforms_for3Drot.m:29-49 with
// the grids of Func_rotate_3Dvol_ROTmat_FourierShear.m:70-90).  For planes of
// unequal sides this is done line by line through global memory:
//   (1) forward transform of every line along a (natural -> scrambled),
//   (2) along b: forward transform, the phase (a's frequency from the line's
//       scrambled position, d's grid from its index), inverse transform,
//   (3) inverse transform along a (scrambled -> natural), real() fused into
//       the fourth shear of a sub-step.
// Each kernel reads and writes the complex volume once; a CTA transforms a
// batch of ROWS lines in shared memory with the radix passes of the position
// kernel.  Lines are batched along the other axis of smallest stride, so
// every global access is coalesced.

// ROWS lines of length L in one CTA's shared memory
template <int L_, int R1_, int ROWS_>
struct LineGeo : Geo<L_, R1_, 256> {
    static constexpr int ROWS = ROWS_;
    static constexpr int FIELD = ROWS_ * Geo<L_, R1_, 256>::S;
};

// the lines of one transform axis: a = transform axis, p = the other axis of
// smaller stride (batched), q = the remaining one
struct LineMap {
    long sa, sp, sq;
    int La, np, nq;
    int pa_is_a;  // shift kernel: 1 if p is the first-transformed axis, 0 if p is the shear axis
};

// the grid value of a frequency index (rot_grid_val) and whether it is Nyquist
__device__ __forceinline__ int grid_of(int k, int n, bool *nyq) { return rot_grid_val(k, n, nyq); }

// MODE 0: forward along the axis (natural -> scrambled); 1: inverse (scrambled
// -> natural, REAL keeps the real part); 2: the shift: forward, phase,
// inverse.  For MODE 2 the lines run along b; (ra1, La_a) give the scrambled
// layout of the first-transformed axis a; nd is the shear axis length; c_a,
// c_b the shear coefficients of a and b.
template <class LG, int MODE, bool REAL>
__global__ void __launch_bounds__(256) k_line(float2 *S, LineMap m, int ra1, int La_a, int nd, double c_a,
                                              double c_b, float scale) {
    constexpr int L = LG::N, R1 = LG::R1, ROWS = LG::ROWS, NT = LG::NT;
    extern __shared__ __align__(16) float2 sm[];
    float2 *buf = sm;
    float2 *tw = buf + LG::FIELD;
    __shared__ double s_row[ROWS];  // per row: 2 g_d c_a g_a / n_d (MODE 2)
    __shared__ double s_gd[ROWS];   // per row: 2 g_d / n_d, or NaN on a Nyquist plane
    for (int i = threadIdx.x; i < L; i += NT) {
        const int k2 = i / R1, n1 = i % R1;
        const long mm = (long)n1 * k2 % L;
        double sn, cs;
        sincospi(-2.0 * (double)mm / (double)L, &sn, &cs);
        tw[i] = make_float2((float)cs, (float)sn);
    }
    const int nbp = (m.np + ROWS - 1) / ROWS;
    const long batches = (long)nbp * m.nq;
    for (long bt = blockIdx.x; bt < batches; bt += gridDim.x) {
        const int bp = (int)(bt % nbp), iq = (int)(bt / nbp);
        __syncthreads();
        if (MODE == 2 && threadIdx.x < ROWS) {
            const int ip = bp * ROWS + threadIdx.x;
            // the line's position along a (scrambled) and its index along d
            const int la = m.pa_is_a ? ip : iq, id = m.pa_is_a ? iq : ip;
            const int ka = la / ra1 + (La_a / ra1) * (la % ra1);
            bool qa, qd;
            const int ga = grid_of(ka, La_a, &qa), gd = grid_of(id, nd, &qd);
            s_gd[threadIdx.x] = (qa || qd) ? NAN : 2.0 * (double)gd / (double)nd;
            s_row[threadIdx.x] = 2.0 * (double)gd * c_a * (double)ga / (double)nd;
        }
        // load the batch (coalesced: along the line when it is contiguous, else across lines)
        for (int i = threadIdx.x; i < ROWS * L; i += NT) {
            int r, k;
            if (m.sa == 1) {
                r = i / L;
                k = i % L;
            } else {
                r = i % ROWS;
                k = i / ROWS;
            }
            const int ip = bp * ROWS + r;
            buf[LG::at(r, k)] = ip < m.np ? S[(long)ip * m.sp + (long)iq * m.sq + (long)k * m.sa] : make_float2(0.f, 0.f);
        }
        __syncthreads();
        if constexpr (MODE == 0 || MODE == 2) {
            row_passA<LG, 0, -1>(buf, tw, NoOp{});
            sync_rows();
            row_passB<LG, -1>(buf);
        }
        if constexpr (MODE == 2) {
            __syncthreads();
            for (int i = threadIdx.x; i < ROWS * L; i += NT) {
                const int r = i / L, lb = i % L;
                const double gdn = s_gd[r];
                float2 f = make_float2(scale, 0.f);
                bool qb;
                const int gb = grid_of(LG::scr(lb), L, &qb);
                if (!qb && !isnan(gdn)) {
                    double t = s_row[r] + gdn * c_b * (double)gb;  // phase / pi
                    t -= 2.0 * rint(0.5 * t);                        // into [-1, 1]
                    float sn, cs;
                    sincospif((float)t, &sn, &cs);
                    f = make_float2(scale * cs, scale * sn);
                }
                float2 &v = buf[LG::at(r, lb)];
                v = cmul(v, f);
            }
            __syncthreads();
        }
        if constexpr (MODE == 1 || MODE == 2) {
            row_passB<LG, +1>(buf);
            sync_rows();
            row_passA<LG, +1, 0>(buf, tw, NoOp{});
        }
        __syncthreads();
        for (int i = threadIdx.x; i < ROWS * L; i += NT) {
            int r, k;
            if (m.sa == 1) {
                r = i / L;
                k = i % L;
            } else {
                r = i % ROWS;
                k = i / ROWS;
            }
            const int ip = bp * ROWS + r;
            if (ip < m.np) {
                float2 v = buf[LG::at(r, k)];
                if (REAL) v.y = 0.f;
                S[(long)ip * m.sp + (long)iq * m.sq + (long)k * m.sa] = v;
            }
        }
    }
}

// one geometry per supported line length (256 threads, radix split L = R1 R2)
#define MSET_LINE_GEOS(X) \
    X(24, 8, 32) X(32, 8, 32) X(48, 16, 16) X(64, 8, 32) X(96, 16, 16) X(128, 16, 16) X(160, 16, 16) \
    X(192, 16, 16) X(256, 16, 16)

bool rot_line_supported(int n) {
#define X(L_, R1_, ROWS_) \
    if (n == L_) return true;
    MSET_LINE_GEOS(X)
#undef X
    return false;
}

static int line_r1(int n) {
#define X(L_, R1_, ROWS_) \
    if (n == L_) return R1_;
    MSET_LINE_GEOS(X)
#undef X
    return 0;
}

template <class LG, int MODE, bool REAL>
static int launch_line_k(float2 *S, const LineMap &m, int ra1, int La_a, int nd, double c_a, double c_b, float scale,
                         int sms, cudaStream_t st) {
    auto k = k_line<LG, MODE, REAL>;
    const size_t sm = sizeof(float2) * ((size_t)LG::FIELD + LG::N);
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return (int)e;
    const long batches = (long)((m.np + LG::ROWS - 1) / LG::ROWS) * m.nq;
    const int grid = (int)std::min<long>(batches, (long)sms * 8);
    k<<<grid, 256, sm, st>>>(S, m, ra1, La_a, nd, c_a, c_b, scale);
    return (int)cudaGetLastError();
}

static int launch_line(int mode, bool real, float2 *S, const LineMap &m, int ra1, int La_a, int nd, double c_a,
                       double c_b, float scale, int sms, cudaStream_t st) {
#define X(L_, R1_, ROWS_)                                                                                    \
    if (m.La == L_) {                                                                                        \
        using LG = LineGeo<L_, R1_, ROWS_>;                                                                  \
        if (mode == 0) return launch_line_k<LG, 0, false>(S, m, ra1, La_a, nd, c_a, c_b, scale, sms, st);    \
        if (mode == 2) return launch_line_k<LG, 2, false>(S, m, ra1, La_a, nd, c_a, c_b, scale, sms, st);    \
        if (real) return launch_line_k<LG, 1, true>(S, m, ra1, La_a, nd, c_a, c_b, scale, sms, st);          \
        return launch_line_k<LG, 1, false>(S, m, ra1, La_a, nd, c_a, c_b, scale, sms, st);                   \
    }
    MSET_LINE_GEOS(X)
#undef X
    return (int)cudaErrorInvalidValue;
}

// lines along axis `ax` (0-based: 0 = x fastest) of an n[0] x n[1] x n[2]
// volume; p = the other axis of smaller stride
static LineMap line_map(const int n[3], int ax) {
    const long st[3] = {1, n[0], (long)n[0] * n[1]};
    int o[2], c = 0;
    for (int i = 0; i < 3; ++i)
        if (i != ax) o[c++] = i;  // o[0] has the smaller stride
    LineMap m;
    m.sa = st[ax];
    m.La = n[ax];
    m.sp = st[o[0]];
    m.np = n[o[0]];
    m.sq = st[o[1]];
    m.nq = n[o[1]];
    m.pa_is_a = 0;
    return m;
}

// one shear along MATLAB dimension dim (1, 2, 3) of an n1 x n2 x n3 complex volume
static int shear_lines(const int n[3], float2 *S, int dim, double ca, double cb, bool real, int sms, cudaStream_t st) {
    const int d = dim - 1;
    // the two transformed axes and their coefficients
    // (dim 1: axis 2 <-> a, axis 3 <-> b; dim 2: axis 1 <-> b, axis 3 <-> a;
    //  dim 3: axis 1 <-> a, axis 2 <-> b: SheerTransforms_for3Drot.m:16-49)
    int ax0, ax1;
    double c0, c1;
    if (d == 0) {
        ax0 = 1; c0 = ca; ax1 = 2; c1 = cb;
    } else if (d == 1) {
        ax0 = 0; c0 = cb; ax1 = 2; c1 = ca;
    } else {
        ax0 = 0; c0 = ca; ax1 = 1; c1 = cb;
    }
    // first-transformed axis: ax0; the shift runs along ax1
    const LineMap ma = line_map(n, ax0);
    LineMap mb = line_map(n, ax1);
    // along ax1 the other two axes are ax0 and d: which one is batched (p)?
    mb.pa_is_a = (mb.sp == (ax0 == 0 ? 1 : ax0 == 1 ? (long)n[0] : (long)n[0] * n[1])) ? 1 : 0;
    const int ra1 = line_r1(n[ax0]);
    const float scale = 1.0f / ((float)n[ax0] * (float)n[ax1]);
    int rc = launch_line(0, false, S, ma, 0, 0, 0, 0, 0, 1.f, sms, st);
    if (!rc) rc = launch_line(2, false, S, mb, ra1, n[ax0], n[d], c0, c1, scale, sms, st);
    if (!rc) rc = launch_line(1, real, S, ma, 0, 0, 0, 0, 0, 1.f, sms, st);
    return rc;
}

// complex S = ifftshift(real vol) / out = fftshift(real(S)) for n1 x n2 x n3
__global__ void k_rot_pre3(const float *vol, float2 *S, int n1, int n2, int n3) {
    const long n12 = (long)n1 * n2, total = n12 * n3;
    const int h1 = (n1 + 1) / 2, h2 = (n2 + 1) / 2, h3 = (n3 + 1) / 2;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
        const int i3 = (int)(i / n12), i2 = (int)((i / n1) % n2), i1 = (int)(i % n1);
        S[(long)((i3 + h3) % n3) * n12 + (long)((i2 + h2) % n2) * n1 + (i1 + h1) % n1] = make_float2(vol[i], 0.f);
    }
}
__global__ void k_rot_post3(const float2 *S, float *out, int n1, int n2, int n3) {
    const long n12 = (long)n1 * n2, total = n12 * n3;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
        const int i3 = (int)(i / n12), i2 = (int)((i / n1) % n2), i1 = (int)(i % n1);
        out[(long)((i3 + n3 / 2) % n3) * n12 + (long)((i2 + n2 / 2) % n2) * n1 + (i1 + n1 / 2) % n1] = S[i].x;
    }
}

int rot_apply3(const RotPlan &pl, int n1, int n2, int n3, const float *vol, float *out, float2 *S, int sms,
               cudaStream_t st) {
    const long total = (long)n1 * n2 * n3;
    if (!pl.active) {
        if (out != vol) return (int)cudaMemcpyAsync(out, vol, sizeof(float) * total, cudaMemcpyDeviceToDevice, st);
        return 0;
    }
    const int n[3] = {n1, n2, n3};
    const int g = (int)std::min<long>((total + 255) / 256, (long)sms * 8);
    k_rot_pre3<<<g, 256, 0, st>>>(vol, S, n1, n2, n3);
    int rc = (int)cudaGetLastError();
    if (rc) return rc;
    for (int s = 0; s < pl.num_step; ++s)
        for (int k = 0; k < 4; ++k) {
            rc = shear_lines(n, S, pl.dim[k], pl.a[k], pl.b[k], k == 3, sms, st);
            if (rc) return rc;
        }
    k_rot_post3<<<g, 256, 0, st>>>(S, out, n1, n2, n3);
    return (int)cudaGetLastError();
}

// ---------------------------------------------------------------------------
// host-side rotation plan (double precision), restating the reference
// ---------------------------------------------------------------------------
namespace {
void quat_rot(const double *v, double theta_deg, double R[3][3]) {  // MatrixQuaternionRot.m:1-11
    const double th = theta_deg * M_PI / 180.0;
    const double nv = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    const double w = std::cos(th / 2), x = -std::sin(th / 2) * v[0] / nv, y = -std::sin(th / 2) * v[1] / nv,
                 z = -std::sin(th / 2) * v[2] / nv;
    R[0][0] = 1 - 2 * y * y - 2 * z * z; R[0][1] = 2 * x * y + 2 * w * z; R[0][2] = 2 * x * z - 2 * w * y;
    R[1][0] = 2 * x * y - 2 * w * z; R[1][1] = 1 - 2 * x * x - 2 * z * z; R[1][2] = 2 * y * z + 2 * w * x;
    R[2][0] = 2 * x * z + 2 * w * y; R[2][1] = 2 * y * z - 2 * w * x; R[2][2] = 1 - 2 * x * x - 2 * y * y;
}
void mul3(const double A[3][3], const double B[3][3], double C[3][3]) {
    double T[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            T[i][j] = 0;
            for (int k = 0; k < 3; ++k) T[i][j] += A[i][k] * B[k][j];
        }
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) C[i][j] = T[i][j];
}
void inverse3(const double A[3][3], double B[3][3]) {
    const double det = A[0][0] * (A[1][1] * A[2][2] - A[1][2] * A[2][1]) -
                       A[0][1] * (A[1][0] * A[2][2] - A[1][2] * A[2][0]) +
                       A[0][2] * (A[1][0] * A[2][1] - A[1][1] * A[2][0]);
    double T[3][3];
    T[0][0] = (A[1][1] * A[2][2] - A[1][2] * A[2][1]) / det;
    T[0][1] = (A[0][2] * A[2][1] - A[0][1] * A[2][2]) / det;
    T[0][2] = (A[0][1] * A[1][2] - A[0][2] * A[1][1]) / det;
    T[1][0] = (A[1][2] * A[2][0] - A[1][0] * A[2][2]) / det;
    T[1][1] = (A[0][0] * A[2][2] - A[0][2] * A[2][0]) / det;
    T[1][2] = (A[0][2] * A[1][0] - A[0][0] * A[1][2]) / det;
    T[2][0] = (A[1][0] * A[2][1] - A[1][1] * A[2][0]) / det;
    T[2][1] = (A[0][1] * A[2][0] - A[0][0] * A[2][1]) / det;
    T[2][2] = (A[0][0] * A[1][1] - A[0][1] * A[1][0]) / det;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) B[i][j] = T[i][j];
}
// My_obtain_quaternion_from_matrix.m:11-39
void quat_from(const double M[3][3], double &qx, double &qy, double &qz, double &qw) {
    const double Tr = M[0][0] + M[1][1] + M[2][2];
    double S;
    if (Tr > 0) {
        S = std::sqrt(Tr + 1) * 2;
        qw = 0.25 * S; qx = (M[2][1] - M[1][2]) / S; qy = (M[0][2] - M[2][0]) / S; qz = (M[1][0] - M[0][1]) / S;
    } else if (M[0][0] > M[1][1] && M[0][0] > M[2][2]) {
        S = std::sqrt(1.0 + M[0][0] - M[1][1] - M[2][2]) * 2;
        qw = (M[2][1] - M[1][2]) / S; qx = 0.25 * S; qy = (M[0][1] + M[1][0]) / S; qz = (M[0][2] + M[2][0]) / S;
    } else if (M[1][1] > M[2][2]) {
        S = std::sqrt(1.0 + M[1][1] - M[0][0] - M[2][2]) * 2;
        qw = (M[0][2] - M[2][0]) / S; qx = (M[0][1] + M[1][0]) / S; qy = 0.25 * S; qz = (M[1][2] + M[2][1]) / S;
    } else {
        S = std::sqrt(1.0 + M[2][2] - M[0][0] - M[1][1]) * 2;
        qw = (M[1][0] - M[0][1]) / S; qx = (M[0][2] + M[2][0]) / S; qy = (M[1][2] + M[2][1]) / S; qz = 0.25 * S;
    }
}
// calculate_S_matrices_for3DFourierShearRot_perm_ver1.m:16-93 and the
// backward variant (W -> -W, coefficients negated); absSum or +inf
double coeffs(double X0, double Y0, double Z0, double W, int perm, bool backward, double co[8]) {
    const double in[3] = {X0, Y0, Z0};
    const double X = in[(0 + perm) % 3], Y = in[(1 + perm) % 3], Z = in[(2 + perm) % 3];
    if (backward) W = -W;
    double a, b, c, d, e, f, g, h;
    if (std::fabs(Y * Z - X * W) > 1e-5 && std::fabs(X * Y - Z * W) > 1e-5) {
        a = (X * X + Y * Y) / (Y * Z - X * W);
        b = (Y * Y - Z * Z) / (X * Y - Z * W) - 2 * (Y * Z * (X * X + Y * Y)) / (X * Y - Z * W) / (Y * Z - X * W);
        c = 2 * Y * Z / (X * Y - Z * W);
        d = 2 * (X * W - Y * Z);
        e = 2 * (X * Y - Z * W);
        f = -2 * X * Y / (Y * Z - X * W);
        g = (X * X - Y * Y) / (Y * Z - X * W) + 2 * X * Y * (Y * Y + Z * Z) / (X * Y - Z * W) / (Y * Z - X * W);
        h = (-1 + X * X + W * W) / (X * Y - Z * W);
    } else if (std::fabs(Y) < 1e-6) {
        a = -X / W; b = Z / W; c = 0; d = 2 * X * W; e = -2 * Z * W; f = 0; g = -X / W; h = Z / W;
    } else {
        return INFINITY;
    }
    const double v[8] = {a, b, c, d, e, f, g, h};
    double s = 0;
    for (int i = 0; i < 8; ++i) {
        co[i] = backward ? -v[i] : v[i];
        s += std::fabs(v[i]);
    }
    return s;
}
}  // namespace

bool rot_plan(const double *v1, const double *v2, const double *v3, double phi, double theta, double psi, bool inverse,
              RotPlan *plan) {
    double R1[3][3], R2[3][3], R3[3][3], R[3][3], M[3][3];
    quat_rot(v1, phi, R1);
    quat_rot(v2, theta, R2);
    quat_rot(v3, psi, R3);
    mul3(R1, R2, R);
    mul3(R, R3, R);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) M[i][j] = R[j][i];  // R = (R1 R2 R3)'
    if (inverse) inverse3(M, M);                      // Func_inv_rot_3Dvol_FourierShear.m:13
    plan->active = std::fabs(theta) > 0.5 || std::fabs(phi) > 0.5 || std::fabs(psi) > 0.5;
    double qx, qy, qz, qw;
    quat_from(M, qx, qy, qz, qw);
    const double Ang = std::acos(qw) * 180.0 / M_PI * 2;
    const double nv = std::sqrt(qx * qx + qy * qy + qz * qz);
    const double Vec[3] = {qx / nv, qy / nv, qz / nv};
    const int numStep = (int)std::floor(Ang / 11.0) + 1;  // rotStepInit = 11
    const double rotStep = Ang / numStep;
    const double w = std::cos(rotStep / 2 * M_PI / 180), sn = std::sin(rotStep / 2 * M_PI / 180);
    const double x = -sn * Vec[0], y = -sn * Vec[1], z = -sn * Vec[2];
    double cf[3][8], cb[3][8], sf[3], sb[3];
    for (int i = 1; i <= 3; ++i) {
        sf[i - 1] = coeffs(x, y, z, w, i, false, cf[i - 1]);
        sb[i - 1] = coeffs(x, y, z, w, i, true, cb[i - 1]);
    }
    int mf = 0, mb = 0;
    for (int i = 1; i < 3; ++i) {
        if (sf[i] < sf[mf]) mf = i;
        if (sb[i] < sb[mb]) mb = i;
    }
    const bool fwd = sf[mf] < sb[mb];
    const int mI = (fwd ? mf : mb) + 1;
    const double *co = fwd ? cf[mf] : cb[mb];
    plan->num_step = numStep;
    // Func_rotate_3Dvol_ROTmat_FourierShear.m:116-128: the four shears of a step
    if (fwd) {
        plan->dim[0] = (mI + 1) % 3 + 1; plan->a[0] = co[6]; plan->b[0] = co[7];
        plan->dim[1] = mI % 3 + 1;       plan->a[1] = co[4]; plan->b[1] = co[5];
        plan->dim[2] = (mI + 2) % 3 + 1; plan->a[2] = co[2]; plan->b[2] = co[3];
        plan->dim[3] = (mI + 1) % 3 + 1; plan->a[3] = co[0]; plan->b[3] = co[1];
    } else {
        plan->dim[0] = (mI + 1) % 3 + 1; plan->a[0] = co[0]; plan->b[0] = co[1];
        plan->dim[1] = (mI + 2) % 3 + 1; plan->a[1] = co[2]; plan->b[1] = co[3];
        plan->dim[2] = mI % 3 + 1;       plan->a[2] = co[4]; plan->b[2] = co[5];
        plan->dim[3] = (mI + 1) % 3 + 1; plan->a[3] = co[6]; plan->b[3] = co[7];
    }
    return plan->active;
}

int rot_twiddles(int n, std::vector<float2> &h) {
    const int r1 = rot_r1(n);
    if (!r1) return -1;
    const int r2 = n / r1;
    h.resize(n);
    for (int k2 = 0; k2 < r2; ++k2)
        for (int n1 = 0; n1 < r1; ++n1) {
            const long m = (long)n1 * k2 % n;
            const double ang = -2.0 * M_PI * (double)m / (double)n;
            h[k2 * r1 + n1] = make_float2((float)std::cos(ang), (float)std::sin(ang));
        }
    return 0;
}

// out = rotation of vol (both device [n][n][n] float, may alias), S = n^3 complex work
int rot_apply(const RotPlan &pl, int n, const float *vol, float *out, float2 *S, const float2 *twn, int sms,
              cudaStream_t st) {
    const long total = (long)n * n * n;
    if (!pl.active) {
        if (out != vol) {
            cudaError_t e = cudaMemcpyAsync(out, vol, sizeof(float) * total, cudaMemcpyDeviceToDevice, st);
            return (int)e;
        }
        return 0;
    }
    const int g = (int)std::min<long>((total + 255) / 256, (long)sms * 8);
    k_rot_pre<<<g, 256, 0, st>>>(vol, S, n);
    int rc = (int)cudaGetLastError();
    if (rc) return rc;
    for (int s = 0; s < pl.num_step; ++s)
        for (int k = 0; k < 4; ++k) {
            rc = shear(n, S, twn, pl.dim[k], pl.a[k], pl.b[k], k == 3, sms, st);
            if (rc) return rc;
        }
    k_rot_post<<<g, 256, 0, st>>>(S, out, n);
    return (int)cudaGetLastError();
}

}  // namespace mset
