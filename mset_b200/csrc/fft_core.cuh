// fft_core.cuh -- shared-memory 2D FFT building blocks for sm_100a.
//
// An N x N complex64 field lives in one CTA's shared memory, row stride
// S = N + N/R1 (one pad element after every R1 elements along x, which makes
// every pass below free of bank conflicts).  A 1D transform of length
// N = R1*R2 is two register passes:
//
//   pass A (per n1, R2 points at x = n1 + R1*j):   R2-point DFT + twiddle
//   pass B (per k2, R1 points at x = j + R1*k2):   R1-point DFT
//
// Natural -> scrambled (NAT2SCR): A then B.  Location L = k1 + R1*k2 then
// holds frequency k = k2 + R2*k1 ("digit-reversed" order).
// Scrambled -> natural (SCR2NAT): B then A (twiddle before the DFT).
//
// A forward transform, a pointwise product and an inverse transform therefore
// need no reordering at all: the propagator, measured amplitudes and probe
// spectrum are stored in the scrambled layout once, at upload.  Both
// directions work with either sign, so the same passes give F and F^{-1}.
//
// The 2D transform is rows (x) then columns (y); the inverse runs columns then
// rows.  The passes that border a pointwise stage are fused with it:
//   row pass A  = [inverse rows A] + op(real space, natural order) + [forward rows A]
//   col pass B  = [forward cols B] + op(Fourier space, scrambled)   + [inverse cols B]
// so one propagation slab costs six shared-memory round trips, with a
// CTA-wide barrier only where row passes meet column passes.
#pragma once
#include <type_traits>
#include <cooperative_groups.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace mset {

// ---------------------------------------------------------------------------
// compile-time trigonometry (Taylor series in double, evaluated by the
// compiler) for the internal twiddles of the register codelets
// ---------------------------------------------------------------------------
constexpr double kPi = 3.14159265358979323846264338327950288;

constexpr double ct_reduce(double x) {
    // x in [0, 2pi) -> [-pi, pi)
    return x >= kPi ? x - 2.0 * kPi : x;
}
constexpr double ct_sin_series(double x) {
    double term = x, sum = x;
    for (int k = 1; k < 30; ++k) {
        term *= -x * x / ((2.0 * k) * (2.0 * k + 1.0));
        sum += term;
    }
    return sum;
}
constexpr double ct_cos_series(double x) {
    double term = 1.0, sum = 1.0;
    for (int k = 1; k < 30; ++k) {
        term *= -x * x / ((2.0 * k - 1.0) * (2.0 * k));
        sum += term;
    }
    return sum;
}
// e^{sign * 2 pi i m / r}
template <int M, int R, int SG>
struct Tw {
    static constexpr double a = ct_reduce(2.0 * kPi * (double)(M % R) / (double)R);
    static constexpr float c = (float)ct_cos_series(a);
    static constexpr float s = (float)(SG * ct_sin_series(a));
};

template <int V>
struct IC {
    static constexpr int value = V;
};
template <int B, int E, class F>
__device__ __forceinline__ void sfor(F &&f) {
    if constexpr (B < E) {
        f(IC<B>{});
        sfor<B + 1, E>(f);
    }
}

// Complex add / subtract with the packed FP32x2 instructions of sm_100
// (add.f32x2 / sub.f32x2 on a 64-bit register pair): one issue slot for both
// components of the interleaved complex value.
__device__ __forceinline__ unsigned long long pk(float2 a) {
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a.x), "f"(a.y));
    return r;
}
__device__ __forceinline__ float2 upk(unsigned long long r) {
    float2 a;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(a.x), "=f"(a.y) : "l"(r));
    return a;
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) {
    unsigned long long r;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(pk(a)), "l"(pk(b)));
    return upk(r);
}
__device__ __forceinline__ float2 csub(float2 a, float2 b) {
    unsigned long long r;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(pk(a)), "l"(pk(b)));
    return upk(r);
}
// Complex multiply with the packed multiply and fused multiply-add of sm_100
// (mul.f32x2 / fma.f32x2): a*b = (a.x b.x, a.y b.x) + (a.y, a.x) (-b.y, b.y),
// two issue slots instead of four (the FP32 pipe does the same work).
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    unsigned long long t, r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(t) : "l"(pk(a)), "l"(pk(make_float2(b.x, b.x))));
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(pk(make_float2(a.y, a.x))), "l"(pk(make_float2(-b.y, b.y))),
        "l"(t));
    return upk(r);
}
// a * conj(b) = (a.x b.x, a.y b.x) + (a.y, a.x) (b.y, -b.y)
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {
    unsigned long long t, r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(t) : "l"(pk(a)), "l"(pk(make_float2(b.x, b.x))));
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(pk(make_float2(a.y, a.x))), "l"(pk(make_float2(b.y, -b.y))),
        "l"(t));
    return upk(r);
}
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
// multiply by i * sg
template <int SG>
__device__ __forceinline__ float2 cmul_i(float2 a) {
    return SG > 0 ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}
template <int M, int R, int SG>
__device__ __forceinline__ float2 twmul(float2 a) {
    constexpr int m = M % R;
    if constexpr (m == 0) {
        return a;
    } else if constexpr (4 * m == R) {
        return cmul_i<SG>(a);
    } else if constexpr (2 * m == R) {
        return make_float2(-a.x, -a.y);
    } else if constexpr (4 * m == 3 * R) {
        return cmul_i<-SG>(a);
    } else {
        return cmul(a, make_float2(Tw<M, R, SG>::c, Tw<M, R, SG>::s));
    }
}

// ---------------------------------------------------------------------------
// register DFT codelets: v[k] <- sum_j v[j] e^{SG 2 pi i jk/R}
// ---------------------------------------------------------------------------
template <int R, int SG>
struct DFT;

template <int SG>
struct DFT<1, SG> {
    static __device__ __forceinline__ void run(float2 *) {}
};
template <int SG>
struct DFT<2, SG> {
    static __device__ __forceinline__ void run(float2 *v) {
        float2 a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    }
};
template <int SG>
struct DFT<3, SG> {
    static __device__ __forceinline__ void run(float2 *v) {
        constexpr float c = -0.5f;
        constexpr float s = (float)(SG * 0.86602540378443864676372317075294);
        float2 a = v[0], b = v[1], d = v[2];
        float2 t = cadd(b, d);
        float2 u = csub(b, d);
        float2 m = make_float2(fmaf(c, t.x, a.x), fmaf(c, t.y, a.y));
        // i*s*u
        float2 w = make_float2(-s * u.y, s * u.x);
        v[0] = cadd(a, t);
        v[1] = cadd(m, w);
        v[2] = csub(m, w);
    }
};
template <int SG>
struct DFT<4, SG> {
    static __device__ __forceinline__ void run(float2 *v) {
        float2 a0 = cadd(v[0], v[2]), a1 = csub(v[0], v[2]);
        float2 b0 = cadd(v[1], v[3]), b1 = cmul_i<SG>(csub(v[1], v[3]));
        v[0] = cadd(a0, b0);
        v[2] = csub(a0, b0);
        v[1] = cadd(a1, b1);
        v[3] = csub(a1, b1);
    }
};
template <int SG>
struct DFT<5, SG> {
    static __device__ __forceinline__ void run(float2 *v) {
        constexpr float c1 = (float)0.30901699437494742410229341718282;   // cos(2pi/5)
        constexpr float c2 = (float)-0.80901699437494742410229341718282;  // cos(4pi/5)
        constexpr float s1 = (float)(SG * 0.95105651629515357211643933337938);
        constexpr float s2 = (float)(SG * 0.58778525229247312916870595463907);
        float2 x0 = v[0];
        float2 t1 = cadd(v[1], v[4]), t2 = cadd(v[2], v[3]);
        float2 u1 = csub(v[1], v[4]), u2 = csub(v[2], v[3]);
        float2 m1 = make_float2(x0.x + c1 * t1.x + c2 * t2.x, x0.y + c1 * t1.y + c2 * t2.y);
        float2 m2 = make_float2(x0.x + c2 * t1.x + c1 * t2.x, x0.y + c2 * t1.y + c1 * t2.y);
        // i*(s1 u1 + s2 u2), i*(s2 u1 - s1 u2)
        float2 n1 = make_float2(s1 * u1.x + s2 * u2.x, s1 * u1.y + s2 * u2.y);
        float2 n2 = make_float2(s2 * u1.x - s1 * u2.x, s2 * u1.y - s1 * u2.y);
        v[0] = cadd(x0, cadd(t1, t2));
        v[1] = make_float2(m1.x - n1.y, m1.y + n1.x);
        v[4] = make_float2(m1.x + n1.y, m1.y - n1.x);
        v[2] = make_float2(m2.x - n2.y, m2.y + n2.x);
        v[3] = make_float2(m2.x + n2.y, m2.y - n2.x);
    }
};

// composite sizes: R = P*Q, six-step in registers
template <int R>
struct Split {
    static constexpr int P = (R % 4 == 0 && R > 4) ? 4 : (R % 2 == 0 ? 2 : (R % 3 == 0 ? 3 : 5));
    static constexpr int Q = R / P;
};
template <int R, int SG>
struct DFT {
    static_assert(R == 6 || R == 8 || R == 10 || R == 12 || R == 16 || R == 9 || R == 15 || R == 20 || R == 32,
                  "unsupported codelet size");
    static __device__ __forceinline__ void run(float2 *v) {
        constexpr int P = Split<R>::P, Q = Split<R>::Q;
        float2 t[R];
        sfor<0, P>([&](auto j1c) {
            constexpr int j1 = decltype(j1c)::value;
            float2 u[Q];
            sfor<0, Q>([&](auto j2c) {
                constexpr int j2 = decltype(j2c)::value;
                u[j2] = v[j1 + P * j2];
            });
            DFT<Q, SG>::run(u);
            sfor<0, Q>([&](auto k2c) {
                constexpr int k2 = decltype(k2c)::value;
                t[j1 * Q + k2] = twmul<j1 * k2, R, SG>(u[k2]);
            });
        });
        sfor<0, Q>([&](auto k2c) {
            constexpr int k2 = decltype(k2c)::value;
            float2 w[P];
            sfor<0, P>([&](auto j1c) {
                constexpr int j1 = decltype(j1c)::value;
                w[j1] = t[j1 * Q + k2];
            });
            DFT<P, SG>::run(w);
            sfor<0, P>([&](auto k1c) {
                constexpr int k1 = decltype(k1c)::value;
                v[k2 + Q * k1] = w[k1];
            });
        });
    }
};

// ---------------------------------------------------------------------------
// geometry of one N x N field in shared memory
// ---------------------------------------------------------------------------
template <int N_, int R1_, int NT_, int MINB_ = 1, bool STAGE_ = false>
struct Geo {
    static constexpr int MINB = MINB_;  // CTAs per SM the register budget is sized for
    static constexpr bool STAGE = STAGE_;  // adjoint's saved-wave rows staged by bulk copies
    static constexpr int N = N_;
    static constexpr int R1 = R1_;
    static constexpr int R2 = N_ / R1_;
    static constexpr int NT = NT_;
    static constexpr int S = N + N / R1;  // padded row stride (elements)
    static constexpr int NRA = N * R1;    // row/col pass-A tasks (R2 points each)
    static constexpr int NRB = N * R2;    // row/col pass-B tasks (R1 points each)
    static constexpr int CL = 1;          // CTAs sharing one field (thread-block cluster)
    static constexpr int ROWS = N;        // rows of the field held by one CTA
    static constexpr int FIELD = ROWS * S;
    static constexpr bool THREE = false;  // the three-phase shape (Geo3)
    static constexpr int CB = R1;         // points of a column-pass-B task
    static constexpr int RY1 = R1;        // the y dimension's factors (the x ones here)
    static_assert(R1 * R2 == N, "N must equal R1*R2");
    __device__ __forceinline__ static int px(int x) { return x + x / R1; }
    __device__ __forceinline__ static int at(int y, int x) { return y * S + px(x); }
    // scrambled location -> frequency index (both dimensions)
    __host__ __device__ __forceinline__ static int scr(int L) { return L / R1 + R2 * (L % R1); }
    __host__ __device__ __forceinline__ static int scrx(int L) { return scr(L); }
    __host__ __device__ __forceinline__ static int scry(int L) { return scr(L); }
    __device__ __forceinline__ static int rank() { return 0; }
    // row of the field held at local row l (yb = ybase(), read once per pass)
    __device__ __forceinline__ static int ybase() { return 0; }
    __device__ __forceinline__ static int gy(int, int l) { return l; }
};

// A field too large for one SM's shared memory, split by rows over a
// thread-block cluster of CL CTAs.  The column transform keeps the single-CTA
// factorisation N = R1*R2 (so the scrambled layout is the single-CTA one),
// and the rows are dealt out by their residue n1 = y mod R1: CTA r holds the
// N1C = R1/CL residues [r*N1C, (r+1)*N1C), row y = n1 + R1*j at local row
// (n1 - r*N1C)*R2 + j.  Row passes and column pass A (R2 points at rows
// n1 + R1*j, one residue) are then CTA-local; only column pass B (R1 points
// at rows j + R1*k2, one of every residue) reads and writes every CTA of the
// cluster through distributed shared memory, each task owned by one thread so
// that the pass is in place.  One distributed pass per column transform, and
// the switch between row passes and column pass A needs only a CTA barrier.
template <int N_, int R1_, int NT_, int CL_, int MINB_ = 1, bool STAGE_ = false>
struct GeoCl : Geo<N_, R1_, NT_, MINB_, STAGE_> {
    using Base = Geo<N_, R1_, NT_, MINB_, STAGE_>;
    static constexpr int CL = CL_;
    static constexpr int ROWS = N_ / CL_;
    static constexpr int N1C = R1_ / CL_;  // residues n1 per CTA
    static constexpr int FIELD = ROWS * Base::S;
    static_assert(R1_ % CL_ == 0 && Base::R2 % CL_ == 0, "column passes must split over the cluster");
    static_assert(N1C * Base::R2 == ROWS, "every CTA holds N1C whole residues");
    __device__ __forceinline__ static int rank() {
        unsigned r;
        asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
        return (int)r;
    }
    __device__ __forceinline__ static int ybase() { return rank() * N1C; }
    __device__ __forceinline__ static int gy(int yb, int l) { return yb + l / Base::R2 + R1_ * (l % Base::R2); }
};

// Three-phase shape of a 128 x 128 field (one CTA of 512 threads).  The
// two-pass shape above costs six shared-memory round trips per propagation
// slab.  Here a 2D transform is three register phases of 16 or 32 points:
//
//   phase 1 (rows)  task (y, n1):  x = n1 + 8 j, j < 16        DFT16 over j
//   phase 2         task (k1, b):  x = a + 8 k1, a < 8         twiddle W^(a k1), DFT8 over a
//                                  y = b + 32 m, m < 4         DFT4 over m, twiddle W^(b k1')
//   phase 3 (cols)  task (x, k1'): y = b + 32 k1', b < 32      DFT32 over b
//
// (natural -> scrambled; the way back runs the phases in reverse with the
// twiddles on the other side of each DFT).  Location Lx = k2 + 8 k1 then
// holds frequency k1 + 16 k2 and Ly = k2' + 32 k1' frequency k1' + 4 k2'.
// The phases bordering a pointwise stage are fused as in the two-pass shape
// (phase 1 = inverse rows + op + forward rows, phase 3 = forward columns + op
// + inverse columns), so a slab costs four round trips.  Warp w's phase-1
// rows {2w, 2w+1} + 32 m are the rows of its phase-2 tasks: phases 1 and 2
// meet at a warp barrier, phases 2 and 3 at a CTA barrier.  Rows are padded
// after every 8 elements and to a stride of 8 mod 16 elements, under which
// the accesses of all three phases are free of bank conflicts with constant
// offsets from one base address per task.  WIDE: two pad elements per 8 (row
// stride 168), so that phase 2 moves its 8 consecutive x values as four
// 16-byte accesses (half the shared-memory instructions of that phase); one
// pad element per 8 (stride 152) otherwise.
template <int MINB_ = 1, bool WIDE_ = false>
struct Geo3 {
    static constexpr bool THREE = true;
    static constexpr bool WIDE = WIDE_;
    static constexpr int MINB = MINB_;
    static constexpr bool STAGE = false;
    static constexpr int N = 128;
    static constexpr int R1 = 8, R2 = 16;   // x: phase-1 task (y, n1) holds x = n1 + R1 j, j < R2
    static constexpr int RY1 = 32, RY2 = 4;  // y: phase 2 radix RY2 at stride RY1, phase 3 radix RY1
    static constexpr int CB = RY1;           // points of a column (phase-3) task
    static constexpr int NT = 512;
    static constexpr int PADX = WIDE_ ? 2 : 1;   // pad elements after every R1
    static constexpr int GS = R1 + PADX;         // stride of x = n1 + R1 j over j
    static constexpr int S = N + PADX * (N / R1) + 8;  // 152 or 168
    static constexpr int CL = 1;
    static constexpr int ROWS = N;
    static constexpr int FIELD = ROWS * S;
    static_assert(S % 16 == 8, "rows 2w and 2w+1 must fall on opposite bank halves");
    __device__ __forceinline__ static int px(int x) { return x + PADX * (x / R1); }
    __device__ __forceinline__ static int at(int y, int x) { return y * S + px(x); }
    __host__ __device__ __forceinline__ static int scrx(int L) { return L / R1 + R2 * (L % R1); }
    __host__ __device__ __forceinline__ static int scry(int L) { return L / RY1 + RY2 * (L % RY1); }
    __device__ __forceinline__ static int rank() { return 0; }
    __device__ __forceinline__ static int ybase() { return 0; }
    __device__ __forceinline__ static int gy(int, int l) { return l; }
};

// twiddle W_N^{n1 k2} with sign (table holds e^{-2 pi i m/N} as [k2][n1])
template <class G, int SG>
__device__ __forceinline__ float2 twN(const float2 *tw, int n1, int k2) {
    float2 w = tw[k2 * G::R1 + n1];
    return SG < 0 ? w : cconj(w);
}

// Work ownership.  Row passes: warp w owns rows [w*RPW, (w+1)*RPW), so the
// two row passes of a transform only need __syncwarp between them.  Column
// passes: warp pair q owns columns [q*CPP, (q+1)*CPP), a named barrier of the
// pair separates them.  Only a switch between row and column passes needs
// the CTA-wide barrier; warps drift apart inside each phase, so one warp's
// global-memory latency overlaps another warp's arithmetic.
template <class G>
struct Own {
    static constexpr int W = G::NT / 32;           // warps
    static constexpr int RPW = G::ROWS / W;         // rows per warp
    static constexpr int CPP = 2 * G::N / W;        // columns per warp pair
    static_assert(G::NT % 64 == 0, "NT must be a multiple of 64");
    static_assert(G::ROWS % W == 0 && (2 * G::N) % W == 0, "rows must split evenly over warps");
    __device__ __forceinline__ static int warp() { return threadIdx.x >> 5; }
    __device__ __forceinline__ static int lane() { return threadIdx.x & 31; }
    __device__ __forceinline__ static int pair() { return threadIdx.x >> 6; }
    __device__ __forceinline__ static int plane() { return threadIdx.x & 63; }
};

__device__ __forceinline__ void sync_rows() { __syncwarp(); }
// barrier of every thread of the cluster, with release / acquire of the
// shared-memory (local and distributed) and global writes before it
__device__ __forceinline__ void cluster_sync() {
    asm volatile("barrier.cluster.arrive.release;\n\tbarrier.cluster.wait.acquire;" ::: "memory");
}
// between column pass A and column pass B
template <class G>
__device__ __forceinline__ void sync_cols() {
    if constexpr (G::CL > 1) {
        // column pass B touches rows of other CTAs
        cluster_sync();
    } else if constexpr (G::THREE) {
        // phase 2 and phase 3 tasks share no rows or columns
        __syncthreads();
    } else {
        // named barrier per warp pair (ids 1..15; 0 is __syncthreads)
        asm volatile("bar.sync %0, 64;" ::"r"(1 + Own<G>::pair()) : "memory");
    }
}
// switch between row passes and column pass A: CTA-local in both geometries
__device__ __forceinline__ void sync_rowcol() { __syncthreads(); }
// every thread of the field (the cluster when it is split)
template <class G>
__device__ __forceinline__ void sync_all() {
    if constexpr (G::CL > 1) cluster_sync();
    else __syncthreads();
}
__device__ __forceinline__ void sync_all() { __syncthreads(); }

// the same shared-memory offset in CTA r of the cluster (generic address)
template <class T>
__device__ __forceinline__ T *peer(T *p, int r) {
    return cooperative_groups::this_cluster().map_shared_rank(p, (unsigned)r);
}
// shared::cluster window address of a local shared-memory pointer in CTA r
__device__ __forceinline__ uint32_t peer_addr(const void *p, int r) {
    const uint32_t a = (uint32_t)__cvta_generic_to_shared(p);
    uint32_t out;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(out) : "r"(a), "r"(r));
    return out;
}
__device__ __forceinline__ float2 ld_cluster(uint32_t addr) {
    float2 v;
    asm volatile("ld.shared::cluster.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "r"(addr));
    return v;
}
__device__ __forceinline__ void st_cluster(uint32_t addr, float2 v) {
    asm volatile("st.shared::cluster.v2.f32 [%0], {%1, %2};" ::"r"(addr), "f"(v.x), "f"(v.y) : "memory");
}

struct NoPre {
    static constexpr bool kAhead = false;
};

// Row pass A.  Task (y, n1) owns x = n1 + R1*j, j < R2.
//   pf(y, n1, pre) : issue the global loads the op needs (before the shared
//                    memory reads, so their latency overlaps them)
//   IN  != 0 : finish a scrambled->natural transform of sign IN
//   op(y, n1, v, pre) : pointwise stage on natural-order real-space values
//   OUT != 0 : start a natural->scrambled transform of sign OUT
struct NoL1 {
    static constexpr int kLines = 0;
    __device__ __forceinline__ void operator()(int, int) const {}
};

// No operand staged in shared memory (see RowStage in mset_kernels_impl.cuh):
// the op takes (y, n1, v, pre).
struct NoStage {
    static constexpr bool kOn = false;
    __device__ __forceinline__ void wait(int) const {}
    __device__ __forceinline__ void refill(int) const {}
    __device__ __forceinline__ const float2 *task(int, int) const { return nullptr; }
};

// Phase 1 of the three-phase shape (Geo3): row pass A without twiddles (they
// belong to phase 2).  Lane l of warp w takes n1 = l % 8 and the rows
// 2w + (l / 8) % 2 + 32 (l / 16) and 64 below it; the callbacks are row pass
// A's.
template <class G, int IN, int OUT, class Pre, class Pf, class Op, class L1, class ST>
__device__ __forceinline__ void rows3(float2 *buf, Pf &&pf, Op &&op, const L1 &, const ST &) {
    static_assert(!ST::kOn && std::decay_t<L1>::kLines == 0, "no staged operands or L1 hints in phase 1");
    constexpr int R1 = G::R1, R2 = G::R2;
    const int lane = threadIdx.x & 31;
    const int n1 = lane % R1;
    const int y0 = 2 * (threadIdx.x >> 5) + ((lane >> 3) & 1) + 32 * (lane >> 4);
    constexpr bool ahead = Pre::kAhead;
    Pre pre, nxt;
    if constexpr (ahead) pf(y0, n1, pre);
#pragma unroll 1
    for (int it = 0; it < 2; ++it) {
        const int y = y0 + 64 * it;
        if constexpr (ahead) {
            if (it == 0) pf(y0 + 64, n1, nxt);
        } else {
            pf(y, n1, pre);
        }
        float2 *row = buf + y * G::S + n1;
        float2 v[R2];
#pragma unroll
        for (int j = 0; j < R2; ++j) v[j] = row[G::GS * j];
        if constexpr (IN != 0) DFT<R2, IN>::run(v);
        op(y, n1, v, pre);
        if constexpr (OUT != 0) DFT<R2, OUT>::run(v);
#pragma unroll
        for (int j = 0; j < R2; ++j) row[G::GS * j] = v[j];
        if constexpr (ahead) pre = nxt;
    }
}

template <class G, int IN, int OUT, class Pre, class Pf, class Op, class L1 = NoL1, class ST = NoStage>
__device__ __forceinline__ void row_passA_pf(float2 *buf, const float2 *tw, Pf &&pf, Op &&op, L1 &&l1 = NoL1{},
                                             const ST &st = ST{}) {
    if constexpr (G::THREE) {
        rows3<G, IN, OUT, Pre>(buf, pf, op, l1, st);
        (void)tw;
    } else {
        using O = Own<G>;
        constexpr int R1 = G::R1, R2 = G::R2;
        constexpr int TASKS = O::RPW * R1;
        static_assert(!ST::kOn || TASKS % 32 == 0, "a staged operand needs whole warp iterations");
        const int yl0 = O::warp() * O::RPW;  // first local row of the warp
        const int yb = G::ybase();           // local row -> row of the field (pf / op)
        // Pre::kAhead: issue the next task's global loads while the current task
        // runs (double-buffered prefetch); otherwise just before its shared reads
        constexpr bool ahead = Pre::kAhead;
        Pre pre, nxt;
        if (ahead && O::lane() < TASKS) pf(G::gy(yb, yl0 + O::lane() / R1), O::lane() % R1, pre);
        // a lane's residue n1 is the same in every task when R1 divides 32, so
        // its twiddles W^(n1 k2) stay in registers for the whole pass instead of
        // being read from shared memory twice per task (while R2 <= 8 leaves
        // room for them)
        constexpr bool kTwReg = (32 % R1 == 0) && R2 <= 8 && (IN != 0 || OUT != 0);
        float2 twr[kTwReg ? R2 : 1];
        if constexpr (kTwReg) {
#pragma unroll
            for (int k2 = 1; k2 < R2; ++k2) twr[k2] = tw[k2 * R1 + O::lane() % R1];
        }
#pragma unroll 1
        for (int tau = O::lane(); tau < TASKS; tau += 32) {
            const int n1 = tau % R1, y = G::gy(yb, yl0 + tau / R1);
            if constexpr (std::decay_t<L1>::kLines > 0) {
                // pull the next iteration's rows of the op's global operands into
                // L1 (hints: no registers, no scoreboard)
                constexpr int LN = std::decay_t<L1>::kLines, RI = 32 / R1;
                const int r0 = yl0 + (tau - O::lane() + 32) / R1;
                if (r0 < yl0 + O::RPW)
                    for (int q = O::lane(); q < RI * LN; q += 32) l1(G::gy(yb, r0 + q / LN), q % LN);
            }
            if constexpr (ahead) {
                if (tau + 32 < TASKS) pf(G::gy(yb, yl0 + (tau + 32) / R1), (tau + 32) % R1, nxt);
            } else {
                pf(y, n1, pre);
            }
            float2 *row = buf + (yl0 + tau / R1) * G::S + n1;
            float2 v[R2];
#pragma unroll
            for (int j = 0; j < R2; ++j) v[j] = row[(R1 + 1) * j];
            auto twi = [&](int k2, auto sg) -> float2 {
                constexpr int SG = decltype(sg)::value;
                if constexpr (kTwReg) return SG < 0 ? twr[k2] : cconj(twr[k2]);
                else return twN<G, SG>(tw, n1, k2);
            };
            if constexpr (IN != 0) {
#pragma unroll
                for (int k2 = 1; k2 < R2; ++k2) v[k2] = cmul(v[k2], twi(k2, std::integral_constant<int, IN>{}));
                DFT<R2, IN>::run(v);
            }
            if constexpr (ST::kOn) {
                // the staged operand rows of this warp iteration: wait for their
                // bulk copy, hand the task its row, refill the stage afterwards
                const int it = (tau - O::lane()) >> 5;
                st.wait(it);
                op(y, n1, v, pre, st.task(it, O::lane()));
                st.refill(it);
            } else {
                op(y, n1, v, pre);
            }
            if constexpr (OUT != 0) {
                DFT<R2, OUT>::run(v);
#pragma unroll
                for (int k2 = 1; k2 < R2; ++k2) v[k2] = cmul(v[k2], twi(k2, std::integral_constant<int, OUT>{}));
            }
#pragma unroll
            for (int j = 0; j < R2; ++j) row[(R1 + 1) * j] = v[j];
            if constexpr (ahead) pre = nxt;
        }
    }
}

// L1 prefetch of the rows the warp's first row-pass-A iteration will read
// (issued a pass or two ahead of it; the later iterations are covered one
// iteration ahead inside row_passA_pf)
template <class G, class L1>
__device__ __forceinline__ void l1_first(const L1 &l1) {
    using O = Own<G>;
    constexpr int LN = L1::kLines;
    if constexpr (LN > 0 && 32 % G::R1 == 0) {
        constexpr int RI = 32 / G::R1;
        const int yl0 = O::warp() * O::RPW, yb = G::ybase();
        for (int q = O::lane(); q < RI * LN; q += 32) l1(G::gy(yb, yl0 + q / LN), q % LN);
    }
}

template <class G, int IN, int OUT, class Op>
__device__ __forceinline__ void row_passA(float2 *buf, const float2 *tw, Op &&op) {
    row_passA_pf<G, IN, OUT, NoPre>(
        buf, tw, [](int, int, NoPre &) {}, [&](int y, int n1, float2 *v, const NoPre &) { op(y, n1, v); });
}

// Row pass B.  Task (y, k2) owns x = j + R1*k2, j < R1.
template <class G, int SG>
__device__ __forceinline__ void row_passB(float2 *buf) {
    using O = Own<G>;
    constexpr int R1 = G::R1, R2 = G::R2;
    constexpr int TASKS = O::RPW * R2;
    const int y0 = O::warp() * O::RPW;
#pragma unroll 1
    for (int tau = O::lane(); tau < TASKS; tau += 32) {
        const int k2 = tau % R2, y = y0 + tau / R2;
        float2 *p = buf + y * G::S + (R1 + 1) * k2;
        float2 v[R1];
#pragma unroll
        for (int j = 0; j < R1; ++j) v[j] = p[j];
        DFT<R1, SG>::run(v);
#pragma unroll
        for (int j = 0; j < R1; ++j) p[j] = v[j];
    }
}

// the R2 twiddles W^(n1 k2) of residue n1 (sign SG): from the transposed
// table twt[n1][k2] two at a time when TT (R2 even), else from tw[k2][n1]
template <class G, int SG, bool TT>
__device__ __forceinline__ void col_twiddles(const float2 *tw, int n1, float2 *w) {
    constexpr int R1 = G::R1, R2 = G::R2;
    if constexpr (TT) {
        const float4 *t4 = reinterpret_cast<const float4 *>(tw + G::N + n1 * R2);
#pragma unroll
        for (int m = 0; m < R2 / 2; ++m) {
            const float4 q = t4[m];
            w[2 * m] = make_float2(q.x, q.y);
            w[2 * m + 1] = make_float2(q.z, q.w);
        }
        if constexpr (SG > 0) {
#pragma unroll
            for (int k2 = 0; k2 < R2; ++k2) w[k2] = cconj(w[k2]);
        }
    } else {
#pragma unroll
        for (int k2 = 1; k2 < R2; ++k2) w[k2] = twN<G, SG>(tw, n1, k2);
    }
    (void)R1;
}

// Column pass A.  Task (x, n1) owns rows y = n1 + R1*j.
//   FWD: natural->scrambled step (DFT then twiddle); else scrambled->natural
//   TT: the transposed twiddle table follows tw (tw + N, [n1][k2])
template <class G, int SG, bool FWD, bool TT = false>
__device__ __forceinline__ void col_passA(float2 *buf, const float2 *tw) {
    using O = Own<G>;
    constexpr int R1 = G::R1, R2 = G::R2;
    if constexpr (G::CL > 1) {
        // CTA-local: task (x, n1) of a residue n1 this CTA holds, element j
        // at local row (n1 - rank*N1C)*R2 + j
        constexpr int TASKS = G::N1C * G::N;
        const int n1b = G::rank() * G::N1C;
#pragma unroll 1
        for (int tau = threadIdx.x; tau < TASKS; tau += G::NT) {
            const int x = tau % G::N, n1l = tau / G::N, n1 = n1b + n1l;
            float2 *p = buf + n1l * R2 * G::S + G::px(x);
            float2 v[R2];
#pragma unroll
            for (int j = 0; j < R2; ++j) v[j] = p[G::S * j];
            float2 w[R2];
            col_twiddles<G, SG, TT>(tw, n1, w);
            if constexpr (FWD) {
                DFT<R2, SG>::run(v);
#pragma unroll
                for (int k2 = 1; k2 < R2; ++k2) v[k2] = cmul(v[k2], w[k2]);
            } else {
#pragma unroll
                for (int k2 = 1; k2 < R2; ++k2) v[k2] = cmul(v[k2], w[k2]);
                DFT<R2, SG>::run(v);
            }
#pragma unroll
            for (int j = 0; j < R2; ++j) p[G::S * j] = v[j];
        }
        return;
    }
    constexpr int TASKS = O::CPP * R1;
    const int x0 = O::pair() * O::CPP;
#pragma unroll 1
    for (int tau = O::plane(); tau < TASKS; tau += 64) {
        const int x = x0 + tau % O::CPP, n1 = tau / O::CPP;
        float2 *p = buf + n1 * G::S + G::px(x);
        float2 v[R2];
#pragma unroll
        for (int j = 0; j < R2; ++j) v[j] = p[R1 * G::S * j];
        float2 w[R2];
        col_twiddles<G, SG, TT>(tw, n1, w);
        if constexpr (FWD) {
            DFT<R2, SG>::run(v);
#pragma unroll
            for (int k2 = 1; k2 < R2; ++k2) v[k2] = cmul(v[k2], w[k2]);
        } else {
#pragma unroll
            for (int k2 = 1; k2 < R2; ++k2) v[k2] = cmul(v[k2], w[k2]);
            DFT<R2, SG>::run(v);
        }
#pragma unroll
        for (int j = 0; j < R2; ++j) p[R1 * G::S * j] = v[j];
    }
}

// Column pass B.  Task (x, k2) owns rows Ly = j + R1*k2 (scrambled).
//   IN  != 0 : finish natural->scrambled (sign IN)
//   op(Ly0, x, v) : pointwise stage on scrambled spectrum, element j at row Ly0 + j
//   OUT != 0 : start scrambled->natural (sign OUT)
template <class G, int IN, int OUT, class Op>
__device__ __forceinline__ void col_passB(float2 *buf, Op &&op) {
    using O = Own<G>;
    constexpr int R1 = G::R1, R2 = G::R2;
    if constexpr (G::THREE) {
        // phase 3: half-warp h of warp w takes the pair q = 2w + h, rows
        // 32 (q / 8) + b and the column groups c and c + D (columns 8 c + i,
        // i < 8) that fall on opposite bank halves: D = 8 with one pad
        // element per 8 columns (9 D = 8 mod 16), D = 4 with two (10 D = 8)
        const int lane = threadIdx.x & 31;
        const int q = 2 * (threadIdx.x >> 5) + (lane >> 4), g = q & 7;
        constexpr int D = G::PADX == 1 ? 8 : 4;
        static_assert((G::GS * D) % 16 == 8, "the two column groups of a half-warp share no bank");
        const int c = D == 8 ? g : (g & 3) + 8 * (g >> 2);
        const int x = 8 * c + (lane & 7) + 8 * D * ((lane >> 3) & 1);
        const int y0 = G::RY1 * (q >> 3);
        float2 *p = buf + y0 * G::S + G::px(x);
        float2 v[G::CB];
#pragma unroll
        for (int j = 0; j < G::CB; ++j) v[j] = p[G::S * j];
        if constexpr (IN != 0) DFT<G::CB, IN>::run(v);
        op(y0, x, v);
        if constexpr (OUT != 0) DFT<G::CB, OUT>::run(v);
#pragma unroll
        for (int j = 0; j < G::CB; ++j) p[G::S * j] = v[j];
    } else if constexpr (G::CL > 1) {
        // distributed: CTA r owns the tasks k2 in [r*K2C, (r+1)*K2C) of every
        // column; element j (row j + R1*k2, residue j) lives in CTA j / N1C at
        // local row (j % N1C)*R2 + k2
        constexpr int K2C = R2 / G::CL;
        constexpr int TASKS = K2C * G::N;
        uint32_t pb[G::CL];  // shared::cluster addresses of the CTAs' fields
#pragma unroll
        for (int r = 0; r < G::CL; ++r) pb[r] = peer_addr(buf, r);
        const int k2b = G::rank() * K2C;
        constexpr uint32_t kRes = sizeof(float2) * R2 * G::S;  // bytes between residues of one CTA
#pragma unroll 1
        for (int tau = threadIdx.x; tau < TASKS; tau += G::NT) {
            const int x = tau % G::N, k2 = k2b + tau / G::N;
            const int y0 = R1 * k2;
            const uint32_t off = sizeof(float2) * (uint32_t)(k2 * G::S + G::px(x));
            float2 v[R1];
#pragma unroll
            for (int j = 0; j < R1; ++j) v[j] = ld_cluster(pb[j / G::N1C] + off + kRes * (j % G::N1C));
            if constexpr (IN != 0) DFT<R1, IN>::run(v);
            op(y0, x, v);
            if constexpr (OUT != 0) DFT<R1, OUT>::run(v);
#pragma unroll
            for (int j = 0; j < R1; ++j) st_cluster(pb[j / G::N1C] + off + kRes * (j % G::N1C), v[j]);
        }
    } else {
        constexpr int TASKS = O::CPP * R2;
        const int x0 = O::pair() * O::CPP;
#pragma unroll 1
        for (int tau = O::plane(); tau < TASKS; tau += 64) {
            const int x = x0 + tau % O::CPP, k2 = tau / O::CPP;
            const int y0 = R1 * k2;
            float2 *p = buf + y0 * G::S + G::px(x);
            float2 v[R1];
#pragma unroll
            for (int j = 0; j < R1; ++j) v[j] = p[G::S * j];
            if constexpr (IN != 0) DFT<R1, IN>::run(v);
            op(y0, x, v);
            if constexpr (OUT != 0) DFT<R1, OUT>::run(v);
#pragma unroll
            for (int j = 0; j < R1; ++j) p[G::S * j] = v[j];
        }
    }
}

// Phase 2 of the three-phase shape: lane l of warp w takes k1 = l % 16 and
// b = 2w + l / 16, element (a, m) at x = a + 8 k1, y = b + 32 m.  FWD: the
// natural -> scrambled step; else scrambled -> natural.  The twiddle tables
// are tw[16 a + k1] = W^(a k1) and tw[N + 32 k1' + b] = W^(b k1') (sign -1).
template <class G, int SG, bool FWD>
__device__ __forceinline__ void mid3(float2 *buf, const float2 *tw) {
    constexpr int RX = G::R1, RY = G::RY2, KX = G::R2;  // 8-point x DFTs, 4-point y DFTs, 16 k1
    const int lane = threadIdx.x & 31;
    const int k1 = lane % KX, b = 2 * (threadIdx.x >> 5) + lane / KX;
    float2 *p = buf + b * G::S + G::GS * k1;
    float2 v[RX * RY];  // v[a + 8 m]
    if constexpr (G::WIDE) {
        // 16-byte pairs (p is 16-byte aligned: S and GS are even)
#pragma unroll
        for (int m = 0; m < RY; ++m)
#pragma unroll
            for (int a = 0; a < RX; a += 2) {
                const float4 t = *reinterpret_cast<const float4 *>(p + G::RY1 * G::S * m + a);
                v[a + RX * m] = make_float2(t.x, t.y);
                v[a + 1 + RX * m] = make_float2(t.z, t.w);
            }
    } else {
#pragma unroll
        for (int m = 0; m < RY; ++m)
#pragma unroll
            for (int a = 0; a < RX; ++a) v[a + RX * m] = p[G::RY1 * G::S * m + a];
    }
    const float2 *twx = tw + k1;
    const float2 *twy = tw + G::N + b;
    auto wx = [&](int a) { const float2 t = twx[KX * a]; return SG < 0 ? t : cconj(t); };
    auto wy = [&](int k) { const float2 t = twy[G::RY1 * k]; return SG < 0 ? t : cconj(t); };
    auto xdft = [&]() {
#pragma unroll
        for (int m = 0; m < RY; ++m) DFT<RX, SG>::run(v + RX * m);
    };
    auto ydft = [&]() {
#pragma unroll
        for (int a = 0; a < RX; ++a) {
            float2 u[RY];
#pragma unroll
            for (int m = 0; m < RY; ++m) u[m] = v[a + RX * m];
            DFT<RY, SG>::run(u);
#pragma unroll
            for (int m = 0; m < RY; ++m) v[a + RX * m] = u[m];
        }
    };
    auto xtw = [&]() {
#pragma unroll
        for (int a = 1; a < RX; ++a) {
            const float2 t = wx(a);
#pragma unroll
            for (int m = 0; m < RY; ++m) v[a + RX * m] = cmul(v[a + RX * m], t);
        }
    };
    auto ytw = [&]() {
#pragma unroll
        for (int k = 1; k < RY; ++k) {
            const float2 t = wy(k);
#pragma unroll
            for (int a = 0; a < RX; ++a) v[a + RX * k] = cmul(v[a + RX * k], t);
        }
    };
    if constexpr (FWD) {
        xtw();
        xdft();
        ydft();
        ytw();
    } else {
        ytw();
        ydft();
        xdft();
        xtw();
    }
    if constexpr (G::WIDE) {
#pragma unroll
        for (int m = 0; m < RY; ++m)
#pragma unroll
            for (int a = 0; a < RX; a += 2)
                *reinterpret_cast<float4 *>(p + G::RY1 * G::S * m + a) =
                    make_float4(v[a + RX * m].x, v[a + RX * m].y, v[a + 1 + RX * m].x, v[a + 1 + RX * m].y);
    } else {
#pragma unroll
        for (int m = 0; m < RY; ++m)
#pragma unroll
            for (int a = 0; a < RX; ++a) p[G::RY1 * G::S * m + a] = v[a + RX * m];
    }
}

// The steps between the row-side pass A and column pass B of a transform:
// natural -> scrambled (mid_fwd: row pass B, column pass A) and back
// (mid_inv), sign SG.  TT: column pass A reads the transposed twiddle table.
template <class G, int SG, bool TT>
__device__ __forceinline__ void mid_fwd(float2 *buf, const float2 *tw) {
    if constexpr (G::THREE) {
        mid3<G, SG, true>(buf, tw);
    } else {
        row_passB<G, SG>(buf);
        sync_rowcol();
        col_passA<G, SG, true, TT>(buf, tw);
    }
}
template <class G, int SG, bool TT>
__device__ __forceinline__ void mid_inv(float2 *buf, const float2 *tw) {
    if constexpr (G::THREE) {
        mid3<G, SG, false>(buf, tw);
    } else {
        col_passA<G, SG, false, TT>(buf, tw);
        sync_rowcol();
        row_passB<G, SG>(buf);
    }
}

struct NoOp {
    template <class... A>
    __device__ __forceinline__ void operator()(A &&...) const {}
};

}  // namespace mset
