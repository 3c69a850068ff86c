// mset_kernels_impl.cuh -- fused per-position multislice forward / adjoint kernels
// for sm_100a.
//
// One CTA owns one probe position at a time; the wave stays in shared memory
// for the whole forward pass, far field and adjoint.  Per slab it costs six
// shared-memory passes forward and six backward (see fft_core.cuh), with the
// transmission exp(i sigma dz sum V), the propagator product, the saved-wave
// store, the gradient product and the far-field residual fused into the
// passes that border them.
//
// Reference semantics (kSeq) follow src/CUDA/mset.cu:80-334 (MSET) and
// :345-546 (SSET): volume, probe and scan position are updated after every
// position, inside the same launch.  kBatch keeps the state fixed and
// accumulates the gradients of every position of every tilt in FP64
// (the batched method).  kErr is run_error_mset/_sset (mset.cu:557-810).
#pragma once
#include <cuda_bf16.h>
#include <utility>
#include "fft_core.cuh"
#include "mset_kernels.cuh"

namespace mset {

// pi as hard-coded in the reference's Fourier shift factor (utility.cu:790)
#define MSET_REF_PI 3.1415926f

template <int NT>
__device__ __forceinline__ void block_sum2(double &a, double &b, double *red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) {
        red[2 * w] = a;
        red[2 * w + 1] = b;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double sa = 0, sb = 0;
        for (int i = 0; i < (NT + 31) / 32; ++i) {
            sa += red[2 * i];
            sb += red[2 * i + 1];
        }
        red[0] = sa;
        red[1] = sb;
    }
    __syncthreads();
    a = red[0];
    b = red[1];
    __syncthreads();
}

// frequency index n(k) of the reference shift factor grid: location k of the
// ifftshifted grid carries n = ((k - ceil(N/2)) mod N) - N/2
// (utility.cu:786-787 followed by circular_shift2D_dev by ceil(N/2)).
__device__ __forceinline__ float shift_grid(int k, int n) {
    const int h = (n + 1) / 2;
    int i = k - h;
    if (i < 0) i += n;
    return (float)i - (float)n * 0.5f;
}

// Bulk prefetch of `bytes` (multiple of 16) starting at a 16-byte aligned
// global address into L2, split over the first threads of the CTA
// (cp.async.bulk.prefetch.L2, no shared memory or registers involved).
__device__ __forceinline__ void prefetch_l2(const void *p, unsigned bytes) {
    constexpr unsigned kChunk = 16384;
    const unsigned nchunk = (bytes + kChunk - 1) / kChunk;
    for (unsigned c = threadIdx.x; c < nchunk; c += blockDim.x) {
        const unsigned off = c * kChunk;
        const unsigned len = min(kChunk, bytes - off);
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"((const char *)p + off), "r"(len)
                     : "memory");
    }
}

template <class G>
struct TPre {
    // double buffer only while the register budget allows it (R2 <= 8)
    static constexpr bool kAhead = G::R2 <= 8;
    float2 t[G::R2];  // transmission of the task's elements
};
template <class G>
struct T1Pre {
    static constexpr bool kAhead = false;  // loaded just before the task's shared-memory reads
    float2 t[G::R2];
};
template <class G>
struct TSPre {
    static constexpr bool kAhead = false;  // two operands: no room for a second buffer
    float2 t[G::R2];  // transmission
    float2 w[G::R2];  // saved wave
};

// L1 prefetch of row y of a row pass A's global operands (transmission slab
// T, then the adjoint's saved wave W), 128-byte line k, issued one task
// iteration ahead by row_passA_pf.  Only as many operands as the L1 left
// beside the shared memory holds with the rows in flight of every CTA on an
// SM (measured): both operands up to 64 KB in flight (n = 128: +1% per mid
// pass), the transmission alone up to 56 KB (n = 160: +2.4%, in the adjoint
// and in the single-buffered forward); none at n = 256 (64 KB per operand:
// -0.4% with the transmission, -3% with both).
template <class G, bool FWD = false, bool TONLY = false>
struct L1Rows {
    static constexpr int kRow = (int)sizeof(float2) * G::N, kLPR = (kRow + 127) / 128;
    static constexpr long kPerOperand = (long)(G::NT / 32) * (32 / G::R1) * kRow * G::MINB;
    static constexpr bool kFits1 = 32 % G::R1 == 0 && kPerOperand <= 56 * 1024;
    // forward: the transmission alone, where registers hold no second buffer;
    // TONLY: the adjoint's transmission alone (its saved wave is staged in
    // shared memory by bulk copies)
    static constexpr int kOperands = FWD ? (!TPre<G>::kAhead && kFits1 ? 1 : 0)
                                   : TONLY ? (kFits1 ? 1 : 0)
                                           : (32 % G::R1 != 0 ? 0 : 2 * kPerOperand <= 65536 ? 2 : kFits1 ? 1 : 0);
    static constexpr int kLines = kOperands * kLPR;
    const char *T, *W;
    __device__ __forceinline__ void operator()(int y, int k) const {
        const char *base = k < kLPR ? T : W;
        if (!base) return;
        const int off = min((k < kLPR ? k : k - kLPR) * 128, kRow - (int)sizeof(float2));
        asm volatile("prefetch.global.L1 [%0];" ::"l"(base + (size_t)y * kRow + off));
    }
};

// the transmission rows of a forward row pass A's first iteration, pulled
// into L1 at the top of the slab (l1_first) where they fit 56 KB per SM:
// -0.9% per mid pass, -1.3% at 160^2, neutral at 256^2 (64 KB, off)
template <class G>
struct L1FirstT {
    static constexpr int kRow = (int)sizeof(float2) * G::N, kLPR = (kRow + 127) / 128;
    static constexpr long kInFlight = (long)(G::NT / 32) * (32 / G::R1) * kRow * G::MINB;
    static constexpr int kLines = kInFlight <= 56 * 1024 ? kLPR : 0;
    const char *T;
    __device__ __forceinline__ void operator()(int y, int k) const {
        if (!T) return;
        asm volatile("prefetch.global.L1 [%0];" ::"l"(T + (size_t)y * kRow + min(k * 128, kRow - (int)sizeof(float2))));
    }
};

// Staging of the adjoint's saved-wave rows in shared memory by bulk copies
// of the TMA engine (cp.async.bulk global -> shared, completion counted on an
// mbarrier).  Row pass A of a slab's adjoint reads, per warp iteration, kRows
// whole rows of the wave saved in the forward; each warp owns two stages of
// kRows rows.  The first two iterations' rows are requested at the top of the
// slab, two passes before they are read; iteration it + 2's rows as soon as
// iteration it has read its stage.  The rows then cost a shared-memory load
// instead of a global load held in registers across the task.  In the
// geometries compiled with STAGE: the 256 x 256 cluster default (one bulk
// copy per row, a CTA's consecutive local rows being 16 field rows apart),
// where it removes most register spills (1.443 s against 1.474 s per pass of
// 3 large tilts).  On the 128 x 128 two-pass shape it traded the global-load
// waits for shared-memory queueing and was not faster (228.2 ms against
// 225.6 ms per mid pass), so that window has no staged shape.
template <class G>
struct StageCfg {
    static constexpr int kRows = 32 % G::R1 == 0 ? 32 / G::R1 : 1;  // rows of one warp iteration
    static constexpr int kIters = Own<G>::RPW * G::R1 / 32;          // warp iterations per row pass
    static constexpr unsigned kRowBytes = (unsigned)(G::N * sizeof(float2));
    static constexpr unsigned kBytes = kRows * kRowBytes;
    static constexpr int kWarps = G::NT / 32;
    // two stages per warp where they fit beside the field and its tables
    // (227 KB per CTA), else one
    static constexpr long kBase = (long)sizeof(float2) * (G::FIELD + 6 * G::N) + 4096;
    static constexpr int kStages = kBase + 2L * kBytes * kWarps <= 227L * 1024 ? 2 : 1;
    static constexpr bool kOn = G::STAGE && 32 % G::R1 == 0 && Own<G>::RPW % kRows == 0 && kIters >= kStages &&
                                kIters % kStages == 0 && kBase + (long)kStages * kBytes * kWarps <= 227L * 1024;
    static constexpr int kStageF2 = kOn ? kStages * kRows * G::N * kWarps : 0;  // stages, float2 units
    static constexpr int kBarF2 = kOn ? kStages * kWarps : 0;                    // one mbarrier (8 B) per stage
};

// bounded wait on an mbarrier phase: false if it did not complete within
// ~4M polls (with back-off), which no bulk copy of a few KB can take
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    for (int i = 0; i < (1 << 22); ++i) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(bar), "r"(parity)
            : "memory");
        if (ok) return true;
        if (i > 64) __nanosleep(64);
    }
    return false;
}

template <class G>
struct RowStage {
    using C = StageCfg<G>;
    static constexpr bool kOn = true;
    static constexpr int S = C::kStages;
    float2 *base;        // this warp's stages [S][kRows][N]
    uint32_t bar;        // shared address of this warp's S mbarriers
    const float2 *src;   // the operand [N][N] in global memory
    int yl0;             // first local row of the warp
    int yb;              // G::ybase() (field rows of a cluster-split CTA)
    unsigned phase;      // completions of each stage's mbarrier before this pass
    unsigned *fault;     // set when a wait gave up (may be null)

    // request the rows of warp iteration it (lane 0; the stage is free):
    // one bulk copy of the contiguous rows, or one per row when the field is
    // split over a cluster (a CTA's consecutive local rows are R1 rows apart)
    __device__ __forceinline__ void issue(int it) const {
        const uint32_t dst = (uint32_t)__cvta_generic_to_shared(base + (it % S) * C::kRows * G::N);
        const uint32_t b = bar + 8u * (uint32_t)(it % S);
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"(C::kBytes) : "memory");
        if constexpr (G::CL == 1) {
            const float2 *g = src + (size_t)(yl0 + it * C::kRows) * G::N;
            asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                         ::"r"(dst), "l"(g), "r"(C::kBytes), "r"(b)
                         : "memory");
        } else {
#pragma unroll
            for (int r = 0; r < C::kRows; ++r) {
                const float2 *g = src + (size_t)G::gy(yb, yl0 + it * C::kRows + r) * G::N;
                asm volatile(
                    "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                        dst + r * C::kRowBytes),
                    "l"(g), "r"(C::kRowBytes), "r"(b)
                    : "memory");
            }
        }
    }
    // the first S iterations, at the top of the slab
    __device__ __forceinline__ void start() const {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncwarp();
        if ((threadIdx.x & 31) == 0)
            for (int it = 0; it < S; ++it) issue(it);
    }
    __device__ __forceinline__ void wait(int it) const {
        const uint32_t b = bar + 8u * (uint32_t)(it % S);
        const unsigned par = (phase + (unsigned)(it / S)) & 1u;
        if (!mbar_wait(b, par)) {
            if (fault && (threadIdx.x & 31) == 0) atomicOr(fault, 1u);
            mbar_wait(b, par);  // let a late copy land before reuse
        }
    }
    // every lane has read the stage of iteration it: reuse it for it + S
    __device__ __forceinline__ void refill(int it) const {
        if (it + S >= C::kIters) return;
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncwarp();
        if ((threadIdx.x & 31) == 0) issue(it + S);
    }
    // the task's row in the stage (lane / R1 = row of the iteration, lane % R1 = n1)
    __device__ __forceinline__ const float2 *task(int it, int lane) const {
        return base + (it % S) * C::kRows * G::N + (lane / G::R1) * G::N + lane % G::R1;
    }
};

// shared-memory layout of the position kernel (float2 units after the field)
template <class G>
struct Smem {
    // TW: twiddles [k2][n1]; TWT (right after): the same transposed, [n1][k2];
    // STG: staged saved-wave rows (16-byte aligned), BAR: their mbarriers
    static constexpr int TW = G::FIELD, TWT = TW + G::N, E1 = TWT + G::N, E2 = E1 + G::N, PY = E2 + G::N,
                         PX = PY + G::N, STG = (PX + G::N + 1) & ~1, BAR = STG + StageCfg<G>::kStageF2,
                         END = BAR + StageCfg<G>::kBarF2;
};
// column pass A reads its twiddles from the transposed table two at a time
// (R2 even): R2/2 16-byte loads per task instead of R2-1 8-byte ones
template <class G>
constexpr bool kColTw = G::R2 % 2 == 0;

template <class G, int METHOD, int ADJ, int MODE>
struct PositionKernel {
    static constexpr int N = G::N, NN = G::N * G::N, R1 = G::R1, R2 = G::R2;
    static constexpr int CB = G::CB;  // points of a column-pass-B task

    // transmission of slab s at (y, x): exp(i sdz sum_{z in slab} V)
    // (mset.cu:134-153 / STEP02_FORWARD_4D.m:12-20; SSET: all z, mset.cu:391-404),
    // read from the precomputed slabs when the tilt has them
    static __device__ __forceinline__ float2 trans(const LaunchArgs &a, const TiltDev &t, int s, int y, int x) {
        // batched passes always run on precomputed slabs
        if constexpr (MODE == kBatch || MODE == kBatchCk || MODE == kSim)
            return t.T[(size_t)s * NN + (size_t)y * N + x];
        if (t.T) return t.T[(size_t)s * NN + (size_t)y * N + x];
        int z0, z1;
        if constexpr (METHOD == kSSET) {
            z0 = 0;
            z1 = a.nz;
        } else {
            z0 = s * a.b;
            z1 = min(z0 + a.b, a.nz);
        }
        const float *p = t.V + (size_t)y * N + x;
        float acc = 0.f;
        for (int z = z0; z < z1; ++z) acc += p[(size_t)z * NN];
        float sn, cs;
        sincosf(a.sdz * acc, &sn, &cs);
        return make_float2(cs, sn);
    }

    // measured amplitude at scrambled location (Ly, Lx): prepared sqrt(I) in
    // scrambled layout, or (kBatchCentred) gathered from the centred pattern
    static __device__ __forceinline__ float meas_amp(const float *amp, const unsigned short *ampb, int Ly, int Lx) {
        if (ampb) {
            // measured counts stored as BF16 (exact for integers <= 256); sqrt in FP32
            const unsigned short b = ampb[(size_t)Ly * N + Lx];
            return sqrtf(__uint_as_float((unsigned)b << 16));
        }
        if constexpr (MODE == kBatchCentred) {
            const int h = (N + 1) / 2;
            int r = G::scry(Ly) - h, c = G::scrx(Lx) - h;
            if (r < 0) r += N;
            if (c < 0) c += N;
            return sqrtf(__ldg(amp + (size_t)r * N + c));
        } else {
            return __ldg(amp + (size_t)Ly * N + Lx);
        }
    }

    // propagator / N^2 at scrambled (Ly, Lx): separable product from shared
    // memory, or the full table in global memory
    static __device__ __forceinline__ float2 prop(const LaunchArgs &a, const float2 *py, const float2 *px, int Ly,
                                                  int Lx) {
        if (a.psep) return cmul(py[Ly], px[Lx]);
        return __ldg(a.pscr + (size_t)Ly * N + Lx);
    }

    // v[j] *= P(y0 + j, x) (CONJ: conj(P)) for the CB rows of a column-pass-B
    // task.  Separable P: Px(x) is read once and Py two rows at a time
    // (16-byte loads; y0 is a multiple of CB, the table 16-byte aligned),
    // 9 shared-memory loads per task instead of 32 (-6% per mid pass)
    template <bool CONJ>
    static __device__ __forceinline__ void apply_prop(const LaunchArgs &a, const float2 *py, const float2 *px,
                                                      int y0, int x, float2 *v) {
        static_assert(CB % 2 == 0, "Py is read in pairs");
        if (a.psep) {
            const float2 pxv = px[x];
            const float4 *q4 = reinterpret_cast<const float4 *>(py + y0);
#pragma unroll
            for (int m = 0; m < CB / 2; ++m) {
                const float4 q = q4[m];
                const float2 p0 = cmul(make_float2(q.x, q.y), pxv), p1 = cmul(make_float2(q.z, q.w), pxv);
                v[2 * m] = CONJ ? cmulc(v[2 * m], p0) : cmul(v[2 * m], p0);
                v[2 * m + 1] = CONJ ? cmulc(v[2 * m + 1], p1) : cmul(v[2 * m + 1], p1);
            }
        } else {
#pragma unroll
            for (int j = 0; j < CB; ++j) {
                const float2 p = prop(a, py, px, y0 + j, x);
                v[j] = CONJ ? cmulc(v[j], p) : cmul(v[j], p);
            }
        }
    }

    // forward through slabs s0 .. s1-1 from the checkpointed wave entering s0,
    // storing the wave after slab s at out[s - s0] (mset.cu:157-183)
    static __device__ __noinline__ void recompute(const LaunchArgs &a, const TiltDev &t, int s0, int s1, float2 *buf,
                                     const float2 *tw, const float2 *py, const float2 *px, const float2 *ckw,
                                     float2 *out) {
        row_passA_pf<G, 0, -1, TPre<G>>(
            buf, tw,
            [&](int y, int n1, TPre<G> &pre) {
#pragma unroll
                for (int j = 0; j < R2; ++j) pre.t[j] = trans(a, t, s0, y, n1 + R1 * j);
            },
            [&](int y, int n1, float2 *v, const TPre<G> &pre) {
                const float2 *w = ckw + (size_t)y * N + n1;
#pragma unroll
                for (int j = 0; j < R2; ++j) v[j] = cmul(w[R1 * j], pre.t[j]);
            });
        sync_rows();
        for (int s = s0; s < s1; ++s) {
            mid_fwd<G, -1, kColTw<G>>(buf, tw);
            sync_cols<G>();
            col_passB<G, -1, +1>(buf, [&](int y0, int x, float2 *v) {
                apply_prop<false>(a, py, px, y0, x, v);
            });
            sync_cols<G>();
            mid_inv<G, +1, kColTw<G>>(buf, tw);
            sync_rows();
            float2 *o = out + (size_t)(s - s0) * NN;
            auto store = [&](int y, int n1, float2 *v) {
                float2 *w = o + (size_t)y * N + n1;
#pragma unroll
                for (int j = 0; j < R2; ++j) w[R1 * j] = v[j];
            };
            if (s + 1 < s1) {
                row_passA_pf<G, +1, -1, TPre<G>>(
                    buf, tw,
                    [&](int y, int n1, TPre<G> &pre) {
#pragma unroll
                        for (int j = 0; j < R2; ++j) pre.t[j] = trans(a, t, s + 1, y, n1 + R1 * j);
                    },
                    [&](int y, int n1, float2 *v, const TPre<G> &pre) {
                        store(y, n1, v);
#pragma unroll
                        for (int j = 0; j < R2; ++j) v[j] = cmul(v[j], pre.t[j]);
                    });
            } else {
                row_passA<G, +1, 0>(buf, tw, store);
            }
            sync_rows();
        }
    }

    static __device__ __forceinline__ void run(const LaunchArgs &a, const TiltDev &t, int p, float2 *buf, float2 *save,
                               double *red, unsigned &stage_phase) {
        const float2 *tw = buf + Smem<G>::TW;
        float2 *e1 = buf + Smem<G>::E1;
        float2 *e2 = buf + Smem<G>::E2;
        const float2 *py = buf + Smem<G>::PY;
        const float2 *px = buf + Smem<G>::PX;
        const int ns = METHOD == kSSET ? 1 : a.ns;
        // checkpointing: keep the wave entering every k-th slab, recompute the
        // waves of a segment right before its adjoint (k = 0: keep them all)
        const int ck = (MODE == kBatchCk && a.ckpt > 0 && a.ckpt < ns) ? a.ckpt : 0;
        const int nseg = ck ? (ns + ck - 1) / ck : 1;
        float2 *recbuf = save + (size_t)nseg * NN;
        float2 *park = save + (size_t)(nseg + ck) * NN;
        float *V = t.V;
        // slab base in a register: generic stores and atomics in the row
        // passes could alias the shared-memory descriptor, which would then be
        // re-read once per task
        const float2 *const Tslab = t.T;
        double *const gslab = t.grad;
        float sxp, syp;
        if constexpr (MODE == kStep) {
            sxp = a.step_x;
            syp = a.step_y;
        } else {
            sxp = t.sx[p];
            syp = t.sy[p];
        }
        const float s1 = syp - a.center, s2 = sxp - a.center;  // mset.cu:121
        // separable Fourier shift factor, indexed by scrambled location
        for (int L = threadIdx.x; L < N; L += G::NT) {
            float sn, cs;
            sincosf(2.0f * MSET_REF_PI * (s1 * shift_grid(G::scry(L), N) / (float)N), &sn, &cs);
            e1[L] = make_float2(cs, sn);
            sincosf(2.0f * MSET_REF_PI * (s2 * shift_grid(G::scrx(L), N) / (float)N), &sn, &cs);
            e2[L] = make_float2(cs, sn);
        }
        sync_all<G>();

        // prefetch of the transmission of slab s for a row-pass task
        auto pf_t = [&](int s) {
            return [&, s](int y, int n1, TPre<G> &pre) {
                if constexpr (MODE == kBatch || MODE == kBatchCk || MODE == kSim) {
                    const float2 *tr = Tslab + (size_t)s * NN + (size_t)y * N + n1;
#pragma unroll
                    for (int j = 0; j < R2; ++j) pre.t[j] = tr[R1 * j];
                } else {
#pragma unroll
                    for (int j = 0; j < R2; ++j) pre.t[j] = trans(a, t, s, y, n1 + R1 * j);
                }
            };
        };

        double err = 0.0;
        // kStep phase 2 (STEP03) starts from a residual and skips the forward
        const bool fwd = MODE != kStep || a.step_phase == 1;
        if (fwd) {
        // ---- incident wave psi0 = F(Q . fs)  (mset.cu:110-131) ----
        col_passB<G, 0, -1>(buf, [&](int y0, int x, float2 *v) {
            const float2 *q = t.Q + (size_t)y0 * N + x;
            const float2 ex = e2[x];
#pragma unroll
            for (int j = 0; j < CB; ++j) v[j] = cmul(cmul(q[(size_t)j * N], e1[y0 + j]), ex);
        });
        sync_cols<G>();
        mid_inv<G, -1, kColTw<G>>(buf, tw);
        sync_rows();
        row_passA_pf<G, -1, -1, TPre<G>>(buf, tw, pf_t(0), [&](int y, int n1, float2 *v, const TPre<G> &pre) {
            if constexpr (MODE != kSim && MODE != kErr) {
                float2 *sv = save + (size_t)y * N + n1;
#pragma unroll
                for (int j = 0; j < R2; ++j) sv[R1 * j] = v[j];
            }
#pragma unroll
            for (int j = 0; j < R2; ++j) v[j] = cmul(v[j], pre.t[j]);
        });
        sync_rows();

        // ---- forward slabs (mset.cu:157-183) ----
        if constexpr (METHOD == kMSET) {
            for (int s = 0; s < ns; ++s) {
                if (Tslab && s + 1 < ns)
                    l1_first<G>(L1FirstT<G>{reinterpret_cast<const char *>(Tslab + (size_t)(s + 1) * NN)});
                mid_fwd<G, -1, kColTw<G>>(buf, tw);
                sync_cols<G>();
                col_passB<G, -1, +1>(buf, [&](int y0, int x, float2 *v) {
                    apply_prop<false>(a, py, px, y0, x, v);
                });
                sync_cols<G>();
                mid_inv<G, +1, kColTw<G>>(buf, tw);
                sync_rows();
                const bool last = s + 1 == ns;
                const int sn = last ? s : s + 1;
                // single-buffered transmission prefetch (R2 > 8): pull the next
                // iteration's rows into L1 as well
                const L1Rows<G, true> l1f{(Tslab && !last)
                                        ? reinterpret_cast<const char *>(Tslab + (size_t)sn * NN)
                                        : nullptr,
                                    nullptr};
                row_passA_pf<G, +1, -1, TPre<G>>(
                    buf, tw,
                    [&](int y, int n1, TPre<G> &pre) {
                        if (!last) pf_t(sn)(y, n1, pre);
                    },
                    [&](int y, int n1, float2 *v, const TPre<G> &pre) {
                        if constexpr (MODE != kSim && MODE != kErr) {
                            const int w = s + 1;
                            float2 *sv = nullptr;
                            if (!ck) {
                                sv = save + (size_t)w * NN;
                            } else if constexpr (MODE == kBatchCk) {
                                if (w % ck == 0 && w < ns) sv = save + (size_t)(w / ck) * NN;
                            }
                            if (sv) {
                                sv += (size_t)y * N + n1;
#pragma unroll
                                for (int j = 0; j < R2; ++j) sv[R1 * j] = v[j];
                            }
                        }
                        if (!last) {
#pragma unroll
                            for (int j = 0; j < R2; ++j) v[j] = cmul(v[j], pre.t[j]);
                        }
                    },
                    l1f);
                sync_rows();
            }
        }

        // ---- far field, error, residual (mset.cu:186-227) ----
        if constexpr (StageCfg<G>::kOn) {
            // the saved waves were written through the generic proxy; the
            // adjoint's bulk copies read them through the async proxy
            asm volatile("fence.proxy.async.global;" ::: "memory");
        }
        mid_fwd<G, -1, kColTw<G>>(buf, tw);
        sync_cols<G>();
        const float *amp = t.amp ? t.amp + (size_t)p * NN : nullptr;
        const unsigned short *ampb = t.ampb ? t.ampb + (size_t)p * NN : nullptr;
        if constexpr (MODE == kSim || MODE == kErr) {
            col_passB<G, -1, 0>(buf, [&](int y0, int x, float2 *v) {
#pragma unroll
                for (int j = 0; j < CB; ++j) {
                    const float a2 = v[j].x * v[j].x + v[j].y * v[j].y;
                    if constexpr (MODE == kSim) {
                        // centred (MATLAB) layout: row r with (r + ceil(N/2)) mod N = ky
                        const int h = (N + 1) / 2;
                        int r = G::scry(y0 + j) - h, c = G::scrx(x) - h;
                        if (r < 0) r += N;
                        if (c < 0) c += N;
                        t.inten[(size_t)p * NN + (size_t)r * N + c] = a2;
                    } else {
                        const float A = sqrtf(a2 + 1e-30f);
                        const float M = meas_amp(amp, ampb, y0 + j, x);
                        const float d = A - M;
                        err += (double)(d * d);
                    }
                }
            });
            if constexpr (MODE == kErr) {
                double dummy = 0.0;
                block_sum2<G::NT>(err, dummy, red);
                if (threadIdx.x == 0) atomicAdd(t.err, err);
            }
            sync_all<G>();
            return;
        } else if constexpr (MODE == kStep) {
            // STEP02 (STEP02_FORWARD_4D.m:36-49): residual (scrambled) and
            // |Psi|^2 (centred) out, error sum; the waves stay in the slots
            col_passB<G, -1, 0>(buf, [&](int y0, int x, float2 *v) {
#pragma unroll
                for (int j = 0; j < CB; ++j) {
                    const float a2 = v[j].x * v[j].x + v[j].y * v[j].y;
                    const float A = sqrtf(a2 + 1e-30f);
                    const float M = meas_amp(amp, ampb, y0 + j, x);
                    const float d = A - M;
                    err += (double)(d * d);
                    a.step_resi[(size_t)(y0 + j) * N + x] = cscale(v[j], 1.0f - M / A);
                    const int h = (N + 1) / 2;
                    int r = G::scry(y0 + j) - h, c = G::scrx(x) - h;
                    if (r < 0) r += N;
                    if (c < 0) c += N;
                    a.step_calc[(size_t)r * N + c] = a2;
                }
            });
            double dummy = 0.0;
            block_sum2<G::NT>(err, dummy, red);
            if (threadIdx.x == 0) atomicAdd(a.step_err, err);
            sync_all<G>();
            return;
        } else {
            col_passB<G, -1, +1>(buf, [&](int y0, int x, float2 *v) {
#pragma unroll
                for (int j = 0; j < CB; ++j) {
                    const float a2 = v[j].x * v[j].x + v[j].y * v[j].y;
                    const float A = sqrtf(a2 + 1e-30f);
                    const float M = meas_amp(amp, ampb, y0 + j, x);
                    const float d = A - M;
                    err += (double)(d * d);
                    float2 r = cscale(v[j], 1.0f - M / A);
                    if constexpr (METHOD == kMSET) {
                        r = cmulc(r, prop(a, py, px, y0 + j, x));  // r * conj(P) / N^2
                    } else {
                        r = cscale(r, 1.0f / (float)NN);
                    }
                    v[j] = r;
                }
            });
            sync_cols<G>();
        }
        } else {
            // STEP03 (STEP03_BACK.m:10-13): the residual r conj(P) / N^2
            // (SSET: r / N^2), inverse column transform started
            col_passB<G, 0, +1>(buf, [&](int y0, int x, float2 *v) {
#pragma unroll
                for (int j = 0; j < CB; ++j) {
                    const float2 r = a.step_resi[(size_t)(y0 + j) * N + x];
                    if constexpr (METHOD == kMSET) v[j] = cmulc(r, prop(a, py, px, y0 + j, x));
                    else v[j] = cscale(r, 1.0f / (float)NN);
                }
            });
            sync_cols<G>();
        }

        // ---- adjoint (mset.cu:232-271; STEP03_BACK.m:12-26) ----
        for (int seg = nseg - 1; seg >= 0; --seg) {
          const int s0 = ck ? seg * ck : 0, s1 = ck ? min(s0 + ck, ns) : ns;
          if constexpr (MODE == kBatchCk) {
            if (ck) {
              // park the adjoint state, recompute the waves s0+1 .. s1 of the
              // segment from its checkpoint, restore the state
              float2 *mine = park + (size_t)G::rank() * G::FIELD;  // this CTA's rows
              sync_all<G>();
              for (int i = threadIdx.x; i < G::FIELD; i += G::NT) mine[i] = buf[i];
              sync_all<G>();
              recompute(a, t, s0, s1, buf, tw, py, px, save + (size_t)seg * NN, recbuf);
              if constexpr (StageCfg<G>::kOn) asm volatile("fence.proxy.async.global;" ::: "memory");
              sync_all<G>();
              for (int i = threadIdx.x; i < G::FIELD; i += G::NT) buf[i] = mine[i];
              sync_all<G>();
            }
          }
          for (int s = s1 - 1; s >= s0; --s) {
            // REF: the wave saved after slab s (mset.cu:248-251); EXACT: the wave entering slab s
            const int ws = (METHOD == kSSET || ADJ == kEXACT) ? s : s + 1;
            const float2 *wave = !ck ? save + (size_t)ws * NN
                                     : (ws == s0 ? save + (size_t)seg * NN : recbuf + (size_t)(ws - s0 - 1) * NN);
            // the saved wave was written long ago (DRAM); have it in L2 by the row pass
            prefetch_l2(wave, (unsigned)(sizeof(float2) * NN));
            constexpr bool kStg = StageCfg<G>::kOn;
            using APre = std::conditional_t<kStg, T1Pre<G>, TSPre<G>>;
            using L1A = std::conditional_t<kStg, L1Rows<G, false, true>, L1Rows<G>>;
            const L1A l1{Tslab ? reinterpret_cast<const char *>(Tslab + (size_t)s * NN) : nullptr,
                         kStg ? nullptr : reinterpret_cast<const char *>(wave)};
            l1_first<G>(l1);  // this slab's first row-pass-A iteration, two passes ahead
            using SG = std::conditional_t<kStg, RowStage<G>, NoStage>;
            SG stg{};
            if constexpr (kStg) {
                constexpr int SS = StageCfg<G>::kStages;
                stg = RowStage<G>{buf + Smem<G>::STG + SS * StageCfg<G>::kRows * N * Own<G>::warp(),
                                  (uint32_t)__cvta_generic_to_shared(buf + Smem<G>::BAR) + 8u * SS * Own<G>::warp(),
                                  wave, Own<G>::warp() * Own<G>::RPW, G::ybase(), stage_phase, a.fault};
                stg.start();
            }
            mid_inv<G, +1, kColTw<G>>(buf, tw);
            sync_rows();
            // the operands are loaded before the task's shared-memory reads:
            // loading them inside the op instead (fewer live registers at
            // R2 = 16) exposes their latency and cost 17-22% at n = 256
            auto pf = [&](int y, int n1, APre &pre) {
                const float2 *sv = wave + (size_t)y * N + n1;
                if constexpr (MODE == kBatch || MODE == kBatchCk) {
                    // the slab row's address once per task (the descriptor
                    // lives in shared memory)
                    const float2 *tr = Tslab + (size_t)s * NN + (size_t)y * N + n1;
#pragma unroll
                    for (int j = 0; j < R2; ++j) {
                        pre.t[j] = tr[R1 * j];
                        if constexpr (!kStg) pre.w[j] = sv[R1 * j];
                    }
                } else {
#pragma unroll
                    for (int j = 0; j < R2; ++j) {
                        pre.t[j] = trans(a, t, s, y, n1 + R1 * j);
                        if constexpr (!kStg) pre.w[j] = sv[R1 * j];
                    }
                }
                (void)sv;
            };
            auto gradop = [&](int y, int n1, float2 *v, const APre &pre, const float2 *wst) {
                // the gradient row's address in a register: a store through a
                // generic pointer could alias the descriptor in shared memory,
                // which would otherwise be re-read after every store
                double *grow = nullptr;
                if constexpr (MODE != kSeq && MODE != kStep) grow = gslab + (size_t)s * NN + (size_t)y * N;
#pragma unroll
                for (int j = 0; j < R2; ++j) {
                    const int x = n1 + R1 * j;
                    const float2 T = pre.t[j];
                    float2 W;
                    if constexpr (kStg) W = wst[R1 * j];
                    else W = pre.w[j];
                    // g = i conj(T) conj(psi) chi
                    const float2 u = cmulc(cmulc(v[j], T), W);
                    const float gre = -u.y;  // Re(i u)
                    if constexpr (MODE == kSeq) {
                        int z0, z1;
                        if constexpr (METHOD == kSSET) {
                            z0 = 0;
                            z1 = a.nz;
                        } else {
                            z0 = s * a.b;
                            z1 = min(z0 + a.b, a.nz);
                        }
                        // RVol += step0 * Re(grad), slab-replicated (mset.cu:273-284)
                        const float du = a.step0 * gre;
                        for (int z = z0; z < z1; ++z) V[(size_t)z * NN + (size_t)y * N + x] += du;
                    } else if constexpr (MODE == kStep) {
                        // STEP03_BACK.m:15-16: g = i u, kept complex
                        a.step_grad[(size_t)s * NN + (size_t)y * N + x] = make_float2(gre, u.x);
                        if (a.step04) {
                            int z0, z1;
                            if constexpr (METHOD == kSSET) {
                                z0 = 0;
                                z1 = a.nz;
                            } else {
                                z0 = s * a.b;
                                z1 = min(z0 + a.b, a.nz);
                            }
                            // Run_MSET_recon.m:155
                            const float du = a.step0 * gre;
                            for (int z = z0; z < z1; ++z) V[(size_t)z * NN + (size_t)y * N + x] += du;
                        }
                    } else {
                        // FP64 sum over positions: a reduction without return
                        // value straight to the global address
                        asm volatile("red.global.add.f64 [%0], %1;" ::"l"(__cvta_generic_to_global(grow + x)),
                                     "d"((double)gre)
                                     : "memory");
                    }
                    v[j] = cmulc(v[j], T);  // chi <- conj(T) chi
                }
            };
            auto run_rowA = [&](auto out) {
                constexpr int OUT = decltype(out)::value;
                if constexpr (kStg) {
                    row_passA_pf<G, +1, OUT, APre>(buf, tw, pf, gradop, l1, stg);
                } else {
                    row_passA_pf<G, +1, OUT, APre>(
                        buf, tw, pf,
                        [&](int y, int n1, float2 *v, const APre &pre) { gradop(y, n1, v, pre, nullptr); }, l1);
                }
            };
            if constexpr (kStg) stage_phase += StageCfg<G>::kIters / StageCfg<G>::kStages;
            if (s > 0) {
                run_rowA(std::integral_constant<int, -1>{});
                sync_rows();
                mid_fwd<G, -1, kColTw<G>>(buf, tw);
                sync_cols<G>();
                col_passB<G, -1, +1>(buf, [&](int y0, int x, float2 *v) {
                    apply_prop<true>(a, py, px, y0, x, v);
                });
                sync_cols<G>();
            } else {
                run_rowA(std::integral_constant<int, 0>{});
                sync_all<G>();
            }
          }
        }
        // buf now holds chi0 (real space, natural order); save[0] holds psi0.

        // ---- scan-position direction, REF: finite differences of conj(psi0)
        //      (mset.cu:316-327; utility.cu:829-876) ----
        double pdx = 0.0, pdy = 0.0;
        if constexpr (ADJ == kREF) {
            const int yb = G::ybase();
            for (int i = threadIdx.x; i < G::ROWS * N; i += G::NT) {
                const int yl = i / N, x = i % N, y = G::gy(yb, yl);
                const float2 c0 = buf[G::at(yl, x)];
                const float2 *f = save + (size_t)y * N + x;
                float2 dx, dy;
                if (x == 0) dx = csub(f[1], f[0]);
                else if (x == N - 1) dx = csub(f[0], f[-1]);
                else dx = cscale(csub(f[1], f[-1]), 0.5f);
                if (y == 0) dy = csub(f[N], f[0]);
                else if (y == N - 1) dy = csub(f[0], f[-N]);
                else dy = cscale(csub(f[N], f[-N]), 0.5f);
                // Re(conj(d) * chi0)
                pdx += (double)(dx.x * c0.x + dx.y * c0.y);
                pdy += (double)(dy.x * c0.x + dy.y * c0.y);
            }
        }
        sync_all<G>();

        // ---- probe direction: d = F^{-1}(chi0) fs(-s), accumulated in the
        //      F^{-1}(probe) domain (mset.cu:288-312) ----
        row_passA<G, 0, +1>(buf, tw, NoOp{});
        sync_rows();
        mid_fwd<G, +1, kColTw<G>>(buf, tw);
        sync_cols<G>();
        const float inv = 1.0f / (float)NN;
        // descriptor fields in registers: the atomics below go through generic
        // pointers that could alias the shared-memory descriptor
        float2 *const Qd = t.Q;
        double *const qacc = t.qacc;
        col_passB<G, +1, 0>(buf, [&](int y0, int x, float2 *v) {
            const float2 ex = e2[x];
            const float kx = 2.0f * MSET_REF_PI * shift_grid(G::scrx(x), N) / (float)N;
#pragma unroll
            for (int j = 0; j < CB; ++j) {
                const size_t li = (size_t)(y0 + j) * N + x;
                const float2 fs = cmul(e1[y0 + j], ex);
                const float2 d = cscale(cmulc(v[j], fs), inv);
                if constexpr (ADJ == kEXACT) {
                    // spectral derivative of psi0 w.r.t. the scan coordinates
                    const float2 qf = cmul(Qd[li], fs);
                    const float ky = 2.0f * MSET_REF_PI * shift_grid(G::scry(y0 + j), N) / (float)N;
                    // X = Q fs (i kappa); -Re(conj(X) Y)
                    const float2 Xx = make_float2(-qf.y * kx, qf.x * kx);
                    const float2 Xy = make_float2(-qf.y * ky, qf.x * ky);
                    pdx -= (double)(Xx.x * v[j].x + Xx.y * v[j].y);
                    pdy -= (double)(Xy.x * v[j].x + Xy.y * v[j].y);
                }
                if constexpr (MODE == kSeq || MODE == kStep) {
                    float2 q = Qd[li];
                    q.x -= a.step1 * d.x;
                    q.y -= a.step1 * d.y;
                    Qd[li] = q;
                } else {
                    atomicAdd(qacc + 2 * li, (double)d.x);
                    atomicAdd(qacc + 2 * li + 1, (double)d.y);
                }
            }
        });
        block_sum2<G::NT>(pdx, pdy, red);
        double dummy = 0.0;
        block_sum2<G::NT>(err, dummy, red);
        if (threadIdx.x == 0) atomicAdd(t.err, err);
        if constexpr (G::CL > 1) {
            // the position sums of every CTA of the cluster, gathered in CTA 0
            if (threadIdx.x == 0) {
                double *dst = peer(red + 2 * (G::NT / 32), 0);
                dst[2 * G::rank()] = pdx;
                dst[2 * G::rank() + 1] = pdy;
            }
            cluster_sync();
            if (G::rank() == 0 && threadIdx.x == 0) {
                const double *part = red + 2 * (G::NT / 32);
                pdx = pdy = 0.0;
                for (int r = 0; r < G::CL; ++r) {
                    pdx += part[2 * r];
                    pdy += part[2 * r + 1];
                }
            }
        }
        if (G::rank() == 0 && threadIdx.x == 0) {
            if constexpr (MODE == kSeq) {
                t.sx[p] = sxp + a.step2 * (float)pdx;  // mset.cu:322
                t.sy[p] = syp + a.step2 * (float)pdy;  // mset.cu:327
            } else if constexpr (MODE == kStep) {
                a.step_pos[0] = sxp + a.step2 * (float)pdx;  // STEP03_BACK.m:37-38
                a.step_pos[1] = syp + a.step2 * (float)pdy;
            } else {
                t.posdir[2 * p] = pdx;
                t.posdir[2 * p + 1] = pdy;
            }
        }
        sync_all<G>();
    }
};

template <class G>
__device__ __forceinline__ void load_tables(float2 *buf, const LaunchArgs &a) {
    float2 *tw = buf + Smem<G>::TW;
    float2 *py = buf + Smem<G>::PY;
    float2 *px = buf + Smem<G>::PX;
    float2 *twt = buf + Smem<G>::TWT;
    for (int i = threadIdx.x; i < G::N; i += G::NT) {
        if constexpr (G::THREE) {
            // the x table [a][k1] and the y table [k1'][b] of phase 2
            tw[i] = a.twn[i];
            twt[i] = a.twn[G::N + i];
        } else {
            tw[i] = a.twn[i];
            twt[(i % G::R1) * G::R2 + i / G::R1] = a.twn[i];  // [k2][n1] -> [n1][k2]
        }
        if (a.psep) {
            py[i] = a.psep[i];
            px[i] = a.psep[G::N + i];
        }
    }
}

template <class G, int METHOD, int ADJ, int MODE>
__global__ void __launch_bounds__(G::NT, G::MINB) k_positions(const LaunchArgs a) {
    extern __shared__ __align__(16) float2 smem[];
    float2 *buf = smem;
    double *red = reinterpret_cast<double *>(buf + Smem<G>::END);
    __shared__ int s_item;
    // the tilt's descriptor lives in shared memory for the whole position:
    // its pointers are read on every pass, and a global read of them would
    // sit in front of every dependent load
    __shared__ TiltDev s_tilt;
    load_tables<G>(buf, a);
    if constexpr (StageCfg<G>::kOn) {
        // two mbarriers per warp for the bulk-staged saved-wave rows (one arrival each)
        if ((threadIdx.x & 31) == 0) {
            constexpr int SS = StageCfg<G>::kStages;
            const uint32_t b = (uint32_t)__cvta_generic_to_shared(buf + Smem<G>::BAR) + 8u * SS * (threadIdx.x >> 5);
            for (int i = 0; i < SS; ++i) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(b + 8u * i) : "memory");
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    unsigned stage_phase = 0;  // completed phases of each staging mbarrier
    // one set of saved-wave slots per field (per cluster when the field is split)
    float2 *save = a.save + (size_t)(blockIdx.x / G::CL) * a.slots * G::N * G::N;
    // (cluster) every CTA has started before any distributed shared-memory access
    sync_all<G>();
    using K = PositionKernel<G, METHOD, ADJ, MODE>;
    if constexpr (MODE == kSeq) {
        if (threadIdx.x == 0) s_tilt = a.tilts[a.seq_tilt];
        sync_all<G>();
        for (int p = 0; p < s_tilt.npos; ++p) K::run(a, s_tilt, p, buf, save, red, stage_phase);
    } else if constexpr (MODE == kStep) {
        if (threadIdx.x == 0) s_tilt = a.tilts[a.seq_tilt];
        sync_all<G>();
        K::run(a, s_tilt, a.step_k, buf, save, red, stage_phase);
    } else {
        int cur = -1;
        for (;;) {
            if constexpr (G::CL > 1) {
                // CTA 0 of the cluster takes the item and hands it to every CTA
                if (G::rank() == 0 && threadIdx.x == 0) {
                    const int v = (int)atomicAdd(a.counter, 1u);
#pragma unroll
                    for (int r = 0; r < G::CL; ++r) *peer(&s_item, r) = v;
                }
                cluster_sync();
            } else {
                if (threadIdx.x == 0) s_item = (int)atomicAdd(a.counter, 1u);
                __syncthreads();
            }
            const int it = s_item;
            __syncthreads();
            if (it >= a.nitems) break;
            const int2 tp = a.items[it];
            if (tp.x != cur) {
                if (threadIdx.x == 0) s_tilt = a.tilts[tp.x];
                __syncthreads();
                cur = tp.x;
            }
            K::run(a, s_tilt, tp.y, buf, save, red, stage_phase);
        }
    }
}

// ---------------------------------------------------------------------------
// preparation kernels
// ---------------------------------------------------------------------------
template <class G>
__global__ void k_prep_amp(const float *meas, float *amp, long npos) {
    // amp[p][Ly][Lx] = sqrt(ifftshift(I)[scr(Ly)][scr(Lx)])  (mset.cu:206-210)
    const long total = npos * (long)G::N * G::N;
    const int h = (G::N + 1) / 2;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
        const long p = i / ((long)G::N * G::N);
        const int l = (int)(i % ((long)G::N * G::N));
        const int Ly = l / G::N, Lx = l % G::N;
        int r = G::scry(Ly) - h, c = G::scrx(Lx) - h;
        if (r < 0) r += G::N;
        if (c < 0) c += G::N;
        amp[i] = sqrtf(meas[p * G::N * G::N + (long)r * G::N + c]);
    }
}

template <class G>
__global__ void k_prep_amp_bf16(const float *meas, unsigned short *ib, long npos) {
    // ib[p][Ly][Lx] = bf16(ifftshift(I)[scr(Ly)][scr(Lx)]), round to nearest even
    const long total = npos * (long)G::N * G::N;
    const int h = (G::N + 1) / 2;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
        const long p = i / ((long)G::N * G::N);
        const int l = (int)(i % ((long)G::N * G::N));
        const int Ly = l / G::N, Lx = l % G::N;
        int r = G::scry(Ly) - h, c = G::scrx(Lx) - h;
        if (r < 0) r += G::N;
        if (c < 0) c += G::N;
        const __nv_bfloat16 v = __float2bfloat16_rn(meas[p * G::N * G::N + (long)r * G::N + c]);
        ib[i] = __bfloat16_as_ushort(v);
    }
}

template <class G>
__global__ void k_prep_prop(const float2 *prop, float2 *pscr) {
    // pscr[Ly][Lx] = ifftshift(prop)[scr(Ly)][scr(Lx)] / N^2  (mex_main.cu:80-83)
    const int h = (G::N + 1) / 2;
    const float inv = 1.0f / (float)(G::N * G::N);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < G::N * G::N; i += gridDim.x * blockDim.x) {
        const int Ly = i / G::N, Lx = i % G::N;
        int r = G::scry(Ly) - h, c = G::scrx(Lx) - h;
        if (r < 0) r += G::N;
        if (c < 0) c += G::N;
        pscr[i] = cscale(prop[r * G::N + c], inv);
    }
}

// Q = F^{-1}(probe) (scrambled) and probe = F(Q) (natural); one CTA, or one
// cluster when the field is split over CTAs.
template <class G, bool TO_Q>
__global__ void __launch_bounds__(G::NT) k_probe_q(const float2 *in, float2 *out, const float2 *twn) {
    extern __shared__ __align__(16) float2 smem[];
    float2 *buf = smem;
    float2 *tw = buf + G::FIELD;
    for (int i = threadIdx.x; i < (G::THREE ? 2 : 1) * G::N; i += G::NT) tw[i] = twn[i];
    sync_all<G>();  // (cluster) every CTA has started before any remote access
    constexpr int N = G::N;
    const int yb = G::ybase();
    if constexpr (TO_Q) {
        for (int i = threadIdx.x; i < G::ROWS * N; i += G::NT)
            buf[G::at(i / N, i % N)] = in[(size_t)G::gy(yb, i / N) * N + i % N];
        __syncthreads();
        row_passA<G, 0, +1>(buf, tw, NoOp{});
        __syncthreads();
        mid_fwd<G, +1, false>(buf, tw);
        sync_all<G>();
        const float inv = 1.0f / (float)(N * N);
        col_passB<G, +1, 0>(buf, [&](int y0, int x, float2 *v) {
#pragma unroll
            for (int j = 0; j < G::CB; ++j) out[(size_t)(y0 + j) * N + x] = cscale(v[j], inv);
        });
    } else {
        col_passB<G, 0, -1>(buf, [&](int y0, int x, float2 *v) {
#pragma unroll
            for (int j = 0; j < G::CB; ++j) v[j] = in[(size_t)(y0 + j) * N + x];
        });
        sync_all<G>();
        mid_inv<G, -1, false>(buf, tw);
        __syncthreads();
        row_passA<G, -1, 0>(buf, tw, [&](int y, int n1, float2 *v) {
#pragma unroll
            for (int j = 0; j < G::R2; ++j) out[(size_t)y * N + n1 + G::R1 * j] = v[j];
        });
    }
    sync_all<G>();  // no CTA leaves while another may still read its shared memory
}


template <class G>
inline size_t smem_bytes() {
    return sizeof(float2) * (size_t)Smem<G>::END + sizeof(double) * 2 * ((G::NT + 31) / 32 + G::CL);
}

// launch of `grid` CTAs, in clusters of G::CL when the field is split
template <class G, class... KA, class... AA>
inline int launch_geo(void (*k)(KA...), int grid, size_t sm, cudaStream_t st, AA &&...args) {
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return (int)e;
    if constexpr (G::CL > 1) {
        if (grid % G::CL) return (int)cudaErrorInvalidValue;
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
        return (int)cudaLaunchKernelEx(&cfg, k, std::forward<AA>(args)...);
    } else {
        k<<<grid, G::NT, sm, st>>>(std::forward<AA>(args)...);
        return (int)cudaGetLastError();
    }
}

template <class G, int METHOD, int ADJ, int MODE>
inline int launch_one(const LaunchArgs &a, int grid, cudaStream_t st) {
    return launch_geo<G>(k_positions<G, METHOD, ADJ, MODE>, grid, smem_bytes<G>(), st, a);
}

// clusters of the batched kernel resident at once (0: not a cluster geometry,
// or the query failed)
template <class G>
int geo_max_clusters() {
    if constexpr (G::CL > 1) {
        auto k = k_positions<G, kMSET, kREF, kBatch>;
        const size_t sm = smem_bytes<G>();
        if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm) != cudaSuccess) return 0;
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(G::CL * 148);
        cfg.blockDim = dim3(G::NT);
        cfg.dynamicSmemBytes = sm;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = G::CL;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        int n = 0;
        if (cudaOccupancyMaxActiveClusters(&n, k, &cfg) != cudaSuccess) return 0;
        return n;
    } else {
        return 0;
    }
}

template <class G>
int geo_positions(int method, int adjoint, int mode, const LaunchArgs &a, int grid, cudaStream_t st) {
    if (mode == kErr || mode == kSim) adjoint = kREF;
#define MSET_L(M, A, MO) \
    if (method == M && adjoint == A && mode == MO) return launch_one<G, M, A, MO>(a, grid, st);
    MSET_L(kMSET, kREF, kSeq) MSET_L(kMSET, kREF, kBatch) MSET_L(kMSET, kEXACT, kSeq) MSET_L(kMSET, kEXACT, kBatch)
    MSET_L(kSSET, kREF, kSeq) MSET_L(kSSET, kREF, kBatch) MSET_L(kSSET, kEXACT, kSeq) MSET_L(kSSET, kEXACT, kBatch)
    MSET_L(kMSET, kREF, kErr) MSET_L(kSSET, kREF, kErr) MSET_L(kMSET, kREF, kSim) MSET_L(kSSET, kREF, kSim)
    MSET_L(kMSET, kREF, kBatchCk) MSET_L(kMSET, kEXACT, kBatchCk)
    MSET_L(kMSET, kREF, kStep) MSET_L(kMSET, kEXACT, kStep) MSET_L(kSSET, kREF, kStep) MSET_L(kSSET, kEXACT, kStep)
#undef MSET_L
    return (int)cudaErrorInvalidValue;
}

// (a geometry whose batched queue is never launched: one cluster per call)
inline int geo_no_clusters() { return 0; }

// the modes that walk one position at a time through one field: the
// reference-semantics pass (kSeq) and the per-position steps (kStep); a
// geometry compiled for these alone splits that one field over a cluster
template <class G>
int geo_positions_seq(int method, int adjoint, int mode, const LaunchArgs &a, int grid, cudaStream_t st) {
#define MSET_L(M, A, MO) \
    if (method == M && adjoint == A && mode == MO) return launch_one<G, M, A, MO>(a, grid, st);
    MSET_L(kMSET, kREF, kSeq) MSET_L(kMSET, kEXACT, kSeq) MSET_L(kSSET, kREF, kSeq) MSET_L(kSSET, kEXACT, kSeq)
    MSET_L(kMSET, kREF, kStep) MSET_L(kMSET, kEXACT, kStep) MSET_L(kSSET, kREF, kStep) MSET_L(kSSET, kEXACT, kStep)
#undef MSET_L
    return (int)cudaErrorInvalidValue;
}

template <class G>
int geo_prep_amp(const float *meas, float *amp, long npos, cudaStream_t st) {
    k_prep_amp<G><<<1184, 256, 0, st>>>(meas, amp, npos);
    return (int)cudaGetLastError();
}

template <class G>
int geo_prep_amp_bf16(const float *meas, unsigned short *ib, long npos, cudaStream_t st) {
    k_prep_amp_bf16<G><<<1184, 256, 0, st>>>(meas, ib, npos);
    return (int)cudaGetLastError();
}

template <class G>
int geo_prep_prop(const float *prop, float2 *pscr, cudaStream_t st) {
    k_prep_prop<G><<<148, 256, 0, st>>>(reinterpret_cast<const float2 *>(prop), pscr);
    return (int)cudaGetLastError();
}

template <class G>
int geo_probe_q(bool to_q, const float2 *in, float2 *out, const float2 *twn, cudaStream_t st) {
    const size_t sm = smem_bytes<G>();
    if (to_q) return launch_geo<G>(k_probe_q<G, true>, G::CL, sm, st, in, out, twn);
    return launch_geo<G>(k_probe_q<G, false>, G::CL, sm, st, in, out, twn);
}

}  // namespace mset

// one translation unit per window size defines its table entry
#define MSET_DEFINE_GEO(N_, R1_, NT_, MINB_) MSET_DEFINE_GEO_T(N_, N_, R1_, (Geo<N_, R1_, NT_, MINB_>))
// another thread / register shape of the same window (same R1, so the same
// scrambled layouts): a choice for the autotuner, table entry kGeo<NAME_>
#define MSET_DEFINE_GEO_VARIANT(NAME_, N_, R1_, NT_, MINB_) \
    MSET_DEFINE_GEO_T(NAME_, N_, R1_, (Geo<N_, R1_, NT_, MINB_>))
// the same window and thread shape with the adjoint's saved-wave rows staged
// in shared memory by bulk copies (StageCfg)
#define MSET_DEFINE_GEO_STAGED(NAME_, N_, R1_, NT_, MINB_) \
    MSET_DEFINE_GEO_T(NAME_, N_, R1_, (Geo<N_, R1_, NT_, MINB_, true>))
// the sequential modes only (geo_positions_seq), with one field split by rows
// over a cluster of CL_ CTAs: table entry kSeqGeo<NAME_>
#define MSET_DEFINE_SEQ_GEO_CL(NAME_, N_, R1_, NT_, CL_)                                \
    namespace mset {                                                                   \
    using SeqGeo##NAME_ = GeoCl<N_, R1_, NT_, CL_>;                                    \
    extern const GeoOps kSeqGeo##NAME_ = {N_,                                          \
                                          R1_,                                         \
                                          SeqGeo##NAME_::RY1,                          \
                                          SeqGeo##NAME_::NT,                           \
                                          SeqGeo##NAME_::CL,                           \
                                          smem_bytes<SeqGeo##NAME_>(),                 \
                                          0,                                           \
                                          &geo_no_clusters,                            \
                                          &geo_positions_seq<SeqGeo##NAME_>,           \
                                          &geo_prep_amp<SeqGeo##NAME_>,                \
                                          &geo_prep_amp_bf16<SeqGeo##NAME_>,           \
                                          &geo_prep_prop<SeqGeo##NAME_>,               \
                                          &geo_probe_q<SeqGeo##NAME_>};                \
    }
// a field split by rows over a cluster of CL_ CTAs
#define MSET_DEFINE_GEO_CL(N_, R1_, NT_, CL_) MSET_DEFINE_GEO_T(N_, N_, R1_, (GeoCl<N_, R1_, NT_, CL_>))
// the same with the adjoint's saved-wave rows staged by bulk copies (StageCfg)
#define MSET_DEFINE_GEO_CL_STAGED(NAME_, N_, R1_, NT_, CL_) \
    MSET_DEFINE_GEO_T(NAME_, N_, R1_, (GeoCl<N_, R1_, NT_, CL_, 1, true>))
#define MSET_DEFINE_GEO_CL_VARIANT(NAME_, N_, R1_, NT_, CL_, MINB_) \
    MSET_DEFINE_GEO_T(NAME_, N_, R1_, (GeoCl<N_, R1_, NT_, CL_, MINB_>))
// the three-phase shape of the 128 x 128 window (Geo3; WIDE_: 16-byte phase-2 accesses)
#define MSET_DEFINE_GEO3(NAME_, WIDE_) MSET_DEFINE_GEO_T(NAME_, 128, 8, (Geo3<1, WIDE_>))
#define MSET_UNPAREN(...) __VA_ARGS__
#define MSET_DEFINE_GEO_T(NAME_, N_, R1_, GT_)                                         \
    namespace mset {                                                                   \
    using Geo##NAME_ = MSET_UNPAREN GT_;                                               \
    extern const GeoOps kGeo##NAME_ = {N_,                                             \
                                       R1_,                                            \
                                       Geo##NAME_::RY1,                                \
                                       Geo##NAME_::NT,                                 \
                                       Geo##NAME_::CL,                                 \
                                       smem_bytes<Geo##NAME_>(),                       \
                                       StageCfg<Geo##NAME_>::kOn ? 1 : 0,              \
                                       &geo_max_clusters<Geo##NAME_>,                  \
                                       &geo_positions<Geo##NAME_>,                     \
                                       &geo_prep_amp<Geo##NAME_>,                      \
                                       &geo_prep_amp_bf16<Geo##NAME_>,                 \
                                       &geo_prep_prop<Geo##NAME_>,                     \
                                       &geo_probe_q<Geo##NAME_>};                      \
    }
