// mset_kernels.cuh -- internal interface between the C-ABI host layer
// (mset_api.cu) and the fused multislice kernels (mset_kernels_impl.cuh, one
// translation unit per window size: geo_<N>.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace mset {

enum Method { kMSET = 1, kSSET = 2 };
enum Adjoint { kREF = 0, kEXACT = 1 };
// what one launch does with each position
enum Mode {
    kSeq = 0,    // reference semantics: update volume, probe and position after every position
    kBatch = 1,  // fixed state, accumulate FP64 gradients over positions
    kErr = 2,    // forward + error only (run_error_mset / run_error_sset)
    kSim = 3,    // forward + write |Psi|^2 (centred layout)
    kBatchCentred = 4,  // kBatch reading the caller's centred intensities (no prepared amplitudes)
    kBatchCk = 5,       // kBatch keeping every k-th wave and recomputing the rest (checkpointing)
    kStep = 6           // one position as the reference's per-position steps: STEP02 (forward;
                        // residual, |Psi|^2 and waves out) or STEP03 (adjoint from a residual)
};

// one tilt: all buffers on the device
struct TiltDev {
    float *V;            // [nz][n][n] beam-frame potential (kSeq: updated in place)
    float2 *Q;           // [n][n] scrambled F^{-1}(probe)  (kSeq: updated in place)
    const float *amp;    // [npos][n][n] scrambled sqrt(ifftshift(I_meas)); kBatchCentred: centred I_meas
    float *sx, *sy;      // [npos] 1-based scan coordinates (kSeq: updated in place)
    double *grad;        // kBatch: [ns][n][n] sum_p Re(g)   (natural layout)
    double *qacc;        // kBatch: [n][n][2] scrambled sum_p F^{-1}(chi0) fs(-s)
    double *posdir;      // kBatch: [npos][2]
    double *err;         // [1] sum over positions and pixels of (A-M)^2
    float *inten;        // kSim: [npos][n][n] centred |Psi|^2
    const float2 *T;     // [ns][n][n] precomputed transmission slabs, or null (computed from V)
    const unsigned short *ampb;  // [npos][n][n] scrambled ifftshift(I_meas) as BF16 bits, or null (use amp)
    int npos;
    int pad_;
};

struct LaunchArgs {
    const TiltDev *tilts;   // device array
    const int2 *items;      // device array of (tilt, position), kBatch/kErr/kSim
    int nitems;
    unsigned *counter;      // work-queue counter (zeroed before the launch)
    float2 *save;           // saved waves per field in flight: [fields][slots][n][n]
    const float2 *pscr;     // propagator / N^2, scrambled layout
    const float2 *psep;     // separable propagator: [2n] = (Py / N, Px / N) scrambled, or null
    const float2 *twn;      // [n] twiddles e^{-2 pi i m/N} as [k2][n1]
    int nz, b, ns;
    float sdz;              // sigma * dz
    float center;           // round((N+1)/2)
    float step0, step1, step2;
    int seq_tilt;           // kSeq: index of the tilt to run
    int ckpt;               // 0: keep every slab's wave; k: keep every k-th, recompute the rest
    int slots;              // saved-wave slots (n x n complex) per field
    // kStep: one position (index step_k of tilt seq_tilt) at scan coordinates
    // (step_x, step_y); phase 1 = STEP02, phase 2 = STEP03
    int step_phase, step_k;
    int step04;             // STEP03 also applies RVol += step0 * Re(grad) (STEP04)
    float step_x, step_y;
    float2 *step_resi;      // [n][n] residual, scrambled (STEP02 writes it, STEP03 reads it)
    float *step_calc;       // [n][n] |Psi|^2, centred (STEP02)
    float2 *step_grad;      // [ns][n][n] complex gradient i conj(T) conj(psi) chi (STEP03)
    float *step_pos;        // [2] updated scan coordinates (STEP03)
    double *step_err;       // [1] += sum over pixels of (A - M)^2 (STEP02; zeroed by the host)
    unsigned *fault;        // [1] set by a kernel whose bounded wait gave up (may be null)
};

// saved-wave slots a CTA needs for ns slabs with checkpoint interval k
__host__ __device__ inline int save_slots(int ns, int k) {
    if (k <= 0 || k >= ns) return ns + 1;
    const int nseg = (ns + k - 1) / k;
    return nseg + k + 2;  // checkpoints, recomputed waves of a segment, parked adjoint state
}

// per-window-size kernel table (one translation unit per size, geo_<N>.cu)
struct GeoOps {
    int n, r1, ry1, nt;  // window, x residues, y residues of the scrambled layout, threads
    int cl;  // CTAs per field (thread-block cluster size; 1: one CTA per position)
    size_t smem;
    int staged;  // the adjoint's saved-wave rows are staged in shared memory by bulk copies
    int (*max_clusters)();  // clusters resident at once (cluster geometries)
    int (*positions)(int method, int adjoint, int mode, const LaunchArgs &a, int grid, cudaStream_t st);
    int (*prep_amp)(const float *meas_centred, float *amp_scr, long npos, cudaStream_t st);
    int (*prep_amp_bf16)(const float *meas_centred, unsigned short *i_scr, long npos, cudaStream_t st);
    int (*prep_prop)(const float *prop_centred, float2 *pscr, cudaStream_t st);
    int (*probe_q)(bool to_q, const float2 *in, float2 *out, const float2 *twn, cudaStream_t st);
};

// host-side launchers (return cudaError_t as int)
struct Plan {
    int n, r1, ry1, nt;
    int cl;
    int staged;        // GeoOps::staged
    int max_clusters;  // cl > 1: clusters resident at once (0: unknown)
    size_t smem;
    int ctas_per_sm;
    const GeoOps *ops;
};
// geometry `variant` (0: default) of window size n; plan_variants(n) of them
// exist, all with the default's scrambled layouts
bool plan_for(int n, Plan *p, int variant = 0);
// the first geometry of window n whose scrambled layouts have r1 x residues
// and ry1 y residues
bool plan_for_layout(int n, int r1, int ry1, Plan *p);
// the cluster geometry of window n for the sequential modes (kSeq, kStep),
// when one is compiled (the sessions of those modes use the one-CTA shape with
// its scrambled layouts, plan_for_layout)
bool plan_seq_for(int n, Plan *p);
int plan_variants(int n);
int launch_positions(const Plan &pl, int method, int adjoint, int mode, const LaunchArgs &a, int grid,
                     cudaStream_t st);
int launch_prep_amp(const Plan &pl, const float *meas_centred, float *amp_scr, long npos, cudaStream_t st);
int launch_prep_amp_bf16(const Plan &pl, const float *meas_centred, unsigned short *i_scr, long npos,
                         cudaStream_t st);
int launch_prep_prop(const Plan &pl, const float *prop_centred, float2 *pscr, cudaStream_t st);
int launch_probe_to_q(const Plan &pl, const float2 *probe, float2 *q, const float2 *twn, cudaStream_t st);
int launch_q_to_probe(const Plan &pl, const float2 *q, float2 *probe, const float2 *twn, cudaStream_t st);
// thread-local error message of the C ABI (mset_last_error)
void set_last_error(const char *msg);

int launch_apply_probe_pos(const TiltDev *tilts_host, int ntilts, int n, float step1, float step2, cudaStream_t st);
int launch_transmission(const TiltDev *tilts_dev, int ntilts, int n, int nz, int b, int ns, float sdz,
                        cudaStream_t st);
int launch_apply_batch(int n, int nz, int b, int ns, int method, float step0, float step1, float step2,
                       const TiltDev *tilts_host, int ntilts, cudaStream_t st);

}  // namespace mset
