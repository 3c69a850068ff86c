/*
 * mset_b200.h -- C ABI of the B200-native MSET multislice hot path.
 *
 * The MEX-compatible entry points keep the argument layout of the reference's
 * CUDA MEX module (jhlee0667/MSET, src/CUDA/mex_main.cu), so a caller that
 * drives `mset_cuda_kernel('upload' | 'run_mset' | 'run_sset' | 'error_mset' |
 * 'error_sset', STEM_data, measured_cells)` can call these instead:
 *
 *   reference mode string                     replacement
 *   'upload'     (mex_main.cu:42-95)          mset_upload / mset_mex_upload
 *   'run_mset'   (mex_main.cu:27-28, 98-155)  mset_run(mode = MSET_MODE_MSET)
 *   'run_sset'   (mex_main.cu:29-30, 98-155)  mset_run(mode = MSET_MODE_SSET)
 *   'error_mset' (mex_main.cu:31-32,157-184)  mset_error(mode = MSET_MODE_MSET)
 *   'error_sset' (mex_main.cu:33-34,157-184)  mset_error(mode = MSET_MODE_SSET)
 *   clear mset_cuda_kernel (Run_MSET_recon.m:174)   mset_destroy / mset_mex_clear
 *
 * and the per-position steps of the reference's CPU path (Run_MSET_recon.m:
 * 136-157): STEP02_FORWARD_4D(_SSET) -> mset_forward_position,
 * STEP03_BACK(_SSET) -> mset_adjoint_position.
 *
 * Array layouts are the MEX ones: MATLAB column-major arrays seen as C arrays
 * with the dimensions reversed (mex_tools.hpp:15-24):
 *   RVol         float [nz][n][n]            (MATLAB size n x n x nz)
 *   init_wave2D  float [n][n][2]             complex interleaved (re, im)
 *   prop2D       float [n][n][2]             centred propagator (the library ifftshifts it)
 *   measured     float [num_scan_pos][n][n]  one pattern per position, centred
 *                (cell element k = position k, mset.cu:201)
 *   scan_xlist / scan_ylist  float [num_scan_pos], 1-based pixels; x pairs with
 *                the fastest (MATLAB dim-1) axis.
 * All pointers in this header are HOST pointers unless a name ends in _dev.
 *
 * Window sizes n with compiled kernels: 24, 32, 48, 64, 96, 128, 160 (one CTA
 * per probe position) and 256 (one position per cluster of 4 CTAs, the field
 * split by rows over their shared memories).
 *
 * Every function returns 0 on success or a negative MSET_E* status; it never
 * aborts.  mset_last_error() gives the message of the calling thread's last
 * failure.  A session is not thread-safe; different sessions are independent.
 */
#ifndef MSET_B200_H
#define MSET_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MSET_MODE_MSET 1 /* multislice (run_main_mset, mset.cu:80-334) */
#define MSET_MODE_SSET 2 /* single slice (run_main_sset, mset.cu:345-546) */

#define MSET_ADJOINT_REF 0   /* reference V-gradient: conj of the wave saved after the slab (mset.cu:248-251) */
#define MSET_ADJOINT_EXACT 1 /* exact adjoint: conj of the wave entering the slab, spectral position derivative */

#define MSET_OK 0
#define MSET_E_ARG -1         /* invalid argument (null pointer, bad size, bad mode) */
#define MSET_E_UNSUPPORTED -2 /* window size without a compiled kernel, non-square window */
#define MSET_E_CUDA -3        /* CUDA runtime error (message in mset_last_error) */
#define MSET_E_STATE -4       /* call out of order (e.g. run before upload) */
#define MSET_E_NOMEM -5       /* device allocation failed */

typedef struct mset_session mset_session;

/* Scalars and arrays of the STEM_data struct fields read by the MEX upload
 * (mex_main.cu:59-75; field names kept). */
typedef struct {
    int32_t n;                 /* lateral size: RVol is n x n x nz (square, mset.cu:83) */
    int32_t nz;                /* depth */
    int32_t num_scan_pos;
    int32_t N_scan_x, N_scan_y;
    float sigma;               /* interaction constant, rad/(V*Angstrom) */
    float potential_pixelsize; /* Angstrom per voxel (slice thickness dz) */
    float alpha, E0;           /* accepted and ignored, as in the reference */
    float step_size[3];        /* object, probe, scan-position step sizes */
    int32_t slice_binning;
    const float *RVol;
    const float *init_wave2D;
    const float *prop2D;
    const float *scan_xlist;
    const float *scan_ylist;
    const float *measured;
} mset_upload_args;

/* ---- session lifetime ---------------------------------------------------- */
int mset_create(int device, mset_session **out);
int mset_destroy(mset_session *s);
const char *mset_last_error(void);
/* version string of the library */
const char *mset_version(void);

/* ---- MEX-compatible entry points ------------------------------------------ */
/* 'upload' (mex_main.cu:42-95): copy the struct fields and the measured
 * patterns to the device, zero the error accumulator.  Device buffers are kept
 * and reused when the next upload has the same sizes. */
int mset_upload(mset_session *s, const mset_upload_args *a);
/* the same with the patterns given as a table of num_scan_pos pointers to
 * n x n single-precision arrays (a->measured is not read): the MEX cell's
 * own arrays, cell k = position k (column-major cell order, mex_main.cu:87
 * borrows the cell the same way), copied to the device without a host-side
 * gather */
int mset_upload_cells(mset_session *s, const mset_upload_args *a, const float *const *measured_cells);
/* 'run_mset' / 'run_sset' (mex_main.cu:98-155): one sequential pass over all
 * positions with the reference's per-position updates of RVol, probe and scan
 * positions.  Outputs (host, caller-allocated): rvol_out [nz][n][n],
 * probe_out [n][n][2], scan_x_out / scan_y_out [num_scan_pos]; error_out may be
 * NULL (the MEX's nlhs == 4) or receives the accumulated error normalised as
 * mex_main.cu:150. */
int mset_run(mset_session *s, int mode, float *rvol_out, float *probe_out, float *scan_x_out,
             float *scan_y_out, float *error_out);
/* same as mset_run with the adjoint formula selectable (MSET_ADJOINT_*) */
int mset_run_ex(mset_session *s, int mode, int adjoint, float *rvol_out, float *probe_out,
                float *scan_x_out, float *scan_y_out, float *error_out);
/* 'error_mset' / 'error_sset' (mex_main.cu:157-184): forward pass over all
 * positions, error accumulated and normalised as mex_main.cu:179. */
int mset_error(mset_session *s, int mode, float *error_out);

/* ---- per-position steps of the reference's CPU path -----------------------
 * STEP02_FORWARD_4D(_SSET) and STEP03_BACK(_SSET) for one position of the
 * uploaded tilt (src/STEP02_FORWARD_4D.m:6-51, src/STEP03_BACK.m:6-39, called
 * from Run_MSET_recon.m:136-157), computed by the same fused kernel as
 * mset_run.  Real-space arrays are MATLAB's centred ones; spectra come back
 * centred (fftshift) as in the MATLAB code.  The probe shift follows the CUDA
 * module (IFFT -> phase -> FFT), which differs from the MATLAB path only on
 * the Nyquist lines of even windows at sub-pixel positions.
 *
 * mset_forward_position (STEP02): position k (0-based; selects the measured
 * pattern) at scan coordinates (row, col) (1-based pixels, STEM_data.row /
 * .col).  Every output may be NULL:
 *   calc_out  float [n][n]          |Psi|^2, centred (calculated_4D_data{k})
 *   resi_out  float [n][n][2]       residual, centred (resi_vec)
 *   waves_out float [ns][n][n][2]   wave after each slab (save_wave_f);
 *                                   SSET: [1][n][n][2], the shifted probe
 *   psi0_out  float [n][n][2]       shifted probe (tmp_probe_wave)
 *   err_out   float                 this position's error term,
 *                                   mean((sqrt(I_meas) - |Psi|)^2) / (N_scan_x N_scan_y)
 * The waves, the residual and (row, col) stay in the session for the
 * adjoint. */
int mset_forward_position(mset_session *s, int mode, int k, float row, float col, float *calc_out,
                          float *resi_out, float *waves_out, float *psi0_out, float *err_out);
/* mset_adjoint_position (STEP03, and STEP04 when update_rvol != 0): back-
 * propagates the residual of the preceding mset_forward_position of the same
 * mode, or resi_in (float [n][n][2], centred) when not NULL.  Updates the
 * session's probe as STEP03 does (probe -= step_size[1] shift(chi0)); with
 * update_rvol also RVol += step_size[0] Re(grad) (Run_MSET_recon.m:155).
 * Outputs (may be NULL):
 *   grad_out   float [nz][n][n][2]  i conj(T) conj(psi) chi per voxel, the slab's
 *                                   value on each of its voxels (STEM_data.grad)
 *   probe_out  float [n][n][2]      the updated probe
 *   rowcol_out float [2]            the updated scan coordinates (row, col)
 * A forward is consumed by one adjoint. */
int mset_adjoint_position(mset_session *s, int mode, int adjoint, const float *resi_in, int update_rvol,
                          float *grad_out, float *probe_out, float *rowcol_out);
/* the session's current volume and probe, as the per-position loop left them
 * on the device (Run_MSET_recon.m:136-157 keeps RVol and probe_wave between
 * positions; here they stay on the GPU, and a caller reads them once per tilt
 * instead of per position).  rvol_out float [nz][n][n], probe_out float
 * [n][n][2]; either may be NULL. */
int mset_read_state(mset_session *s, float *rvol_out, float *probe_out);
/* The sequential pass (mset_run) and the per-position steps walk one position
 * at a time, so one position's field is all the parallel work there is.
 * Where a cluster geometry is compiled for the window (n = 128: 8 CTAs of 16
 * rows), that field is split over a thread-block cluster (distributed shared
 * memory) and each position runs on several SMs; results are those of the
 * one-CTA kernel up to the order of the cluster's partial sums.
 * mset_set_sequential_split(s, 0) keeps one CTA per field; on by default.
 * mset_sequential_split returns the CTAs per field the sequential modes use. */
int mset_set_sequential_split(mset_session *s, int on);
int mset_sequential_split(mset_session *s);

/* global-session shims with the MEX's lifetime (one implicit session per
 * process, recreated by every upload, mex_main.cu:13, 56) */
int mset_mex_upload(const mset_upload_args *a);
int mset_mex_upload_cells(const mset_upload_args *a, const float *const *measured_cells);
int mset_mex_run(int mode, float *rvol_out, float *probe_out, float *scan_x_out, float *scan_y_out,
                 float *error_out);
int mset_mex_error(int mode, float *error_out);
int mset_mex_clear(void);
/* the implicit session (NULL before the first mset_mex_upload), for the
 * per-position steps and the other session calls from a MEX gateway */
mset_session *mset_mex_session(void);

/* ---- batched method --------------------------------------------------------
 * Every position of every tilt sees the same volume, probe and positions; the
 * gradients of all positions are accumulated in FP64 in one persistent launch.
 * Tilt j has its own beam-frame volume V_j, probe, scan positions and measured
 * patterns, all resident on the device. */
typedef struct {
    int32_t n, nz, slice_binning;
    int32_t method;  /* MSET_MODE_* */
    int32_t adjoint; /* MSET_ADJOINT_* */
    float sigma, potential_pixelsize;
    float step_size[3];
    int32_t ntilts;
    const int32_t *npos; /* [ntilts] positions per tilt */
    const float *prop2D; /* [n][n][2] centred propagator */
} mset_batch_args;

int mset_batch_setup(mset_session *s, const mset_batch_args *a);
/* tilt j: probe [n][n][2], scan_x/scan_y [npos_j], measured [npos_j][n][n]
 * (centred), volume [nz][n][n] in the tilt's beam frame (NULL keeps the
 * current one). */
int mset_batch_set_tilt(mset_session *s, int j, const float *probe, const float *scan_x,
                        const float *scan_y, const float *measured, const float *volume);
int mset_batch_set_volume(mset_session *s, int j, const float *volume);
/* one batched pass: forward + adjoint of every position of every tilt.
 * Outputs (host, any may be NULL: results then stay on the device):
 *   grad_out   [ntilts][ns][n][n] double: sum over positions of Re(g) per slab
 *   probe_out  [ntilts][n][n][2] double: sum over positions of F^{-1}(chi0) fs(-s),
 *              standard FFT order; its forward FFT is sum_p shift_{-s_p}(chi0_p),
 *              the probe direction of mset.cu:288-309 summed over positions
 *   posdir_out [sum npos][2] double: scan-position directions
 *   err_out    [ntilts] double: sum over positions and pixels of (A - M)^2 */
int mset_batch_gradient(mset_session *s, double *grad_out, double *probe_out, double *posdir_out,
                        double *err_out);
/* forward-only pass: err_out [ntilts] as above */
int mset_batch_error(mset_session *s, double *err_out);
/* forward-only pass writing |Psi|^2 (centred layout) of every position:
 * inten_out [sum npos][n][n] */
int mset_batch_simulate(mset_session *s, float *inten_out);
/* apply the last batched gradient: V_j += step0 * G_j, probe_j -= step1 * P_j,
 * positions += step2 * posdir */
int mset_batch_apply(mset_session *s);
/* read back tilt j's state: volume [nz][n][n], probe [n][n][2], scan_x/y [npos_j] */
int mset_batch_get_tilt(mset_session *s, int j, float *volume, float *probe, float *scan_x, float *scan_y);
/* device-side timing helpers for benchmarks: run the batched gradient pass
 * `reps` times on resident data and return the mean device time per pass in
 * milliseconds measured with CUDA events on the session stream */
int mset_batch_time(mset_session *s, int reps, double *ms_per_pass);
/* the plain form of the same pass, device-timed over reps: one launch per
 * tilt with one CTA per position (no persistent queue across tilts, no CUDA
 * graph, no checkpointing; saved waves for every position of the largest
 * tilt), the same kernel and results; the comparator of the batched form */
int mset_batch_time_plain(mset_session *s, int reps, double *ms_per_pass);
/* number of kernel launches issued by one mset_batch_gradient call */
int mset_batch_launch_count(mset_session *s);

/* storage of the measured patterns of a batched session: on != 0 keeps the
 * counts as BF16 (2 bytes per pixel instead of 4; integers up to 256 are
 * exact, larger counts are rounded to 8 significant bits) and takes the square
 * root in FP32 when they are read; the loss accumulates in FP32 per pixel and
 * FP64 per position.  Applies to measured patterns set after the call. */
int mset_batch_set_amplitude_bf16(mset_session *s, int on);

/* checkpointing of the batched pass: keep the wave entering every k-th slab
 * and recompute a segment's waves right before its adjoint (one extra forward
 * per slab, (ceil(ns/k) + k + 2) instead of (ns + 1) saved n x n waves per
 * resident CTA); k = 0 or k >= ns keeps every wave */
int mset_batch_set_checkpoint(mset_session *s, int k);

/* results of the last batched pass (mset_batch_gradient's outputs, any NULL)
 * without running a pass: for sessions run through a group */
int mset_batch_read_gradient(mset_session *s, double *grad, double *probe, double *posdir, double *err);

/* ---- autotuner ------------------------------------------------------------------
 * Has no counterpart in the reference (its per-position launches have no batch
 * shape).  Times the batched pass on a sample of the session's own positions
 * (up to 4 x SMs x resident CTAs) for every shape whose saved-wave storage fits
 * mem_budget_bytes (0: no limit) and keeps the fastest, or among shapes within
 * 1% of it the one using less memory.  Shape = kernel thread shape (two or
 * three compiled shapes for 64, 96, 128, 160 and 256: threads per CTA and the
 * register budget that goes with them, row padding, or the saved waves staged
 * by bulk copies) x persistent CTAs (SMs x CTAs per
 * SM, i.e. positions in flight) x checkpoint interval k in {0, 2, 4, 8, 16}
 * (k < slabs; k = 0 keeps every wave).  The choice stays with the session
 * (mset_batch_set_checkpoint overrides k).  MSET_E_NOMEM when no shape fits. */
typedef struct {
    int32_t grid;           /* persistent CTAs */
    int32_t ctas_per_sm;
    int32_t checkpoint;     /* k */
    int32_t candidates;     /* shapes timed */
    double us_per_position; /* measured device time per position at this shape */
    double save_bytes;      /* saved-wave storage at this shape */
    int32_t threads;        /* threads per CTA of the chosen kernel shape */
    int32_t staged;         /* 1: the shape stages the adjoint's saved-wave rows in
                               shared memory by bulk copies (TMA engine) */
} mset_tune_result;
int mset_batch_tune(mset_session *s, double mem_budget_bytes, mset_tune_result *out);
/* compiled kernel shapes of window size n that share the default shape's
 * scrambled Fourier layout (threads per CTA, register budget, padding or
 * staging; same results), and the choice of one for a session (0: default;
 * resets the tuned batch shape) */
int mset_batch_variants(int n);
int mset_batch_set_variant(mset_session *s, int variant);
/* the shape the next batched pass uses (candidates = 0; us_per_position = 0
 * when the session was not tuned) */
int mset_batch_get_tune(mset_session *s, mset_tune_result *out);

/* ---- groups: several tilt series of uneven size in one pass --------------------
 * Has no counterpart in the reference.  A group holds batched sessions of any
 * window sizes, slab counts, scan counts and tilt counts on one device; one
 * group pass runs every member's gradient pass (the member's own persistent
 * kernel over all its positions) and leaves the results on the device
 * (mset_batch_read_gradient).  Schedules: SERIAL, the members' kernels one after
 * another, each with all SMs; CONCURRENT, all members' kernels at once on
 * forked streams with the SMs split in proportion to each member's work
 * (mset_split_ctas), so that they finish together.  With use_graph the pass is
 * captured once as one CUDA graph and replayed (re-captured when a member's
 * buffers or shape change).  Sessions must outlive the group. */
#define MSET_GROUP_SERIAL 0
#define MSET_GROUP_CONCURRENT 1
typedef struct mset_group mset_group;
int mset_group_create(int device, mset_group **out);
int mset_group_destroy(mset_group *g);
int mset_group_add(mset_group *g, mset_session *s);
int mset_group_set_schedule(mset_group *g, int schedule);
/* tunes every member (the budget split in proportion to the members' full
 * saved-wave storage), then times both schedules and keeps the faster */
int mset_group_tune(mset_group *g, double mem_budget_bytes, int *schedule_out);
int mset_group_gradient(mset_group *g, int use_graph);
int mset_group_time(mset_group *g, int reps, int use_graph, double *ms_per_pass);
/* SM split of the concurrent schedule: one SM per member plus the remaining
 * SMs by largest remainder of work[i] / sum(work); grid_out[i] = SMs_i x
 * ctas_per_sm[i].  Pure host function. */
int mset_split_ctas(int count, const double *work, const int *ctas_per_sm, int sms, int *grid_out);

/* ---- batched iteration ---------------------------------------------------------
 * One iteration of the batched method on a cubic lab-frame volume rec (nv^3,
 * nv == nz, nv <= n, lateral zero-padding to the window):
 *   V_j  = pad(Func_inv_rot(rec, angles_j))          (STEP01_ROTATION.m:13)
 *   forward + loss + adjoint of every position of every tilt (one launch)
 *   rec += step0 * sum_j Func_rot(G_j)                (Run_MSET_recon.m:155, 179)
 *   positivity (Run_MSET_recon.m:183-185), TV / TV-FISTA of rec / max(rec)
 *   rescaled by max(rec) (Run_MSET_recon.m:267-270)
 *   probe_j -= step1 * sum_p shift_{-s}(chi0), positions += step2 * posdir
 * Every step is stream-ordered on the device; with use_graph the iteration is
 * captured once as a CUDA graph and replayed. */
typedef struct {
    int32_t nv;          /* reconstruction volume edge */
    const float *angles; /* [ntilts][3] (phi, theta, psi) in degrees (STEM_data.tilt_angles) */
    const float *vec1, *vec2, *vec3; /* rotation axes (main.m:25-27: [0 0 1], [0 1 0], [1 0 0]) */
    int32_t use_positivity;
    int32_t use_tv;
    double tv_lambda;
    int32_t tv_iter;
    int32_t tv_fista; /* 1: TV_FISTA_method, 0: TV_method */
} mset_iter_args;

int mset_batch_iteration_setup(mset_session *s, const mset_iter_args *a);
/* the same for a reconstruction of any shape [nv3][nv2][nv1] (a->nv is not
 * read): nv3 = the session's depth nz, nv1, nv2 <= n with n - nv1 and n - nv2
 * even (laterally centred in the window), each side a rotation line length
 * (mset_rotate_volume_nd) unless the volume is cubic; rec in / out of
 * mset_batch_set_rec / get_rec is then [nv3][nv2][nv1] */
int mset_batch_iteration_setup_nd(mset_session *s, const mset_iter_args *a, int nv1, int nv2, int nv3);
/* lab-frame volume in / out: host [nv][nv][nv] float ([nv3][nv2][nv1] after
 * mset_batch_iteration_setup_nd) */
int mset_batch_set_rec(mset_session *s, const float *rec);
int mset_batch_get_rec(mset_session *s, float *rec);
/* niter iterations; err_out [niter][ntilts] (sum of (A-M)^2 of the pass before
 * each update), tv_err_out [niter]; both nullable */
int mset_batch_iterate(mset_session *s, int niter, int use_graph, double *err_out, double *tv_err_out);
/* niter iterations with the backtracking line search of the reference's
 * reconstruction loop (Run_MSET_recon.m:106-252): each iteration saves rec,
 * probes and positions, applies one update without TV, runs the error pass of
 * the new state (mean over tilts of err / positions / n^2, mex_main.cu:179);
 * if that is not below the previous iteration's mean error (1e31 at the
 * start) the state is restored and all three step sizes are multiplied by
 * bls_parameter, until the object step falls below bls_parameter^5 times its
 * value at the call (then the call stops early, state restored).  After an
 * accepted update, TV as configured.  The session's step sizes stay reduced.
 * mean_err_out [niter] and step_out [niter][3] (nullable) hold the accepted
 * iterations' errors and step sizes; iters_out (nullable) their count.
 * Host-driven: one host synchronisation per trial. */
int mset_batch_iterate_bls(mset_session *s, int niter, double bls_parameter, double *mean_err_out,
                           float *step_out, int *iters_out);
/* captures the iteration graph, then times niter replays with CUDA events on
 * the session stream (the state advances by niter iterations) */
int mset_batch_iterate_time(mset_session *s, int niter, double *ms_per_iter);
/* one phase of an iteration, for tilt sharding over GPUs: phase 1 ends with
 * this session's lab-frame gradient sum in the FP64 device buffer of
 * mset_batch_device_info; the caller all-reduces it (NCCL, on the session
 * stream) and runs phase 2, the update.  Asynchronous on the session stream. */
int mset_batch_iterate_phase(mset_session *s, int phase, int use_graph);
/* device buffers and stream of the iteration: gacc [nv^3] double, the session
 * cudaStream_t, the per-tilt error sums [ntilts] double; any pointer may be NULL */
int mset_batch_device_info(mset_session *s, void **gacc_dev, size_t *gacc_count, void **stream,
                           double **err_dev);

/* ---- Fourier-shear tilt rotation --------------------------------------------
 * Func_rot_3Dvol_FourierShear (inverse = 0) and Func_inv_rot_3Dvol_FourierShear
 * (inverse = 1) (func_lib/Func_rot_3Dvol_FourierShear.m:5-19,
 * Func_inv_rot_3Dvol_FourierShear.m:5-20, Func_rotate_3Dvol_ROTmat_FourierShear.m:14-134):
 * rotation by the quaternion axes vec1..vec3 and angles (phi, theta, psi) in
 * degrees, split into sub-rotations of at most 11 degrees of four Fourier
 * shears each.  vol_in / vol_out: host [n][n][n] float (MATLAB n x n x n),
 * may alias.  All angles within 0.5 degrees: copied unchanged, as the
 * reference does.  Cubic volumes with n in {24, 32, 48, 64, 96, 128, 160, 256}
 * (256: each plane split over a 4-CTA thread-block cluster). */
int mset_rotate_volume(mset_session *s, const float *vol_in, float *vol_out, int n, const float *vec1,
                       const float *vec2, const float *vec3, double phi, double theta, double psi, int inverse);
/* The same rotation of a volume of any shape: vol_in / vol_out host
 * [n3][n2][n1] float (MATLAB n1 x n2 x n3), every side one of 24, 32, 48, 64,
 * 96, 128, 160, 192, 256 (e.g. 256 x 256 x 192).  The grids, the Nyquist
 * zeroing and the coefficient of each axis follow the reference for unequal
 * sides (Func_rotate_3Dvol_ROTmat_FourierShear.m:70-90,
 * SheerTransforms_for3Drot.m:16-49); each shear runs as batched 1D transforms
 * (forward along one plane axis, phase + both directions along the other,
 * inverse along the first). */
int mset_rotate_volume_nd(mset_session *s, const float *vol_in, float *vol_out, int n1, int n2, int n3,
                          const float *vec1, const float *vec2, const float *vec3, double phi, double theta,
                          double psi, int inverse);

/* ---- TV regularisation -------------------------------------------------------
 * TV_FISTA_method (fista = 1, func_lib/TV_FISTA_method.m:5-38) or TV_method
 * (fista = 0, func_lib/TV_method.m:5-28) on a 3D volume: niter projected
 * gradient iterations on the dual field (tau = 1/12, periodic differences),
 * output = input - lambda div(P), tv_error = lambda * sum |grad(output)|.
 * vol: host [n3][n2][n1] float, replaced by the output.  Dual variables in
 * FP32 (the reference's arithmetic is single once it meets the single input),
 * FISTA momentum step in FP64, error in FP64. */
int mset_tv(mset_session *s, float *vol, int n1, int n2, int n3, double lambda, int niter, int fista,
            double *tv_error);

/* ---- allocation-free batched pass -------------------------------------------
 * Has no counterpart in the reference.  For callers that cannot allocate
 * device memory (work issued while a CUDA graph is being captured, device
 * memory owned by a framework allocator or by MATLAB gpuArrays, real-time
 * pipelines that forbid allocation after start-up): one batched forward +
 * adjoint pass over the npos positions of ONE tilt, every input and output a
 * caller-owned DEVICE pointer, no cudaMalloc / cudaFree or allocating library
 * call.  Its scratch (saved waves, prepared propagator and probe spectrum,
 * probe accumulator, work counter) is a fixed 64 MiB device array inside the
 * library, held by every GPU that loads the library until the process exits.
 *   n in {24, 64, 128}; 0 < npos <= 131072; sizes whose (ns + 1) saved waves
 *   of n x n complex64 do not fit beside the fixed part of the 64 MiB are
 *   rejected with MSET_E_UNSUPPORTED (n = 128 allows ns up to ~500).
 * Inputs (device): rvol [nz][n][n] float, probe [n][n][2] float, prop2D
 * [n][n][2] centred, scan_x/scan_y [npos], measured [npos][n][n] centred
 * intensities, finite and non-negative (not checked here: mset_upload refuses
 * negative, NaN or infinite counts, this pass reads the caller's device
 * buffer as it is, and such counts give NaN gradients and errors).
 * Outputs (device), all overwritten: grad [ns][n][n] double,
 * probe_out [n][n][2] double (standard FFT order), posdir [npos][2] double,
 * err [1] double -- the same quantities mset_batch_gradient returns.
 * Work is queued on `stream` (a cudaStream_t, NULL = legacy default stream)
 * and is asynchronous.  The first call on a device resolves the scratch
 * array's device address (cudaGetSymbolAddress), and so does the first call
 * after the device's primary context was reset; make those calls before any
 * stream capture.  Every call shares the scratch array, so calls whose
 * work overlaps on the GPU (other streams, other host threads) race: order
 * them on one stream. */
int mset_batch_gradient_noalloc(int device, void *stream, int n, int nz, int slice_binning, int method,
                                int adjoint, float sigma, float potential_pixelsize, int npos,
                                const float *rvol_dev, const float *probe_dev, const float *prop2D_dev,
                                const float *scan_x_dev, const float *scan_y_dev, const float *measured_dev,
                                double *grad_dev, double *probe_out_dev, double *posdir_dev, double *err_dev);

#ifdef __cplusplus
}
#endif
#endif /* MSET_B200_H */
