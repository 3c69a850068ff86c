// mset_api.cu -- C ABI (include/mset_b200.h): sessions, validation, device
// buffers, the MEX-compatible modes and the batched method.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/mset_b200.h"
#include "mset_kernels.cuh"
#include "mset_rotate.cuh"
#include "mset_volume.cuh"

using namespace mset;

namespace {

thread_local std::string g_err;

int fail(int code, const char *fmt, ...) {
    char b[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(b, sizeof b, fmt, ap);
    va_end(ap);
    g_err = b;
    return code;
}

int cuda_fail(cudaError_t e, const char *where) {
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();  // not sticky: clear it so that later calls see a clean state
        return fail(MSET_E_NOMEM, "%s: out of device memory", where);
    }
    return fail(MSET_E_CUDA, "%s: %s", where, cudaGetErrorString(e));
}

// NVTX range around an entry point (visible in Nsight timelines; no cost
// without a tool attached)
struct Range {
    explicit Range(const char *name) { nvtxRangePushA(name); }
    ~Range() { nvtxRangePop(); }
};

#define CK(call)                                                    \
    do {                                                            \
        cudaError_t e_ = (call);                                    \
        if (e_ != cudaSuccess) return cuda_fail(e_, #call);         \
    } while (0)

#define CKL(rc, what)                                                                 \
    do {                                                                              \
        int rc_ = (rc);                                                               \
        if (rc_ != 0) return cuda_fail((cudaError_t)rc_, what);                       \
    } while (0)

template <class T>
struct DevBuf {
    T *p = nullptr;
    size_t n = 0;
    ~DevBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    // (re)allocate when the element count changes; contents undefined
    cudaError_t ensure(size_t count) {
        if (count == n && p) return cudaSuccess;
        release();
        if (count == 0) return cudaSuccess;
        cudaError_t e = cudaMalloc((void **)&p, sizeof(T) * count);
        if (e == cudaSuccess) n = count;
        return e;
    }
};

}  // namespace

namespace mset {
void set_last_error(const char *msg) { g_err = msg; }
}  // namespace mset

struct TiltBufs {
    DevBuf<float2> T;  // batched method: precomputed transmission slabs
    DevBuf<float> V;
    DevBuf<float2> Q;
    DevBuf<float> amp;
    DevBuf<unsigned short> ampb;  // BF16 counts (batched sessions with BF16 storage)
    DevBuf<float> sx, sy;
    DevBuf<double> grad, qacc, posdir;
    int npos = 0;
};

struct mset_session {
    int device = 0;
    cudaStream_t st = nullptr;
    int sms = 0;
    // geometry
    int n = 0, nz = 0, b = 1, ns = 0;
    int method = kMSET, adjoint = kREF;
    float sigma = 0, dz = 0, step[3] = {0, 0, 0};
    int nsx = 0, nsy = 0;
    Plan plan{};
    // sequential modes (kSeq, kStep): one field split over a thread-block
    // cluster, where such a geometry is compiled for n (seq_split: in use)
    Plan seq_plan{};
    bool has_seq = false;
    bool seq_split = true;
    bool ready = false;
    bool batch = false;
    // tilts (1 for the MEX-style session)
    std::vector<TiltBufs> tilts;
    std::vector<int> npos;
    std::vector<int> pos_off;
    int total_pos = 0;
    // shared buffers
    DevBuf<float2> pscr, psep, twn, save, tmpc;
    bool sep = false;  // propagator is numerically separable: P = Py (x) Px
    DevBuf<float> meas_tmp;
    DevBuf<double> err;
    DevBuf<TiltDev> d_tilts;
    DevBuf<int2> items;
    DevBuf<unsigned> counter;
    DevBuf<unsigned> fault;  // [1] set by a position kernel whose bounded wait gave up
    DevBuf<float> inten;
    int save_slots = 0;
    int ckpt = 0;  // checkpoint interval of the batched pass (0: keep every wave)
    int amp_bf16 = 0;  // batched sessions: measured counts stored as BF16
    int tuned_grid = 0;  // CTAs of the batched pass picked by the tuner (0: every resident CTA)
    double tuned_us_per_pos = 0;  // tuner's measured cost of one position at tuned_grid
    std::vector<TiltDev> h_tilts;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // batched iteration (rotate -> pass -> rotate back -> update -> TV)
    bool it_ready = false;
    int nv = 0;                  // cubic reconstruction: its edge; else 0
    int nv1 = 0, nv2 = 0, nv3 = 0;  // reconstruction [nv3][nv2][nv1] (x fastest)
    std::vector<RotPlan> plan_inv, plan_fwd;
    DevBuf<float> rec, gvol;
    DevBuf<float> bls_rec, bls_pos;  // line search: state before the tried update
    DevBuf<float2> bls_q;
    DevBuf<double> gacc, err_hist, tv_hist;
    DevBuf<unsigned> it_counter, mx_bits;
    DevBuf<float> mx;
    int it_pos = 1, it_tv = 0, it_tv_iter = 0, it_tv_fista = 1;
    double it_tv_lambda = 0;
    int hist_cap = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    cudaGraph_t phase_graph[2] = {nullptr, nullptr};
    cudaGraphExec_t phase_exec[2] = {nullptr, nullptr};
    int grid_cache = 0;
    // TV work buffers
    DevBuf<float> tv_in, tv_out, tv_P, tv_Y, tv_D;
    DevBuf<double> tv_err;
    // rotation work buffers
    // per-position steps (mset_forward_position / mset_adjoint_position)
    DevBuf<float2> step_resi, step_grad;
    DevBuf<float> step_calc, step_pos;
    DevBuf<double> step_err;
    int step_k = -1, step_mode = 0;  // position and method of the pending STEP02 (-1: none)
    float step_x = 0, step_y = 0;
    DevBuf<float> rot_vol;
    DevBuf<float2> rot_S, rot_tw;
    int rot_n = 0;
};

namespace {

int set_device(mset_session *s) {
    CK(cudaSetDevice(s->device));
    return 0;
}

// e^{-2 pi i m / n} in double, rounded to float
float2 twiddle(long m, int n) {
    const double a = -2.0 * M_PI * (double)(m % n) / (double)n;
    return make_float2((float)std::cos(a), (float)std::sin(a));
}

// twiddle tables of the plan's shape: e^{-2 pi i n1 k2 / N} as [k2][n1]
// (two-pass shape), or the three-phase shape's x table [a][k1] (a < r1) and
// y table [k1'][b] (b < ry1) one after the other
int upload_twiddles(mset_session *s) {
    const int n = s->plan.n, r1 = s->plan.r1, r2 = n / r1;
    const bool three = s->plan.ry1 != s->plan.r1;
    std::vector<float2> h(three ? 2 * n : n);
    if (three) {
        const int ry1 = s->plan.ry1, ry2 = n / ry1;
        for (int a = 0; a < r1; ++a)
            for (int k1 = 0; k1 < r2; ++k1) h[a * r2 + k1] = twiddle((long)a * k1, n);
        for (int k = 0; k < ry2; ++k)
            for (int b = 0; b < ry1; ++b) h[n + k * ry1 + b] = twiddle((long)b * k, n);
    } else {
        for (int k2 = 0; k2 < r2; ++k2)
            for (int n1 = 0; n1 < r1; ++n1) h[k2 * r1 + n1] = twiddle((long)n1 * k2, n);
    }
    CK(s->twn.ensure(h.size()));
    CK(cudaMemcpyAsync(s->twn.p, h.data(), sizeof(float2) * h.size(), cudaMemcpyHostToDevice, s->st));
    return 0;
}

// frequency index held at scrambled location L of a dimension with r residues
int scrambled_freq(int L, int n, int r) { return L / r + (n / r) * (L % r); }

// sequential: the session serves the sequential entry points (upload / run /
// per-position steps), whose one-CTA shape takes the scrambled layouts of the
// window's cluster geometry for that pass when one is compiled
int ensure_geometry(mset_session *s, int n, int nz, int b, float sigma, float dz, const float *prop,
                    bool sequential) {
    if (n <= 1 || nz <= 0 || b <= 0) return fail(MSET_E_ARG, "invalid sizes n=%d nz=%d slice_binning=%d", n, nz, b);
    Plan pl;
    if (!plan_for(n, &pl))
        return fail(MSET_E_UNSUPPORTED,
                    "window size %d has no compiled kernel (supported: 24, 32, 48, 64, 96, 128, 160, 256)", n);
    if (b > nz) b = nz;  // STEP00_INIT.m:126-128
    Plan sq{};
    bool has_seq = plan_seq_for(n, &sq);
    if (sequential && has_seq && (sq.r1 != pl.r1 || sq.ry1 != pl.ry1)) {
        Plan alt;
        if (plan_for_layout(n, sq.r1, sq.ry1, &alt)) pl = alt;
    }
    has_seq = has_seq && sq.r1 == pl.r1 && sq.ry1 == pl.ry1;
    if (pl.cl > 1) pl.max_clusters = pl.ops->max_clusters();
    s->plan = pl;
    s->seq_plan = sq;
    s->has_seq = has_seq;
    s->n = n;
    s->nz = nz;
    s->b = b;
    s->ns = (nz + b - 1) / b;
    s->sigma = sigma;
    s->dz = dz;
    const size_t n2 = (size_t)n * n;
    CK(s->pscr.ensure(n2));
    CK(s->tmpc.ensure(n2 * 2));
    int rc = upload_twiddles(s);
    if (rc) return rc;
    // propagator: host centred -> device -> scrambled / N^2
    CK(cudaMemcpyAsync(s->tmpc.p, prop, sizeof(float2) * n2, cudaMemcpyHostToDevice, s->st));
    CKL(launch_prep_prop(pl, reinterpret_cast<const float *>(s->tmpc.p), s->pscr.p, s->st), "prep_prop");
    // The Fresnel propagator exp(-i pi lambda dz (qx^2 + qy^2)) is a product
    // Py(ky) Px(kx) (Func_generate_propagator.m:36); when the caller's table
    // is separable to FP32 rounding, the kernels keep the two vectors in
    // shared memory instead of reading the n x n table.
    {
        const int h = (n + 1) / 2;
        std::vector<double> re(n2), im(n2);
        double mx = 0;
        for (int r = 0; r < n; ++r)
            for (int c = 0; c < n; ++c) {
                const size_t o = (size_t)((r + h) % n) * n + (c + h) % n;
                re[o] = prop[2 * ((size_t)r * n + c)];
                im[o] = prop[2 * ((size_t)r * n + c) + 1];
                mx = std::max(mx, std::hypot(re[o], im[o]));
            }
        const double a0 = re[0], b0 = im[0], d0 = a0 * a0 + b0 * b0;
        s->sep = d0 > 1e-6 * mx * mx;
        double e = 0;
        for (int ky = 0; ky < n && s->sep; ++ky)
            for (int kx = 0; kx < n; ++kx) {
                // u[ky] v[kx] with u = P[:, 0], v = P[0, :] / P[0][0]
                const double ur = re[(size_t)ky * n], ui = im[(size_t)ky * n];
                const double vr = (re[kx] * a0 + im[kx] * b0) / d0, vi = (im[kx] * a0 - re[kx] * b0) / d0;
                const double pr = ur * vr - ui * vi, pi = ur * vi + ui * vr;
                e = std::max(e, std::hypot(pr - re[(size_t)ky * n + kx], pi - im[(size_t)ky * n + kx]));
            }
        s->sep = s->sep && e <= 2e-6 * mx;
        if (s->sep) {
            std::vector<float2> h2(2 * n);
            for (int L = 0; L < n; ++L) {
                const int ky = scrambled_freq(L, n, pl.ry1), kx = scrambled_freq(L, n, pl.r1);
                h2[L] = make_float2((float)(re[(size_t)ky * n] / n), (float)(im[(size_t)ky * n] / n));
                const double vr = (re[kx] * a0 + im[kx] * b0) / d0, vi = (im[kx] * a0 - re[kx] * b0) / d0;
                h2[n + L] = make_float2((float)(vr / n), (float)(vi / n));
            }
            CK(s->psep.ensure(2 * n));
            CK(cudaMemcpyAsync(s->psep.p, h2.data(), sizeof(float2) * 2 * n, cudaMemcpyHostToDevice, s->st));
            CK(cudaStreamSynchronize(s->st));
        }
    }
    CK(s->err.ensure(64));
    CK(s->counter.ensure(1));
    return 0;
}

// saved-wave storage for a launch of `grid` CTAs: one slot set per field in
// flight (per CTA, or per cluster when a field is split over a cluster)
int ensure_save(mset_session *s, int grid) {
    const size_t per = (size_t)save_slots(s->ns, s->ckpt) * s->n * s->n;
    const size_t fields = (size_t)std::max(1, grid / std::max(1, s->plan.cl));
    if (s->save.n >= per * fields) return 0;
    cudaError_t e = s->save.ensure(per * fields);
    if (e != cudaSuccess) return cuda_fail(e, "allocating saved-wave buffers");
    s->save_slots = (int)fields;
    return 0;
}

int upload_tilt_probe(mset_session *s, TiltBufs &t, const float *probe) {
    const size_t n2 = (size_t)s->n * s->n;
    CK(t.Q.ensure(n2));
    CK(cudaMemcpyAsync(s->tmpc.p, probe, sizeof(float2) * n2, cudaMemcpyHostToDevice, s->st));
    CKL(launch_probe_to_q(s->plan, s->tmpc.p, t.Q.p, s->twn.p, s->st), "probe_to_q");
    return 0;
}

// measured patterns from one contiguous [npos][n][n] buffer, or (cells != NULL)
// from a table of npos pointers to n x n patterns: the MEX cell's own arrays,
// as the reference borrows them (mex_main.cu:87), with no host-side gather
int upload_tilt_measured(mset_session *s, TiltBufs &t, const float *meas, const float *const *cells = nullptr) {
    const size_t n2 = (size_t)s->n * s->n;
    const size_t cnt = n2 * t.npos;
    if (cnt == 0) return 0;
    // intensities are square-rooted in the loss: a negative, NaN or infinite
    // count would turn every gradient of the pass into NaN
    for (int p = 0; p < t.npos; ++p) {
        const float *m = cells ? cells[p] : meas + (size_t)p * n2;
        if (!m) return fail(MSET_E_ARG, "measured pattern %d is a null pointer", p);
        for (size_t i = 0; i < n2; ++i)
            if (!(m[i] >= 0.f) || m[i] == INFINITY)
                return fail(MSET_E_ARG, "measured pattern %d has a negative, NaN or infinite value at pixel %zu (%g)",
                            p, i, (double)m[i]);
    }
    CK(s->meas_tmp.ensure(std::max(s->meas_tmp.n, cnt)));
    if (cells) {
        for (int p = 0; p < t.npos; ++p)
            CK(cudaMemcpyAsync(s->meas_tmp.p + (size_t)p * n2, cells[p], sizeof(float) * n2, cudaMemcpyHostToDevice,
                               s->st));
    } else {
        CK(cudaMemcpyAsync(s->meas_tmp.p, meas, sizeof(float) * cnt, cudaMemcpyHostToDevice, s->st));
    }
    if (s->batch && s->amp_bf16) {
        t.amp.release();
        CK(t.ampb.ensure(cnt));
        CKL(launch_prep_amp_bf16(s->plan, s->meas_tmp.p, t.ampb.p, t.npos, s->st), "prep_amp_bf16");
    } else {
        t.ampb.release();
        CK(t.amp.ensure(cnt));
        CKL(launch_prep_amp(s->plan, s->meas_tmp.p, t.amp.p, t.npos, s->st), "prep_amp");
    }
    return 0;
}

int refresh_tilt_table(mset_session *s) {
    const int J = (int)s->tilts.size();
    s->h_tilts.assign(J, TiltDev{});
    for (int j = 0; j < J; ++j) {
        TiltBufs &t = s->tilts[j];
        TiltDev &d = s->h_tilts[j];
        d.V = t.V.p;
        d.Q = t.Q.p;
        d.amp = t.amp.p;
        d.ampb = t.ampb.p;
        d.sx = t.sx.p;
        d.sy = t.sy.p;
        d.grad = t.grad.p;
        d.qacc = t.qacc.p;
        d.posdir = t.posdir.p;
        d.err = s->err.p + j;
        d.inten = s->inten.p ? s->inten.p + (size_t)s->pos_off[j] * s->n * s->n : nullptr;
        d.T = s->batch ? t.T.p : nullptr;
        d.npos = t.npos;
    }
    CK(s->d_tilts.ensure(J));
    CK(cudaMemcpyAsync(s->d_tilts.p, s->h_tilts.data(), sizeof(TiltDev) * J, cudaMemcpyHostToDevice, s->st));
    return 0;
}

int persistent_grid(mset_session *s, int items) {
    const int cl = std::max(1, s->plan.cl);
    if (cl > 1) {
        // a field split over a cluster: as many clusters as fit at once
        int fields = s->plan.max_clusters > 0 ? s->plan.max_clusters : s->sms / cl;
        if (s->tuned_grid > 0) fields = std::min(fields, s->tuned_grid / cl);
        return std::max(1, std::min(fields, items)) * cl;
    }
    if (s->tuned_grid > 0) return std::max(1, std::min(s->tuned_grid, items));
    // CTAs resident per SM for this kernel's shared memory and threads
    const size_t per_sm_smem = 227 * 1024;
    int by_smem = (int)(per_sm_smem / (s->plan.smem + 1024));
    int by_thr = 2048 / s->plan.nt;
    int c = std::max(1, std::min(by_smem, by_thr));
    int g = s->sms * c;
    return std::max(1, std::min(g, items));
}

LaunchArgs base_args(mset_session *s) {
    LaunchArgs a{};
    a.tilts = s->d_tilts.p;
    a.items = s->items.p;
    a.nitems = s->total_pos;
    a.counter = s->counter.p;
    a.save = s->save.p;
    a.pscr = s->pscr.p;
    a.psep = s->sep ? s->psep.p : nullptr;
    a.twn = s->twn.p;
    a.nz = s->nz;
    a.b = s->b;
    a.ns = s->ns;
    a.sdz = s->sigma * s->dz;
    a.center = (float)std::round((s->n + 1.0f) / 2.0f);  // mset.cu:83
    a.step0 = s->step[0];
    a.step1 = s->step[1];
    a.step2 = s->step[2];
    a.seq_tilt = 0;
    a.ckpt = s->ckpt;
    a.slots = save_slots(s->ns, s->ckpt);
    a.fault = s->fault.p;
    return a;
}

// The position kernel waits, with a bound, for the bulk copies that stage
// its operands in shared memory; a wait that gave up sets the session's
// fault word.  Read (and clear) it where a call hands results back.
// the plan of the sequential modes: the cluster geometry when compiled and
// enabled, else the session's own
const Plan &seq_plan(const mset_session *s) { return (s->has_seq && s->seq_split) ? s->seq_plan : s->plan; }

int take_fault(mset_session *s) {
    if (!s->fault.p) return 0;
    unsigned f = 0;
    CK(cudaMemcpyAsync(&f, s->fault.p, sizeof(unsigned), cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    if (!f) return 0;
    CK(cudaMemsetAsync(s->fault.p, 0, sizeof(unsigned), s->st));
    CK(cudaStreamSynchronize(s->st));
    return fail(MSET_E_CUDA, "a bulk copy into shared memory did not complete within the position kernel's "
                             "bounded wait; the results of this call are invalid");
}

int effective_mode(const mset_session *s, int method, int mode) {
    return (mode == kBatch && method == kMSET && s->ckpt > 0 && s->ckpt < s->ns) ? kBatchCk : mode;
}

// host-side preparation of a queue launch with `grid` CTAs (not capturable:
// allocation and a pageable copy of the tilt table)
int queue_prepare(mset_session *s, int mode, int grid) {
    if (mode != kSim)
        for (const TiltBufs &t : s->tilts)
            if (t.npos > 0 && !t.amp.p && !t.ampb.p)
                return fail(MSET_E_STATE, "measured patterns not set for every tilt");
    int rc = ensure_save(s, grid);
    if (rc) return rc;
    return refresh_tilt_table(s);
}

// capturable part: reset the work counter and launch over the first nitems items
int queue_enqueue(mset_session *s, int method, int adjoint, int mode, int grid, int nitems) {
    CK(cudaMemsetAsync(s->counter.p, 0, sizeof(unsigned), s->st));
    LaunchArgs a = base_args(s);
    a.nitems = nitems;
    CKL(launch_positions(s->plan, method, adjoint, effective_mode(s, method, mode), a, grid, s->st),
        "position kernel launch");
    return 0;
}

int launch_queue(mset_session *s, int method, int adjoint, int mode) {
    const int grid = persistent_grid(s, s->total_pos);
    int rc = queue_prepare(s, mode, grid);
    if (rc) return rc;
    return queue_enqueue(s, method, adjoint, mode, grid, s->total_pos);
}

int check_mode(int mode) {
    if (mode != MSET_MODE_MSET && mode != MSET_MODE_SSET)
        return fail(MSET_E_ARG, "The running mode is not correct (choose 'run_mset', 'run_sset', 'error_mset' or 'error_sset')");
    return 0;
}

}  // namespace

extern "C" {

const char *mset_last_error(void) { return g_err.c_str(); }
const char *mset_version(void) { return "mset_b200 0.1 (sm_100a)"; }

int mset_create(int device, mset_session **out) {
    if (!out) return fail(MSET_E_ARG, "null output pointer");
    *out = nullptr;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) return fail(MSET_E_CUDA, "no CUDA device available (%s)", cudaGetErrorString(e));
    if (device < 0 || device >= ndev) return fail(MSET_E_ARG, "device %d out of range (%d devices)", device, ndev);
    mset_session *s = new mset_session();
    s->device = device;
    e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&s->sms, cudaDevAttrMultiProcessorCount, device);
    if (e == cudaSuccess) e = cudaEventCreate(&s->ev0);
    if (e == cudaSuccess) e = cudaEventCreate(&s->ev1);
    if (e == cudaSuccess) e = s->fault.ensure(1);
    if (e == cudaSuccess) e = cudaMemset(s->fault.p, 0, sizeof(unsigned));
    if (e != cudaSuccess) {
        delete s;
        return cuda_fail(e, "session setup");
    }
    *out = s;
    return 0;
}

int mset_destroy(mset_session *s) {
    if (!s) return 0;
    cudaSetDevice(s->device);
    if (s->st) cudaStreamSynchronize(s->st);
    if (s->graph_exec) cudaGraphExecDestroy(s->graph_exec);
    if (s->graph) cudaGraphDestroy(s->graph);
    for (int p = 0; p < 2; ++p) {
        if (s->phase_exec[p]) cudaGraphExecDestroy(s->phase_exec[p]);
        if (s->phase_graph[p]) cudaGraphDestroy(s->phase_graph[p]);
    }
    s->tilts.clear();
    if (s->ev0) cudaEventDestroy(s->ev0);
    if (s->ev1) cudaEventDestroy(s->ev1);
    if (s->st) cudaStreamDestroy(s->st);
    delete s;
    return 0;
}

static int upload_impl(mset_session *s, const mset_upload_args *a, const float *const *cells) {
    if (!s || !a) return fail(MSET_E_ARG, "null argument");
    if (!a->RVol || !a->init_wave2D || !a->prop2D || (!a->scan_xlist && a->num_scan_pos) ||
        (!a->scan_ylist && a->num_scan_pos) || (!a->measured && !cells && a->num_scan_pos))
        return fail(MSET_E_ARG, "null array in upload arguments");
    if (a->num_scan_pos < 0) return fail(MSET_E_ARG, "num_scan_pos < 0");
    if (a->N_scan_x <= 0 || a->N_scan_y <= 0) return fail(MSET_E_ARG, "N_scan_x and N_scan_y must be positive");
    if (a->slice_binning <= 0) return fail(MSET_E_ARG, "slice_binning must be a positive integer");
    int rc = set_device(s);
    if (rc) return rc;
    s->ready = false;
    s->batch = false;
    s->step_k = -1;
    s->ckpt = 0;  // the sequential kernels keep every slab's wave
    rc = ensure_geometry(s, a->n, a->nz, a->slice_binning, a->sigma, a->potential_pixelsize, a->prop2D, true);
    if (rc) return rc;
    s->step[0] = a->step_size[0];
    s->step[1] = a->step_size[1];
    s->step[2] = a->step_size[2];
    s->nsx = a->N_scan_x;
    s->nsy = a->N_scan_y;
    s->tilts.resize(1);
    TiltBufs &t = s->tilts[0];
    t.npos = a->num_scan_pos;
    s->npos.assign(1, t.npos);
    s->pos_off.assign(1, 0);
    s->total_pos = t.npos;
    const size_t n2 = (size_t)s->n * s->n;
    CK(t.V.ensure(n2 * s->nz));
    CK(cudaMemcpyAsync(t.V.p, a->RVol, sizeof(float) * n2 * s->nz, cudaMemcpyHostToDevice, s->st));
    rc = upload_tilt_probe(s, t, a->init_wave2D);
    if (rc) return rc;
    CK(t.sx.ensure(std::max(1, t.npos)));
    CK(t.sy.ensure(std::max(1, t.npos)));
    if (t.npos) {
        CK(cudaMemcpyAsync(t.sx.p, a->scan_xlist, sizeof(float) * t.npos, cudaMemcpyHostToDevice, s->st));
        CK(cudaMemcpyAsync(t.sy.p, a->scan_ylist, sizeof(float) * t.npos, cudaMemcpyHostToDevice, s->st));
    }
    rc = upload_tilt_measured(s, t, a->measured, cells);
    if (rc) return rc;
    // work list for the forward-only pass
    std::vector<int2> it(std::max(1, t.npos));
    for (int p = 0; p < t.npos; ++p) it[p] = make_int2(0, p);
    CK(s->items.ensure(it.size()));
    CK(cudaMemcpyAsync(s->items.p, it.data(), sizeof(int2) * it.size(), cudaMemcpyHostToDevice, s->st));
    CK(cudaMemsetAsync(s->err.p, 0, sizeof(double) * 64, s->st));  // mset.cu:38
    CK(cudaStreamSynchronize(s->st));
    s->ready = true;
    return 0;
}

int mset_upload(mset_session *s, const mset_upload_args *a) { return upload_impl(s, a, nullptr); }

int mset_upload_cells(mset_session *s, const mset_upload_args *a, const float *const *measured_cells) {
    if (!measured_cells && a && a->num_scan_pos) return fail(MSET_E_ARG, "null pattern table");
    return upload_impl(s, a, measured_cells);
}

int mset_run_ex(mset_session *s, int mode, int adjoint, float *rvol_out, float *probe_out, float *scan_x_out,
                float *scan_y_out, float *error_out) {
    if (!s) return fail(MSET_E_ARG, "null session");
    int rc = check_mode(mode);
    if (rc) return rc;
    if (adjoint != MSET_ADJOINT_REF && adjoint != MSET_ADJOINT_EXACT) return fail(MSET_E_ARG, "bad adjoint mode");
    if (!s->ready || s->batch) return fail(MSET_E_STATE, "run called before upload");
    if (!rvol_out || !probe_out || !scan_x_out || !scan_y_out) return fail(MSET_E_ARG, "null output array");
    rc = set_device(s);
    if (rc) return rc;
    // the pass overwrites the saved waves and updates V, probe and positions:
    // a pending STEP02 can no longer be followed by its STEP03
    s->step_k = -1;
    rc = ensure_save(s, 1);
    if (rc) return rc;
    rc = refresh_tilt_table(s);
    if (rc) return rc;
    LaunchArgs a = base_args(s);
    const Plan &sp = seq_plan(s);
    CKL(launch_positions(sp, mode, adjoint, kSeq, a, std::max(1, sp.cl), s->st), "sequential position kernel launch");
    TiltBufs &t = s->tilts[0];
    const size_t n2 = (size_t)s->n * s->n;
    CKL(launch_q_to_probe(s->plan, t.Q.p, s->tmpc.p, s->twn.p, s->st), "q_to_probe");
    CK(cudaMemcpyAsync(rvol_out, t.V.p, sizeof(float) * n2 * s->nz, cudaMemcpyDeviceToHost, s->st));
    CK(cudaMemcpyAsync(probe_out, s->tmpc.p, sizeof(float2) * n2, cudaMemcpyDeviceToHost, s->st));
    if (t.npos) {
        CK(cudaMemcpyAsync(scan_x_out, t.sx.p, sizeof(float) * t.npos, cudaMemcpyDeviceToHost, s->st));
        CK(cudaMemcpyAsync(scan_y_out, t.sy.p, sizeof(float) * t.npos, cudaMemcpyDeviceToHost, s->st));
    }
    double e = 0;
    CK(cudaMemcpyAsync(&e, s->err.p, sizeof(double), cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    if (error_out) *error_out = (float)(e / ((double)s->nsx * s->nsy) / (double)n2);  // mex_main.cu:150
    return take_fault(s);
}

int mset_run(mset_session *s, int mode, float *rvol_out, float *probe_out, float *scan_x_out, float *scan_y_out,
             float *error_out) {
    Range range_("mset_run");
    return mset_run_ex(s, mode, MSET_ADJOINT_REF, rvol_out, probe_out, scan_x_out, scan_y_out, error_out);
}

int mset_error(mset_session *s, int mode, float *error_out) {
    Range range_("mset_error");
    if (!s) return fail(MSET_E_ARG, "null session");
    int rc = check_mode(mode);
    if (rc) return rc;
    if (!s->ready || s->batch) return fail(MSET_E_STATE, "error called before upload");
    if (!error_out) return fail(MSET_E_ARG, "null output");
    rc = set_device(s);
    if (rc) return rc;
    if (s->total_pos > 0) {
        rc = launch_queue(s, mode, kREF, kErr);
        if (rc) return rc;
    }
    double e = 0;
    CK(cudaMemcpyAsync(&e, s->err.p, sizeof(double), cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    const double n2 = (double)s->n * s->n;
    *error_out = (float)(e / ((double)s->nsx * s->nsy) / n2);  // mex_main.cu:179
    return 0;
}

// ---- per-position steps (STEP02_FORWARD_4D / STEP03_BACK) ---------------------

// centred (MATLAB fftshift) index of scrambled location L: frequency scr(L)
// moved by floor(n/2)
static int centred_of_scrambled(int L, int n, int r) {
    const int k = scrambled_freq(L, n, r);
    int c = k - (n + 1) / 2;
    return c < 0 ? c + n : c;
}

int mset_forward_position(mset_session *s, int mode, int k, float row, float col, float *calc_out,
                          float *resi_out, float *waves_out, float *psi0_out, float *err_out) {
    Range range_("mset_forward_position");
    if (!s) return fail(MSET_E_ARG, "null session");
    int rc = check_mode(mode);
    if (rc) return rc;
    if (!s->ready || s->batch) return fail(MSET_E_STATE, "forward_position called before upload");
    TiltBufs &t = s->tilts[0];
    if (k < 0 || k >= t.npos) return fail(MSET_E_ARG, "position %d out of range (%d positions)", k, t.npos);
    if (!std::isfinite(row) || !std::isfinite(col)) return fail(MSET_E_ARG, "non-finite scan coordinates");
    rc = set_device(s);
    if (rc) return rc;
    s->step_k = -1;
    rc = ensure_save(s, 1);
    if (!rc) rc = refresh_tilt_table(s);
    if (rc) return rc;
    const int n = s->n;
    const size_t n2 = (size_t)n * n;
    const int ns = mode == MSET_MODE_SSET ? 1 : s->ns;
    CK(s->step_resi.ensure(n2));
    CK(s->step_calc.ensure(n2));
    CK(s->step_err.ensure(1));
    CK(cudaMemsetAsync(s->step_err.p, 0, sizeof(double), s->st));
    LaunchArgs a = base_args(s);
    a.step_phase = 1;
    a.step_k = k;
    a.step_x = row;
    a.step_y = col;
    a.step_resi = s->step_resi.p;
    a.step_calc = s->step_calc.p;
    a.step_err = s->step_err.p;
    const Plan &sp = seq_plan(s);
    CKL(launch_positions(sp, mode, kREF, kStep, a, std::max(1, sp.cl), s->st), "STEP02 launch");
    // the waves of field 0: slot 0 = psi0, slot s + 1 = wave after slab s
    std::vector<float2> resi(resi_out ? n2 : 0);
    if (resi_out)
        CK(cudaMemcpyAsync(resi.data(), s->step_resi.p, sizeof(float2) * n2, cudaMemcpyDeviceToHost, s->st));
    if (calc_out) CK(cudaMemcpyAsync(calc_out, s->step_calc.p, sizeof(float) * n2, cudaMemcpyDeviceToHost, s->st));
    if (waves_out) {
        // STEP02_FORWARD_4D.m:33 (after each slab); SSET: psi0 (STEP02_FORWARD_4D_SSET.m:16)
        const float2 *src = s->save.p + (mode == MSET_MODE_SSET ? 0 : n2);
        CK(cudaMemcpyAsync(waves_out, src, sizeof(float2) * n2 * ns, cudaMemcpyDeviceToHost, s->st));
    }
    if (psi0_out) CK(cudaMemcpyAsync(psi0_out, s->save.p, sizeof(float2) * n2, cudaMemcpyDeviceToHost, s->st));
    double e = 0;
    CK(cudaMemcpyAsync(&e, s->step_err.p, sizeof(double), cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    if (resi_out) {
        float2 *ro = reinterpret_cast<float2 *>(resi_out);
        for (int Ly = 0; Ly < n; ++Ly) {
            const int r = centred_of_scrambled(Ly, n, s->plan.ry1);
            for (int Lx = 0; Lx < n; ++Lx)
                ro[(size_t)r * n + centred_of_scrambled(Lx, n, s->plan.r1)] = resi[(size_t)Ly * n + Lx];
        }
    }
    // mean over the pattern / (N_scan_x N_scan_y)  (STEP02_FORWARD_4D.m:46-48)
    if (err_out) *err_out = (float)(e / (double)n2 / ((double)s->nsx * s->nsy));
    s->step_k = k;
    s->step_mode = mode;
    s->step_x = row;
    s->step_y = col;
    return 0;
}

int mset_adjoint_position(mset_session *s, int mode, int adjoint, const float *resi_in, int update_rvol,
                          float *grad_out, float *probe_out, float *rowcol_out) {
    Range range_("mset_adjoint_position");
    if (!s) return fail(MSET_E_ARG, "null session");
    int rc = check_mode(mode);
    if (rc) return rc;
    if (adjoint != MSET_ADJOINT_REF && adjoint != MSET_ADJOINT_EXACT) return fail(MSET_E_ARG, "bad adjoint mode");
    if (!s->ready || s->batch) return fail(MSET_E_STATE, "adjoint_position called before upload");
    if (s->step_k < 0 || s->step_mode != mode)
        return fail(MSET_E_STATE, "adjoint_position needs a preceding forward_position of the same mode");
    rc = set_device(s);
    if (rc) return rc;
    const int n = s->n;
    const size_t n2 = (size_t)n * n;
    const int ns = mode == MSET_MODE_SSET ? 1 : s->ns;
    if (resi_in) {
        const float2 *ri = reinterpret_cast<const float2 *>(resi_in);
        std::vector<float2> scr(n2);
        for (int Ly = 0; Ly < n; ++Ly) {
            const int r = centred_of_scrambled(Ly, n, s->plan.ry1);
            for (int Lx = 0; Lx < n; ++Lx)
                scr[(size_t)Ly * n + Lx] = ri[(size_t)r * n + centred_of_scrambled(Lx, n, s->plan.r1)];
        }
        CK(cudaMemcpyAsync(s->step_resi.p, scr.data(), sizeof(float2) * n2, cudaMemcpyHostToDevice, s->st));
        CK(cudaStreamSynchronize(s->st));
    }
    CK(s->step_grad.ensure(n2 * ns));
    CK(s->step_pos.ensure(2));
    LaunchArgs a = base_args(s);
    a.step_phase = 2;
    a.step_k = s->step_k;
    a.step_x = s->step_x;
    a.step_y = s->step_y;
    a.step04 = update_rvol ? 1 : 0;
    a.step_resi = s->step_resi.p;
    a.step_grad = s->step_grad.p;
    a.step_pos = s->step_pos.p;
    const Plan &sp = seq_plan(s);
    CKL(launch_positions(sp, mode, adjoint, kStep, a, std::max(1, sp.cl), s->st), "STEP03 launch");
    TiltBufs &t = s->tilts[0];
    std::vector<float2> g(grad_out ? n2 * ns : 0);
    if (grad_out)
        CK(cudaMemcpyAsync(g.data(), s->step_grad.p, sizeof(float2) * n2 * ns, cudaMemcpyDeviceToHost, s->st));
    if (probe_out) {
        CKL(launch_q_to_probe(s->plan, t.Q.p, s->tmpc.p, s->twn.p, s->st), "q_to_probe");
        CK(cudaMemcpyAsync(probe_out, s->tmpc.p, sizeof(float2) * n2, cudaMemcpyDeviceToHost, s->st));
    }
    if (rowcol_out) CK(cudaMemcpyAsync(rowcol_out, s->step_pos.p, sizeof(float) * 2, cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    if (grad_out) {
        // the slab's value on each of its voxels (STEP03_BACK.m:18-22; SSET: every z,
        // STEP03_BACK_SSET.m:13-14)
        float2 *go = reinterpret_cast<float2 *>(grad_out);
        for (int z = 0; z < s->nz; ++z) {
            const int sl = mode == MSET_MODE_SSET ? 0 : z / s->b;
            std::memcpy(go + (size_t)z * n2, g.data() + (size_t)sl * n2, sizeof(float2) * n2);
        }
    }
    s->step_k = -1;
    return take_fault(s);
}

int mset_set_sequential_split(mset_session *s, int on) {
    if (!s) return fail(MSET_E_ARG, "null session");
    s->seq_split = on != 0;
    return 0;
}

int mset_sequential_split(mset_session *s) {
    if (!s) return fail(MSET_E_ARG, "null session");
    return (s->has_seq && s->seq_split) ? seq_plan(s).cl : 1;
}

int mset_read_state(mset_session *s, float *rvol_out, float *probe_out) {
    if (!s) return fail(MSET_E_ARG, "null session");
    if (!s->ready || s->batch) return fail(MSET_E_STATE, "read_state called before upload");
    int rc = set_device(s);
    if (rc) return rc;
    TiltBufs &t = s->tilts[0];
    const size_t n2 = (size_t)s->n * s->n;
    if (rvol_out) CK(cudaMemcpyAsync(rvol_out, t.V.p, sizeof(float) * n2 * s->nz, cudaMemcpyDeviceToHost, s->st));
    if (probe_out) {
        CKL(launch_q_to_probe(s->plan, t.Q.p, s->tmpc.p, s->twn.p, s->st), "q_to_probe");
        CK(cudaMemcpyAsync(probe_out, s->tmpc.p, sizeof(float2) * n2, cudaMemcpyDeviceToHost, s->st));
    }
    CK(cudaStreamSynchronize(s->st));
    return 0;
}

// ---- global-session shims --------------------------------------------------
static mset_session *g_mex = nullptr;

int mset_mex_upload(const mset_upload_args *a) {
    if (!g_mex) {
        int rc = mset_create(0, &g_mex);
        if (rc) return rc;
    }
    return mset_upload(g_mex, a);
}
int mset_mex_upload_cells(const mset_upload_args *a, const float *const *measured_cells) {
    if (!g_mex) {
        int rc = mset_create(0, &g_mex);
        if (rc) return rc;
    }
    return mset_upload_cells(g_mex, a, measured_cells);
}
int mset_mex_run(int mode, float *rvol_out, float *probe_out, float *scan_x_out, float *scan_y_out, float *error_out) {
    if (!g_mex) return fail(MSET_E_STATE, "run called before upload");
    return mset_run(g_mex, mode, rvol_out, probe_out, scan_x_out, scan_y_out, error_out);
}
int mset_mex_error(int mode, float *error_out) {
    if (!g_mex) return fail(MSET_E_STATE, "error called before upload");
    return mset_error(g_mex, mode, error_out);
}
int mset_mex_clear(void) {
    int rc = mset_destroy(g_mex);
    g_mex = nullptr;
    return rc;
}
mset_session *mset_mex_session(void) { return g_mex; }

// ---- batched method ---------------------------------------------------------
int mset_batch_setup(mset_session *s, const mset_batch_args *a) {
    if (!s || !a || !a->prop2D || !a->npos) return fail(MSET_E_ARG, "null argument");
    if (a->ntilts <= 0) return fail(MSET_E_ARG, "ntilts must be positive");
    if (a->method != MSET_MODE_MSET && a->method != MSET_MODE_SSET) return fail(MSET_E_ARG, "bad method");
    if (a->adjoint != MSET_ADJOINT_REF && a->adjoint != MSET_ADJOINT_EXACT) return fail(MSET_E_ARG, "bad adjoint");
    int rc = set_device(s);
    if (rc) return rc;
    s->ready = false;
    rc = ensure_geometry(s, a->n, a->nz, a->slice_binning, a->sigma, a->potential_pixelsize, a->prop2D, false);
    if (rc) return rc;
    s->method = a->method;
    s->adjoint = a->adjoint;
    s->batch = true;
    for (int i = 0; i < 3; ++i) s->step[i] = a->step_size[i];
    s->nsx = s->nsy = 1;
    const int J = a->ntilts;
    s->tilts.resize(J);
    s->npos.assign(a->npos, a->npos + J);
    s->pos_off.assign(J, 0);
    s->total_pos = 0;
    const size_t n2 = (size_t)s->n * s->n;
    const int nsg = a->method == MSET_MODE_SSET ? 1 : s->ns;
    std::vector<int2> it;
    for (int j = 0; j < J; ++j) {
        if (a->npos[j] < 0) return fail(MSET_E_ARG, "negative position count for tilt %d", j);
        s->pos_off[j] = s->total_pos;
        s->total_pos += a->npos[j];
        TiltBufs &t = s->tilts[j];
        t.npos = a->npos[j];
        CK(t.V.ensure(n2 * s->nz));
        CK(t.T.ensure(n2 * nsg));
        CK(t.Q.ensure(n2));
        CK(t.sx.ensure(std::max(1, t.npos)));
        CK(t.sy.ensure(std::max(1, t.npos)));
        CK(t.grad.ensure(n2 * nsg));
        CK(t.qacc.ensure(n2 * 2));
        CK(t.posdir.ensure(2 * std::max(1, t.npos)));
        CK(cudaMemsetAsync(t.V.p, 0, sizeof(float) * n2 * s->nz, s->st));
        for (int p = 0; p < t.npos; ++p) it.push_back(make_int2(j, p));
    }
    // position-major order inside each tilt; tilts follow each other so the
    // active gradient accumulators stay in L2
    if (it.empty()) it.push_back(make_int2(0, 0));
    CK(s->items.ensure(it.size()));
    CK(cudaMemcpyAsync(s->items.p, it.data(), sizeof(int2) * it.size(), cudaMemcpyHostToDevice, s->st));
    if ((size_t)J > 64) {
        CK(s->err.ensure(J));
    }
    CK(cudaStreamSynchronize(s->st));
    s->batch = true;
    s->ready = true;
    return 0;
}

static int batch_ok(mset_session *s) {
    if (!s) return fail(MSET_E_ARG, "null session");
    if (!s->ready || !s->batch) return fail(MSET_E_STATE, "batched call before mset_batch_setup");
    return set_device(s);
}

int mset_batch_set_tilt(mset_session *s, int j, const float *probe, const float *scan_x, const float *scan_y,
                        const float *measured, const float *volume) {
    int rc = batch_ok(s);
    if (rc) return rc;
    if (j < 0 || j >= (int)s->tilts.size()) return fail(MSET_E_ARG, "tilt index %d out of range", j);
    TiltBufs &t = s->tilts[j];
    if (probe) {
        rc = upload_tilt_probe(s, t, probe);
        if (rc) return rc;
    }
    if (t.npos) {
        if (scan_x) CK(cudaMemcpyAsync(t.sx.p, scan_x, sizeof(float) * t.npos, cudaMemcpyHostToDevice, s->st));
        if (scan_y) CK(cudaMemcpyAsync(t.sy.p, scan_y, sizeof(float) * t.npos, cudaMemcpyHostToDevice, s->st));
        if (measured) {
            rc = upload_tilt_measured(s, t, measured);
            if (rc) return rc;
        }
    }
    if (volume) {
        CK(cudaMemcpyAsync(t.V.p, volume, sizeof(float) * (size_t)s->n * s->n * s->nz, cudaMemcpyHostToDevice,
                           s->st));
    }
    CK(cudaStreamSynchronize(s->st));
    return 0;
}

int mset_batch_set_volume(mset_session *s, int j, const float *volume) {
    if (!volume) return fail(MSET_E_ARG, "null volume");
    return mset_batch_set_tilt(s, j, nullptr, nullptr, nullptr, nullptr, volume);
}

static int batch_zero(mset_session *s) {
    const size_t n2 = (size_t)s->n * s->n;
    const int nsg = s->method == MSET_MODE_SSET ? 1 : s->ns;
    for (auto &t : s->tilts) {
        CK(cudaMemsetAsync(t.grad.p, 0, sizeof(double) * n2 * nsg, s->st));
        CK(cudaMemsetAsync(t.qacc.p, 0, sizeof(double) * n2 * 2, s->st));
    }
    CK(cudaMemsetAsync(s->err.p, 0, sizeof(double) * s->tilts.size(), s->st));
    return 0;
}

// transmission slabs of every tilt from the current volumes
static int batch_transmission_enqueue(mset_session *s) {
    const int nsg = s->method == MSET_MODE_SSET ? 1 : s->ns;
    const int b = s->method == MSET_MODE_SSET ? s->nz : s->b;
    CKL(launch_transmission(s->d_tilts.p, (int)s->tilts.size(), s->n, s->nz, b, nsg, s->sigma * s->dz, s->st),
        "transmission");
    return 0;
}

static int batch_transmission(mset_session *s) {
    int rc = refresh_tilt_table(s);
    if (rc) return rc;
    return batch_transmission_enqueue(s);
}

static int batch_pass(mset_session *s) {
    int rc = batch_zero(s);
    if (rc) return rc;
    if (s->total_pos == 0) return 0;
    rc = batch_transmission(s);
    if (rc) return rc;
    return launch_queue(s, s->method, s->adjoint, kBatch);
}

// The plain form of the pass: one launch per tilt with one CTA per position
// (no persistent work queue across tilts, no CUDA graph), every slab's wave
// kept (no checkpointing); the same kernel and arithmetic as batch_pass.
static int plain_pass(mset_session *s) {
    int rc = batch_zero(s);
    if (rc) return rc;
    if (s->total_pos == 0) return 0;
    rc = batch_transmission(s);
    if (rc) return rc;
    const int cl = std::max(1, s->plan.cl);
    for (size_t j = 0; j < s->tilts.size(); ++j) {
        const int np = s->tilts[j].npos;
        if (np == 0) continue;
        CK(cudaMemsetAsync(s->counter.p, 0, sizeof(unsigned), s->st));
        LaunchArgs a = base_args(s);
        a.items = s->items.p + s->pos_off[j];
        a.nitems = np;
        a.ckpt = 0;
        a.slots = save_slots(s->ns, 0);
        CKL(launch_positions(s->plan, s->method, s->adjoint, kBatch, a, np * cl, s->st), "plain position launch");
    }
    return 0;
}

int mset_batch_time_plain(mset_session *s, int reps, double *ms_per_pass) {
    Range range_("mset_batch_time_plain");
    int rc = batch_ok(s);
    if (rc) return rc;
    if (reps <= 0 || !ms_per_pass) return fail(MSET_E_ARG, "bad arguments");
    int maxp = 0;
    for (const TiltBufs &t : s->tilts) maxp = std::max(maxp, t.npos);
    // saved waves for one field per position of the largest tilt, all slabs
    const int ck = s->ckpt;
    s->ckpt = 0;
    rc = queue_prepare(s, kBatch, std::max(1, maxp) * std::max(1, s->plan.cl));
    if (!rc) rc = plain_pass(s);  // warm-up
    if (rc) {
        s->ckpt = ck;
        return rc;
    }
    cudaError_t e = cudaEventRecord(s->ev0, s->st);
    for (int r = 0; r < reps && e == cudaSuccess && !rc; ++r) rc = plain_pass(s);
    if (e == cudaSuccess) e = cudaEventRecord(s->ev1, s->st);
    if (e == cudaSuccess) e = cudaEventSynchronize(s->ev1);
    s->ckpt = ck;
    if (rc) return rc;
    if (e != cudaSuccess) return cuda_fail(e, "timing the plain pass");
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, s->ev0, s->ev1));
    *ms_per_pass = ms / reps;
    return take_fault(s);
}

int mset_batch_gradient(mset_session *s, double *grad_out, double *probe_out, double *posdir_out, double *err_out) {
    Range range_("mset_batch_gradient");
    int rc = batch_ok(s);
    if (rc) return rc;
    rc = batch_pass(s);
    if (rc) return rc;
    return mset_batch_read_gradient(s, grad_out, probe_out, posdir_out, err_out);
}

int mset_batch_read_gradient(mset_session *s, double *grad_out, double *probe_out, double *posdir_out,
                             double *err_out) {
    int rc = batch_ok(s);
    if (rc) return rc;
    const size_t n2 = (size_t)s->n * s->n;
    const int nsg = s->method == MSET_MODE_SSET ? 1 : s->ns;
    const int J = (int)s->tilts.size();
    for (int j = 0; j < J; ++j) {
        TiltBufs &t = s->tilts[j];
        if (grad_out)
            CK(cudaMemcpyAsync(grad_out + (size_t)j * nsg * n2, t.grad.p, sizeof(double) * nsg * n2,
                               cudaMemcpyDeviceToHost, s->st));
        if (probe_out) {
            // device layout is scrambled; the caller gets standard FFT order
            std::vector<double> tmp(2 * n2);
            CK(cudaMemcpyAsync(tmp.data(), t.qacc.p, sizeof(double) * 2 * n2, cudaMemcpyDeviceToHost, s->st));
            CK(cudaStreamSynchronize(s->st));
            const int n = s->n;
            double *o = probe_out + (size_t)j * 2 * n2;
            for (int ly = 0; ly < n; ++ly)
                for (int lx = 0; lx < n; ++lx) {
                    const int ky = scrambled_freq(ly, n, s->plan.ry1), kx = scrambled_freq(lx, n, s->plan.r1);
                    o[2 * ((size_t)ky * n + kx)] = tmp[2 * ((size_t)ly * n + lx)];
                    o[2 * ((size_t)ky * n + kx) + 1] = tmp[2 * ((size_t)ly * n + lx) + 1];
                }
        }
        if (posdir_out && t.npos)
            CK(cudaMemcpyAsync(posdir_out + 2 * (size_t)s->pos_off[j], t.posdir.p, sizeof(double) * 2 * t.npos,
                               cudaMemcpyDeviceToHost, s->st));
    }
    if (err_out) CK(cudaMemcpyAsync(err_out, s->err.p, sizeof(double) * J, cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    return take_fault(s);
}

int mset_batch_error(mset_session *s, double *err_out) {
    Range range_("mset_batch_error");
    int rc = batch_ok(s);
    if (rc) return rc;
    CK(cudaMemsetAsync(s->err.p, 0, sizeof(double) * s->tilts.size(), s->st));
    if (s->total_pos) {
        rc = batch_transmission(s);
        if (rc) return rc;
        rc = launch_queue(s, s->method, kREF, kErr);
        if (rc) return rc;
    }
    if (err_out) CK(cudaMemcpyAsync(err_out, s->err.p, sizeof(double) * s->tilts.size(), cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    return 0;
}

int mset_batch_simulate(mset_session *s, float *inten_out) {
    Range range_("mset_batch_simulate");
    int rc = batch_ok(s);
    if (rc) return rc;
    if (!inten_out) return fail(MSET_E_ARG, "null output");
    const size_t n2 = (size_t)s->n * s->n;
    CK(s->inten.ensure(std::max<size_t>(1, n2 * s->total_pos)));
    if (s->total_pos) {
        rc = batch_transmission(s);
        if (rc) return rc;
        rc = launch_queue(s, s->method, kREF, kSim);
        if (rc) return rc;
        CK(cudaMemcpyAsync(inten_out, s->inten.p, sizeof(float) * n2 * s->total_pos, cudaMemcpyDeviceToHost, s->st));
    }
    CK(cudaStreamSynchronize(s->st));
    s->inten.release();
    return refresh_tilt_table(s);
}

int mset_batch_apply(mset_session *s) {
    int rc = batch_ok(s);
    if (rc) return rc;
    rc = refresh_tilt_table(s);
    if (rc) return rc;
    CKL(launch_apply_batch(s->n, s->nz, s->b, s->ns, s->method, s->step[0], s->step[1], s->step[2],
                           s->h_tilts.data(), (int)s->tilts.size(), s->st),
        "apply");
    CK(cudaStreamSynchronize(s->st));
    return 0;
}

int mset_batch_get_tilt(mset_session *s, int j, float *volume, float *probe, float *scan_x, float *scan_y) {
    int rc = batch_ok(s);
    if (rc) return rc;
    if (j < 0 || j >= (int)s->tilts.size()) return fail(MSET_E_ARG, "tilt index %d out of range", j);
    TiltBufs &t = s->tilts[j];
    const size_t n2 = (size_t)s->n * s->n;
    if (volume) CK(cudaMemcpyAsync(volume, t.V.p, sizeof(float) * n2 * s->nz, cudaMemcpyDeviceToHost, s->st));
    if (probe) {
        CKL(launch_q_to_probe(s->plan, t.Q.p, s->tmpc.p, s->twn.p, s->st), "q_to_probe");
        CK(cudaMemcpyAsync(probe, s->tmpc.p, sizeof(float2) * n2, cudaMemcpyDeviceToHost, s->st));
    }
    if (scan_x && t.npos) CK(cudaMemcpyAsync(scan_x, t.sx.p, sizeof(float) * t.npos, cudaMemcpyDeviceToHost, s->st));
    if (scan_y && t.npos) CK(cudaMemcpyAsync(scan_y, t.sy.p, sizeof(float) * t.npos, cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    return 0;
}

int mset_batch_time(mset_session *s, int reps, double *ms_per_pass) {
    int rc = batch_ok(s);
    if (rc) return rc;
    if (reps <= 0 || !ms_per_pass) return fail(MSET_E_ARG, "bad arguments");
    CK(cudaEventRecord(s->ev0, s->st));
    for (int r = 0; r < reps; ++r) {
        rc = batch_pass(s);
        if (rc) return rc;
    }
    CK(cudaEventRecord(s->ev1, s->st));
    CK(cudaEventSynchronize(s->ev1));
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, s->ev0, s->ev1));
    *ms_per_pass = ms / reps;
    return take_fault(s);
}

// ---- Fourier-shear rotation -------------------------------------------------
// work buffers of a rotation of an n1 x n2 x n3 volume: a cubic one rotates
// plane by plane (k_shear), any other shape line by line (rot_apply3)
static int rot_prepare3(mset_session *s, int n1, int n2, int n3) {
    if (n1 == n2 && n2 == n3) {
        if (!rot_supported(n1))
            return fail(MSET_E_UNSUPPORTED, "rotation of a %d^3 volume has no compiled kernel "
                                            "(supported: 24, 32, 48, 64, 96, 128, 160, 256)", n1);
    } else if (!rot_line_supported(n1) || !rot_line_supported(n2) || !rot_line_supported(n3)) {
        return fail(MSET_E_UNSUPPORTED, "rotation of a %d x %d x %d volume: every side must be one of 24, 32, 48, "
                                        "64, 96, 128, 160, 192, 256", n1, n2, n3);
    }
    const size_t nvox = (size_t)n1 * n2 * n3;
    CK(s->rot_vol.ensure(std::max(s->rot_vol.n, nvox)));
    CK(s->rot_S.ensure(std::max(s->rot_S.n, nvox)));
    return 0;
}

static int rot_prepare(mset_session *s, int n) {
    int rc = rot_prepare3(s, n, n, n);
    if (rc) return rc;
    if (s->rot_n != n) {
        std::vector<float2> h;
        rot_twiddles(n, h);
        CK(s->rot_tw.ensure(n));
        CK(cudaMemcpyAsync(s->rot_tw.p, h.data(), sizeof(float2) * n, cudaMemcpyHostToDevice, s->st));
        CK(cudaStreamSynchronize(s->st));
        s->rot_n = n;
    }
    return 0;
}

// rotation of the reconstruction-shaped volume src into dst (may alias)
static int rotate_rec(mset_session *s, const RotPlan &pl, const float *src, float *dst) {
    if (s->nv > 0) return rot_apply(pl, s->nv, src, dst, s->rot_S.p, s->rot_tw.p, s->sms, s->st);
    return rot_apply3(pl, s->nv1, s->nv2, s->nv3, src, dst, s->rot_S.p, s->sms, s->st);
}

int mset_rotate_volume_nd(mset_session *s, const float *vol_in, float *vol_out, int n1, int n2, int n3,
                          const float *vec1, const float *vec2, const float *vec3, double phi, double theta,
                          double psi, int inverse) {
    Range range_("mset_rotate_volume_nd");
    if (!s || !vol_in || !vol_out || !vec1 || !vec2 || !vec3) return fail(MSET_E_ARG, "null argument");
    if (n1 <= 1 || n2 <= 1 || n3 <= 1) return fail(MSET_E_ARG, "bad volume size %d x %d x %d", n1, n2, n3);
    int rc = set_device(s);
    if (rc) return rc;
    if (!rot_line_supported(n1) || !rot_line_supported(n2) || !rot_line_supported(n3))
        return fail(MSET_E_UNSUPPORTED, "rotation of a %d x %d x %d volume: every side must be one of 24, 32, 48, "
                                        "64, 96, 128, 160, 192, 256", n1, n2, n3);
    const size_t nvox = (size_t)n1 * n2 * n3;
    CK(s->rot_vol.ensure(std::max(s->rot_vol.n, nvox)));
    CK(s->rot_S.ensure(std::max(s->rot_S.n, nvox)));
    const double v1[3] = {vec1[0], vec1[1], vec1[2]}, v2[3] = {vec2[0], vec2[1], vec2[2]},
                 v3[3] = {vec3[0], vec3[1], vec3[2]};
    RotPlan pl;
    rot_plan(v1, v2, v3, phi, theta, psi, inverse != 0, &pl);
    CK(cudaMemcpyAsync(s->rot_vol.p, vol_in, sizeof(float) * nvox, cudaMemcpyHostToDevice, s->st));
    CKL(rot_apply3(pl, n1, n2, n3, s->rot_vol.p, s->rot_vol.p, s->rot_S.p, s->sms, s->st), "rotation");
    CK(cudaMemcpyAsync(vol_out, s->rot_vol.p, sizeof(float) * nvox, cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    return 0;
}

int mset_rotate_volume(mset_session *s, const float *vol_in, float *vol_out, int n, const float *vec1,
                       const float *vec2, const float *vec3, double phi, double theta, double psi, int inverse) {
    Range range_("mset_rotate_volume");
    if (!s || !vol_in || !vol_out || !vec1 || !vec2 || !vec3) return fail(MSET_E_ARG, "null argument");
    if (n <= 1) return fail(MSET_E_ARG, "bad volume size %d", n);
    int rc = set_device(s);
    if (rc) return rc;
    rc = rot_prepare(s, n);
    if (rc) return rc;
    const double v1[3] = {vec1[0], vec1[1], vec1[2]}, v2[3] = {vec2[0], vec2[1], vec2[2]},
                 v3[3] = {vec3[0], vec3[1], vec3[2]};
    RotPlan pl;
    rot_plan(v1, v2, v3, phi, theta, psi, inverse != 0, &pl);
    const size_t n3 = (size_t)n * n * n;
    CK(cudaMemcpyAsync(s->rot_vol.p, vol_in, sizeof(float) * n3, cudaMemcpyHostToDevice, s->st));
    CKL(rot_apply(pl, n, s->rot_vol.p, s->rot_vol.p, s->rot_S.p, s->rot_tw.p, s->sms, s->st), "rotation");
    CK(cudaMemcpyAsync(vol_out, s->rot_vol.p, sizeof(float) * n3, cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    return 0;
}

// ---- TV / TV-FISTA ----------------------------------------------------------
int mset_tv(mset_session *s, float *vol, int n1, int n2, int n3, double lambda, int niter, int fista,
            double *tv_error) {
    Range range_("mset_tv");
    if (!s || !vol) return fail(MSET_E_ARG, "null argument");
    if (n1 <= 0 || n2 <= 0 || n3 <= 0 || niter < 0 || !(lambda > 0))
        return fail(MSET_E_ARG, "need positive sizes, niter >= 0 and lambda > 0");
    int rc = set_device(s);
    if (rc) return rc;
    const size_t V = (size_t)n1 * n2 * n3;
    CK(s->tv_in.ensure(V));
    CK(s->tv_out.ensure(V));
    CK(s->tv_P.ensure(3 * V));
    CK(s->tv_Y.ensure(3 * V));
    CK(s->tv_D.ensure(V));
    CK(s->tv_err.ensure(1));
    CK(cudaMemcpyAsync(s->tv_in.p, vol, sizeof(float) * V, cudaMemcpyHostToDevice, s->st));
    CK(cudaMemsetAsync(s->tv_err.p, 0, sizeof(double), s->st));
    TvArgs a{s->tv_in.p, s->tv_out.p, s->tv_P.p, s->tv_Y.p, s->tv_D.p, n1, n2, n3, lambda, niter, fista ? 1 : 0,
             s->tv_err.p};
    CKL(tv_prox(a, s->st), "tv");
    CK(cudaMemcpyAsync(vol, s->tv_out.p, sizeof(float) * V, cudaMemcpyDeviceToHost, s->st));
    double e = 0;
    CK(cudaMemcpyAsync(&e, s->tv_err.p, sizeof(double), cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    if (tv_error) *tv_error = e;
    return 0;
}

// ---- batched iteration ------------------------------------------------------
static void drop_graph(mset_session *s) {
    if (s->graph_exec) cudaGraphExecDestroy(s->graph_exec);
    if (s->graph) cudaGraphDestroy(s->graph);
    s->graph_exec = nullptr;
    s->graph = nullptr;
    for (int p = 0; p < 2; ++p) {
        if (s->phase_exec[p]) cudaGraphExecDestroy(s->phase_exec[p]);
        if (s->phase_graph[p]) cudaGraphDestroy(s->phase_graph[p]);
        s->phase_exec[p] = nullptr;
        s->phase_graph[p] = nullptr;
    }
}

namespace {
// history slot: hist[k * J + j] = err[j], k from a device counter, so the
// same captured graph appends on every replay
__global__ void k_record_err(const double *err, int J, double *hist, int cap, unsigned *counter, const double *tv_err,
                             double *tv_hist) {
    const unsigned k = *counter;
    if (k < (unsigned)cap) {
        for (int j = threadIdx.x; j < J; j += blockDim.x) hist[(size_t)k * J + j] = err[j];
        if (threadIdx.x == 0 && tv_err) tv_hist[k] = *tv_err;
    }
    __syncthreads();
    if (threadIdx.x == 0) *counter = k + 1;
}
}  // namespace

int mset_batch_iteration_setup_nd(mset_session *s, const mset_iter_args *a, int nv1, int nv2, int nv3) {
    int rc = batch_ok(s);
    if (rc) return rc;
    if (!a || !a->angles || !a->vec1 || !a->vec2 || !a->vec3) return fail(MSET_E_ARG, "null argument");
    if (nv3 != s->nz)
        return fail(MSET_E_ARG, "the reconstruction depth nv3 (%d) must equal the session depth nz (%d)", nv3, s->nz);
    if (nv1 > s->n || nv2 > s->n)
        return fail(MSET_E_ARG, "the reconstruction (%d x %d laterally) exceeds the window (%d)", nv1, nv2, s->n);
    if ((s->n - nv1) % 2 || (s->n - nv2) % 2)
        return fail(MSET_E_ARG, "window minus volume sides must be even (centred padding)");
    if (a->use_tv && (!(a->tv_lambda > 0) || a->tv_iter < 0)) return fail(MSET_E_ARG, "bad TV parameters");
    const bool cubic = nv1 == nv2 && nv2 == nv3;
    rc = cubic ? rot_prepare(s, nv1) : rot_prepare3(s, nv1, nv2, nv3);
    if (rc) return rc;
    const int J = (int)s->tilts.size();
    const double v1[3] = {a->vec1[0], a->vec1[1], a->vec1[2]}, v2[3] = {a->vec2[0], a->vec2[1], a->vec2[2]},
                 v3[3] = {a->vec3[0], a->vec3[1], a->vec3[2]};
    s->plan_inv.resize(J);
    s->plan_fwd.resize(J);
    for (int j = 0; j < J; ++j) {
        const float *an = a->angles + 3 * j;
        rot_plan(v1, v2, v3, an[0], an[1], an[2], true, &s->plan_inv[j]);   // Func_inv_rot (STEP01_ROTATION.m:13)
        rot_plan(v1, v2, v3, an[0], an[1], an[2], false, &s->plan_fwd[j]);  // Func_rot (Run_MSET_recon.m:179)
    }
    const size_t V = (size_t)nv1 * nv2 * nv3;
    CK(s->rec.ensure(V));
    CK(s->gvol.ensure(V));
    CK(s->gacc.ensure(V));
    CK(s->it_counter.ensure(1));
    CK(s->mx_bits.ensure(1));
    CK(s->mx.ensure(1));
    CK(cudaMemsetAsync(s->rec.p, 0, sizeof(float) * V, s->st));
    s->nv = cubic ? nv1 : 0;
    s->nv1 = nv1;
    s->nv2 = nv2;
    s->nv3 = nv3;
    s->it_pos = a->use_positivity ? 1 : 0;
    s->it_tv = a->use_tv ? 1 : 0;
    s->it_tv_iter = a->tv_iter;
    s->it_tv_fista = a->tv_fista ? 1 : 0;
    s->it_tv_lambda = a->tv_lambda;
    if (s->it_tv) {
        CK(s->tv_in.ensure(V));
        CK(s->tv_out.ensure(V));
        CK(s->tv_P.ensure(3 * V));
        CK(s->tv_Y.ensure(3 * V));
        CK(s->tv_D.ensure(V));
        CK(s->tv_err.ensure(1));
    }
    CK(cudaStreamSynchronize(s->st));
    drop_graph(s);
    s->it_ready = true;
    return 0;
}

int mset_batch_iteration_setup(mset_session *s, const mset_iter_args *a) {
    if (!a) return fail(MSET_E_ARG, "null argument");
    return mset_batch_iteration_setup_nd(s, a, a->nv, a->nv, a->nv);
}

int mset_batch_set_rec(mset_session *s, const float *rec) {
    int rc = batch_ok(s);
    if (rc) return rc;
    if (!s->it_ready) return fail(MSET_E_STATE, "mset_batch_iteration_setup first");
    if (!rec) return fail(MSET_E_ARG, "null volume");
    CK(cudaMemcpyAsync(s->rec.p, rec, sizeof(float) * (size_t)s->nv1 * s->nv2 * s->nv3, cudaMemcpyHostToDevice, s->st));
    CK(cudaStreamSynchronize(s->st));
    return 0;
}

int mset_batch_get_rec(mset_session *s, float *rec) {
    int rc = batch_ok(s);
    if (rc) return rc;
    if (!s->it_ready) return fail(MSET_E_STATE, "mset_batch_iteration_setup first");
    if (!rec) return fail(MSET_E_ARG, "null volume");
    CK(cudaMemcpyAsync(rec, s->rec.p, sizeof(float) * (size_t)s->nv1 * s->nv2 * s->nv3, cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    return 0;
}

// everything of one iteration, stream-ordered, no host synchronisation and
// no pageable copies: safe to capture into a CUDA graph.  Phase 1: beam-frame
// volumes, the batched pass and the lab-frame gradient sum over this
// session's tilts (gacc); phase 2: the update from gacc.  A caller that
// shards tilts over GPUs all-reduces gacc between the phases.
static int record_phase(mset_session *s, int phase, bool with_tv = true, bool with_hist = true) {
    const int J = (int)s->tilts.size();
    const int n = s->n;
    const long V = (long)s->nv1 * s->nv2 * s->nv3;
    const int nsg = s->method == MSET_MODE_SSET ? 1 : s->ns;
    const int bvox = s->method == MSET_MODE_SSET ? s->nz : s->b;
    const size_t n2 = (size_t)n * n;
    if (phase == 2) goto update;
    // 1. beam-frame volumes V_j = pad(Func_inv_rot(rec, angles_j))
    for (int j = 0; j < J; ++j) {
        CKL(rotate_rec(s, s->plan_inv[j], s->rec.p, s->gvol.p), "rotation");
        CKL(vol_pad(s->gvol.p, s->tilts[j].V.p, s->nv1, s->nv2, s->nv3, n, s->st), "pad");
    }
    // 2. the batched pass over all positions of all tilts
    for (auto &t : s->tilts) {
        CK(cudaMemsetAsync(t.grad.p, 0, sizeof(double) * n2 * nsg, s->st));
        CK(cudaMemsetAsync(t.qacc.p, 0, sizeof(double) * n2 * 2, s->st));
    }
    CK(cudaMemsetAsync(s->err.p, 0, sizeof(double) * J, s->st));
    CKL(launch_transmission(s->d_tilts.p, J, n, s->nz, bvox, nsg, s->sigma * s->dz, s->st), "transmission");
    CK(cudaMemsetAsync(s->counter.p, 0, sizeof(unsigned), s->st));
    {
        LaunchArgs la = base_args(s);
        const int mode = (s->method == kMSET && s->ckpt > 0 && s->ckpt < s->ns) ? kBatchCk : kBatch;
        CKL(launch_positions(s->plan, s->method, s->adjoint, mode, la, s->grid_cache, s->st), "position kernel");
    }
    // 3. gradient back to the lab frame: sum_j Func_rot(G_j)
    for (int j = 0; j < J; ++j) {
        CKL(vol_slab_to_volume(s->tilts[j].grad.p, s->gvol.p, s->nv1, s->nv2, s->nv3, n, bvox, s->st),
            "slab_to_volume");
        CKL(rotate_rec(s, s->plan_fwd[j], s->gvol.p, s->gvol.p), "rotation");
        CKL(vol_accumulate(s->gvol.p, s->gacc.p, V, j == 0, s->st), "accumulate");
    }
    if (phase == 1) return 0;
update:
    // 4. object update, positivity (Run_MSET_recon.m:183-185), TV (:267-270)
    CKL(vol_update(s->rec.p, s->gacc.p, V, s->step[0], s->st), "update");
    if (s->it_pos) CKL(vol_positivity(s->rec.p, V, s->st), "positivity");
    if (s->it_tv && with_tv) {
        CKL(vol_max(s->rec.p, V, s->mx_bits.p, s->mx.p, s->st), "max");
        CKL(vol_scale(s->rec.p, s->tv_in.p, V, s->mx.p, s->st), "scale");
        CK(cudaMemsetAsync(s->tv_err.p, 0, sizeof(double), s->st));
        const TvArgs ta{s->tv_in.p, s->tv_out.p, s->tv_P.p, s->tv_Y.p, s->tv_D.p, s->nv1, s->nv2, s->nv3,
                        s->it_tv_lambda, s->it_tv_iter, s->it_tv_fista, s->tv_err.p};
        CKL(tv_prox(ta, s->st), "tv");
        CKL(vol_mul(s->tv_out.p, s->rec.p, V, s->mx.p, s->st), "rescale");
    }
    // 5. probe and scan positions
    CKL(launch_apply_probe_pos(s->h_tilts.data(), J, n, s->step[1], s->step[2], s->st), "apply");
    if (!with_hist) return 0;
    // 6. error history
    k_record_err<<<1, 64, 0, s->st>>>(s->err.p, J, s->err_hist.p, s->hist_cap, s->it_counter.p,
                                      s->it_tv ? s->tv_err.p : nullptr, s->tv_hist.p);
    CK(cudaGetLastError());
    return 0;
}

int mset_batch_iterate(mset_session *s, int niter, int use_graph, double *err_out, double *tv_err_out) {
    Range range_("mset_batch_iterate");
    int rc = batch_ok(s);
    if (rc) return rc;
    if (!s->it_ready) return fail(MSET_E_STATE, "mset_batch_iteration_setup first");
    if (niter < 0) return fail(MSET_E_ARG, "niter < 0");
    const int J = (int)s->tilts.size();
    // everything that allocates or copies from the host happens here, before
    // the iterations (and before any capture)
    const int grid = persistent_grid(s, std::max(1, s->total_pos));
    rc = ensure_save(s, grid);
    if (rc) return rc;
    s->grid_cache = grid;
    rc = refresh_tilt_table(s);
    if (rc) return rc;
    const int cap = std::max(1, niter);
    if (s->hist_cap < cap) {
        CK(s->err_hist.ensure((size_t)cap * J));
        CK(s->tv_hist.ensure(cap));
        s->hist_cap = cap;
        drop_graph(s);
    }
    CK(cudaMemsetAsync(s->it_counter.p, 0, sizeof(unsigned), s->st));
    CK(cudaStreamSynchronize(s->st));
    if (use_graph) {
        if (!s->graph_exec) {
            CK(cudaStreamBeginCapture(s->st, cudaStreamCaptureModeRelaxed));
            rc = record_phase(s, 1);
            if (!rc) rc = record_phase(s, 2);
            cudaGraph_t g = nullptr;
            cudaError_t e = cudaStreamEndCapture(s->st, &g);
            if (rc) {
                if (g) cudaGraphDestroy(g);
                return rc;
            }
            if (e != cudaSuccess) return cuda_fail(e, "graph capture");
            s->graph = g;
            CK(cudaGraphInstantiate(&s->graph_exec, g, 0));
        }
        for (int k = 0; k < niter; ++k) CK(cudaGraphLaunch(s->graph_exec, s->st));
    } else {
        for (int k = 0; k < niter; ++k) {
            rc = record_phase(s, 1);
            if (!rc) rc = record_phase(s, 2);
            if (rc) return rc;
        }
    }
    if (err_out && niter)
        CK(cudaMemcpyAsync(err_out, s->err_hist.p, sizeof(double) * niter * J, cudaMemcpyDeviceToHost, s->st));
    if (tv_err_out && niter)
        CK(cudaMemcpyAsync(tv_err_out, s->tv_hist.p, sizeof(double) * niter, cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    return take_fault(s);
}

// TV / TV-FISTA of rec / max(rec), rescaled by max(rec) (Run_MSET_recon.m:267-270)
static int record_tv(mset_session *s) {
    const long V = (long)s->nv1 * s->nv2 * s->nv3;
    CKL(vol_max(s->rec.p, V, s->mx_bits.p, s->mx.p, s->st), "max");
    CKL(vol_scale(s->rec.p, s->tv_in.p, V, s->mx.p, s->st), "scale");
    CK(cudaMemsetAsync(s->tv_err.p, 0, sizeof(double), s->st));
    const TvArgs ta{s->tv_in.p, s->tv_out.p, s->tv_P.p, s->tv_Y.p, s->tv_D.p, s->nv1, s->nv2, s->nv3,
                    s->it_tv_lambda, s->it_tv_iter, s->it_tv_fista, s->tv_err.p};
    CKL(tv_prox(ta, s->st), "tv");
    CKL(vol_mul(s->tv_out.p, s->rec.p, V, s->mx.p, s->st), "rescale");
    return 0;
}

// error pass of the current state over every tilt: V_j = pad(Func_inv_rot(rec)),
// forward only (run_error_mset, mset.cu:557-696), sums into s->err
static int record_error_phase(mset_session *s) {
    const int J = (int)s->tilts.size();
    const int n = s->n;
    const int nsg = s->method == MSET_MODE_SSET ? 1 : s->ns;
    const int bvox = s->method == MSET_MODE_SSET ? s->nz : s->b;
    for (int j = 0; j < J; ++j) {
        CKL(rotate_rec(s, s->plan_inv[j], s->rec.p, s->gvol.p), "rotation");
        CKL(vol_pad(s->gvol.p, s->tilts[j].V.p, s->nv1, s->nv2, s->nv3, n, s->st), "pad");
    }
    CK(cudaMemsetAsync(s->err.p, 0, sizeof(double) * J, s->st));
    CKL(launch_transmission(s->d_tilts.p, J, n, s->nz, bvox, nsg, s->sigma * s->dz, s->st), "transmission");
    CK(cudaMemsetAsync(s->counter.p, 0, sizeof(unsigned), s->st));
    LaunchArgs la = base_args(s);
    CKL(launch_positions(s->plan, s->method, kREF, kErr, la, s->grid_cache, s->st), "error pass");
    return 0;
}

// copy of the state a line-search step may have to undo: rec, probes, positions
static int bls_state(mset_session *s, bool save) {
    const size_t n2 = (size_t)s->n * s->n;
    const long V = (long)s->nv1 * s->nv2 * s->nv3;
    if (save) CK(cudaMemcpyAsync(s->bls_rec.p, s->rec.p, sizeof(float) * V, cudaMemcpyDeviceToDevice, s->st));
    else CK(cudaMemcpyAsync(s->rec.p, s->bls_rec.p, sizeof(float) * V, cudaMemcpyDeviceToDevice, s->st));
    for (size_t j = 0; j < s->tilts.size(); ++j) {
        TiltBufs &t = s->tilts[j];
        float2 *q = s->bls_q.p + j * n2;
        float *px = s->bls_pos.p + 2 * (size_t)s->pos_off[j], *py = px + t.npos;
        const size_t pb = sizeof(float) * t.npos;
        if (save) {
            CK(cudaMemcpyAsync(q, t.Q.p, sizeof(float2) * n2, cudaMemcpyDeviceToDevice, s->st));
            if (t.npos) {
                CK(cudaMemcpyAsync(px, t.sx.p, pb, cudaMemcpyDeviceToDevice, s->st));
                CK(cudaMemcpyAsync(py, t.sy.p, pb, cudaMemcpyDeviceToDevice, s->st));
            }
        } else {
            CK(cudaMemcpyAsync(t.Q.p, q, sizeof(float2) * n2, cudaMemcpyDeviceToDevice, s->st));
            if (t.npos) {
                CK(cudaMemcpyAsync(t.sx.p, px, pb, cudaMemcpyDeviceToDevice, s->st));
                CK(cudaMemcpyAsync(t.sy.p, py, pb, cudaMemcpyDeviceToDevice, s->st));
            }
        }
    }
    return 0;
}

static void drop_phase_graphs(mset_session *s) {
    for (int p = 0; p < 2; ++p) {
        if (s->phase_exec[p]) cudaGraphExecDestroy(s->phase_exec[p]);
        if (s->phase_graph[p]) cudaGraphDestroy(s->phase_graph[p]);
        s->phase_exec[p] = nullptr;
        s->phase_graph[p] = nullptr;
    }
}

int mset_batch_iterate_bls(mset_session *s, int niter, double bls_parameter, double *mean_err_out,
                           float *step_out, int *iters_out) {
    Range range_("mset_batch_iterate_bls");
    int rc = batch_ok(s);
    if (rc) return rc;
    if (!s->it_ready) return fail(MSET_E_STATE, "mset_batch_iteration_setup first");
    if (niter < 0) return fail(MSET_E_ARG, "niter < 0");
    if (!(bls_parameter > 0.0 && bls_parameter < 1.0)) return fail(MSET_E_ARG, "bls_parameter must be in (0, 1)");
    if (iters_out) *iters_out = 0;
    const int J = (int)s->tilts.size();
    const size_t n2 = (size_t)s->n * s->n;
    const long V = (long)s->nv1 * s->nv2 * s->nv3;
    const int grid = persistent_grid(s, std::max(1, s->total_pos));
    rc = ensure_save(s, grid);
    if (rc) return rc;
    s->grid_cache = grid;
    rc = refresh_tilt_table(s);
    if (rc) return rc;
    CK(s->bls_rec.ensure(V));
    CK(s->bls_q.ensure(std::max<size_t>(1, n2 * J)));
    CK(s->bls_pos.ensure(std::max<size_t>(1, 2 * (size_t)s->total_pos)));
    // the step sizes change below: graphs captured with the old ones are stale
    drop_graph(s);
    const float step0_orig = s->step[0];
    const double floor0 = std::pow(bls_parameter, 5) * (double)step0_orig;
    double old_mean = 1e31;
    std::vector<double> err(J);
    int done = 0;
    bool stop = false;
    for (int i = 0; i < niter && !stop; ++i) {
        rc = bls_state(s, true);
        if (rc) return rc;
        double mean = 0;
        for (;;) {
            // one update (rotations, pass, gradient sum, update, positivity,
            // probe and position steps), then the error of the new state
            rc = record_phase(s, 1);
            if (!rc) rc = record_phase(s, 2, false, false);
            if (!rc) rc = record_error_phase(s);
            if (rc) return rc;
            CK(cudaMemcpyAsync(err.data(), s->err.p, sizeof(double) * J, cudaMemcpyDeviceToHost, s->st));
            CK(cudaStreamSynchronize(s->st));
            mean = 0;
            for (int j = 0; j < J; ++j)
                mean += s->npos[j] ? err[j] / s->npos[j] / (double)n2 : 0.0;  // mex_main.cu:179
            mean /= J;
            if (old_mean > mean) break;                 // accepted (Run_MSET_recon.m:240)
            rc = bls_state(s, false);                   // rejected: undo, shrink every step
            if (rc) return rc;
            for (int k = 0; k < 3; ++k) s->step[k] = (float)(bls_parameter * s->step[k]);
            if ((double)s->step[0] < floor0) {          // Run_MSET_recon.m:250-253
                stop = true;
                break;
            }
        }
        if (stop) break;
        if (s->it_tv) {
            rc = record_tv(s);
            if (rc) return rc;
        }
        if (mean_err_out) mean_err_out[i] = mean;
        if (step_out)
            for (int k = 0; k < 3; ++k) step_out[3 * i + k] = s->step[k];
        old_mean = mean;
        ++done;
    }
    CK(cudaStreamSynchronize(s->st));
    if (iters_out) *iters_out = done;
    return take_fault(s);
}

int mset_batch_iterate_phase(mset_session *s, int phase, int use_graph) {
    Range range_("mset_batch_iterate_phase");
    int rc = batch_ok(s);
    if (rc) return rc;
    if (!s->it_ready) return fail(MSET_E_STATE, "mset_batch_iteration_setup first");
    if (phase != 1 && phase != 2) return fail(MSET_E_ARG, "phase must be 1 or 2");
    if (phase == 1 || !s->grid_cache) {
        const int grid = persistent_grid(s, std::max(1, s->total_pos));
        rc = ensure_save(s, grid);
        if (rc) return rc;
        if (grid != s->grid_cache) drop_phase_graphs(s);
        s->grid_cache = grid;
        rc = refresh_tilt_table(s);
        if (rc) return rc;
        if (s->hist_cap < 1) {
            CK(s->err_hist.ensure(s->tilts.size()));
            CK(s->tv_hist.ensure(1));
            s->hist_cap = 1;
        }
    }
    // the history slot of a single phase call is always the first
    CK(cudaMemsetAsync(s->it_counter.p, 0, sizeof(unsigned), s->st));
    if (use_graph) {
        cudaGraphExec_t &ex = s->phase_exec[phase - 1];
        if (!ex) {
            CK(cudaStreamBeginCapture(s->st, cudaStreamCaptureModeRelaxed));
            rc = record_phase(s, phase);
            cudaGraph_t g = nullptr;
            cudaError_t e = cudaStreamEndCapture(s->st, &g);
            if (rc) {
                if (g) cudaGraphDestroy(g);
                return rc;
            }
            if (e != cudaSuccess) return cuda_fail(e, "graph capture");
            s->phase_graph[phase - 1] = g;
            CK(cudaGraphInstantiate(&ex, g, 0));
        }
        CK(cudaGraphLaunch(ex, s->st));
    } else {
        rc = record_phase(s, phase);
        if (rc) return rc;
    }
    return 0;
}

int mset_batch_device_info(mset_session *s, void **gacc_dev, size_t *gacc_count, void **stream,
                           double **err_dev) {
    int rc = batch_ok(s);
    if (rc) return rc;
    if (!s->it_ready) return fail(MSET_E_STATE, "mset_batch_iteration_setup first");
    if (gacc_dev) *gacc_dev = s->gacc.p;
    if (gacc_count) *gacc_count = (size_t)s->nv1 * s->nv2 * s->nv3;
    if (stream) *stream = (void *)s->st;
    if (err_dev) *err_dev = s->err.p;
    return 0;
}

int mset_batch_iterate_time(mset_session *s, int niter, double *ms_per_iter) {
    int rc = batch_ok(s);
    if (rc) return rc;
    if (!ms_per_iter || niter <= 0) return fail(MSET_E_ARG, "bad arguments");
    rc = mset_batch_iterate(s, 1, 1, nullptr, nullptr);  // capture + one replay
    if (rc) return rc;
    CK(cudaEventRecord(s->ev0, s->st));
    for (int k = 0; k < niter; ++k) CK(cudaGraphLaunch(s->graph_exec, s->st));
    CK(cudaEventRecord(s->ev1, s->st));
    CK(cudaEventSynchronize(s->ev1));
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, s->ev0, s->ev1));
    *ms_per_iter = ms / niter;
    return take_fault(s);
}

int mset_batch_set_amplitude_bf16(mset_session *s, int on) {
    int rc = batch_ok(s);
    if (rc) return rc;
    s->amp_bf16 = on ? 1 : 0;
    return 0;
}

int mset_batch_set_checkpoint(mset_session *s, int k) {
    int rc = batch_ok(s);
    if (rc) return rc;
    if (k < 0) return fail(MSET_E_ARG, "checkpoint interval must be >= 0");
    s->ckpt = k;
    s->grid_cache = 0;
    drop_graph(s);
    return 0;
}

int mset_batch_launch_count(mset_session *s) {
    if (!s) return fail(MSET_E_ARG, "null session");
    return 2;  // transmission slabs + position kernel
}

}  // extern "C"

// ---- autotuner ----------------------------------------------------------------
// The batched pass has two shape parameters that trade memory for speed: the
// number of persistent CTAs (positions in flight; each owns a saved-wave slot
// set) and the checkpoint interval k (slots per CTA: ns + 1 at k = 0,
// ceil(ns/k) + k + 2 otherwise, with the forward of each segment recomputed in
// the adjoint).  The tuner times every (CTAs per SM, k) pair whose saved-wave
// storage fits the memory budget on a sample of the session's own positions
// and keeps the fastest; among shapes within 1% of it, the one using less
// memory.
namespace {

int occupancy_limit(const mset_session *s) {
    if (s->plan.cl > 1) return 1;  // one CTA of a cluster per SM
    const int by_smem = (int)((227 * 1024) / (s->plan.smem + 1024));
    const int by_thr = 2048 / s->plan.nt;
    return std::max(1, std::min(by_smem, by_thr));
}

double save_bytes(const mset_session *s, int grid, int k) {
    const int fields = std::max(1, grid / std::max(1, s->plan.cl));
    return (double)fields * save_slots(s->ns, k) * s->n * s->n * sizeof(float2);
}

// one warm launch, then `reps` timed launches over the first nitems positions
int time_queue(mset_session *s, int grid, int nitems, int reps, double *ms) {
    int rc = queue_prepare(s, kBatch, grid);
    if (rc) return rc;
    rc = queue_enqueue(s, s->method, s->adjoint, kBatch, grid, nitems);
    if (rc) return rc;
    CK(cudaEventRecord(s->ev0, s->st));
    for (int r = 0; r < reps; ++r) {
        rc = queue_enqueue(s, s->method, s->adjoint, kBatch, grid, nitems);
        if (rc) return rc;
    }
    CK(cudaEventRecord(s->ev1, s->st));
    CK(cudaEventSynchronize(s->ev1));
    float t = 0;
    CK(cudaEventElapsedTime(&t, s->ev0, s->ev1));
    *ms = t / reps;
    return 0;
}

int tune_session(mset_session *s, double budget, mset_tune_result *out) {
    std::vector<int> ks{0};
    if (s->method == MSET_MODE_MSET)
        for (int k : {2, 4, 8, 16})
            if (k < s->ns) ks.push_back(k);
    const int k_in = s->ckpt;
    const Plan plan_in = s->plan;
    // the same positions for every shape: as many as the widest grid of any
    // variant keeps busy four times over
    int occ_max = 1;
    for (int v = 0; v < plan_variants(s->n); ++v) {
        Plan pl;
        if (plan_for(s->n, &pl, v)) {
            s->plan = pl;
            occ_max = std::max(occ_max, occupancy_limit(s));
        }
    }
    s->plan = plan_in;
    const int sample = std::min(s->total_pos, 4 * s->sms * occ_max);
    int rc = batch_zero(s);
    if (!rc) rc = batch_transmission(s);
    if (rc) return rc;
    int best_grid = 0, best_k = 0, timed = 0;
    double best_us = 0, best_bytes = 0;
    Plan best_plan = plan_in;
    const int tuned_in = s->tuned_grid;
    for (int v = 0; v < plan_variants(s->n); ++v) {
        Plan pl;
        if (!plan_for(s->n, &pl, v)) continue;
        if (pl.cl > 1) pl.max_clusters = pl.ops->max_clusters();
        s->plan = pl;
        const int occ = occupancy_limit(s);
        int last_grid = 0;
        for (int c = 1; c <= occ; ++c) {
            s->tuned_grid = 0;
            const int grid = s->plan.cl > 1 ? persistent_grid(s, s->total_pos)
                                            : std::max(1, std::min(s->sms * c, s->total_pos));
            s->tuned_grid = tuned_in;
            if (grid == last_grid) break;
            last_grid = grid;
            for (int k : ks) {
                const double bytes = save_bytes(s, grid, k);
                if (budget > 0 && bytes > budget) continue;
                s->ckpt = k;
                double ms = 0;
                rc = time_queue(s, grid, sample, 2, &ms);
                if (rc) {
                    s->ckpt = k_in;
                    s->plan = plan_in;
                    return rc;
                }
                ++timed;
                const double us = ms * 1e3 / sample;
                const bool faster = !best_grid || us < 0.99 * best_us;
                const bool tie_smaller = best_grid && us <= 1.01 * best_us && bytes < best_bytes;
                if (faster || tie_smaller) {
                    if (faster || us < best_us) best_us = us;
                    best_grid = grid;
                    best_k = k;
                    best_bytes = bytes;
                    best_plan = s->plan;
                }
            }
        }
    }
    s->plan = best_plan;
    if (!best_grid) {
        s->plan = plan_in;
        s->ckpt = k_in;
        return fail(MSET_E_NOMEM, "no batch shape of the %d^2 window fits the memory budget of %.0f bytes", s->n,
                    budget);
    }
    s->ckpt = best_k;
    s->tuned_grid = best_grid;
    s->tuned_us_per_pos = best_us;
    s->grid_cache = 0;
    drop_graph(s);
    s->save.release();
    rc = ensure_save(s, best_grid);
    if (rc) return rc;
    rc = batch_zero(s);  // the sample passes left partial sums
    if (rc) return rc;
    CK(cudaStreamSynchronize(s->st));
    if (out) {
        out->grid = best_grid;
        out->ctas_per_sm = (best_grid + s->sms - 1) / s->sms;
        out->checkpoint = best_k;
        out->candidates = timed;
        out->us_per_position = best_us;
        out->save_bytes = best_bytes;
        out->threads = s->plan.nt;
    out->staged = s->plan.staged;
    }
    return 0;
}

}  // namespace

// ---- groups of batched sessions -------------------------------------------------
struct mset_group {
    int device = 0;
    cudaStream_t st = nullptr;
    cudaEvent_t fork = nullptr, ev0 = nullptr, ev1 = nullptr;
    std::vector<mset_session *> m;
    std::vector<cudaEvent_t> done;
    int schedule = MSET_GROUP_SERIAL;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<const void *> sig;  // pointers and shapes the captured graph was built on
};

namespace {

void group_drop_graph(mset_group *g) {
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    g->exec = nullptr;
    g->graph = nullptr;
    g->sig.clear();
}

// work of a member in SM-time units: the tuner's measured cost, else a model
// proportional to slabs x n^2 log2 n per position
double member_work(const mset_session *s) {
    if (s->tuned_us_per_pos > 0) return s->total_pos * s->tuned_us_per_pos;
    return (double)s->total_pos * s->ns * s->n * s->n * std::log2((double)s->n) * 1e-6;
}

int group_grids(mset_group *g, std::vector<int> &grids) {
    const int M = (int)g->m.size();
    grids.assign(M, 0);
    if (g->schedule == MSET_GROUP_SERIAL) {
        for (int i = 0; i < M; ++i) grids[i] = persistent_grid(g->m[i], std::max(1, g->m[i]->total_pos));
        return 0;
    }
    std::vector<double> w(M);
    std::vector<int> occ(M);
    for (int i = 0; i < M; ++i) {
        mset_session *s = g->m[i];
        w[i] = member_work(s);
        occ[i] = s->tuned_grid > 0 ? std::max(1, (s->tuned_grid + s->sms - 1) / s->sms) : occupancy_limit(s);
    }
    int rc = mset_split_ctas(M, w.data(), occ.data(), g->m[0]->sms, grids.data());
    if (rc) return rc;
    for (int i = 0; i < M; ++i) {
        const int cl = std::max(1, g->m[i]->plan.cl);
        grids[i] = std::max(1, std::min(grids[i] / cl, std::max(1, g->m[i]->total_pos))) * cl;
    }
    return 0;
}

// the capturable part of one group pass on g->st
int group_enqueue(mset_group *g, const std::vector<int> &grids) {
    CK(cudaEventRecord(g->fork, g->st));
    const int M = (int)g->m.size();
    for (int i = 0; i < M; ++i) {
        mset_session *s = g->m[i];
        const bool after_prev = g->schedule == MSET_GROUP_SERIAL && i > 0;
        CK(cudaStreamWaitEvent(s->st, after_prev ? g->done[i - 1] : g->fork, 0));
        int rc = batch_zero(s);
        if (rc) return rc;
        if (s->total_pos) {
            rc = batch_transmission_enqueue(s);
            if (!rc) rc = queue_enqueue(s, s->method, s->adjoint, kBatch, grids[i], s->total_pos);
            if (rc) return rc;
        }
        CK(cudaEventRecord(g->done[i], s->st));
    }
    for (int i = 0; i < M; ++i) CK(cudaStreamWaitEvent(g->st, g->done[i], 0));
    return 0;
}

int group_prepare(mset_group *g, std::vector<int> &grids) {
    if (g->m.empty()) return fail(MSET_E_STATE, "empty group");
    CK(cudaSetDevice(g->device));
    int rc = group_grids(g, grids);
    if (rc) return rc;
    std::vector<const void *> sig;
    sig.push_back(reinterpret_cast<const void *>((intptr_t)g->schedule));
    for (size_t i = 0; i < g->m.size(); ++i) {
        mset_session *s = g->m[i];
        rc = queue_prepare(s, kBatch, grids[i]);
        if (rc) return rc;
        for (const void *p : {(const void *)s->d_tilts.p, (const void *)s->save.p, (const void *)s->items.p,
                              (const void *)s->counter.p, (const void *)s->err.p})
            sig.push_back(p);
        sig.push_back(reinterpret_cast<const void *>((intptr_t)grids[i]));
        sig.push_back(s->plan.ops);
        sig.push_back(reinterpret_cast<const void *>((intptr_t)s->ckpt));
        sig.push_back(reinterpret_cast<const void *>((intptr_t)s->total_pos));
        for (const TiltBufs &t : s->tilts) {
            sig.push_back(t.grad.p);
            sig.push_back(t.qacc.p);
        }
    }
    if (sig != g->sig) group_drop_graph(g);
    g->sig.swap(sig);
    return 0;
}

int group_launch(mset_group *g, const std::vector<int> &grids, bool use_graph) {
    if (!use_graph) return group_enqueue(g, grids);
    if (!g->exec) {
        CK(cudaStreamBeginCapture(g->st, cudaStreamCaptureModeRelaxed));
        int rc = group_enqueue(g, grids);
        cudaGraph_t gr = nullptr;
        cudaError_t e = cudaStreamEndCapture(g->st, &gr);
        if (rc) {
            if (gr) cudaGraphDestroy(gr);
            return rc;
        }
        if (e != cudaSuccess) return cuda_fail(e, "capturing the group pass");
        g->graph = gr;
        e = cudaGraphInstantiate(&g->exec, gr, 0);
        if (e != cudaSuccess) {
            group_drop_graph(g);
            return cuda_fail(e, "instantiating the group pass");
        }
    }
    CK(cudaGraphLaunch(g->exec, g->st));
    return 0;
}

}  // namespace

extern "C" {

int mset_batch_tune(mset_session *s, double mem_budget_bytes, mset_tune_result *out) {
    Range range_("mset_batch_tune");
    int rc = batch_ok(s);
    if (rc) return rc;
    if (mem_budget_bytes < 0) return fail(MSET_E_ARG, "negative memory budget");
    if (s->total_pos == 0) return fail(MSET_E_STATE, "no positions to tune on");
    return tune_session(s, mem_budget_bytes, out);
}

int mset_batch_variants(int n) { return plan_variants(n); }

int mset_batch_set_variant(mset_session *s, int variant) {
    int rc = batch_ok(s);
    if (rc) return rc;
    Plan pl;
    if (variant < 0 || !plan_for(s->n, &pl, variant))
        return fail(MSET_E_ARG, "window %d has %d kernel shapes, not %d", s->n, plan_variants(s->n), variant + 1);
    if (pl.cl > 1) pl.max_clusters = pl.ops->max_clusters();
    s->plan = pl;
    s->tuned_grid = 0;
    s->tuned_us_per_pos = 0;
    s->grid_cache = 0;
    drop_graph(s);
    return 0;
}

int mset_batch_get_tune(mset_session *s, mset_tune_result *out) {
    int rc = batch_ok(s);
    if (rc) return rc;
    if (!out) return fail(MSET_E_ARG, "null output");
    const int grid = persistent_grid(s, std::max(1, s->total_pos));
    out->grid = grid;
    out->ctas_per_sm = (grid + s->sms - 1) / s->sms;
    out->checkpoint = s->ckpt;
    out->candidates = 0;
    out->us_per_position = s->tuned_us_per_pos;
    out->save_bytes = save_bytes(s, grid, s->ckpt);
    out->threads = s->plan.nt;
    out->staged = s->plan.staged;
    return 0;
}

int mset_split_ctas(int count, const double *work, const int *ctas_per_sm, int sms, int *grid_out) {
    if (count <= 0 || !work || !ctas_per_sm || !grid_out || sms <= 0) return fail(MSET_E_ARG, "bad arguments");
    if (count > sms) return fail(MSET_E_ARG, "more members (%d) than SMs (%d)", count, sms);
    double tot = 0;
    for (int i = 0; i < count; ++i) {
        if (!(work[i] >= 0) || ctas_per_sm[i] <= 0) return fail(MSET_E_ARG, "bad work or occupancy of member %d", i);
        tot += work[i];
    }
    // one SM each, the rest by largest remainder of the work share
    std::vector<int> sm(count, 1);
    const int spare = sms - count;
    std::vector<std::pair<double, int>> rem;
    int given = 0;
    for (int i = 0; i < count; ++i) {
        const double share = tot > 0 ? spare * work[i] / tot : (double)spare / count;
        const int whole = (int)std::floor(share);
        sm[i] += whole;
        given += whole;
        rem.push_back({share - whole, i});
    }
    std::stable_sort(rem.begin(), rem.end(), [](const std::pair<double, int> &a, const std::pair<double, int> &b) {
        return a.first > b.first;
    });
    for (int r = 0; r < spare - given; ++r) sm[rem[r].second] += 1;
    for (int i = 0; i < count; ++i) grid_out[i] = sm[i] * ctas_per_sm[i];
    return 0;
}

int mset_group_create(int device, mset_group **out) {
    if (!out) return fail(MSET_E_ARG, "null output pointer");
    *out = nullptr;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDeviceCount");
    if (device < 0 || device >= ndev) return fail(MSET_E_ARG, "device %d out of range", device);
    mset_group *g = new mset_group;
    g->device = device;
    e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&g->st, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&g->fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreate(&g->ev0);
    if (e == cudaSuccess) e = cudaEventCreate(&g->ev1);
    if (e != cudaSuccess) {
        mset_group_destroy(g);
        return cuda_fail(e, "group setup");
    }
    *out = g;
    return 0;
}

int mset_group_destroy(mset_group *g) {
    if (!g) return 0;
    cudaSetDevice(g->device);
    if (g->st) cudaStreamSynchronize(g->st);
    group_drop_graph(g);
    for (cudaEvent_t e : g->done) cudaEventDestroy(e);
    if (g->fork) cudaEventDestroy(g->fork);
    if (g->ev0) cudaEventDestroy(g->ev0);
    if (g->ev1) cudaEventDestroy(g->ev1);
    if (g->st) cudaStreamDestroy(g->st);
    delete g;
    return 0;
}

int mset_group_add(mset_group *g, mset_session *s) {
    if (!g) return fail(MSET_E_ARG, "null group");
    int rc = batch_ok(s);
    if (rc) return rc;
    if (s->device != g->device) return fail(MSET_E_ARG, "session on device %d, group on %d", s->device, g->device);
    for (mset_session *o : g->m)
        if (o == s) return fail(MSET_E_ARG, "session already in the group");
    CK(cudaSetDevice(g->device));
    cudaEvent_t e = nullptr;
    CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    g->m.push_back(s);
    g->done.push_back(e);
    group_drop_graph(g);
    return 0;
}

int mset_group_set_schedule(mset_group *g, int schedule) {
    if (!g) return fail(MSET_E_ARG, "null group");
    if (schedule != MSET_GROUP_SERIAL && schedule != MSET_GROUP_CONCURRENT)
        return fail(MSET_E_ARG, "unknown schedule %d", schedule);
    if (schedule != g->schedule) group_drop_graph(g);
    g->schedule = schedule;
    return 0;
}

int mset_group_gradient(mset_group *g, int use_graph) {
    Range range_("mset_group_gradient");
    if (!g) return fail(MSET_E_ARG, "null group");
    std::vector<int> grids;
    int rc = group_prepare(g, grids);
    if (rc) return rc;
    rc = group_launch(g, grids, use_graph != 0);
    if (rc) return rc;
    CK(cudaStreamSynchronize(g->st));
    for (mset_session *m : g->m)
        if ((rc = take_fault(m)) != 0) return rc;
    return 0;
}

int mset_group_time(mset_group *g, int reps, int use_graph, double *ms_per_pass) {
    if (!g || reps <= 0 || !ms_per_pass) return fail(MSET_E_ARG, "bad arguments");
    std::vector<int> grids;
    int rc = group_prepare(g, grids);
    if (rc) return rc;
    rc = group_launch(g, grids, use_graph != 0);  // warm (and capture)
    if (rc) return rc;
    CK(cudaEventRecord(g->ev0, g->st));
    for (int r = 0; r < reps; ++r) {
        rc = group_launch(g, grids, use_graph != 0);
        if (rc) return rc;
    }
    CK(cudaEventRecord(g->ev1, g->st));
    CK(cudaEventSynchronize(g->ev1));
    float t = 0;
    CK(cudaEventElapsedTime(&t, g->ev0, g->ev1));
    *ms_per_pass = t / reps;
    for (mset_session *m : g->m)
        if ((rc = take_fault(m)) != 0) return rc;
    return 0;
}

int mset_group_tune(mset_group *g, double mem_budget_bytes, int *schedule_out) {
    Range range_("mset_group_tune");
    if (!g) return fail(MSET_E_ARG, "null group");
    if (g->m.empty()) return fail(MSET_E_STATE, "empty group");
    if (mem_budget_bytes < 0) return fail(MSET_E_ARG, "negative memory budget");
    // the budget is split in proportion to each member's full-storage need
    double need = 0;
    for (mset_session *s : g->m) need += save_bytes(s, persistent_grid(s, std::max(1, s->total_pos)), 0);
    for (mset_session *s : g->m) {
        if (s->total_pos == 0) continue;
        const double own = save_bytes(s, persistent_grid(s, std::max(1, s->total_pos)), 0);
        const double b = mem_budget_bytes > 0 ? mem_budget_bytes * own / std::max(need, 1.0) : 0;
        CK(cudaSetDevice(s->device));
        s->tuned_grid = 0;
        int rc = tune_session(s, b, nullptr);
        if (rc) return rc;
    }
    // both schedules, timed on full passes
    double best = 0;
    int best_sched = MSET_GROUP_SERIAL;
    for (int sched : {MSET_GROUP_SERIAL, MSET_GROUP_CONCURRENT}) {
        int rc = mset_group_set_schedule(g, sched);
        if (rc) return rc;
        double ms = 0;
        rc = mset_group_time(g, 2, 0, &ms);
        if (rc) return rc;
        if (sched == MSET_GROUP_SERIAL || ms < best) {
            best = ms;
            best_sched = sched;
        }
    }
    int rc = mset_group_set_schedule(g, best_sched);
    if (rc) return rc;
    if (schedule_out) *schedule_out = best_sched;
    return 0;
}

}  // extern "C"
