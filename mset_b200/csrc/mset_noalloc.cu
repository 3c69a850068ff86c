// mset_noalloc.cu -- an allocation-free variant of the batched gradient pass
// for one tilt (mset_batch_gradient_noalloc in include/mset_b200.h).
//
// Some callers cannot call cudaMalloc: code that runs while a CUDA graph is
// being captured, hosts whose device memory is owned by a framework allocator
// or by MATLAB gpuArrays, and real-time pipelines that forbid allocation after
// start-up.  They pass their own device buffers for every input and output;
// the scratch this pass needs (saved waves, the prepared propagator and probe
// spectrum, the probe accumulator, the work counter) lives in one file-scope
// device array of fixed size, which every GPU that loads the library holds
// until the process exits.
#include <cuda.h>

#include <algorithm>
#include <cmath>
#include <mutex>

#include "../../include/mset_b200.h"
#include "mset_kernels_impl.cuh"

namespace {

using namespace mset;

// fixed scratch: 64 MiB per device
constexpr size_t kScratchBytes = size_t(64) << 20;
constexpr int kMaxPositions = 1 << 17;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// device address of g_noalloc_scratch, resolved once per device with that
// device current (the host-side symbol is only a stand-in, not a device
// address), together with the id of the context it was resolved in: after a
// device reset the module is loaded again in a new primary context and the
// array may sit elsewhere, so a changed id resolves it again
std::mutex g_mu;
void *g_scratch_ptr[64] = {};
unsigned long long g_scratch_ctx[64] = {};

// id of the context current on this thread (cuCtxGetId through the runtime's
// driver entry points, so the library needs no link to libcuda); 0 when it
// cannot be had, and then the address is resolved on every call
unsigned long long current_context_id() {
    using PfnGetCurrent = CUresult (*)(CUcontext *);
    using PfnGetId = CUresult (*)(CUcontext, unsigned long long *);
    static PfnGetCurrent get_current = nullptr;
    static PfnGetId get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<PfnGetCurrent>(f);
        f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<PfnGetId>(f);
    });
    if (!get_current || !get_id) return 0;
    CUcontext c = nullptr;
    unsigned long long id = 0;
    if (get_current(&c) != CUDA_SUCCESS || !c || get_id(c, &id) != CUDA_SUCCESS) return 0;
    return id;
}

size_t align256(size_t v) { return (v + 255) & ~size_t(255); }

int err(int code, const char *msg) {
    set_last_error(msg);
    return code;
}

__global__ void k_noalloc_twiddles(float2 *twn, int n, int r1) {
    const int r2 = n / r1;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const int k2 = i / r1, n1 = i % r1;
        const long m = (long)n1 * k2 % n;
        double s, c;
        sincospi(-2.0 * (double)m / (double)n, &s, &c);
        twn[i] = make_float2((float)c, (float)s);
    }
    (void)r2;
}

__global__ void k_noalloc_setup(TiltDev *table, TiltDev t, int2 *items, int npos) {
    if (blockIdx.x == 0 && threadIdx.x == 0) *table = t;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npos; i += gridDim.x * blockDim.x)
        items[i] = make_int2(0, i);
}

// scrambled accumulator -> standard FFT order
__global__ void k_noalloc_unscramble(const double *qacc, double *out, int n, int r1) {
    const int r2 = n / r1;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n * n; i += gridDim.x * blockDim.x) {
        const int ly = i / n, lx = i % n;
        const int ky = ly / r1 + r2 * (ly % r1), kx = lx / r1 + r2 * (lx % r1);
        out[2 * ((size_t)ky * n + kx)] = qacc[2 * (size_t)i];
        out[2 * ((size_t)ky * n + kx) + 1] = qacc[2 * (size_t)i + 1];
    }
}

template <class G>
int run_geo(int method, int adjoint, const LaunchArgs &a, int grid, cudaStream_t st) {
#define MSET_NA(M, A) \
    if (method == M && adjoint == A) return launch_one<G, M, A, kBatchCentred>(a, grid, st);
    MSET_NA(kMSET, kREF) MSET_NA(kMSET, kEXACT) MSET_NA(kSSET, kREF) MSET_NA(kSSET, kEXACT)
#undef MSET_NA
    return (int)cudaErrorInvalidValue;
}

struct NaGeo {
    int n, r1, nt, minb;
    size_t smem;
    int (*run)(int, int, const LaunchArgs &, int, cudaStream_t);
    int (*prep_prop)(const float *, float2 *, cudaStream_t);
    int (*probe_q)(bool, const float2 *, float2 *, const float2 *, cudaStream_t);
};

#define MSET_NA_GEO(N_, R1_, NT_, MINB_)                                                                 \
    {N_, R1_, NT_, MINB_, smem_bytes<Geo<N_, R1_, NT_, MINB_>>(), &run_geo<Geo<N_, R1_, NT_, MINB_>>, \
     &geo_prep_prop<Geo<N_, R1_, NT_, MINB_>>, &geo_probe_q<Geo<N_, R1_, NT_, MINB_>>}

const NaGeo kNaGeos[] = {MSET_NA_GEO(24, 8, 64, 8), MSET_NA_GEO(64, 8, 256, 2), MSET_NA_GEO(128, 16, 512, 1)};

}  // namespace

extern "C" int mset_batch_gradient_noalloc(int device, void *stream, int n, int nz, int slice_binning, int method,
                                           int adjoint, float sigma, float potential_pixelsize, int npos,
                                           const float *rvol_dev, const float *probe_dev, const float *prop2D_dev,
                                           const float *scan_x_dev, const float *scan_y_dev,
                                           const float *measured_dev, double *grad_dev, double *probe_out_dev,
                                           double *posdir_dev, double *err_dev) {
    const NaGeo *g = nullptr;
    for (const NaGeo &c : kNaGeos)
        if (c.n == n) g = &c;
    if (!g) return err(MSET_E_UNSUPPORTED, "mset_batch_gradient_noalloc: window size must be 24, 64 or 128");
    if (nz <= 0 || slice_binning <= 0 || npos <= 0 || npos > kMaxPositions)
        return err(MSET_E_ARG, "mset_batch_gradient_noalloc: need nz > 0, slice_binning > 0, 0 < npos <= 131072");
    if ((method != MSET_MODE_MSET && method != MSET_MODE_SSET) ||
        (adjoint != MSET_ADJOINT_REF && adjoint != MSET_ADJOINT_EXACT))
        return err(MSET_E_ARG, "mset_batch_gradient_noalloc: bad method or adjoint");
    if (!rvol_dev || !probe_dev || !prop2D_dev || !scan_x_dev || !scan_y_dev || !measured_dev || !grad_dev ||
        !probe_out_dev || !posdir_dev || !err_dev)
        return err(MSET_E_ARG, "mset_batch_gradient_noalloc: null device pointer");
    if (device < 0 || device >= 64) return err(MSET_E_ARG, "mset_batch_gradient_noalloc: device out of range");
    const int b = slice_binning > nz ? nz : slice_binning;
    const int ns = (nz + b - 1) / b;
    const size_t n2 = (size_t)n * n;

    // scratch layout
    const size_t off_twn = 0;
    const size_t off_pscr = align256(off_twn + sizeof(float2) * n);
    const size_t off_q = align256(off_pscr + sizeof(float2) * n2);
    const size_t off_qacc = align256(off_q + sizeof(float2) * n2);
    const size_t off_tab = align256(off_qacc + sizeof(double) * 2 * n2);
    const size_t off_cnt = align256(off_tab + sizeof(TiltDev));
    const size_t off_items = align256(off_cnt + sizeof(unsigned));
    const size_t off_save = align256(off_items + sizeof(int2) * npos);
    const size_t slot = sizeof(float2) * (size_t)(ns + 1) * n2;
    if (off_save + slot > kScratchBytes)
        return err(MSET_E_UNSUPPORTED,
                   "mset_batch_gradient_noalloc: (ns + 1) saved waves of n x n complex exceed the 64 MiB scratch");
    const int slots = (int)((kScratchBytes - off_save) / slot);

    int prev = 0;
    cudaError_t e = cudaGetDevice(&prev);
    if (e != cudaSuccess) return err(MSET_E_CUDA, cudaGetErrorString(e));
    e = cudaSetDevice(device);
    if (e != cudaSuccess) return err(MSET_E_CUDA, cudaGetErrorString(e));
    int rc = 0;
    unsigned char *base = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        const unsigned long long ctx = current_context_id();
        if (!g_scratch_ptr[device] || ctx == 0 || ctx != g_scratch_ctx[device]) {
            void *ptr = nullptr;
            e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
            if (e != cudaSuccess) {
                cudaSetDevice(prev);
                return err(MSET_E_CUDA, cudaGetErrorString(e));
            }
            g_scratch_ptr[device] = ptr;
            g_scratch_ctx[device] = ctx;
        }
        base = static_cast<unsigned char *>(g_scratch_ptr[device]);
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    float2 *twn = reinterpret_cast<float2 *>(base + off_twn);
    float2 *pscr = reinterpret_cast<float2 *>(base + off_pscr);
    float2 *q = reinterpret_cast<float2 *>(base + off_q);
    double *qacc = reinterpret_cast<double *>(base + off_qacc);
    TiltDev *tab = reinterpret_cast<TiltDev *>(base + off_tab);
    unsigned *cnt = reinterpret_cast<unsigned *>(base + off_cnt);
    int2 *items = reinterpret_cast<int2 *>(base + off_items);
    float2 *save = reinterpret_cast<float2 *>(base + off_save);

    int sms = 0;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess || sms <= 0) {
        cudaSetDevice(prev);
        return err(MSET_E_CUDA, e != cudaSuccess ? cudaGetErrorString(e) : "no multiprocessors reported");
    }
    const int by_smem = (int)((227 * 1024) / (g->smem + 1024));
    const int per_sm = std::max(1, std::min(std::min(by_smem, 2048 / g->nt), g->minb));
    const int grid = std::max(1, std::min(std::min(slots, sms * per_sm), npos));

    TiltDev t{};
    t.V = const_cast<float *>(rvol_dev);
    t.Q = q;
    t.amp = measured_dev;
    t.sx = const_cast<float *>(scan_x_dev);
    t.sy = const_cast<float *>(scan_y_dev);
    t.grad = grad_dev;
    t.qacc = qacc;
    t.posdir = posdir_dev;
    t.err = err_dev;
    t.npos = npos;

    do {
        k_noalloc_twiddles<<<1, 256, 0, st>>>(twn, n, g->r1);
        if ((e = cudaGetLastError()) != cudaSuccess) break;
        k_noalloc_setup<<<(npos + 255) / 256, 256, 0, st>>>(tab, t, items, npos);
        if ((e = cudaGetLastError()) != cudaSuccess) break;
        if ((rc = g->prep_prop(prop2D_dev, pscr, st)) != 0) break;
        if ((rc = g->probe_q(true, reinterpret_cast<const float2 *>(probe_dev), q, twn, st)) != 0) break;
        const int nsg = method == MSET_MODE_SSET ? 1 : ns;
        if ((e = cudaMemsetAsync(grad_dev, 0, sizeof(double) * nsg * n2, st)) != cudaSuccess) break;
        if ((e = cudaMemsetAsync(qacc, 0, sizeof(double) * 2 * n2, st)) != cudaSuccess) break;
        if ((e = cudaMemsetAsync(err_dev, 0, sizeof(double), st)) != cudaSuccess) break;
        if ((e = cudaMemsetAsync(cnt, 0, sizeof(unsigned), st)) != cudaSuccess) break;
        LaunchArgs a{};
        a.tilts = tab;
        a.items = items;
        a.nitems = npos;
        a.counter = cnt;
        a.save = save;
        a.pscr = pscr;
        a.twn = twn;
        a.nz = nz;
        a.b = b;
        a.ns = ns;
        a.sdz = sigma * potential_pixelsize;
        a.center = (float)std::round((n + 1.0f) / 2.0f);
        a.ckpt = 0;
        a.slots = ns + 1;  // one scratch slot of (ns + 1) waves per CTA, as sized above
        if ((rc = g->run(method, adjoint, a, grid, st)) != 0) break;
        k_noalloc_unscramble<<<64, 256, 0, st>>>(qacc, probe_out_dev, n, g->r1);
        e = cudaGetLastError();
    } while (0);
    cudaSetDevice(prev);
    if (rc != 0) e = (cudaError_t)rc;
    if (e != cudaSuccess) return err(MSET_E_CUDA, cudaGetErrorString(e));
    return 0;
}
