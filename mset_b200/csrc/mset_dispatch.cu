// mset_dispatch.cu -- window-size dispatch and the size-independent
// kernels of the batched update.
#include <algorithm>
#include "mset_kernels.cuh"


namespace mset {

// every compiled geometry; the first entry of a window size is its default,
// the others with the same scrambled layouts are alternative thread shapes
// the autotuner may pick (at n = 256 the default stages the adjoint's
// saved-wave rows by bulk copies: 1.443 s against 1.474 s per pass of 3 large
// tilts on one B200).  At n = 128 the default is the three-phase shape; the
// two-pass shape 128 after it has the layout of the sequential cluster
// geometry 128c8 and serves the sequential entry points.
#define MSET_GEOS(X) X(24) X(32) X(48) X(64) X(64v2) X(96) X(96v2) X(128t) X(128w) X(128) X(160) X(160v2) X(256s) X(256) X(256v2)
#define X(N_) extern const GeoOps kGeo##N_;
MSET_GEOS(X)
#undef X

static const GeoOps *const kAllGeos[] = {
#define X(N_) &kGeo##N_,
    MSET_GEOS(X)
#undef X
};

// the reference-semantics pass and the per-position steps walk one position
// at a time through one field; these geometries split that field over a
// thread-block cluster so one position uses several SMs
#define MSET_SEQ_GEOS(X) X(128c8)
#define X(N_) extern const GeoOps kSeqGeo##N_;
MSET_SEQ_GEOS(X)
#undef X
static const GeoOps *const kSeqGeos[] = {
#define X(N_) &kSeqGeo##N_,
    MSET_SEQ_GEOS(X)
#undef X
};

static void fill_plan(const GeoOps *g, Plan *p) {
    p->n = g->n;
    p->r1 = g->r1;
    p->ry1 = g->ry1;
    p->nt = g->nt;
    p->cl = g->cl;
    p->staged = g->staged;
    p->max_clusters = 0;
    p->smem = g->smem;
    p->ctas_per_sm = 0;
    p->ops = g;
}

bool plan_seq_for(int n, Plan *p) {
    for (const GeoOps *g : kSeqGeos)
        if (g->n == n) {
            fill_plan(g, p);
            p->staged = 0;
            return true;
        }
    return false;
}

static bool same_layout(const GeoOps *a, const GeoOps *b) { return a->r1 == b->r1 && a->ry1 == b->ry1; }

static const GeoOps *default_geo(int n) {
    for (const GeoOps *g : kAllGeos)
        if (g->n == n) return g;
    return nullptr;
}

// the shapes of window n with the default's scrambled layouts, default first
static const GeoOps *find_geo(int n, int variant) {
    const GeoOps *d = default_geo(n);
    if (!d) return nullptr;
    for (const GeoOps *g : kAllGeos)
        if (g->n == n && same_layout(g, d) && variant-- == 0) return g;
    return nullptr;
}

int plan_variants(int n) {
    const GeoOps *d = default_geo(n);
    int c = 0;
    for (const GeoOps *g : kAllGeos) c += d && g->n == n && same_layout(g, d);
    return c;
}

bool plan_for(int n, Plan *p, int variant) {
    const GeoOps *g = find_geo(n, variant);
    if (!g) return false;
    fill_plan(g, p);
    return true;
}

bool plan_for_layout(int n, int r1, int ry1, Plan *p) {
    for (const GeoOps *g : kAllGeos)
        if (g->n == n && g->r1 == r1 && g->ry1 == ry1) {
            fill_plan(g, p);
            return true;
        }
    return false;
}

int launch_positions(const Plan &pl, int method, int adjoint, int mode, const LaunchArgs &a, int grid,
                     cudaStream_t st) {
    return pl.ops->positions(method, adjoint, mode, a, grid, st);
}
int launch_prep_amp(const Plan &pl, const float *meas, float *amp, long npos, cudaStream_t st) {
    return pl.ops->prep_amp(meas, amp, npos, st);
}
int launch_prep_amp_bf16(const Plan &pl, const float *meas, unsigned short *ib, long npos, cudaStream_t st) {
    return pl.ops->prep_amp_bf16(meas, ib, npos, st);
}
int launch_prep_prop(const Plan &pl, const float *prop, float2 *pscr, cudaStream_t st) {
    return pl.ops->prep_prop(prop, pscr, st);
}
int launch_probe_to_q(const Plan &pl, const float2 *probe, float2 *q, const float2 *twn, cudaStream_t st) {
    return pl.ops->probe_q(true, probe, q, twn, st);
}
int launch_q_to_probe(const Plan &pl, const float2 *q, float2 *probe, const float2 *twn, cudaStream_t st) {
    return pl.ops->probe_q(false, q, probe, twn, st);
}

// batched update: V += step0 * G (slab-replicated), Q -= step1 * qacc,
// positions += step2 * posdir
__global__ void k_apply_volume(float *V, const double *g, int n2, int nz, int b, float step0) {
    const long total = (long)nz * n2;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
        const int z = (int)(i / n2);
        const int l = (int)(i % n2);
        const int s = z / b;
        V[i] += step0 * (float)g[(long)s * n2 + l];
    }
}
__global__ void k_apply_probe(float2 *Q, const double *qacc, int n2, float step1) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n2; i += gridDim.x * blockDim.x) {
        float2 q = Q[i];
        q.x -= step1 * (float)qacc[2 * i];
        q.y -= step1 * (float)qacc[2 * i + 1];
        Q[i] = q;
    }
}
__global__ void k_apply_pos(float *sx, float *sy, const double *pd, int npos, float step2) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npos; i += gridDim.x * blockDim.x) {
        sx[i] += step2 * (float)pd[2 * i];
        sy[i] += step2 * (float)pd[2 * i + 1];
    }
}

// transmission slabs of every tilt: T[s][y][x] = exp(i sdz sum_{z in slab s} V)
// (mset.cu:134-153), once per pass so the position kernel reads one complex
// value instead of recomputing it in the forward and the adjoint
__global__ void k_transmission(const TiltDev *tilts, int ntilts, int n2, int nz, int b, int ns, float sdz) {
    const long per = (long)ns * n2;
    const long total = per * ntilts;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
        const int j = (int)(i / per);
        const long r = i % per;
        const int s = (int)(r / n2);
        const int l = (int)(r % n2);
        const TiltDev &t = tilts[j];
        const int z0 = s * b, z1 = min(z0 + b, nz);
        float acc = 0.f;
        for (int z = z0; z < z1; ++z) acc += __ldg(t.V + (size_t)z * n2 + l);
        float sn, cs;
        sincosf(sdz * acc, &sn, &cs);
        const_cast<float2 *>(t.T)[r] = make_float2(cs, sn);
    }
}

int launch_transmission(const TiltDev *tilts, int ntilts, int n, int nz, int b, int ns, float sdz, cudaStream_t st) {
    const long total = (long)ntilts * ns * n * n;
    const int grid = (int)std::min<long>((total + 255) / 256, 148L * 16);
    k_transmission<<<grid, 256, 0, st>>>(tilts, ntilts, n * n, nz, b, ns, sdz);
    return (int)cudaGetLastError();
}

int launch_apply_batch(int n, int nz, int b, int ns, int method, float step0, float step1, float step2,
                       const TiltDev *tilts, int ntilts, cudaStream_t st) {
    (void)ns;
    const int n2 = n * n;
    const int bb = method == kSSET ? nz : b;
    for (int j = 0; j < ntilts; ++j) {
        const TiltDev &t = tilts[j];
        k_apply_volume<<<592, 256, 0, st>>>(t.V, t.grad, n2, nz, bb, step0);
        k_apply_probe<<<64, 256, 0, st>>>(t.Q, t.qacc, n2, step1);
        k_apply_pos<<<8, 256, 0, st>>>(t.sx, t.sy, t.posdir, t.npos, step2);
    }
    return (int)cudaGetLastError();
}

int launch_apply_probe_pos(const TiltDev *tilts, int ntilts, int n, float step1, float step2, cudaStream_t st) {
    for (int j = 0; j < ntilts; ++j) {
        const TiltDev &t = tilts[j];
        k_apply_probe<<<64, 256, 0, st>>>(t.Q, t.qacc, n * n, step1);
        if (t.npos) k_apply_pos<<<8, 256, 0, st>>>(t.sx, t.sy, t.posdir, t.npos, step2);
    }
    return (int)cudaGetLastError();
}

}  // namespace mset
