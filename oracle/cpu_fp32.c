/*
 * cpu_fp32.c -- single-precision CPU port of the reference's per-position
 * multislice forward + adjoint, for the timed CPU baseline.
 *
 * TEST INFRASTRUCTURE ONLY.  bench.py times it as the CPU baseline (the
 * reference's own CPU path is MATLAB code in single precision,
 * STEP00_INIT.m:224 and Run_MSET_recon.m:131 cast the volume and probe to
 * single; MATLAB is not available here); tests/test_cpu_fp32.py checks it
 * against the FP64 oracle.  Nothing in the product path (mset_b200/) links,
 * loads or calls it.
 *
 * Per position it follows the same steps as mset_oracle.c's position() and
 * the reference it cites (src/CUDA/mset.cu:107-327, STEP02_FORWARD_4D.m:6-51,
 * STEP03_BACK.m:6-39): shifted probe psi0 = F(F^{-1}(probe) fs), transmission
 * of every slab, propagation F^{-1}(P F(T psi)), far field, amplitude
 * residual, back-propagation with the reference formula for the volume
 * gradient (mset.cu:248-251), probe direction and finite-difference position
 * direction (utility.cu:829-876).  Arithmetic in float; the batched sums over
 * positions (volume gradient, probe direction, error) in double, as the
 * batched method on the GPU keeps them.  Transmission slabs are computed once
 * per call (the batched method's order); positions run in parallel over
 * OpenMP threads, each with its own float gradient buffer.
 *
 * cpu32_sequential_tilt is the same position in the reference's own order
 * (run_main_mset, mset.cu:80-334; Run_MSET_recon.m:136-157 on the CPU path):
 * one position after the other on one thread, each starting from the volume,
 * probe and coordinates the previous ones updated, with the transmission
 * rebuilt from the current volume per position (mset.cu:134-153).
 *
 * FFT: iterative radix-2 (window edge a power of two), twiddles computed in
 * double and stored as float.
 */
#define _GNU_SOURCE
#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef float _Complex cf;

#define REF_PI_F 3.1415926f /* utility.cu:790 */

typedef struct {
    int n, logn;
    cf *w;     /* w[k] = exp(-2 pi i k / n), k < n/2 */
    int *rev;  /* bit reversal permutation */
} plan32;

static int plan32_init(plan32 *p, int n) {
    int l = 0;
    while ((1 << l) < n) ++l;
    if ((1 << l) != n) return -1;
    p->n = n;
    p->logn = l;
    p->w = malloc(sizeof(cf) * (size_t)(n / 2 > 0 ? n / 2 : 1));
    p->rev = malloc(sizeof(int) * (size_t)n);
    for (int k = 0; k < n / 2; ++k) {
        double a = -2.0 * M_PI * (double)k / (double)n;
        p->w[k] = (float)cos(a) + I * (float)sin(a);
    }
    for (int i = 0; i < n; ++i) {
        int r = 0;
        for (int b = 0; b < l; ++b) r |= ((i >> b) & 1) << (l - 1 - b);
        p->rev[i] = r;
    }
    return 0;
}

static void plan32_free(plan32 *p) {
    free(p->w);
    free(p->rev);
}

/* in-place unnormalised 1D FFT of x[0..n) (contiguous), sign -1 or +1 */
static void fft1(const plan32 *p, cf *x, int sign) {
    const int n = p->n;
    for (int i = 0; i < n; ++i) {
        const int r = p->rev[i];
        if (r > i) {
            cf t = x[i];
            x[i] = x[r];
            x[r] = t;
        }
    }
    for (int len = 2; len <= n; len <<= 1) {
        const int half = len >> 1, step = n / len;
        for (int i = 0; i < n; i += len)
            for (int j = 0; j < half; ++j) {
                cf w = p->w[j * step];
                if (sign > 0) w = conjf(w);
                const cf u = x[i + j], v = x[i + j + half] * w;
                x[i + j] = u + v;
                x[i + j + half] = u - v;
            }
    }
}

/* 2D FFT of a [n][n] array: rows, then columns through a line buffer */
static void fft2(const plan32 *p, cf *a, int sign, cf *line) {
    const int n = p->n;
    for (int r = 0; r < n; ++r) fft1(p, a + (size_t)r * n, sign);
    for (int c = 0; c < n; ++c) {
        for (int r = 0; r < n; ++r) line[r] = a[(size_t)r * n + c];
        fft1(p, line, sign);
        for (int r = 0; r < n; ++r) a[(size_t)r * n + c] = line[r];
    }
}

static void ifft2n(const plan32 *p, cf *a, cf *line) {
    const size_t n2 = (size_t)p->n * p->n;
    fft2(p, a, +1, line);
    const float s = 1.0f / (float)n2;
    for (size_t i = 0; i < n2; ++i) a[i] *= s;
}

/* circular shift by ceil(n/2) (utility.cu:609-630 as used at mex_main.cu:80) */
static size_t ishift(int r, int c, int n) {
    const int h = (n + 1) / 2;
    return (size_t)((r + h) % n) * n + (size_t)((c + h) % n);
}

/* Fourier shift factor in standard order (utility.cu:776-800, mset.cu:122) */
static void shift_factor(int n, float s1, float s2, cf *out) {
    const int h = (n + 1) / 2;
    for (int k1 = 0; k1 < n; ++k1) {
        const float n1 = (float)(((k1 - h) % n + n) % n) - 0.5f * (float)n;
        for (int k2 = 0; k2 < n; ++k2) {
            const float nn2 = (float)(((k2 - h) % n + n) % n) - 0.5f * (float)n;
            const float ph = 2.0f * REF_PI_F * (s1 * n1 / (float)n + s2 * nn2 / (float)n);
            out[(size_t)k1 * n + k2] = cosf(ph) + I * sinf(ph);
        }
    }
}

/* Batched forward + adjoint over npos positions of one tilt (reference
 * adjoint formula), single precision.  Inputs as mset_oracle.c's
 * orc_batched_tilt: rvol [nz][n][n], probe / prop [n][n][2] (prop centred),
 * measured [npos][n][n] centred.  Outputs: grad [ns][n][n] (sum of Re g over
 * positions), probe_acc [n][n][2] (sum of the probe directions, standard
 * order), pos_dir [npos][2], err_sum [1].  Returns 0, or -1 for a window that
 * is not a power of two or bad sizes. */
int cpu32_batched_tilt(int n, int nz, int binning, double sigma, double dz, int npos, const float *rvol,
                       const float *probe, const float *prop_centred, const float *scan_x, const float *scan_y,
                       const float *measured, double *grad, double *probe_acc, double *pos_dir, double *err_sum,
                       int nthreads) {
    if (n < 2 || nz <= 0 || binning <= 0 || npos < 0) return -1;
    plan32 pl;
    if (plan32_init(&pl, n)) return -1;
    const size_t n2 = (size_t)n * n;
    const int ns = (nz + binning - 1) / binning; /* STEP00_INIT.m:185 */
    cf *P = malloc(sizeof(cf) * n2), *Q = malloc(sizeof(cf) * n2), *T = malloc(sizeof(cf) * n2 * ns);
    for (int r = 0; r < n; ++r)
        for (int c = 0; c < n; ++c) {
            const size_t i = (size_t)r * n + c;
            P[ishift(r, c, n)] = prop_centred[2 * i] + I * prop_centred[2 * i + 1]; /* mex_main.cu:80 */
            Q[i] = probe[2 * i] + I * probe[2 * i + 1];
        }
    {
        cf *line = malloc(sizeof(cf) * n);
        ifft2n(&pl, Q, line); /* F^{-1}(probe), hoisted out of the position loop */
        free(line);
    }
    const float sdz = (float)(sigma * dz);
    for (int s = 0; s < ns; ++s) { /* mset.cu:134-153 */
        const int z0 = s * binning, z1 = z0 + binning < nz ? z0 + binning : nz;
        for (size_t i = 0; i < n2; ++i) {
            float acc = 0.f;
            for (int z = z0; z < z1; ++z) acc += rvol[(size_t)z * n2 + i];
            T[(size_t)s * n2 + i] = cosf(sdz * acc) + I * sinf(sdz * acc);
        }
    }
    memset(grad, 0, sizeof(double) * n2 * ns);
    memset(probe_acc, 0, sizeof(double) * 2 * n2);
    double err_total = 0.0;
    const float center = roundf((n + 1.0f) / 2.0f); /* mset.cu:83 */
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
#pragma omp parallel reduction(+ : err_total)
    {
        cf *w = malloc(sizeof(cf) * n2), *fs = malloc(sizeof(cf) * n2), *psi0 = malloc(sizeof(cf) * n2);
        cf *waves = malloc(sizeof(cf) * n2 * (ns + 1)), *line = malloc(sizeof(cf) * n), *d = malloc(sizeof(cf) * n2);
        float *gl = calloc(n2 * ns, sizeof(float));
        double *pl_acc = calloc(2 * n2, sizeof(double));
#pragma omp for schedule(dynamic, 1)
        for (int p = 0; p < npos; ++p) {
            const float s1 = scan_y[p] - center, s2 = scan_x[p] - center; /* mset.cu:121 */
            shift_factor(n, s1, s2, fs);
            for (size_t i = 0; i < n2; ++i) psi0[i] = Q[i] * fs[i];
            fft2(&pl, psi0, -1, line);
            memcpy(w, psi0, sizeof(cf) * n2);
            for (int s = 0; s < ns; ++s) { /* mset.cu:157-183 */
                const cf *Ts = T + (size_t)s * n2;
                for (size_t i = 0; i < n2; ++i) w[i] *= Ts[i];
                fft2(&pl, w, -1, line);
                for (size_t i = 0; i < n2; ++i) w[i] *= P[i];
                ifft2n(&pl, w, line);
                memcpy(waves + (size_t)(s + 1) * n2, w, sizeof(cf) * n2);
            }
            fft2(&pl, w, -1, line); /* far field, residual (mset.cu:186-227) */
            const float *meas = measured + (size_t)p * n2;
            double e = 0.0;
            for (int r = 0; r < n; ++r)
                for (int c = 0; c < n; ++c) {
                    const size_t k = ishift(r, c, n);
                    const float a2 = crealf(w[k]) * crealf(w[k]) + cimagf(w[k]) * cimagf(w[k]);
                    const float A = sqrtf(a2 + 1e-30f), M = sqrtf(meas[(size_t)r * n + c]);
                    e += (double)((A - M) * (A - M));
                    w[k] *= 1.0f - M / A;
                }
            err_total += e;
            for (int s = ns - 1; s >= 0; --s) { /* mset.cu:232-271 */
                const cf *Ts = T + (size_t)s * n2;
                const cf *psi = waves + (size_t)(s + 1) * n2; /* mset.cu:248-251 */
                for (size_t i = 0; i < n2; ++i) w[i] *= conjf(P[i]);
                ifft2n(&pl, w, line);
                float *g = gl + (size_t)s * n2;
                for (size_t i = 0; i < n2; ++i) {
                    g[i] += crealf(I * conjf(Ts[i]) * conjf(psi[i]) * w[i]);
                    w[i] *= conjf(Ts[i]);
                }
                if (s > 0) fft2(&pl, w, -1, line);
            }
            /* probe direction F^{-1}(chi0) fs(-s) (mset.cu:288-309), kept in the
             * F^{-1}(probe) domain as the batched method accumulates it */
            memcpy(d, w, sizeof(cf) * n2);
            ifft2n(&pl, d, line);
            for (size_t i = 0; i < n2; ++i) {
                const cf v = d[i] * conjf(fs[i]);
                pl_acc[2 * i] += crealf(v);
                pl_acc[2 * i + 1] += cimagf(v);
            }
            /* position direction, finite differences of conj(psi0) (utility.cu:829-876) */
            double px = 0.0, py = 0.0;
            for (int i1 = 0; i1 < n; ++i1)
                for (int i2 = 0; i2 < n; ++i2) {
                    const size_t i = (size_t)i1 * n + i2;
                    const cf *f = psi0;
                    cf dx, dy;
                    if (i2 == 0) dx = conjf(f[i + 1]) - conjf(f[i]);
                    else if (i2 == n - 1) dx = conjf(f[i]) - conjf(f[i - 1]);
                    else dx = (conjf(f[i + 1]) - conjf(f[i - 1])) * 0.5f;
                    if (i1 == 0) dy = conjf(f[i + n]) - conjf(f[i]);
                    else if (i1 == n - 1) dy = conjf(f[i]) - conjf(f[i - n]);
                    else dy = (conjf(f[i + n]) - conjf(f[i - n])) * 0.5f;
                    px += (double)crealf(dx * w[i]);
                    py += (double)crealf(dy * w[i]);
                }
            pos_dir[2 * p] = px;
            pos_dir[2 * p + 1] = py;
        }
#pragma omp critical
        {
            for (size_t i = 0; i < n2 * ns; ++i) grad[i] += (double)gl[i];
            for (size_t i = 0; i < 2 * n2; ++i) probe_acc[i] += pl_acc[i];
        }
        free(w);
        free(fs);
        free(psi0);
        free(waves);
        free(line);
        free(d);
        free(gl);
        free(pl_acc);
    }
    /* the probe direction in the probe's own (Fourier) domain: F of the sum
     * equals the oracle's sum of F(F^{-1}(chi0) fs(-s)) (mset.cu:288-309) */
    {
        cf *acc = malloc(sizeof(cf) * n2), *line = malloc(sizeof(cf) * n);
        for (size_t i = 0; i < n2; ++i) acc[i] = (float)probe_acc[2 * i] + I * (float)probe_acc[2 * i + 1];
        fft2(&pl, acc, -1, line);
        for (size_t i = 0; i < n2; ++i) {
            probe_acc[2 * i] = crealf(acc[i]);
            probe_acc[2 * i + 1] = cimagf(acc[i]);
        }
        free(acc);
        free(line);
    }
    *err_sum = err_total;
    free(P);
    free(Q);
    free(T);
    plan32_free(&pl);
    return 0;
}

/* Far-field intensities |Psi|^2 (centred, as the reference's measured
 * patterns are stored) of npos positions at the volume rvol, single
 * precision: the forward half of cpu32_batched_tilt (mset.cu:107-190), for
 * simulating a sample's measured patterns on the host. */
int cpu32_simulate(int n, int nz, int binning, double sigma, double dz, int npos, const float *rvol,
                   const float *probe, const float *prop_centred, const float *scan_x, const float *scan_y,
                   float *inten, int nthreads) {
    if (n < 2 || nz <= 0 || binning <= 0 || npos < 0) return -1;
    plan32 pl;
    if (plan32_init(&pl, n)) return -1;
    const size_t n2 = (size_t)n * n;
    const int ns = (nz + binning - 1) / binning;
    cf *P = malloc(sizeof(cf) * n2), *Q = malloc(sizeof(cf) * n2), *T = malloc(sizeof(cf) * n2 * ns);
    for (int r = 0; r < n; ++r)
        for (int c = 0; c < n; ++c) {
            const size_t i = (size_t)r * n + c;
            P[ishift(r, c, n)] = prop_centred[2 * i] + I * prop_centred[2 * i + 1];
            Q[i] = probe[2 * i] + I * probe[2 * i + 1];
        }
    {
        cf *line = malloc(sizeof(cf) * n);
        ifft2n(&pl, Q, line);
        free(line);
    }
    const float sdz = (float)(sigma * dz);
    for (int s = 0; s < ns; ++s) {
        const int z0 = s * binning, z1 = z0 + binning < nz ? z0 + binning : nz;
        for (size_t i = 0; i < n2; ++i) {
            float acc = 0.f;
            for (int z = z0; z < z1; ++z) acc += rvol[(size_t)z * n2 + i];
            T[(size_t)s * n2 + i] = cosf(sdz * acc) + I * sinf(sdz * acc);
        }
    }
    const float center = roundf((n + 1.0f) / 2.0f);
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
#pragma omp parallel
    {
        cf *w = malloc(sizeof(cf) * n2), *fs = malloc(sizeof(cf) * n2), *line = malloc(sizeof(cf) * n);
#pragma omp for schedule(dynamic, 1)
        for (int p = 0; p < npos; ++p) {
            shift_factor(n, scan_y[p] - center, scan_x[p] - center, fs);
            for (size_t i = 0; i < n2; ++i) w[i] = Q[i] * fs[i];
            fft2(&pl, w, -1, line);
            for (int s = 0; s < ns; ++s) {
                const cf *Ts = T + (size_t)s * n2;
                for (size_t i = 0; i < n2; ++i) w[i] *= Ts[i];
                fft2(&pl, w, -1, line);
                for (size_t i = 0; i < n2; ++i) w[i] *= P[i];
                ifft2n(&pl, w, line);
            }
            fft2(&pl, w, -1, line);
            float *o = inten + (size_t)p * n2;
            for (int r = 0; r < n; ++r)
                for (int c = 0; c < n; ++c) {
                    const cf v = w[ishift(r, c, n)];
                    o[(size_t)r * n + c] = crealf(v) * crealf(v) + cimagf(v) * cimagf(v);
                }
        }
        free(w);
        free(fs);
        free(line);
    }
    free(P);
    free(Q);
    free(T);
    plan32_free(&pl);
    return 0;
}

/* Sequential tilt pass with reference semantics (MSET, reference adjoint
 * formula), single precision on one thread: for each position in order the
 * forward and adjoint of cpu32_batched_tilt, then RVol += step0 Re(g)
 * replicated over each slab's voxels (mset.cu:265-284), probe -= step1
 * F(F^{-1}(chi0) fs(-s)) (mset.cu:288-312), scan coordinates += step2 times
 * the finite-difference position direction (mset.cu:316-327).  rvol, probe,
 * scan_x, scan_y are updated in place; err_sum receives sum_p sum_px
 * (A - M)^2.  Sums over pixels (error, position direction) in double. */
int cpu32_sequential_tilt(int n, int nz, int binning, double sigma, double dz, const double *step, int npos,
                          float *rvol, float *probe, const float *prop_centred, float *scan_x, float *scan_y,
                          const float *measured, double *err_sum) {
    if (n < 2 || nz <= 0 || binning <= 0 || npos < 0) return -1;
    plan32 pl;
    if (plan32_init(&pl, n)) return -1;
    const size_t n2 = (size_t)n * n;
    const int ns = (nz + binning - 1) / binning;
    cf *P = malloc(sizeof(cf) * n2), *T = malloc(sizeof(cf) * n2 * ns), *Q = malloc(sizeof(cf) * n2);
    cf *w = malloc(sizeof(cf) * n2), *fs = malloc(sizeof(cf) * n2), *psi0 = malloc(sizeof(cf) * n2);
    cf *waves = malloc(sizeof(cf) * n2 * (ns + 1)), *line = malloc(sizeof(cf) * n), *d = malloc(sizeof(cf) * n2);
    float *g = malloc(sizeof(float) * n2 * ns);
    for (int r = 0; r < n; ++r)
        for (int c = 0; c < n; ++c) {
            const size_t i = (size_t)r * n + c;
            P[ishift(r, c, n)] = prop_centred[2 * i] + I * prop_centred[2 * i + 1];
        }
    const float sdz = (float)(sigma * dz);
    const float center = roundf((n + 1.0f) / 2.0f);
    const float st0 = (float)step[0], st1 = (float)step[1], st2 = (float)step[2];
    double err_total = 0.0;
    for (int p = 0; p < npos; ++p) {
        for (int s = 0; s < ns; ++s) { /* transmission from the current volume (mset.cu:134-153) */
            const int z0 = s * binning, z1 = z0 + binning < nz ? z0 + binning : nz;
            for (size_t i = 0; i < n2; ++i) {
                float acc = 0.f;
                for (int z = z0; z < z1; ++z) acc += rvol[(size_t)z * n2 + i];
                T[(size_t)s * n2 + i] = cosf(sdz * acc) + I * sinf(sdz * acc);
            }
        }
        /* psi0 = F(F^{-1}(probe) fs) with the current probe (mset.cu:110-131) */
        for (size_t i = 0; i < n2; ++i) Q[i] = probe[2 * i] + I * probe[2 * i + 1];
        ifft2n(&pl, Q, line);
        const float s1 = scan_y[p] - center, s2 = scan_x[p] - center;
        shift_factor(n, s1, s2, fs);
        for (size_t i = 0; i < n2; ++i) psi0[i] = Q[i] * fs[i];
        fft2(&pl, psi0, -1, line);
        memcpy(w, psi0, sizeof(cf) * n2);
        for (int s = 0; s < ns; ++s) { /* mset.cu:157-183 */
            const cf *Ts = T + (size_t)s * n2;
            for (size_t i = 0; i < n2; ++i) w[i] *= Ts[i];
            fft2(&pl, w, -1, line);
            for (size_t i = 0; i < n2; ++i) w[i] *= P[i];
            ifft2n(&pl, w, line);
            memcpy(waves + (size_t)(s + 1) * n2, w, sizeof(cf) * n2);
        }
        fft2(&pl, w, -1, line); /* far field, residual (mset.cu:186-227) */
        const float *meas = measured + (size_t)p * n2;
        for (int r = 0; r < n; ++r)
            for (int c = 0; c < n; ++c) {
                const size_t k = ishift(r, c, n);
                const float a2 = crealf(w[k]) * crealf(w[k]) + cimagf(w[k]) * cimagf(w[k]);
                const float A = sqrtf(a2 + 1e-30f), M = sqrtf(meas[(size_t)r * n + c]);
                err_total += (double)((A - M) * (A - M));
                w[k] *= 1.0f - M / A;
            }
        for (int s = ns - 1; s >= 0; --s) { /* mset.cu:232-271 */
            const cf *Ts = T + (size_t)s * n2;
            const cf *psi = waves + (size_t)(s + 1) * n2; /* mset.cu:248-251 */
            for (size_t i = 0; i < n2; ++i) w[i] *= conjf(P[i]);
            ifft2n(&pl, w, line);
            float *gs = g + (size_t)s * n2;
            for (size_t i = 0; i < n2; ++i) {
                gs[i] = crealf(I * conjf(Ts[i]) * conjf(psi[i]) * w[i]);
                w[i] *= conjf(Ts[i]);
            }
            if (s > 0) fft2(&pl, w, -1, line);
        }
        /* position direction from conj(psi0) and chi0 (utility.cu:829-876) */
        double px = 0.0, py = 0.0;
        for (int i1 = 0; i1 < n; ++i1)
            for (int i2 = 0; i2 < n; ++i2) {
                const size_t i = (size_t)i1 * n + i2;
                const cf *f = psi0;
                cf dx, dy;
                if (i2 == 0) dx = conjf(f[i + 1]) - conjf(f[i]);
                else if (i2 == n - 1) dx = conjf(f[i]) - conjf(f[i - 1]);
                else dx = (conjf(f[i + 1]) - conjf(f[i - 1])) * 0.5f;
                if (i1 == 0) dy = conjf(f[i + n]) - conjf(f[i]);
                else if (i1 == n - 1) dy = conjf(f[i]) - conjf(f[i - n]);
                else dy = (conjf(f[i + n]) - conjf(f[i - n])) * 0.5f;
                px += (double)crealf(dx * w[i]);
                py += (double)crealf(dy * w[i]);
            }
        /* probe direction F(F^{-1}(chi0) fs(-s)) and the probe update (mset.cu:288-312) */
        memcpy(d, w, sizeof(cf) * n2);
        ifft2n(&pl, d, line);
        for (size_t i = 0; i < n2; ++i) d[i] *= conjf(fs[i]);
        fft2(&pl, d, -1, line);
        for (size_t i = 0; i < n2; ++i) {
            probe[2 * i] -= st1 * crealf(d[i]);
            probe[2 * i + 1] -= st1 * cimagf(d[i]);
        }
        /* object update, slab-replicated (mset.cu:265-284) */
        for (int s = 0; s < ns; ++s) {
            const int z0 = s * binning, z1 = z0 + binning < nz ? z0 + binning : nz;
            const float *gs = g + (size_t)s * n2;
            for (int z = z0; z < z1; ++z)
                for (size_t i = 0; i < n2; ++i) rvol[(size_t)z * n2 + i] += st0 * gs[i];
        }
        scan_x[p] += st2 * (float)px; /* mset.cu:322 */
        scan_y[p] += st2 * (float)py; /* mset.cu:327 */
    }
    *err_sum = err_total;
    free(P);
    free(T);
    free(Q);
    free(w);
    free(fs);
    free(psi0);
    free(waves);
    free(line);
    free(d);
    free(g);
    plan32_free(&pl);
    return 0;
}
