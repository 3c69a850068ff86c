/*
 * mset_oracle.c -- FP64 CPU restatement of the MSET multislice hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker the CUDA library is
 * compared against; nothing in the product path (mset_b200/) links, loads or
 * calls it.  Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline /
 * reference leg may use it.
 *
 * Every routine follows the reference (jhlee0667/MSET) as cited at its head.
 * Arithmetic is done in double precision with an own mixed-radix FFT
 * (unnormalised forward e^{-i}, inverse e^{+i}, as cuFFT / MATLAB fftn).
 *
 * Layout (identical to the reference MEX boundary, src/CUDA/mex_tools.hpp:15-24
 * reverses MATLAB dims into C order):
 *   volume      float/double [nz][n][n]   (x = fastest = MATLAB dim 1)
 *   2D fields   complex      [n][n]       interleaved (re, im)
 *   measured    float        [P][n][n]    MATLAB-centred layout (not ifftshifted)
 *   scan_x/y    1-based pixel coordinates; x pairs with the fast axis
 *               (src/CUDA/mset.cu:121, utility.cu:776-800).
 *
 * Parity pins: tests/golden/ holds vectors produced by the reference's own
 * CUDA code (src/CUDA/mset.cu compiled with a project mex shim, run on a B200);
 * tests/test_oracle_golden.py checks this file against them.
 */
#define _GNU_SOURCE
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef double _Complex cd;

/* pi as hard-coded in the reference's Fourier shift factor (utility.cu:790). */
#define REF_PI 3.1415926

/* ------------------------------------------------------------------------- */
/* Mixed-radix FFT (recursive decimation in time, any n; radices 4,2,3,5,    */
/* then any remaining prime by direct DFT).                                  */
/* ------------------------------------------------------------------------- */
typedef struct {
    int n;
    int nf;
    int fac[40];
    cd *w; /* w[t] = exp(-2 pi i t / n) */
} fftplan;

static void plan_init(fftplan *p, int n) {
    p->n = n;
    p->nf = 0;
    int m = n;
    while (m % 4 == 0) { p->fac[p->nf++] = 4; m /= 4; }
    while (m % 2 == 0) { p->fac[p->nf++] = 2; m /= 2; }
    for (int r = 3; m > 1; r += 2) {
        while (m % r == 0) { p->fac[p->nf++] = r; m /= r; }
    }
    if (p->nf == 0) p->fac[p->nf++] = 1;
    p->w = (cd *)malloc(sizeof(cd) * (size_t)n);
    for (int t = 0; t < n; ++t) {
        double a = -2.0 * M_PI * (double)t / (double)n;
        p->w[t] = cos(a) + I * sin(a);
    }
}

static void plan_free(fftplan *p) { free(p->w); p->w = NULL; }

static inline cd tw(const fftplan *p, long e, int sign) {
    long t = e % p->n;
    if (t < 0) t += p->n;
    cd v = p->w[t];
    return sign < 0 ? v : conj(v);
}

static void fft_rec(const fftplan *pl, const cd *in, long is, cd *out, int n,
                    const int *fac, long wstep, int sign) {
    int p = fac[0];
    if (p == 1) { out[0] = in[0]; return; }
    int m = n / p;
    if (m == 1) {
        for (int k = 0; k < p; ++k) {
            cd s = 0;
            for (int j = 0; j < p; ++j) s += in[j * is] * tw(pl, (long)j * k * wstep * m, sign);
            out[k] = s;
        }
        return;
    }
    for (int j = 0; j < p; ++j) fft_rec(pl, in + j * is, is * p, out + j * m, m, fac + 1, wstep * p, sign);
    cd tmp[64];
    cd *t = p <= 64 ? tmp : (cd *)malloc(sizeof(cd) * p);
    for (int k = 0; k < m; ++k) {
        for (int j = 0; j < p; ++j) t[j] = out[j * m + k] * tw(pl, (long)j * k * wstep, sign);
        for (int q = 0; q < p; ++q) {
            cd s = 0;
            for (int j = 0; j < p; ++j) s += t[j] * tw(pl, (long)j * q * m * wstep, sign);
            out[q * m + k] = s;
        }
    }
    if (t != tmp) free(t);
}

/* in-place 1D FFT of x[0], x[stride], ... (n points) */
static void fft1(const fftplan *pl, cd *x, long stride, int sign, cd *buf_in, cd *buf_out) {
    int n = pl->n;
    for (int i = 0; i < n; ++i) buf_in[i] = x[i * stride];
    fft_rec(pl, buf_in, 1, buf_out, n, pl->fac, 1, sign);
    for (int i = 0; i < n; ++i) x[i * stride] = buf_out[i];
}

/* unnormalised 2D FFT of a [n1][n2] array, sign -1 forward, +1 inverse */
static void fft2(const fftplan *p1, const fftplan *p2, cd *a, int sign, cd *b1, cd *b2) {
    int n1 = p1->n, n2 = p2->n;
    for (int r = 0; r < n1; ++r) fft1(p2, a + (long)r * n2, 1, sign, b1, b2);
    for (int c = 0; c < n2; ++c) fft1(p1, a + c, n2, sign, b1, b2);
}

/* exported: unnormalised 2D FFT on interleaved doubles */
int orc_fft2(double *a, int n1, int n2, int sign) {
    fftplan p1, p2;
    plan_init(&p1, n1);
    plan_init(&p2, n2);
    int mx = n1 > n2 ? n1 : n2;
    cd *b1 = malloc(sizeof(cd) * mx), *b2 = malloc(sizeof(cd) * mx);
    fft2(&p1, &p2, (cd *)a, sign, b1, b2);
    free(b1); free(b2);
    plan_free(&p1); plan_free(&p2);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* Per-position model                                                        */
/* ------------------------------------------------------------------------- */
enum { ORC_MSET = 1, ORC_SSET = 2 };
enum { ORC_REF = 0, ORC_EXACT = 1 };

typedef struct {
    int n, nz, b, ns;
    double sigma, dz;
    fftplan pl;
    cd *pstd;   /* ifftshift(prop2D), standard FFT order (mex_main.cu:80) */
    cd *b1, *b2;
} model;

/* ifftshift = circular shift by ceil(n/2) along both axes
 * (utility.cu:609-630 called with ceil(dims/2), mex_main.cu:80). */
static inline long ishift_index(int r, int c, int n) {
    int h = (n + 1) / 2;
    return (long)((r + h) % n) * n + (c + h) % n;
}

static void model_init(model *m, int n, int nz, int b, double sigma, double dz, const float *prop_centered) {
    m->n = n; m->nz = nz; m->b = b;
    m->ns = (nz + b - 1) / b; /* numPlanes = ceil(Nz/b), STEP00_INIT.m:185 */
    m->sigma = sigma; m->dz = dz;
    plan_init(&m->pl, n);
    long n2 = (long)n * n;
    m->pstd = malloc(sizeof(cd) * n2);
    if (prop_centered) {
        for (int r = 0; r < n; ++r)
            for (int c = 0; c < n; ++c) {
                long i = (long)r * n + c;
                m->pstd[ishift_index(r, c, n)] = prop_centered[2 * i] + I * prop_centered[2 * i + 1];
            }
    }
    m->b1 = malloc(sizeof(cd) * n);
    m->b2 = malloc(sizeof(cd) * n);
}

static void model_free(model *m) {
    plan_free(&m->pl);
    free(m->pstd); free(m->b1); free(m->b2);
}

/* thread-private FFT scratch for OpenMP use */
typedef struct { cd *b1, *b2; } scratch;

static void fft2m(const model *m, cd *a, int sign, scratch *s) {
    fft2(&m->pl, &m->pl, a, sign, s->b1, s->b2);
}

static void ifft2n(const model *m, cd *a, scratch *s) {
    long n2 = (long)m->n * m->n;
    fft2m(m, a, +1, s);
    double sc = 1.0 / (double)n2;
    for (long i = 0; i < n2; ++i) a[i] *= sc;
}

/* Fourier shift factor in standard FFT order (utility.cu:776-800 followed by
 * the ifftshift at mset.cu:122): exp(i 2 pi (s1 n1/N + s2 n2/N)) with
 * n = idx - N/2 before the shift. */
static void shift_factor(int n, double s1, double s2, cd *out, double *n1v, double *n2v) {
    int h = (n + 1) / 2;
    for (int k1 = 0; k1 < n; ++k1) {
        int i1 = ((k1 - h) % n + n) % n;
        double n1 = (double)i1 - (double)n / 2.0;
        if (n1v) n1v[k1] = n1;
        for (int k2 = 0; k2 < n; ++k2) {
            int i2 = ((k2 - h) % n + n) % n;
            double nn2 = (double)i2 - (double)n / 2.0;
            if (n2v && k1 == 0) n2v[k2] = nn2;
            double ph = 2.0 * REF_PI * (s1 * n1 / n + s2 * nn2 / n);
            out[(long)k1 * n + k2] = cos(ph) + I * sin(ph);
        }
    }
}

/* psi0 = FFT(IFFT(probe) . fs(s))  (mset.cu:110-131;
 * Func_generate_probe_wave_scan_sub_pixel.m:4-27).  s1 pairs with the slow
 * axis (scan_y), s2 with the fast axis (scan_x). */
static void probe_shift(const model *m, const cd *probe, double s1, double s2, cd *out, cd *fsbuf, scratch *sc) {
    long n2 = (long)m->n * m->n;
    memcpy(out, probe, sizeof(cd) * n2);
    ifft2n(m, out, sc);
    shift_factor(m->n, s1, s2, fsbuf, NULL, NULL);
    for (long i = 0; i < n2; ++i) out[i] *= fsbuf[i];
    fft2m(m, out, -1, sc);
}

/* Per-position result container */
typedef struct {
    cd *psi0;      /* incident (shifted) probe, N^2 */
    cd *waves;     /* ns+1 waves: waves[0] = psi0 (SSET: psi0); waves[s+1] = wave after slab s */
    cd *trans;     /* ns transmission slabs */
    cd *far;       /* far field Psi, N^2 */
    double *errpx; /* (A-M)^2 per pixel, N^2 (standard order) */
    cd *grad;      /* ns slab gradients g_s (complex) */
    cd *chi0;      /* back-propagated wave at the entrance, N^2 */
    cd *probe_dir; /* shift_{-s}(chi0), N^2 */
    double pos_dir[2]; /* x, y */
    double err;    /* sum over pixels of (A-M)^2 */
} posres;

static void posres_alloc(posres *r, const model *m) {
    long n2 = (long)m->n * m->n;
    r->psi0 = malloc(sizeof(cd) * n2);
    r->waves = malloc(sizeof(cd) * n2 * (m->ns + 1));
    r->trans = malloc(sizeof(cd) * n2 * m->ns);
    r->far = malloc(sizeof(cd) * n2);
    r->errpx = malloc(sizeof(double) * n2);
    r->grad = malloc(sizeof(cd) * n2 * m->ns);
    r->chi0 = malloc(sizeof(cd) * n2);
    r->probe_dir = malloc(sizeof(cd) * n2);
}

static void posres_free(posres *r) {
    free(r->psi0); free(r->waves); free(r->trans); free(r->far); free(r->errpx);
    free(r->grad); free(r->chi0); free(r->probe_dir);
}

/* Transmission slabs T_s = exp(i sigma dz sum_{z in slab s} V_z)
 * (mset.cu:134-153; STEP02_FORWARD_4D.m:12-20).  SSET: one slab over the whole
 * depth (mset.cu:391-404; STEP02_FORWARD_4D_SSET.m:9). */
static void transmission(const model *m, int method, const double *V, cd *T) {
    long n2 = (long)m->n * m->n;
    int ns = method == ORC_SSET ? 1 : m->ns;
    int b = method == ORC_SSET ? m->nz : m->b;
    for (int s = 0; s < ns; ++s) {
        int z0 = s * b, z1 = z0 + b < m->nz ? z0 + b : m->nz;
        for (long i = 0; i < n2; ++i) {
            double acc = 0;
            for (int z = z0; z < z1; ++z) acc += V[(long)z * n2 + i];
            double ph = m->sigma * m->dz * acc;
            T[(long)s * n2 + i] = cos(ph) + I * sin(ph);
        }
    }
}

/* One position: forward, far field, residual, adjoint, probe and position
 * directions.  Follows mset.cu:107-327 (MSET) / 372-546 (SSET) and
 * STEP02_FORWARD_4D.m / STEP03_BACK.m.  amp_std = sqrt(ifftshift(I_meas)) in
 * standard order (mset.cu:206-210).  If do_adjoint == 0 only the forward and
 * error are computed (run_error_mset, mset.cu:557-696). */
static void position(const model *m, int method, int admode, const double *V, const cd *probe,
                     double scan_x, double scan_y, const double *amp_std, int do_adjoint,
                     posres *r, scratch *sc) {
    int n = m->n;
    long n2 = (long)n * n;
    int ns = method == ORC_SSET ? 1 : m->ns;
    double c = round((n + 1.0) / 2.0); /* pot_array_centers, mset.cu:83 */
    double s1 = scan_y - c, s2 = scan_x - c;
    cd *fs = malloc(sizeof(cd) * n2);
    probe_shift(m, probe, s1, s2, r->psi0, fs, sc);
    transmission(m, method, V, r->trans);

    cd *w = malloc(sizeof(cd) * n2);
    memcpy(w, r->psi0, sizeof(cd) * n2);
    memcpy(r->waves, w, sizeof(cd) * n2);
    for (int s = 0; s < ns; ++s) {
        const cd *T = r->trans + (long)s * n2;
        for (long i = 0; i < n2; ++i) w[i] *= T[i];
        if (method == ORC_MSET) {
            fft2m(m, w, -1, sc);
            for (long i = 0; i < n2; ++i) w[i] *= m->pstd[i];
            ifft2n(m, w, sc);
        }
        memcpy(r->waves + (long)(s + 1) * n2, w, sizeof(cd) * n2);
    }
    /* far field, error and residual (mset.cu:186-227) */
    fft2m(m, w, -1, sc);
    memcpy(r->far, w, sizeof(cd) * n2);
    double err = 0;
    for (long i = 0; i < n2; ++i) {
        double a2 = creal(w[i]) * creal(w[i]) + cimag(w[i]) * cimag(w[i]);
        double A = sqrt(a2 + 1e-30);
        double M = amp_std[i];
        double e = (A - M) * (A - M);
        r->errpx[i] = e;
        err += e;
        w[i] = w[i] * (1.0 - M / A);
    }
    r->err = err;
    if (!do_adjoint) { free(w); free(fs); return; }

    /* adjoint (mset.cu:232-271; STEP03_BACK.m:12-26) */
    if (method == ORC_MSET) {
        for (int s = ns - 1; s >= 0; --s) {
            const cd *T = r->trans + (long)s * n2;
            for (long i = 0; i < n2; ++i) w[i] *= conj(m->pstd[i]);
            ifft2n(m, w, sc);
            /* REF: wave saved after slab s (mset.cu:248-251); EXACT: wave entering slab s */
            const cd *psi = r->waves + (long)(admode == ORC_EXACT ? s : s + 1) * n2;
            cd *g = r->grad + (long)s * n2;
            for (long i = 0; i < n2; ++i) g[i] = I * conj(T[i]) * conj(psi[i]) * w[i];
            for (long i = 0; i < n2; ++i) w[i] *= conj(T[i]);
            if (s > 0) fft2m(m, w, -1, sc);
        }
        /* the reference transforms forward then inverse (mset.cu:259, 266): identity */
    } else {
        ifft2n(m, w, sc);
        const cd *T = r->trans;
        for (long i = 0; i < n2; ++i) r->grad[i] = I * conj(T[i]) * conj(r->psi0[i]) * w[i];
        for (long i = 0; i < n2; ++i) w[i] *= conj(T[i]);
    }
    memcpy(r->chi0, w, sizeof(cd) * n2);

    /* probe direction: shift back by -s (mset.cu:288-309) */
    probe_shift(m, r->chi0, -s1, -s2, r->probe_dir, fs, sc);

    /* position direction (mset.cu:316-327; utility.cu:829-876) */
    if (admode == ORC_REF) {
        double px = 0, py = 0;
        for (int i1 = 0; i1 < n; ++i1)
            for (int i2 = 0; i2 < n; ++i2) {
                long i = (long)i1 * n + i2;
                cd dx, dy;
                const cd *f = r->psi0;
                if (i2 == 0) dx = conj(f[i + 1]) - conj(f[i]);
                else if (i2 == n - 1) dx = conj(f[i]) - conj(f[i - 1]);
                else dx = (conj(f[i + 1]) - conj(f[i - 1])) / 2.0;
                if (i1 == 0) dy = conj(f[i + n]) - conj(f[i]);
                else if (i1 == n - 1) dy = conj(f[i]) - conj(f[i - n]);
                else dy = (conj(f[i + n]) - conj(f[i - n])) / 2.0;
                px += creal(dx * r->chi0[i]);
                py += creal(dy * r->chi0[i]);
            }
        r->pos_dir[0] = px;
        r->pos_dir[1] = py;
    } else {
        /* spectral derivative of psi0 w.r.t. the scan coordinates */
        double *n1v = malloc(sizeof(double) * n), *n2v = malloc(sizeof(double) * n);
        shift_factor(n, s1, s2, fs, n1v, n2v);
        cd *q = malloc(sizeof(cd) * n2), *dxw = malloc(sizeof(cd) * n2), *dyw = malloc(sizeof(cd) * n2);
        memcpy(q, probe, sizeof(cd) * n2);
        ifft2n(m, q, sc);
        for (int k1 = 0; k1 < n; ++k1)
            for (int k2 = 0; k2 < n; ++k2) {
                long i = (long)k1 * n + k2;
                cd base = q[i] * fs[i];
                dxw[i] = base * (I * 2.0 * REF_PI * n2v[k2] / n);
                dyw[i] = base * (I * 2.0 * REF_PI * n1v[k1] / n);
            }
        fft2m(m, dxw, -1, sc);
        fft2m(m, dyw, -1, sc);
        double px = 0, py = 0;
        for (long i = 0; i < n2; ++i) {
            px -= creal(conj(dxw[i]) * r->chi0[i]);
            py -= creal(conj(dyw[i]) * r->chi0[i]);
        }
        r->pos_dir[0] = px;
        r->pos_dir[1] = py;
        free(n1v); free(n2v); free(q); free(dxw); free(dyw);
    }
    free(w); free(fs);
}

static void amp_from_measured(int n, const float *meas, double *amp) {
    for (int r = 0; r < n; ++r)
        for (int c = 0; c < n; ++c) {
            long i = (long)r * n + c;
            amp[ishift_index(r, c, n)] = sqrt((double)meas[i]);
        }
}

static void to_cd(const float *f, cd *o, long n) {
    for (long i = 0; i < n; ++i) o[i] = f[2 * i] + I * f[2 * i + 1];
}

/* ------------------------------------------------------------------------- */
/* Exported entry points                                                     */
/* ------------------------------------------------------------------------- */

/* Sequential tilt pass with reference semantics: run_main_mset / run_main_sset
 * (update != 0) or run_error_mset / run_error_sset (update == 0).
 * rvol, probe, scan_x, scan_y are updated in place (FP64 internally, stored
 * back as float).  err_sum receives sum_p sum_px (A-M)^2 (the caller
 * normalises as mex_main.cu:150/179). */
int orc_run_tilt(int n, int nz, int binning, double sigma, double dz, const double *step,
                 int method, int admode, int update, int npos,
                 float *rvol, float *probe, const float *prop_centered,
                 float *scan_x, float *scan_y, const float *measured, double *err_sum) {
    if (n <= 1 || nz <= 0 || binning <= 0 || npos < 0) return -1;
    model m;
    model_init(&m, n, nz, binning, sigma, dz, prop_centered);
    long n2 = (long)n * n, nv = n2 * nz;
    double *V = malloc(sizeof(double) * nv);
    for (long i = 0; i < nv; ++i) V[i] = rvol[i];
    cd *P = malloc(sizeof(cd) * n2);
    to_cd(probe, P, n2);
    double *sx = malloc(sizeof(double) * (npos > 0 ? npos : 1)), *sy = malloc(sizeof(double) * (npos > 0 ? npos : 1));
    for (int p = 0; p < npos; ++p) { sx[p] = scan_x[p]; sy[p] = scan_y[p]; }
    double *amp = malloc(sizeof(double) * n2);
    posres r;
    posres_alloc(&r, &m);
    scratch sc = {m.b1, m.b2};
    double errs = 0;
    int ns = method == ORC_SSET ? 1 : m.ns;
    int bb = method == ORC_SSET ? nz : binning;
    for (int p = 0; p < npos; ++p) {
        amp_from_measured(n, measured + (long)p * n2, amp);
        position(&m, method, admode, V, P, sx[p], sy[p], amp, update, &r, &sc);
        errs += r.err;
        if (!update) continue;
        /* object update: RVol += step0 * Re(grad), slab-replicated (mset.cu:273-284) */
        for (int s = 0; s < ns; ++s) {
            int z0 = s * bb, z1 = z0 + bb < nz ? z0 + bb : nz;
            const cd *g = r.grad + (long)s * n2;
            for (int z = z0; z < z1; ++z)
                for (long i = 0; i < n2; ++i) V[(long)z * n2 + i] += step[0] * creal(g[i]);
        }
        /* probe update (mset.cu:311-312) */
        for (long i = 0; i < n2; ++i) P[i] -= step[1] * r.probe_dir[i];
        /* scan position update (mset.cu:322, 327) */
        sx[p] += step[2] * r.pos_dir[0];
        sy[p] += step[2] * r.pos_dir[1];
    }
    for (long i = 0; i < nv; ++i) rvol[i] = (float)V[i];
    for (long i = 0; i < n2; ++i) { probe[2 * i] = (float)creal(P[i]); probe[2 * i + 1] = (float)cimag(P[i]); }
    for (int p = 0; p < npos; ++p) { scan_x[p] = (float)sx[p]; scan_y[p] = (float)sy[p]; }
    *err_sum = errs;
    posres_free(&r);
    free(V); free(P); free(sx); free(sy); free(amp);
    model_free(&m);
    return 0;
}

/* One position with double inputs (for finite differences and per-position
 * parity).  Any output pointer may be NULL.
 *   V [nz][n][n], probe/prop interleaved complex, amp_std = sqrt(ifftshift(I))
 *   psi0_out, far_out, chi0_out, probe_dir_out: interleaved complex N^2
 *   grad_out: ns slabs interleaved complex; pos_dir_out: 2 doubles; err_out: 1
 *   waves_out: ns+1 waves interleaved complex, [0] = psi0, [s+1] = wave after
 *   slab s (save_wave_f of STEP02_FORWARD_4D.m:33; SSET: psi0 and T psi0) */
int orc_position(int n, int nz, int binning, double sigma, double dz, int method, int admode,
                 const double *V, const double *probe, const double *prop_centered_d,
                 double scan_x, double scan_y, const double *amp_std,
                 double *psi0_out, double *far_out, double *err_out, double *grad_out,
                 double *chi0_out, double *probe_dir_out, double *pos_dir_out, double *waves_out) {
    long n2 = (long)n * n;
    float *propf = malloc(sizeof(float) * 2 * n2);
    model m;
    model_init(&m, n, nz, binning, sigma, dz, NULL);
    /* keep the double-precision propagator */
    for (int r = 0; r < n; ++r)
        for (int c = 0; c < n; ++c) {
            long i = (long)r * n + c;
            m.pstd[ishift_index(r, c, n)] = prop_centered_d[2 * i] + I * prop_centered_d[2 * i + 1];
        }
    free(propf);
    posres r;
    posres_alloc(&r, &m);
    scratch sc = {m.b1, m.b2};
    position(&m, method, admode, V, (const cd *)probe, scan_x, scan_y, amp_std, 1, &r, &sc);
    int ns = method == ORC_SSET ? 1 : m.ns;
    if (psi0_out) memcpy(psi0_out, r.psi0, sizeof(cd) * n2);
    if (far_out) memcpy(far_out, r.far, sizeof(cd) * n2);
    if (err_out) *err_out = r.err;
    if (grad_out) memcpy(grad_out, r.grad, sizeof(cd) * n2 * ns);
    if (chi0_out) memcpy(chi0_out, r.chi0, sizeof(cd) * n2);
    if (probe_dir_out) memcpy(probe_dir_out, r.probe_dir, sizeof(cd) * n2);
    if (pos_dir_out) { pos_dir_out[0] = r.pos_dir[0]; pos_dir_out[1] = r.pos_dir[1]; }
    if (waves_out) memcpy(waves_out, r.waves, sizeof(cd) * n2 * (ns + 1));
    posres_free(&r);
    model_free(&m);
    return 0;
}

/* Loss of one position (sum over pixels of (A-M)^2) for finite differences. */
double orc_position_loss(int n, int nz, int binning, double sigma, double dz, int method,
                         const double *V, const double *probe, const double *prop_centered_d,
                         double scan_x, double scan_y, const double *amp_std) {
    double e = 0;
    long n2 = (long)n * n;
    model m;
    model_init(&m, n, nz, binning, sigma, dz, NULL);
    for (int r = 0; r < n; ++r)
        for (int c = 0; c < n; ++c) {
            long i = (long)r * n + c;
            m.pstd[ishift_index(r, c, n)] = prop_centered_d[2 * i] + I * prop_centered_d[2 * i + 1];
        }
    posres r;
    posres_alloc(&r, &m);
    scratch sc = {m.b1, m.b2};
    position(&m, method, ORC_REF, V, (const cd *)probe, scan_x, scan_y, amp_std, 0, &r, &sc);
    e = r.err;
    posres_free(&r);
    model_free(&m);
    (void)n2;
    return e;
}

/* Batched tilt pass (the batched method: every position of the tilt sees the
 * same volume, probe and positions).  Accumulates
 *   grad_slab[ns][n][n]  += sum_p Re(g_{p,s})                (FP64)
 *   probe_acc[n][n] (cplx)+= sum_p shift_{-s_p}(chi0_p)      (FP64)
 *   pos_dir[p][2]         = position directions per position
 *   err_sum               += sum_p sum_px (A-M)^2
 * Positions run in parallel (OpenMP, nthreads <= 0 = all) with one partial
 * accumulator per thread, summed in thread order: the result is deterministic
 * for a given thread count. */
int orc_batched_tilt(int n, int nz, int binning, double sigma, double dz, int method, int admode,
                     int npos, const float *rvol, const float *probe, const float *prop_centered,
                     const float *scan_x, const float *scan_y, const float *measured,
                     double *grad_slab, double *probe_acc, double *pos_dir, double *err_sum,
                     int nthreads) {
    model m;
    model_init(&m, n, nz, binning, sigma, dz, prop_centered);
    long n2 = (long)n * n, nv = n2 * nz;
    int ns = method == ORC_SSET ? 1 : m.ns;
    double *V = malloc(sizeof(double) * nv);
    for (long i = 0; i < nv; ++i) V[i] = rvol[i];
    cd *P = malloc(sizeof(cd) * n2);
    to_cd(probe, P, n2);
    double *errs = calloc(npos > 0 ? npos : 1, sizeof(double));
    int nth = 1;
#ifdef _OPENMP
    nth = nthreads > 0 ? nthreads : omp_get_max_threads();
#endif
    double *gpart = calloc((size_t)nth * ns * n2, sizeof(double));
    cd *ppart = calloc((size_t)nth * n2, sizeof(cd));
#pragma omp parallel num_threads(nth)
    {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        posres r;
        posres_alloc(&r, &m);
        scratch sc = {malloc(sizeof(cd) * n), malloc(sizeof(cd) * n)};
        double *amp = malloc(sizeof(double) * n2);
        double *gp = gpart + (size_t)tid * ns * n2;
        cd *pp = ppart + (size_t)tid * n2;
#pragma omp for schedule(static)
        for (int p = 0; p < npos; ++p) {
            amp_from_measured(n, measured + (long)p * n2, amp);
            position(&m, method, admode, V, P, scan_x[p], scan_y[p], amp, 1, &r, &sc);
            errs[p] = r.err;
            for (long i = 0; i < (long)ns * n2; ++i) gp[i] += creal(r.grad[i]);
            for (long i = 0; i < n2; ++i) pp[i] += r.probe_dir[i];
            pos_dir[2 * p] = r.pos_dir[0];
            pos_dir[2 * p + 1] = r.pos_dir[1];
        }
        posres_free(&r);
        free(sc.b1); free(sc.b2); free(amp);
    }
    for (int t = 0; t < nth; ++t) {
        for (long i = 0; i < (long)ns * n2; ++i) grad_slab[i] += gpart[(size_t)t * ns * n2 + i];
        for (long i = 0; i < n2; ++i) {
            cd v = ppart[(size_t)t * n2 + i];
            probe_acc[2 * i] += creal(v);
            probe_acc[2 * i + 1] += cimag(v);
        }
    }
    double e = 0;
    for (int p = 0; p < npos; ++p) e += errs[p];
    *err_sum += e;
    free(errs); free(gpart); free(ppart); free(V); free(P);
    model_free(&m);
    return 0;
}

int orc_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ------------------------------------------------------------------------- */
/* Fourier-shear 3D rotation (Welling et al. 2006) as in the reference:      */
/*   func_lib/Func_rot_3Dvol_FourierShear.m:5-19,                            */
/*   Func_inv_rot_3Dvol_FourierShear.m:5-20, MatrixQuaternionRot.m:1-11,     */
/*   Func_rotate_3Dvol_ROTmat_FourierShear.m:14-134,                         */
/*   My_obtain_quaternion_from_matrix.m:11-39,                               */
/*   calculate_S_matrices_for3DFourierShearRot_perm_ver1.m:16-93,            */
/*   ..._backward_ver1.m:16-91, SheerTransforms_for3Drot.m:16-49.            */
/* Volume layout: C [n3][n2][n1] = MATLAB (n1, n2, n3).                      */
/* ------------------------------------------------------------------------- */
static void quat_rot(const double *v, double theta_deg, double R[3][3]) {
    double th = theta_deg * M_PI / 180.0;
    double nv = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    double w = cos(th / 2), x = -sin(th / 2) * v[0] / nv, y = -sin(th / 2) * v[1] / nv, z = -sin(th / 2) * v[2] / nv;
    R[0][0] = 1 - 2 * y * y - 2 * z * z; R[0][1] = 2 * x * y + 2 * w * z; R[0][2] = 2 * x * z - 2 * w * y;
    R[1][0] = 2 * x * y - 2 * w * z; R[1][1] = 1 - 2 * x * x - 2 * z * z; R[1][2] = 2 * y * z + 2 * w * x;
    R[2][0] = 2 * x * z + 2 * w * y; R[2][1] = 2 * y * z - 2 * w * x; R[2][2] = 1 - 2 * x * x - 2 * y * y;
}

static void matmul3(double A[3][3], double B[3][3], double C[3][3]) {
    double T[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            T[i][j] = 0;
            for (int k = 0; k < 3; ++k) T[i][j] += A[i][k] * B[k][j];
        }
    memcpy(C, T, sizeof T);
}

static void inv3(double A[3][3], double B[3][3]) {
    double det = A[0][0] * (A[1][1] * A[2][2] - A[1][2] * A[2][1]) - A[0][1] * (A[1][0] * A[2][2] - A[1][2] * A[2][0]) +
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
    memcpy(B, T, sizeof T);
}

static void quat_from_matrix(double M[3][3], double *qx, double *qy, double *qz, double *qw) {
    double Tr = M[0][0] + M[1][1] + M[2][2], S;
    if (Tr > 0) {
        S = sqrt(Tr + 1) * 2;
        *qw = 0.25 * S; *qx = (M[2][1] - M[1][2]) / S; *qy = (M[0][2] - M[2][0]) / S; *qz = (M[1][0] - M[0][1]) / S;
    } else if (M[0][0] > M[1][1] && M[0][0] > M[2][2]) {
        S = sqrt(1.0 + M[0][0] - M[1][1] - M[2][2]) * 2;
        *qw = (M[2][1] - M[1][2]) / S; *qx = 0.25 * S; *qy = (M[0][1] + M[1][0]) / S; *qz = (M[0][2] + M[2][0]) / S;
    } else if (M[1][1] > M[2][2]) {
        S = sqrt(1.0 + M[1][1] - M[0][0] - M[2][2]) * 2;
        *qw = (M[0][2] - M[2][0]) / S; *qx = (M[0][1] + M[1][0]) / S; *qy = 0.25 * S; *qz = (M[1][2] + M[2][1]) / S;
    } else {
        S = sqrt(1.0 + M[2][2] - M[0][0] - M[1][1]) * 2;
        *qw = (M[1][0] - M[0][1]) / S; *qx = (M[0][2] + M[2][0]) / S; *qy = (M[1][2] + M[2][1]) / S; *qz = 0.25 * S;
    }
}

/* shear coefficients a..h for one permutation; returns absSum (INF if singular) */
static double shear_coeffs(double X0, double Y0, double Z0, double W, int perm, int backward, double co[8]) {
    double in[3] = {X0, Y0, Z0};
    /* circshift([X,Y,Z], [0 -perm]): element i takes in[(i + perm) mod 3] */
    double X = in[(0 + perm) % 3], Y = in[(1 + perm) % 3], Z = in[(2 + perm) % 3];
    if (backward) W = -W;
    double a, b, c, d, e, f, g, h;
    if (fabs(Y * Z - X * W) > 1e-5 && fabs(X * Y - Z * W) > 1e-5) {
        a = (X * X + Y * Y) / (Y * Z - X * W);
        b = (Y * Y - Z * Z) / (X * Y - Z * W) - 2 * (Y * Z * (X * X + Y * Y)) / (X * Y - Z * W) / (Y * Z - X * W);
        c = 2 * Y * Z / (X * Y - Z * W);
        d = 2 * (X * W - Y * Z);
        e = 2 * (X * Y - Z * W);
        f = -2 * X * Y / (Y * Z - X * W);
        g = (X * X - Y * Y) / (Y * Z - X * W) + 2 * X * Y * (Y * Y + Z * Z) / (X * Y - Z * W) / (Y * Z - X * W);
        h = (-1 + X * X + W * W) / (X * Y - Z * W);
    } else if (fabs(Y) < 1e-6) {
        a = -X / W; b = Z / W; c = 0; d = 2 * X * W; e = -2 * Z * W; f = 0; g = -X / W; h = Z / W;
    } else {
        return INFINITY;
    }
    double v[8] = {a, b, c, d, e, f, g, h};
    double s = 0;
    for (int i = 0; i < 8; ++i) {
        co[i] = backward ? -v[i] : v[i];
        s += fabs(v[i]);
    }
    return s;
}

/* grid value after ifftshift(k - round((n+1)/2)) with the Nyquist index zeroed
 * (Func_rotate_3Dvol_ROTmat_FourierShear.m:70-90); *nyq = 1 at that index */
static double rot_grid(int i, int n, int *nyq) {
    int h = (n + 1) / 2;          /* ceil(n/2) */
    int k = (i - h) % n; if (k < 0) k += n;  /* ifftshift: out[i] = v[(i - ceil(n/2)) mod n] */
    double c = floor((n + 1) / 2.0 + 0.5);
    double val = (double)(k + 1) - c;
    *nyq = (n % 2 == 0) && (i == (int)c - 1);
    return *nyq ? 0.0 : val;
}

typedef struct { int n[3]; fftplan pl[3]; cd *buf1, *buf2; } rotctx;

/* one shear along MATLAB dimension dim (1, 2, 3) with coefficients (ca, cb) */
static void shear(rotctx *r, cd *V, int dim, double ca, double cb) {
    int n1 = r->n[0], n2 = r->n[1], n3 = r->n[2];
    long s1 = 1, s2 = n1, s3 = (long)n1 * n2;
    int other[2];
    if (dim == 1) { other[0] = 3; other[1] = 2; }
    else if (dim == 2) { other[0] = 3; other[1] = 1; }
    else { other[0] = 2; other[1] = 1; }
    long st[4] = {0, s1, s2, s3};
    int nn[4] = {0, n1, n2, n3};
    /* forward FFTs along the two other dims */
    for (int o = 0; o < 2; ++o) {
        int d = other[o];
        /* loop over all lines along d */
        for (long base = 0; base < (long)n1 * n2 * n3; ++base) {
            int i1 = base % n1, i2 = (base / n1) % n2, i3 = base / ((long)n1 * n2);
            int idx[4] = {0, i1, i2, i3};
            if (idx[d] != 0) continue;
            fft1(&r->pl[d - 1], V + base, st[d], -1, r->buf1, r->buf2);
        }
    }
    for (int i3 = 0; i3 < n3; ++i3)
        for (int i2 = 0; i2 < n2; ++i2)
            for (int i1 = 0; i1 < n1; ++i1) {
                int q1, q2, q3;
                double g1 = rot_grid(i1, n1, &q1), g2 = rot_grid(i2, n2, &q2), g3 = rot_grid(i3, n3, &q3);
                if (q1 || q2 || q3) continue; /* nx = ny = nz = 0 on any Nyquist plane: phase 0 */
                double ph;
                if (dim == 1) ph = 2 * M_PI * ((double)n2 / n1 * ca * g2 / n2 + (double)n3 / n1 * cb * g3 / n3) * g1;
                else if (dim == 2) ph = 2 * M_PI * ((double)n1 / n2 * cb * g1 / n1 + (double)n3 / n2 * ca * g3 / n3) * g2;
                else ph = 2 * M_PI * ((double)n1 / n3 * ca * g1 / n1 + (double)n2 / n3 * cb * g2 / n2) * g3;
                V[(long)i3 * s3 + (long)i2 * s2 + i1] *= cos(ph) + I * sin(ph);
            }
    for (int o = 0; o < 2; ++o) {
        int d = other[o];
        double sc = 1.0 / nn[d];
        for (long base = 0; base < (long)n1 * n2 * n3; ++base) {
            int i1 = base % n1, i2 = (base / n1) % n2, i3 = base / ((long)n1 * n2);
            int idx[4] = {0, i1, i2, i3};
            if (idx[d] != 0) continue;
            fft1(&r->pl[d - 1], V + base, st[d], +1, r->buf1, r->buf2);
            for (int k = 0; k < nn[d]; ++k) V[base + k * st[d]] *= sc;
        }
    }
}

/* Func_rotate_3Dvol_ROTmat_FourierShear(vol, MAT, rotStepInit), MAT row-major */
static void rotate_rotmat(double *vol, int n1, int n2, int n3, double M[3][3], double rotStepInit) {
    double qx, qy, qz, qw;
    quat_from_matrix(M, &qx, &qy, &qz, &qw);
    double Ang = acos(qw) * 180.0 / M_PI * 2;
    double nv = sqrt(qx * qx + qy * qy + qz * qz);
    double Vec[3] = {qx / nv, qy / nv, qz / nv};
    int numStep = (int)floor(Ang / rotStepInit) + 1;
    double rotStep = Ang / numStep;
    double w = cos(rotStep / 2 * M_PI / 180), x = -sin(rotStep / 2 * M_PI / 180) * Vec[0],
           y = -sin(rotStep / 2 * M_PI / 180) * Vec[1], z = -sin(rotStep / 2 * M_PI / 180) * Vec[2];
    double cf[3][8], cb[3][8], sf[3], sb[3];
    for (int i = 1; i <= 3; ++i) {
        sf[i - 1] = shear_coeffs(x, y, z, w, i, 0, cf[i - 1]);
        sb[i - 1] = shear_coeffs(x, y, z, w, i, 1, cb[i - 1]);
    }
    int mf = 0, mb = 0;
    for (int i = 1; i < 3; ++i) {
        if (sf[i] < sf[mf]) mf = i;
        if (sb[i] < sb[mb]) mb = i;
    }
    int fwd = sf[mf] < sb[mb];
    int mI = (fwd ? mf : mb) + 1; /* MATLAB 1-based index */
    double *co = fwd ? cf[mf] : cb[mb];
    rotctx r;
    r.n[0] = n1; r.n[1] = n2; r.n[2] = n3;
    int mx = n1 > n2 ? n1 : n2; if (n3 > mx) mx = n3;
    for (int d = 0; d < 3; ++d) plan_init(&r.pl[d], r.n[d]);
    r.buf1 = malloc(sizeof(cd) * mx);
    r.buf2 = malloc(sizeof(cd) * mx);
    long nv3 = (long)n1 * n2 * n3;
    cd *S = malloc(sizeof(cd) * nv3);
    /* SheerVol = ifftshift(initVol) */
    int h1 = (n1 + 1) / 2, h2 = (n2 + 1) / 2, h3 = (n3 + 1) / 2;
    for (int i3 = 0; i3 < n3; ++i3)
        for (int i2 = 0; i2 < n2; ++i2)
            for (int i1 = 0; i1 < n1; ++i1)
                S[(long)((i3 + h3) % n3) * n1 * n2 + (long)((i2 + h2) % n2) * n1 + (i1 + h1) % n1] =
                    vol[(long)i3 * n1 * n2 + (long)i2 * n1 + i1];
    for (int st = 0; st < numStep; ++st) {
        if (fwd) {
            shear(&r, S, (mI + 1) % 3 + 1, co[6], co[7]);
            shear(&r, S, mI % 3 + 1, co[4], co[5]);
            shear(&r, S, (mI + 2) % 3 + 1, co[2], co[3]);
            shear(&r, S, (mI + 1) % 3 + 1, co[0], co[1]);
        } else {
            shear(&r, S, (mI + 1) % 3 + 1, co[0], co[1]);
            shear(&r, S, (mI + 2) % 3 + 1, co[2], co[3]);
            shear(&r, S, mI % 3 + 1, co[4], co[5]);
            shear(&r, S, (mI + 1) % 3 + 1, co[6], co[7]);
        }
        for (long i = 0; i < nv3; ++i) S[i] = creal(S[i]);
    }
    /* RotVol = fftshift(SheerVol): out[(i + floor(n/2)) mod n] = S[i] */
    for (int i3 = 0; i3 < n3; ++i3)
        for (int i2 = 0; i2 < n2; ++i2)
            for (int i1 = 0; i1 < n1; ++i1)
                vol[(long)((i3 + n3 / 2) % n3) * n1 * n2 + (long)((i2 + n2 / 2) % n2) * n1 + (i1 + n1 / 2) % n1] =
                    creal(S[(long)i3 * n1 * n2 + (long)i2 * n1 + i1]);
    free(S); free(r.buf1); free(r.buf2);
    for (int d = 0; d < 3; ++d) plan_free(&r.pl[d]);
}

/* rotation matrix of Func_rot_3Dvol_FourierShear (inverse = 0) or
 * Func_inv_rot_3Dvol_FourierShear (inverse = 1); returns 0 when all angles
 * are within 0.5 degrees (the reference then returns the volume unchanged) */
int orc_rotation_matrix(const double *v1, const double *v2, const double *v3, double phi, double theta, double psi,
                        int inverse, double *Mout) {
    double R1[3][3], R2[3][3], R3[3][3], R[3][3], Rt[3][3];
    quat_rot(v1, phi, R1);
    quat_rot(v2, theta, R2);
    quat_rot(v3, psi, R3);
    matmul3(R1, R2, R);
    matmul3(R, R3, R);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) Rt[i][j] = R[j][i];
    if (inverse) inv3(Rt, Rt);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) Mout[3 * i + j] = Rt[i][j];
    return (fabs(theta) > 0.5 || fabs(phi) > 0.5 || fabs(psi) > 0.5) ? 1 : 0;
}

/* Func_rot_3Dvol_FourierShear / Func_inv_rot_3Dvol_FourierShear with
 * rotStepInit = 11 (Func_rot_3Dvol_FourierShear.m:15); vol in place (double) */
int orc_rot3d(double *vol, int n1, int n2, int n3, const double *v1, const double *v2, const double *v3, double phi,
              double theta, double psi, int inverse) {
    double M[9];
    if (!orc_rotation_matrix(v1, v2, v3, phi, theta, psi, inverse, M)) return 0;
    double MM[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) MM[i][j] = M[3 * i + j];
    rotate_rotmat(vol, n1, n2, n3, MM, 11.0);
    return 1;
}

/* the shear plan of a rotation, for checking a GPU implementation:
 * out[0] = numStep, out[1] = forward (1) / backward (0), out[2] = mI (1-based),
 * out[3..10] = coefficients a..h */
int orc_rotation_plan(const double *M9, double rotStepInit, double *out) {
    double M[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) M[i][j] = M9[3 * i + j];
    double qx, qy, qz, qw;
    quat_from_matrix(M, &qx, &qy, &qz, &qw);
    double Ang = acos(qw) * 180.0 / M_PI * 2;
    double nv = sqrt(qx * qx + qy * qy + qz * qz);
    double Vec[3] = {qx / nv, qy / nv, qz / nv};
    int numStep = (int)floor(Ang / rotStepInit) + 1;
    double rotStep = Ang / numStep;
    double w = cos(rotStep / 2 * M_PI / 180), x = -sin(rotStep / 2 * M_PI / 180) * Vec[0],
           y = -sin(rotStep / 2 * M_PI / 180) * Vec[1], z = -sin(rotStep / 2 * M_PI / 180) * Vec[2];
    double cf[3][8], cb[3][8], sf[3], sb[3];
    for (int i = 1; i <= 3; ++i) {
        sf[i - 1] = shear_coeffs(x, y, z, w, i, 0, cf[i - 1]);
        sb[i - 1] = shear_coeffs(x, y, z, w, i, 1, cb[i - 1]);
    }
    int mf = 0, mb = 0;
    for (int i = 1; i < 3; ++i) {
        if (sf[i] < sf[mf]) mf = i;
        if (sb[i] < sb[mb]) mb = i;
    }
    int fwd = sf[mf] < sb[mb];
    out[0] = numStep;
    out[1] = fwd;
    out[2] = (fwd ? mf : mb) + 1;
    for (int i = 0; i < 8; ++i) out[3 + i] = fwd ? cf[mf][i] : cb[mb][i];
    return 0;
}
