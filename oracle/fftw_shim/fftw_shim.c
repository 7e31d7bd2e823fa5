/*
 * CPU FFT implementing the FFTW3 API subset declared in fftw3.h.
 *
 * TEST INFRASTRUCTURE ONLY (see fftw3.h).  It backs two things: the
 * reference sources compiled as-is under oracle/_ref, and the oracle
 * restatement in oracle/gabe_oracle.c.  The product library uses cuFFT.
 *
 * Method: mixed-radix Stockham autosort FFT (radices 4, 2, 3, 5 and a
 * direct DFT for any other prime factor), the textbook decimation-in-time
 * formulation with twiddles exp(sign*2*pi*i*t/n) tabulated once per length
 * from libm cos/sin.  Multi-dimensional transforms are row-column: the last
 * (contiguous) dimension first for r2c, last for c2r, with pairs of real rows
 * packed into one complex transform (x + i*y) and separated through the
 * Hermitian symmetry of each half.
 */
#include "fftw3.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static int g_nthreads = 1;

void fftw_plan_with_nthreads(int nthreads) { g_nthreads = nthreads > 0 ? nthreads : 1; }
int fftw_init_threads(void) { return 1; }
void fftw_cleanup_threads(void) {}
int gabe_fft_get_nthreads(void) { return g_nthreads; }

void *fftw_malloc(size_t n) {
    void *p = NULL;
    if (posix_memalign(&p, 64, n ? n : 64) != 0) return NULL;
    return p;
}
void fftw_free(void *p) { free(p); }

/* ------------------------------------------------------------------ */
/* 1-D complex plan                                                    */
/* ------------------------------------------------------------------ */
typedef struct {
    int n;
    int nstage;
    int radix[40];
    double *tw; /* n complex entries exp(-2*pi*i*t/n); backward uses conj */
} line_plan;

static void line_plan_init(line_plan *lp, int n) {
    lp->n = n;
    lp->nstage = 0;
    int m = n;
    while (m % 4 == 0) { lp->radix[lp->nstage++] = 4; m /= 4; }
    while (m % 2 == 0) { lp->radix[lp->nstage++] = 2; m /= 2; }
    while (m % 3 == 0) { lp->radix[lp->nstage++] = 3; m /= 3; }
    while (m % 5 == 0) { lp->radix[lp->nstage++] = 5; m /= 5; }
    for (int p = 7; m > 1; p += 2) {
        while (m % p == 0) { lp->radix[lp->nstage++] = p; m /= p; }
    }
    lp->tw = (double *)malloc(sizeof(double) * 2 * (size_t)(n > 0 ? n : 1));
    for (int t = 0; t < n; t++) {
        double ang = 2.0 * M_PI * (double)t / (double)n;
        lp->tw[2 * t] = cos(ang);
        lp->tw[2 * t + 1] = -sin(ang);
    }
}

static void line_plan_free(line_plan *lp) { free(lp->tw); lp->tw = NULL; }

/* y = DFT_R(v) with sign; v, y have R complex entries. */
static void small_dft(int R, const double *v, double *y, int sign, const line_plan *lp) {
    if (R == 2) {
        y[0] = v[0] + v[2]; y[1] = v[1] + v[3];
        y[2] = v[0] - v[2]; y[3] = v[1] - v[3];
        return;
    }
    if (R == 4) {
        double a0r = v[0] + v[4], a0i = v[1] + v[5];
        double a1r = v[0] - v[4], a1i = v[1] - v[5];
        double b0r = v[2] + v[6], b0i = v[3] + v[7];
        double b1r = v[2] - v[6], b1i = v[3] - v[7];
        /* multiply b1 by sign*i */
        double cr = -sign * b1i, ci = sign * b1r;
        y[0] = a0r + b0r; y[1] = a0i + b0i;
        y[4] = a0r - b0r; y[5] = a0i - b0i;
        y[2] = a1r + cr;  y[3] = a1i + ci;
        y[6] = a1r - cr;  y[7] = a1i - ci;
        return;
    }
    /* generic direct DFT using the length-n table: exp(sign*2*pi*i*q*r/R)
     * = tw[(q*r*(n/R)) mod n] (conjugated for sign=+1). */
    int n = lp->n, step = n / R;
    for (int q = 0; q < R; q++) {
        double sr = 0.0, si = 0.0;
        for (int r = 0; r < R; r++) {
            int t = (int)(((long long)q * r * step) % n);
            double wr = lp->tw[2 * t], wi = lp->tw[2 * t + 1];
            if (sign > 0) wi = -wi;
            sr += v[2 * r] * wr - v[2 * r + 1] * wi;
            si += v[2 * r] * wi + v[2 * r + 1] * wr;
        }
        y[2 * q] = sr; y[2 * q + 1] = si;
    }
}

/* In-place transform of one line (interleaved complex, length n) using the
 * caller's scratch of 2n doubles. */
static void line_fft(const line_plan *lp, double *x, double *scratch, int sign) {
    int n = lp->n;
    if (n <= 1) return;
    double *src = x, *dst = scratch;
    int Ns = 1;
    double v[2 * 64], y[2 * 64];
    for (int s = 0; s < lp->nstage; s++) {
        int R = lp->radix[s];
        int nb = n / R;
        for (int j = 0; j < nb; j++) {
            int k = j % Ns;
            for (int r = 0; r < R; r++) {
                double xr = src[2 * (j + r * nb)], xi = src[2 * (j + r * nb) + 1];
                int t = (int)(((long long)r * k * (n / (Ns * R))) % n);
                double wr = lp->tw[2 * t], wi = lp->tw[2 * t + 1];
                if (sign > 0) wi = -wi;
                v[2 * r] = xr * wr - xi * wi;
                v[2 * r + 1] = xr * wi + xi * wr;
            }
            small_dft(R, v, y, sign, lp);
            int idxD = (j / Ns) * Ns * R + k;
            for (int r = 0; r < R; r++) {
                dst[2 * (idxD + r * Ns)] = y[2 * r];
                dst[2 * (idxD + r * Ns) + 1] = y[2 * r + 1];
            }
        }
        Ns *= R;
        double *t = src; src = dst; dst = t;
    }
    if (src != x) memcpy(x, src, sizeof(double) * 2 * (size_t)n);
}

void gabe_fft_c2c_1d(int n, double *data, int sign) {
    line_plan lp;
    line_plan_init(&lp, n);
    double *scr = (double *)malloc(sizeof(double) * 2 * (size_t)n);
    line_fft(&lp, data, scr, sign);
    free(scr);
    line_plan_free(&lp);
}

/* ------------------------------------------------------------------ */
/* 3-D plans                                                           */
/* ------------------------------------------------------------------ */
struct gabe_fft_plan_s {
    int kind; /* 0 = r2c, 1 = c2r */
    int n0, n1, n2, nz;
    double *in_r;        /* r2c default input  */
    fftw_complex *in_c;  /* c2r default input  */
    double *out_r;       /* c2r default output */
    fftw_complex *out_c; /* r2c default output */
    line_plan p0, p1, p2;
};

static fftw_plan plan_common(int kind, int n0, int n1, int n2) {
    fftw_plan p = (fftw_plan)calloc(1, sizeof(*p));
    p->kind = kind;
    p->n0 = n0; p->n1 = n1; p->n2 = n2; p->nz = n2 / 2 + 1;
    line_plan_init(&p->p0, n0);
    line_plan_init(&p->p1, n1);
    line_plan_init(&p->p2, n2);
    return p;
}

fftw_plan fftw_plan_dft_r2c_3d(int n0, int n1, int n2, double *in, fftw_complex *out, unsigned flags) {
    (void)flags;
    fftw_plan p = plan_common(0, n0, n1, n2);
    p->in_r = in; p->out_c = out;
    return p;
}

fftw_plan fftw_plan_dft_c2r_3d(int n0, int n1, int n2, fftw_complex *in, double *out, unsigned flags) {
    (void)flags;
    fftw_plan p = plan_common(1, n0, n1, n2);
    p->in_c = in; p->out_r = out;
    return p;
}

void fftw_destroy_plan(fftw_plan p) {
    if (!p) return;
    line_plan_free(&p->p0);
    line_plan_free(&p->p1);
    line_plan_free(&p->p2);
    free(p);
}

#define BATCH 8

/* Complex transforms along a strided axis of a [outer][len][inner] complex
 * array (inner contiguous): lines are indexed by (outer, inner). */
static void strided_pass(const line_plan *lp, double *data, int outer, int len, int inner, int sign) {
    int nbatch = (inner + BATCH - 1) / BATCH;
    long long ntask = (long long)outer * nbatch;
#pragma omp parallel num_threads(g_nthreads)
    {
        double *buf = (double *)malloc(sizeof(double) * 2 * (size_t)len * BATCH);
        double *scr = (double *)malloc(sizeof(double) * 2 * (size_t)len);
#pragma omp for schedule(static)
        for (long long task = 0; task < ntask; task++) {
            int o = (int)(task / nbatch);
            int b0 = (int)(task % nbatch) * BATCH;
            int nb = inner - b0 < BATCH ? inner - b0 : BATCH;
            double *base = data + 2 * ((size_t)o * len * inner + b0);
            for (int m = 0; m < len; m++)
                for (int b = 0; b < nb; b++) {
                    buf[2 * ((size_t)b * len + m)] = base[2 * ((size_t)m * inner + b)];
                    buf[2 * ((size_t)b * len + m) + 1] = base[2 * ((size_t)m * inner + b) + 1];
                }
            for (int b = 0; b < nb; b++) line_fft(lp, buf + 2 * (size_t)b * len, scr, sign);
            for (int m = 0; m < len; m++)
                for (int b = 0; b < nb; b++) {
                    base[2 * ((size_t)m * inner + b)] = buf[2 * ((size_t)b * len + m)];
                    base[2 * ((size_t)m * inner + b) + 1] = buf[2 * ((size_t)b * len + m) + 1];
                }
        }
        free(buf);
        free(scr);
    }
}

static void r2c_rows(const line_plan *lp, const double *in, double *out, long long nrows, int n, int nz) {
    long long npairs = (nrows + 1) / 2;
#pragma omp parallel num_threads(g_nthreads)
    {
        double *z = (double *)malloc(sizeof(double) * 2 * (size_t)n);
        double *scr = (double *)malloc(sizeof(double) * 2 * (size_t)n);
#pragma omp for schedule(static)
        for (long long pr = 0; pr < npairs; pr++) {
            long long r0 = 2 * pr, r1 = r0 + 1;
            const double *x0 = in + (size_t)r0 * n;
            const double *x1 = r1 < nrows ? in + (size_t)r1 * n : NULL;
            for (int m = 0; m < n; m++) {
                z[2 * m] = x0[m];
                z[2 * m + 1] = x1 ? x1[m] : 0.0;
            }
            line_fft(lp, z, scr, -1);
            double *X0 = out + 2 * (size_t)r0 * nz;
            double *X1 = x1 ? out + 2 * (size_t)r1 * nz : NULL;
            for (int k = 0; k < nz; k++) {
                int kk = (n - k) % n;
                double zr = z[2 * k], zi = z[2 * k + 1];
                double cr = z[2 * kk], ci = -z[2 * kk + 1]; /* conj(Z[n-k]) */
                X0[2 * k] = 0.5 * (zr + cr);
                X0[2 * k + 1] = 0.5 * (zi + ci);
                if (X1) {
                    /* (Z - conj Z')/(2i) */
                    double dr = zr - cr, di = zi - ci;
                    X1[2 * k] = 0.5 * di;
                    X1[2 * k + 1] = -0.5 * dr;
                }
            }
        }
        free(z);
        free(scr);
    }
}

static void c2r_rows(const line_plan *lp, const double *in, double *out, long long nrows, int n, int nz) {
    long long npairs = (nrows + 1) / 2;
#pragma omp parallel num_threads(g_nthreads)
    {
        double *z = (double *)malloc(sizeof(double) * 2 * (size_t)n);
        double *scr = (double *)malloc(sizeof(double) * 2 * (size_t)n);
#pragma omp for schedule(static)
        for (long long pr = 0; pr < npairs; pr++) {
            long long r0 = 2 * pr, r1 = r0 + 1;
            const double *X0 = in + 2 * (size_t)r0 * nz;
            const double *X1 = r1 < nrows ? in + 2 * (size_t)r1 * nz : NULL;
            for (int k = 0; k < nz; k++) {
                double ar = X0[2 * k], ai = X0[2 * k + 1];
                double br = X1 ? X1[2 * k] : 0.0, bi = X1 ? X1[2 * k + 1] : 0.0;
                int self_conj = (k == 0) || (2 * k == n);
                if (self_conj) { ai = 0.0; bi = 0.0; }
                /* Z[k] = A + iB */
                z[2 * k] = ar - bi;
                z[2 * k + 1] = ai + br;
                if (k > 0 && 2 * k < n) {
                    /* Z[n-k] = conj(A) + i conj(B) */
                    z[2 * (n - k)] = ar + bi;
                    z[2 * (n - k) + 1] = -ai + br;
                }
            }
            line_fft(lp, z, scr, +1);
            double *x0 = out + (size_t)r0 * n;
            double *x1 = X1 ? out + (size_t)r1 * n : NULL;
            for (int m = 0; m < n; m++) {
                x0[m] = z[2 * m];
                if (x1) x1[m] = z[2 * m + 1];
            }
        }
        free(z);
        free(scr);
    }
}

void fftw_execute_dft_r2c(const fftw_plan p, double *in, fftw_complex *out) {
    int n0 = p->n0, n1 = p->n1, n2 = p->n2, nz = p->nz;
    double *o = (double *)out;
    r2c_rows(&p->p2, in, o, (long long)n0 * n1, n2, nz);
    strided_pass(&p->p1, o, n0, n1, nz, -1);
    strided_pass(&p->p0, o, 1, n0, n1 * nz, -1);
}

void fftw_execute_dft_c2r(const fftw_plan p, fftw_complex *in, double *out) {
    int n0 = p->n0, n1 = p->n1, n2 = p->n2, nz = p->nz;
    size_t nc = (size_t)n0 * n1 * nz;
    double *tmp = (double *)fftw_malloc(sizeof(double) * 2 * nc);
    memcpy(tmp, in, sizeof(double) * 2 * nc);
    strided_pass(&p->p0, tmp, 1, n0, n1 * nz, +1);
    strided_pass(&p->p1, tmp, n0, n1, nz, +1);
    c2r_rows(&p->p2, tmp, out, (long long)n0 * n1, n2, nz);
    fftw_free(tmp);
}

void fftw_execute(const fftw_plan p) {
    if (p->kind == 0)
        fftw_execute_dft_r2c(p, p->in_r, p->out_c);
    else
        fftw_execute_dft_c2r(p, p->in_c, p->out_r);
}
