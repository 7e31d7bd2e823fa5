/*
 * gabe_oracle.c -- CPU restatement of GABE's lattice-evolution path (FP64).
 *
 * TEST INFRASTRUCTURE ONLY; see gabe_oracle.h.  Compiled with
 * -ffp-contract=off so that every multiply and add rounds separately, as the
 * reference's x86-64 build (no FMA) does.  Sums run serially in the
 * reference's loop order with one partial per field, which is what the
 * reference's OpenMP reductions produce with one thread, so with the same
 * inputs this code reproduces a parallelize=0 reference build bit for bit.
 */
#include "gabe_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "fftw_shim/fftw3.h"

#define IDX(N, i, j, k) ((((size_t)(i)) * (N) + (j)) * (N) + (k))

static inline int incr(int i, int N) { return i == N - 1 ? 0 : i + 1; }
static inline int decr(int i, int N) { return i == 0 ? N - 1 : i - 1; }
static inline double pw2(double x) { return x * x; }

/* ------------------------------------------------------------------ */
/* model                                                               */
/* ------------------------------------------------------------------ */
void ora_model_constants(ora_params *p, double c0, double c1)
{
    memset(p->mc, 0, sizeof(p->mc));
    if (p->model == ORA_MODEL_QUADRATIC) {
        /* COUP = gsq/mphi/mphi (g2model.cpp:64) and the folded constant
         * 0.5*gsq/mphi/mphi of the potential (g2model.cpp:68). */
        double mphi = c0, gsq = c1;
        p->mc[0] = gsq / mphi / mphi;
        p->mc[1] = 0.5 * gsq / mphi / mphi;
    } else {
        double lam = c0, g = c1;
        p->mc[0] = lam;
        p->mc[1] = g;
        p->mc[2] = 0.25 * lam;
        p->mc[3] = 0.5 * g;
        p->mc[4] = 3. * lam;
    }
}

double ora_potential(const ora_params *p, double P, double C)
{
    if (p->model == ORA_MODEL_QUADRATIC)
        return (0.5 * P * P + p->mc[1] * P * P * C * C); /* g2model.cpp:66-69 */
    return p->mc[2] * P * P * P * P + p->mc[3] * P * P * C * C;
}

double ora_dvdf(const ora_params *p, int fld, double P, double C)
{
    if (p->model == ORA_MODEL_QUADRATIC) { /* g2model.cpp:72-87 */
        if (fld == 0) return (P + p->mc[0] * C * C * P);
        return (p->mc[0] * P * P * C);
    }
    if (fld == 0) return p->mc[0] * P * P * P + p->mc[1] * C * C * P;
    return p->mc[1] * P * P * C;
}

static double eff_mass(const ora_params *p, int fld, const double *f)
{
    /* effMass (g2model.cpp:89-108; lphi4 variant in ref_cfg) */
    int N = p->N;
    size_t n3 = (size_t)N * N * N;
    const double *P = f, *C = f + n3;
    double m = 0.;
    double gridsize = (double)(N * N * N);
    for (size_t x = 0; x < n3; x++) {
        if (p->model == ORA_MODEL_QUADRATIC) {
            if (fld == 0) m += (1. + p->mc[0] * C[x] * C[x]);
            else m += (p->mc[0] * P[x] * P[x]);
        } else {
            if (fld == 0) m += p->mc[4] * P[x] * P[x] + p->mc[1] * C[x] * C[x];
            else m += p->mc[1] * P[x] * P[x];
        }
    }
    return m / gridsize;
}

/* ------------------------------------------------------------------ */
/* stencils and energies                                              */
/* ------------------------------------------------------------------ */
static inline double laplacian(const double *f, int N, double dx, int i, int j, int k)
{
    /* g2functions.cpp:35-43 */
    return (f[IDX(N, incr(i, N), j, k)] + f[IDX(N, decr(i, N), j, k)]
            + f[IDX(N, i, incr(j, N), k)] + f[IDX(N, i, decr(j, N), k)]
            + f[IDX(N, i, j, incr(k, N))] + f[IDX(N, i, j, decr(k, N))]
            - 6. * f[IDX(N, i, j, k)]) / (dx * dx);
}

void ora_calc_energy(const ora_params *p, const double *f, const double *df, double a_s, double out[4])
{
    int N = p->N;
    size_t n3 = (size_t)N * N * N;
    double dx = p->L / ((double)N);
    double gridsize = (double)(N * N * N);
    /* avgKin (g2functions.cpp:153-165): one reduction per field */
    double kin = 0.;
    for (int fld = 0; fld < p->nflds; fld++) {
        double part = 0.;
        const double *d = df + fld * n3;
        for (size_t x = 0; x < n3; x++) part += d[x] * d[x];
        kin = kin + part;
    }
    kin = kin / gridsize / 2.;
    /* avgPot (g2functions.cpp:139-150) */
    double pot = 0.;
    for (size_t x = 0; x < n3; x++) pot += ora_potential(p, f[x], f[n3 + x]);
    pot = pot / gridsize;
    /* avgGrad (g2functions.cpp:124-136) */
    double grad = 0.;
    for (int fld = 0; fld < p->nflds; fld++) {
        double part = 0.;
        const double *g = f + fld * n3;
        for (int i = 0; i < N; i++)
            for (int j = 0; j < N; j++)
                for (int k = 0; k < N; k++)
                    part -= g[IDX(N, i, j, k)] * laplacian(g, N, dx, i, j, k);
        grad = grad + part;
    }
    grad = grad / gridsize / 2. / a_s / a_s;
    out[0] = kin;
    out[1] = pot;
    out[2] = grad;
    out[3] = kin + pot + grad; /* calcEnergy, g2functions.cpp:168-174 */
}

double ora_adf(double edrho_s, double a_s)
{
    return sqrt(8. * M_PI / 3. * edrho_s) * a_s; /* g2functions.cpp:188-191 */
}

static void set_energy(const ora_params *p, const double *f, const double *df, ora_scalars *sc, int s)
{
    double e[4];
    ora_calc_energy(p, f, df, sc->a[s], e);
    sc->edkin[s] = e[0];
    sc->edpot[s] = e[1];
    sc->edgrad[s] = e[2];
    sc->edrho[s] = e[3];
}

/* ------------------------------------------------------------------ */
/* initial conditions                                                  */
/* ------------------------------------------------------------------ */
static void rand_init(const ora_params *p, double *f, double *df, double d2vdf2, double H0,
                      double rescale_B, double *fk, double *fkd, double *inic, fftw_plan pf, fftw_plan pd)
{
    /* randInit (g2init.cpp:68-189): field_full_rand 1 without (variant 0) or
     * with (1) the spectral cut-off, or field_full_rand 0 (2) */
    const int var = p->ic_variant;
    int N = p->N, nz = N / 2 + 1;
    double L = p->L;
    double dk2 = 4. * M_PI * M_PI / L / L;
    for (int i = 0; i < N; i++) {
        double i2 = (i < (N / 2 + 1) ? (i * i) : ((N - i) * (N - i)));
        for (int j = 0; j < N; j++) {
            double j2 = (j < (N / 2 + 1) ? (j * j) : ((N - j) * (N - j)));
            for (int k = 0; k < nz; k++) {
                double k2 = (k * k);
                size_t x = (size_t)k + (size_t)nz * ((size_t)j + (size_t)N * i);
                if (i + j + k == 0) {
                    fk[2 * x] = 0.; fk[2 * x + 1] = 0.;
                    fkd[2 * x] = 0.; fkd[2 * x + 1] = 0.;
                    continue;
                }
                double wk = sqrt(dk2 * ((double)i2 + (double)j2 + (double)k2) + d2vdf2);
                if (var == 2) { /* :155-163 */
                    fk[2 * x] = rescale_B * sqrt(1 / (2. * wk * L * L * L)) *
                                (1. - tanh(p->spec_smooth * (sqrt(i2 + j2 + k2) - N * p->spec_cut))) / 2.;
                    fk[2 * x + 1] = 0.;
                    fkd[2 * x] = -H0 * fk[2 * x];
                    fkd[2 * x + 1] = 0.;
                    continue;
                }
                double u, th, r1[2], r2[2];
                u = (double)rand() / (double)RAND_MAX;
                th = 2. * M_PI * (double)rand() / (double)RAND_MAX;
                if (var == 1) { /* :120-131 */
                    const double cut = p->spec_smooth * (sqrt(i2 + j2 + k2) - N * p->spec_cut);
                    r1[0] = rescale_B * cos(th) * sqrt(-log(u) / (2. * wk * L * L * L)) * (1. - tanh(cut)) / 2.;
                    r1[1] = rescale_B * sin(th) * sqrt(-log(u) / (2. * wk * L * L * L)) * (1. - tanh(cut)) / 2.;
                    u = (double)rand() / (double)RAND_MAX;
                    th = 2. * M_PI * (double)rand() / (double)RAND_MAX;
                    r2[0] = rescale_B * cos(th) * sqrt(-log(u) / (2. * wk * L * L * L)) * (1. - tanh(cut)) / 2.;
                    r2[1] = rescale_B * sin(th) * sqrt(-log(u) / (2. * wk * L * L * L)) * (1. - tanh(cut)) / 2.;
                } else { /* :135-143 */
                    r1[0] = rescale_B * cos(th) * sqrt(-log(u) / (2. * wk * L * L * L));
                    r1[1] = rescale_B * sin(th) * sqrt(-log(u) / (2. * wk * L * L * L));
                    u = (double)rand() / (double)RAND_MAX;
                    th = 2. * M_PI * (double)rand() / (double)RAND_MAX;
                    r2[0] = rescale_B * cos(th) * sqrt(-log(u) / (2. * wk * L * L * L));
                    r2[1] = rescale_B * sin(th) * sqrt(-log(u) / (2. * wk * L * L * L));
                }
                fk[2 * x] = (r1[0] + r2[0]) / sqrt(2.);
                fk[2 * x + 1] = (r1[1] + r2[1]) / sqrt(2.);
                fkd[2 * x] = (r2[1] - r1[1]) * wk / sqrt(2.) - H0 * fk[2 * x];
                fkd[2 * x + 1] = (r1[0] - r2[0]) * wk / sqrt(2.) - H0 * fk[2 * x + 1];
            }
        }
    }
    size_t n3 = (size_t)N * N * N;
    fftw_execute(pf);
    for (size_t x = 0; x < n3; x++) f[x] += inic[x];
    fftw_execute(pd);
    for (size_t x = 0; x < n3; x++) df[x] += inic[x];
}

void ora_init(const ora_params *p, int seed, const double f0[2], const double df0[2], double rescale_B,
              double *field, double *dfield, ora_scalars *sc)
{
    int N = p->N;
    size_t n3 = (size_t)N * N * N;
    memset(sc, 0, sizeof(*sc));
    /* initfields, first call: homogeneous values (g2model.cpp:122-129) */
    for (int fld = 0; fld < p->nflds; fld++)
        for (size_t x = 0; x < n3; x++) {
            field[fld * n3 + x] = f0[fld];
            dfield[fld * n3 + x] = df0[fld];
        }
    /* initexpansion (g2init.cpp:16-43) */
    if (p->expansion == 0) {
        sc->a[0] = 1;
        sc->adot[0] = 0;
        sc->a[1] = 1;
        sc->adot[1] = 0;
        set_energy(p, field, dfield, sc, 0);
    } else {
        sc->a[0] = 1;
        set_energy(p, field, dfield, sc, 0);
        sc->adot[0] = ora_adf(sc->edrho[0], sc->a[0]);
    }
    /* initfields, second call: fluctuations (g2model.cpp:132-140) */
    int nz = N / 2 + 1;
    size_t nc = (size_t)N * N * nz;
    double *inic = (double *)fftw_malloc(sizeof(double) * n3);
    double *fk = (double *)fftw_malloc(sizeof(double) * 2 * nc);
    double *fkd = (double *)fftw_malloc(sizeof(double) * 2 * nc);
    fftw_plan pf = fftw_plan_dft_c2r_3d(N, N, N, (fftw_complex *)fk, inic, FFTW_MEASURE);
    fftw_plan pd = fftw_plan_dft_c2r_3d(N, N, N, (fftw_complex *)fkd, inic, FFTW_MEASURE);
    srand(seed);
    double H0 = sqrt(8. * M_PI / 3. * sc->edrho[0]);
    for (int fld = 0; fld < p->nflds; fld++) {
        double m2 = eff_mass(p, fld, field);
        rand_init(p, field + fld * n3, dfield + fld * n3, m2, H0, rescale_B, fk, fkd, inic, pf, pd);
    }
    fftw_destroy_plan(pf);
    fftw_destroy_plan(pd);
    fftw_free(inic);
    fftw_free(fk);
    fftw_free(fkd);
    set_energy(p, field, dfield, sc, 0);
}

/* ------------------------------------------------------------------ */
/* tensor perturbations                                                */
/* ------------------------------------------------------------------ */
static inline double delfld(const double *f, int N, int i, int j, int k, int n)
{
    /* g2evolutionpert.cpp:31-44 */
    if (n == 1) return (f[IDX(N, incr(i, N), j, k)] - f[IDX(N, decr(i, N), j, k)]) / 2;
    if (n == 2) return (f[IDX(N, i, incr(j, N), k)] - f[IDX(N, i, decr(j, N), k)]) / 2;
    return (f[IDX(N, i, j, incr(k, N))] - f[IDX(N, i, j, decr(k, N))]) / 2;
}

static void stress_point(const ora_params *p, const double *fs, int i, int j, int k, double out[6])
{
    /* jtg_stresstensor for (1,1),(1,2),(1,3),(2,2),(2,3),(3,3)
     * (g2evolutionpert.cpp:48-132) */
    int N = p->N;
    size_t n3 = (size_t)N * N * N;
    double dx = p->L / ((double)N);
    double dn = (double)(1 / pw2(dx));
    for (int c = 0; c < 6; c++) out[c] = 0.0;
    for (int m = 0; m < p->nflds; m++) {
        const double *f = fs + m * n3;
        double d1 = delfld(f, N, i, j, k, 1);
        double d2 = delfld(f, N, i, j, k, 2);
        double d3 = delfld(f, N, i, j, k, 3);
        out[0] += (2. / 3.) * dn * d1 * d1 - (1. / 3.) * dn * d2 * d2 - (1. / 3.) * dn * d3 * d3;
        out[1] += dn * d1 * d2;
        out[2] += (dn * d1 * d3);
        out[3] += -(1. / 3.) * dn * d1 * d1 + (2. / 3.) * dn * d2 * d2 - (1. / 3.) * dn * d3 * d3;
        out[4] += (dn * d2 * d3);
        out[5] += -(1. / 3.) * dn * d1 * d1 - (1. / 3.) * dn * d2 * d2 + (2. / 3.) * dn * d3 * d3;
    }
}

void ora_tt_point(const int n[3], double nm, const double S[12], double T[12])
{
    /* Lambda_ij,lm S_lm times nm = dx^3, written term by term in the
     * reference's order (g2evolutionpert.cpp:203-310) so rounding agrees.
     * S/T hold (re,im) of components 11,12,13,22,23,33. */
    double m2 = pw2((double)n[0]) + pw2((double)n[1]) + pw2((double)n[2]);
    double z = ((double)n[2]) / sqrt(m2);
    double x = ((double)n[0]) / sqrt(m2);
    double y = ((double)n[1]) / sqrt(m2);
    for (int c = 0; c < 2; c++) {
        double s0 = S[0 + c], s1 = S[2 + c], s2 = S[4 + c], s3 = S[6 + c], s4 = S[8 + c], s5 = S[10 + c];
        /* T11 */
        T[0 + c] = .5 * pw2(1 - x * x) * nm * s0 - (1 - x * x) * x * y * nm * s1
                   - (1 - x * x) * x * z * nm * s2 + pw2(x * y) * nm * s3
                   - .5 * (1 - x * x) * (1 - y * y) * nm * s3 + (1 + x * x) * y * z * nm * s4
                   + pw2(x * z) * nm * s5 - .5 * (1 - x * x) * (1 - z * z) * nm * s5;
        /* T22 */
        T[6 + c] = .5 * pw2(1 - y * y) * nm * s3 - (1 - y * y) * x * y * nm * s1
                   - (1 - y * y) * y * z * nm * s4 + pw2(x * y) * nm * s0
                   - .5 * (1 - x * x) * (1 - y * y) * nm * s0 + (1 + y * y) * x * z * nm * s2
                   + pw2(y * z) * nm * s5 - .5 * (1 - y * y) * (1 - z * z) * nm * s5;
        /* T33 */
        T[10 + c] = .5 * pw2(1 - z * z) * nm * s5 - (1 - z * z) * x * z * nm * s2
                    - (1 - z * z) * y * z * nm * s4 + pw2(x * z) * nm * s0
                    - .5 * (1 - x * x) * (1 - z * z) * nm * s0 + (1 + z * z) * x * y * nm * s1
                    + pw2(y * z) * nm * s3 - .5 * (1 - y * y) * (1 - z * z) * nm * s3;
        /* T12 */
        T[2 + c] = -.5 * x * y * (1 - x * x) * nm * s0 - .5 * x * y * (1 - y * y) * nm * s3
                   + .5 * x * y * (1 + z * z) * nm * s5 + (1 - x * x) * (1 - y * y) * nm * s1
                   - y * z * (1 - x * x) * nm * s2 - x * z * (1 - y * y) * nm * s4;
        /* T13 */
        T[4 + c] = -.5 * x * z * (1 - x * x) * nm * s0 + .5 * x * z * (1 + y * y) * nm * s3
                   - .5 * x * z * (1 - z * z) * nm * s5 + (1 - x * x) * (1 - z * z) * nm * s2
                   - y * z * (1 - x * x) * nm * s1 - x * y * (1 - z * z) * nm * s4;
        /* T23 */
        T[8 + c] = +.5 * y * z * (1 + x * x) * nm * s0 - .5 * y * z * (1 - y * y) * nm * s3
                   - .5 * y * z * (1 - z * z) * nm * s5 + (1 - y * y) * (1 - z * z) * nm * s4
                   - x * y * (1 - z * z) * nm * s2 - x * z * (1 - y * y) * nm * s1;
    }
}

void ora_fft_stresstensor(const ora_params *p, const double *fs, double *T)
{
    /* g2evolutionpert.cpp:135-339 */
    int N = p->N, nz = N / 2 + 1;
    size_t n3 = (size_t)N * N * N, M = (size_t)N * N * nz;
    double *src = (double *)fftw_malloc(sizeof(double) * 6 * n3);
    double *out = (double *)fftw_malloc(sizeof(double) * 2 * 6 * M);
    for (int i = 0; i < N; i++)
        for (int j = 0; j < N; j++)
            for (int k = 0; k < N; k++) {
                double o[6];
                stress_point(p, fs, i, j, k, o);
                for (int c = 0; c < 6; c++) src[c * n3 + IDX(N, i, j, k)] = o[c];
            }
    fftw_plan pl = fftw_plan_dft_r2c_3d(N, N, N, src, (fftw_complex *)out, FFTW_MEASURE);
    for (int c = 0; c < 6; c++)
        fftw_execute_dft_r2c(pl, src + c * n3, (fftw_complex *)(out + 2 * c * M));
    fftw_destroy_plan(pl);
    double dx = p->L / ((double)N);
    double normmm = pow(dx, 3);
    /* component c of the reference's T_gw planar order: 11re,11im,12re,... */
    for (int i = 0; i < N; i++) {
        int px = (i <= N / 2 ? i : i - N);
        for (int j = 0; j < N; j++) {
            int py = (j <= N / 2 ? j : j - N);
            for (int k = 0; k < nz; k++) {
                size_t x = ((size_t)i * N + j) * nz + k;
                double S[12], Tt[12];
                for (int c = 0; c < 6; c++) {
                    S[2 * c] = out[2 * (c * M + x)];
                    S[2 * c + 1] = out[2 * (c * M + x) + 1];
                }
                int n[3] = {px, py, k};
                ora_tt_point(n, normmm, S, Tt);
                for (int c = 0; c < 12; c++) T[c * M + x] = Tt[c];
            }
        }
    }
    for (int c = 0; c < 12; c++) T[c * M] = 0; /* g2evolutionpert.cpp:319-321 */
    fftw_free(src);
    fftw_free(out);
}

static void evolve_perts(const ora_params *p, int s, int snew, double deet, const double *field,
                         double *h, double *l, double *T, const ora_scalars *sc)
{
    /* evolve_perts + derivs (g2evolutionpert.cpp:343-516) */
    int N = p->N, nz = N / 2 + 1;
    size_t n3 = (size_t)N * N * N, M = (size_t)N * N * nz;
    double *Ts = T + (size_t)s * 12 * M;
    ora_fft_stresstensor(p, field + (size_t)s * p->nflds * n3, Ts);
    double as = sc->a[s], ads = sc->adot[s];
    double norm = (4. * M_PI * M_PI / p->L / p->L / as / as);
    double omega = (8. * M_PI) / as / as;
    double *hs = h + (size_t)s * 12 * M, *ls = l + (size_t)s * 12 * M;
    double *hn = h + (size_t)snew * 12 * M, *ln = l + (size_t)snew * 12 * M;
    for (int i = 0; i < N; i++) {
        int ii = (i <= N / 2 ? i : i - N);
        for (int j = 0; j < N; j++) {
            int jj = (j <= N / 2 ? j : j - N);
            for (int k = 0; k < nz; k++) {
                size_t x = ((size_t)i * N + j) * nz + k;
                double kk = (pw2((double)ii) + pw2((double)jj) + pw2((double)k)) * norm;
                double hd[12], ld[12];
                for (int c = 0; c < 12; c++) {
                    ld[c] = -kk * hs[c * M + x] - 3. * ads / as * ls[c * M + x] + 2. * omega * Ts[c * M + x];
                    hd[c] = ls[c * M + x];
                }
                for (int c = 0; c < 12; c++) {
                    hn[c * M + x] = h[c * M + x] + deet * hd[c];
                    ln[c * M + x] = l[c * M + x] + deet * ld[c];
                }
            }
        }
    }
}

/* ------------------------------------------------------------------ */
/* step                                                                */
/* ------------------------------------------------------------------ */
void ora_step(const ora_params *p, double *field, double *dfield, double *h, double *l, double *T_gw,
              ora_scalars *sc)
{
    int N = p->N, F = p->nflds;
    size_t n3 = (size_t)N * N * N;
    double dx = p->L / ((double)N), dt = p->dt;
    double *f0 = field, *f1 = field + F * n3, *d0 = dfield, *d1 = dfield + F * n3;
    int own_T = 0;
    if (p->gws && !T_gw) {
        T_gw = (double *)malloc(sizeof(double) * 2 * 12 * (size_t)N * N * (N / 2 + 1));
        own_T = 1;
    }
    /* stage 1 (g2functions.cpp:236-244) */
    for (int fld = 0; fld < F; fld++)
        for (int i = 0; i < N; i++)
            for (int j = 0; j < N; j++)
                for (int k = 0; k < N; k++) {
                    size_t x = IDX(N, i, j, k);
                    const double *g = f0 + fld * n3;
                    double dd = laplacian(g, N, dx, i, j, k) / sc->a[0] / sc->a[0]
                                - ora_dvdf(p, fld, f0[x], f0[n3 + x])
                                - 3 * sc->adot[0] / sc->a[0] * d0[fld * n3 + x];
                    f1[fld * n3 + x] = f0[fld * n3 + x] + .5 * dt * d0[fld * n3 + x];
                    d1[fld * n3 + x] = d0[fld * n3 + x] + .5 * dt * dd;
                }
    const int ex = p->expansion, gw = p->gws && ex == 1;
    if (gw) evolve_perts(p, 0, 1, 0.5 * dt, field, h, l, T_gw, sc); /* :247 */
    if (ex != 0) {
        /* :250-252 (type 2: :286-288) */
        sc->a[1] = sc->a[0] + .5 * dt * sc->adot[0];
        set_energy(p, f1, d1, sc, 1);
        sc->adot[1] = ora_adf(sc->edrho[1], sc->a[1]);
    }
    /* stage 2 (g2functions.cpp:254-262) */
    for (int fld = 0; fld < F; fld++)
        for (int i = 0; i < N; i++)
            for (int j = 0; j < N; j++)
                for (int k = 0; k < N; k++) {
                    size_t x = IDX(N, i, j, k);
                    const double *g = f1 + fld * n3;
                    double dd = laplacian(g, N, dx, i, j, k) / sc->a[1] / sc->a[1]
                                - ora_dvdf(p, fld, f1[x], f1[n3 + x])
                                - 3 * sc->adot[1] / sc->a[1] * d1[fld * n3 + x];
                    f0[fld * n3 + x] = f0[fld * n3 + x] + dt * d1[fld * n3 + x];
                    d0[fld * n3 + x] = d0[fld * n3 + x] + dt * dd;
                }
    if (gw) evolve_perts(p, 1, 0, dt, field, h, l, T_gw, sc); /* :265 */
    if (ex != 0) {
        /* :268-270 (type 2: :299-301) */
        sc->a[0] = sc->a[0] + dt * sc->adot[1];
        set_energy(p, f0, d0, sc, 0);
        sc->adot[0] = ora_adf(sc->edrho[0], sc->a[0]);
    } else {
        set_energy(p, f0, d0, sc, 0); /* :231 */
    }
    if (own_T) free(T_gw);
}

/* ------------------------------------------------------------------ */
/* spectra                                                             */
/* ------------------------------------------------------------------ */
int ora_spectra_numbins(int N) { return ((int)(sqrt(3.) * N / 2 + 1)); }

static double gw_power(const double *l0, size_t M, size_t x)
{
    /* weights of g2spectra.cpp:133-144 */
    double w[12] = {1, 1, 2, 2, 2, 2, 1, 1, 2, 2, 1, 1};
    double s = 0.;
    for (int c = 0; c < 12; c++) {
        double v = l0[c * M + x];
        s = (c == 0) ? pw2(v) : s + w[c] * pw2(v);
    }
    return s;
}

int ora_spectra(const ora_params *p, const double *field0, const double *l0, double edrho0, double *out)
{
    /* specOut (g2spectra.cpp:23-234) */
    int N = p->N, nz = N / 2 + 1, F = p->nflds;
    size_t n3 = (size_t)N * N * N, M = (size_t)N * N * nz;
    double L = p->L;
    const double spec_norm = pow(L / (double)N, 6.) * pow(2. * M_PI / L, 3.);
    const int nb = ora_spectra_numbins(N);
    int ncol = 1 + 2 * F + (p->gws ? 3 : 0);
    double *pw = (double *)calloc((size_t)nb, sizeof(double));
    double *np = (double *)calloc((size_t)nb, sizeof(double));
    double *in = (double *)fftw_malloc(sizeof(double) * n3);
    double *o = (double *)fftw_malloc(sizeof(double) * 2 * M);
    fftw_plan pl = fftw_plan_dft_r2c_3d(N, N, N, in, (fftw_complex *)o, FFTW_MEASURE);
    for (int b = 0; b < nb; b++) out[(size_t)b * ncol] = 2. * M_PI * b / L;
    for (int fld = 0; fld < F; fld++) {
        memcpy(in, field0 + fld * n3, sizeof(double) * n3);
        fftw_execute(pl);
        memset(pw, 0, sizeof(double) * nb);
        memset(np, 0, sizeof(double) * nb);
        for (int i = 0; i < N; i++) {
            int px = (i <= N / 2 ? i : i - N);
            for (int j = 0; j < N; j++) {
                int py = (j <= N / 2 ? j : j - N);
                for (int k = 1; k < N / 2; k++) {
                    size_t x = k + (size_t)nz * (j + (size_t)N * i);
                    int b = (int)sqrt(pw2(px) + pw2(py) + pw2(k));
                    pw[b] += 2. * (pw2(o[2 * x]) + pw2(o[2 * x + 1]));
                    np[b] += 2;
                }
                int kk[2] = {0, N / 2};
                for (int q = 0; q < 2; q++) {
                    size_t x = kk[q] + (size_t)nz * (j + (size_t)N * i);
                    int b = (int)sqrt(pw2(px) + pw2(py) + pw2(kk[q]));
                    pw[b] += (pw2(o[2 * x]) + pw2(o[2 * x + 1]));
                    np[b] += 1;
                }
            }
        }
        for (int b = 0; b < nb; b++) {
            double *row = out + (size_t)b * ncol;
            if (np[b] > 0) {
                row[1 + 2 * fld] = pw[b] * spec_norm / ((double)np[b]);
                row[2 + 2 * fld] = pow((double)b * 2. * M_PI / L, 3) * pw[b] * spec_norm / ((double)np[b]) / 2. / M_PI / M_PI;
            } else {
                row[1 + 2 * fld] = 0.;
                row[2 + 2 * fld] = 0.;
            }
        }
    }
    fftw_destroy_plan(pl);
    fftw_free(in);
    fftw_free(o);
    if (p->gws) {
        double hub = sqrt(8. * M_PI / 3.) * sqrt(edrho0);
        double dp = 2. * M_PI / (double)L;
        double norm1 = 4.e-5 / pow(100., .333) / 24. / M_PI / M_PI / pow(L, 3.) / pw2(hub);
        memset(pw, 0, sizeof(double) * nb);
        int *npg = (int *)calloc((size_t)nb, sizeof(int));
        for (int i = 0; i < N; i++) {
            int px = (i <= N / 2 ? i : i - N);
            for (int j = 0; j < N; j++) {
                int py = (j <= N / 2 ? j : j - N);
                for (int k = 1; k < N / 2; k++) {
                    size_t x = ((size_t)i * N + j) * nz + k;
                    int b = (int)sqrt(pw2(px) + pw2(py) + pw2(k));
                    npg[b] += 2;
                    pw[b] += 2. * gw_power(l0, M, x);
                }
                /* kz = 0 and kz = N/2 rows; the reference reads l at kz=N/2 for both */
                size_t x0 = ((size_t)i * N + j) * nz + (p->gw_spec_quirk ? N / 2 : 0);
                size_t xN = ((size_t)i * N + j) * nz + N / 2;
                int b0 = (int)sqrt(pw2(px) + pw2(py) + pw2(0));
                npg[b0] += 1;
                pw[b0] += gw_power(l0, M, x0);
                int bN = (int)sqrt(pw2(px) + pw2(py) + pw2(N / 2));
                npg[bN] += 1;
                pw[bN] += gw_power(l0, M, xN);
            }
        }
        for (int b = 0; b < nb; b++) {
            double *row = out + (size_t)b * ncol;
            if (npg[b] > 0) {
                row[1 + 2 * F] = pw[b] * spec_norm / ((double)npg[b]);
                row[2 + 2 * F] = norm1 * pow((double)b * 2 * M_PI / L, 3.) * pw[b] / (double)npg[b];
            } else {
                row[1 + 2 * F] = 0.;
                row[2 + 2 * F] = 0.;
            }
            row[3 + 2 * F] = dp * (double)b;
        }
        free(npg);
    }
    free(pw);
    free(np);
    return nb;
}
