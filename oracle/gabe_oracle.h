/*
 * gabe_oracle.h -- CPU restatement of GABE's lattice-evolution path (FP64).
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py may load liboracle.so, and only as the
 * checker.  The CUDA library never links or calls it.
 *
 * Every function cites the reference code it restates.  State layout is the
 * reference's: field/dfield [2 stages][nflds][N][N][N] (g2main.cpp:49,99),
 * h/l/T_gw [2 stages][12][N][N][N/2+1] (g2main.cpp:53-55), k fastest.
 *
 * Pinned against the reference itself: tests/golden holds dumps written by
 * the reference sources compiled under oracle/_ref (oracle/Makefile), and
 * tests/test_oracle_golden.py checks this restatement against them.
 */
#ifndef GABE_ORACLE_H
#define GABE_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

enum { ORA_MODEL_QUADRATIC = 0, ORA_MODEL_LPHI4 = 1 };

typedef struct {
    int N;
    int nflds;        /* must be 2 */
    double L, dt;
    int model;        /* ORA_MODEL_* */
    int gws;          /* 0/1 */
    int gw_spec_quirk;/* 1: read l at kz=N/2 for the kz=0 plane as g2spectra.cpp:149-164 does */
    int expansion;    /* expansion_type 0, 1 or 2 (g2parameters.h:62); callers set it */
    /* model constants, see ora_model_constants() */
    double mc[6];
    /* initial spectrum (randInit, g2init.cpp:117-165): 0 field_full_rand 1
     * without cut-off; 1 field_full_rand 1 with spec_cut_off/spec_smooth;
     * 2 field_full_rand 0 (deterministic amplitudes) with the cut-off */
    int ic_variant;
    int ic_pad;
    double spec_cut, spec_smooth;
} ora_params;

typedef struct {
    double a[2], adot[2], edkin[2], edpot[2], edgrad[2], edrho[2];
} ora_scalars;

/* Fill p->mc for a model.  Quadratic (reference g2model.cpp:64-87):
 * mphi, gsq.  lphi4 (oracle/ref_cfg/g2model_lphi4.cpp): lam_pr, gsq_pr. */
void ora_model_constants(ora_params *p, double c0, double c1);

double ora_potential(const ora_params *p, double phi, double chi);
double ora_dvdf(const ora_params *p, int fld, double phi, double chi);

/* calcEnergy(s) on one stage's arrays (g2functions.cpp:124-174):
 * out = {kin, pot, grad, rho}. */
void ora_calc_energy(const ora_params *p, const double *f, const double *df, double a_s, double out[4]);

/* adf (g2functions.cpp:188-191). */
double ora_adf(double edrho_s, double a_s);

/* The reference initialisation sequence initfields(); initexpansion();
 * initfields() (g2main.cpp:111-118, g2model.cpp:113-144, g2init.cpp:16-189)
 * with srand(seed) and rand() in single-thread order.  Writes stage 0 of
 * field/dfield and the scalars.  expansion_type 0 starts from a = 1,
 * adot = 0 in both stages (g2init.cpp:18-24); expansion_type 2 leaves the
 * start to the user (g2init.cpp:32-41) and is started here as type 1. */
void ora_init(const ora_params *p, int seed, const double f0[2], const double df0[2],
              double rescale_B, double *field, double *dfield, ora_scalars *sc);

/* One step() (g2functions.cpp:201-304): expansion_type 1 (:234-271)
 * including evolve_perts (g2evolutionpert.cpp:343-455) when p->gws;
 * expansion_type 0 (:207-232: a and adot fixed, no tensor modes, only
 * calcEnergy(0) at the end); expansion_type 2 (:272-302: type 1's update
 * without the tensor modes).  T_gw may be NULL (then allocated internally). */
void ora_step(const ora_params *p, double *field, double *dfield, double *h, double *l,
              double *T_gw, ora_scalars *sc);

/* fft_stresstensor(s) (g2evolutionpert.cpp:135-339): writes T_gw stage s
 * (12 x N*N*(N/2+1)) from field stage s. */
void ora_fft_stresstensor(const ora_params *p, const double *field_s, double *T_s);

/* The reference's explicit TT projection for one k-point times nm (= dx^3)
 * (g2evolutionpert.cpp:203-310).  S and T are 6 complex values (re,im) in
 * the order 11,12,13,22,23,33; n = integer wave vector. */
void ora_tt_point(const int n[3], double nm, const double S[12], double T[12]);

/* specOut (g2spectra.cpp:23-234): out has numbins rows and
 * 1 + 2*nflds (+3 with gws) columns: k, P_phi, D2_phi, P_chi, D2_chi
 * [, P_gw, Omega_gw, p].  Returns numbins. */
int ora_spectra_numbins(int N);
int ora_spectra(const ora_params *p, const double *field0, const double *l0, double edrho0, double *out);

#ifdef __cplusplus
}
#endif

#endif
