/*
 * Build-time knobs for compiling the reference sources as the oracle.
 *
 * TEST INFRASTRUCTURE ONLY.  This header takes the place of the reference's
 * g2parameters.h (same names, same meaning; reference g2parameters.h:19-100)
 * when oracle/Makefile compiles the unmodified reference .cpp files with
 * `-Ioracle/ref_cfg -I<reference> -I-`, so every configuration is a
 * recompile with different -D values instead of an edited copy.
 *
 *   GABE_N        lattice points per side             (reference :57)
 *   GABE_L        box side in program units           (reference :58)
 *   GABE_DT       time step                           (reference :61)
 *   GABE_GWS      0/1 tensor perturbations            (reference :55)
 *   GABE_MODEL    0 = shipped m^2 phi^2 + g^2 phi^2 chi^2 model
 *                     (reference g2model.cpp, constants :44-48, B = mphi)
 *                 1 = lambda phi^4 + g^2 phi^2 chi^2 in the reference's
 *                     rescaling convention (oracle/ref_cfg/g2model_lphi4.cpp)
 *   GABE_PARALLEL 0 -> one thread, deterministic rand() order (reference :53,97-100)
 *   GABE_SEED     randseed                            (reference :56)
 *   GABE_ENDTIME, GABE_SLICEWAIT, GABE_FIELD_OUTDIM, GABE_VAR_OUTPUT
 *   GABE_EXPANSION expansion_type                     (reference :62)
 *   GABE_FULL_RAND field_full_rand                    (reference :72)
 *   GABE_SPEC_CUT, GABE_SPEC_SMOOTH  spec_cut_off, spec_smooth (reference :73-74)
 *   GABE_FFTW_FLAG fftw_flag, 1 = long double         (reference :19-38)
 *                 run length and output knobs (reference :60,80,84,86) for
 *                 builds that use the reference's own g2main.cpp/g2output.cpp
 *
 * tot_num_thrds becomes a run-time value (env GABE_REF_THREADS) so one
 * binary can be timed with every host core.
 */
#include <math.h>

#ifndef GABE_FFTW_FLAG
#define GABE_FFTW_FLAG 0
#endif
#define fftw_flag GABE_FFTW_FLAG
#if fftw_flag == 1
/* long double state (reference :19-38); only the compile check of the
 * drop-in translation unit builds this form: the FFT shim is double only */
#define gNum long double
#define exp expl
#define sqrt sqrtl
#define cbrt cbrtl
#define log logl
#else
#define gNum double
#endif

#ifndef GABE_N
#define GABE_N 64
#endif
#ifndef GABE_L
#define GABE_L 20.
#endif
#ifndef GABE_DT
#define GABE_DT 0.01
#endif
#ifndef GABE_GWS
#define GABE_GWS 0
#endif
#ifndef GABE_MODEL
#define GABE_MODEL 1
#endif
#ifndef GABE_PARALLEL
#define GABE_PARALLEL 0
#endif
#ifndef GABE_SEED
#define GABE_SEED 44463132
#endif
#ifndef GABE_ENDTIME
#define GABE_ENDTIME 1.e9 /* the harness fixes the step count itself */
#endif
#ifndef GABE_SLICEWAIT
#define GABE_SLICEWAIT 1
#endif
#ifndef GABE_FIELD_OUTDIM
#define GABE_FIELD_OUTDIM 0
#endif
#ifndef GABE_VAR_OUTPUT
#define GABE_VAR_OUTPUT 0
#endif

#define num_flds 2

#if GABE_MODEL == 0
/* shipped model: V = m^2 phi^2/2 + g^2 phi^2 chi^2/2, program units B = m */
const gNum mphi = 1.e-6;
const gNum phi0 = 0.193;
const gNum gsq = 2.5e-7;
const gNum f0[2] = {phi0, 0.};
const gNum df0[2] = {-0.142231, 0.};
const gNum rescale_B = mphi;
#else
/* lambda phi^4 + g^2 phi^2 chi^2, program units B = sqrt(lambda) phi0:
 * V_pr = lam_pr phi^4/4 + gsq_pr phi^2 chi^2/2 with lam_pr = 1/phi0^2,
 * gsq_pr = (g^2/lambda)/phi0^2. */
const gNum lambda_phys = 9.e-14;
const gNum g2_over_lambda = 100.;
const gNum phi0 = 0.342;
const gNum lam_pr = 1. / (phi0 * phi0);
const gNum gsq_pr = g2_over_lambda / (phi0 * phi0);
const gNum f0[2] = {phi0, 0.};
const gNum df0[2] = {0., 0.};
const gNum rescale_B = sqrt(lambda_phys) * phi0;
/* names the shipped g2model.cpp would expect; unused by the lphi4 model */
const gNum mphi = rescale_B;
const gNum gsq = g2_over_lambda * lambda_phys;
#endif

#define parallelize GABE_PARALLEL
int gabe_ref_threads(void);
#define tot_num_thrds (gabe_ref_threads())
#define calc_gws GABE_GWS
const int randseed = GABE_SEED;
const int N = GABE_N;
const gNum L = GABE_L;
const gNum starttime = 0.;
const gNum endtime = GABE_ENDTIME;
const gNum dt = GABE_DT;
#ifndef GABE_EXPANSION
#define GABE_EXPANSION 1
#endif
#define expansion_type GABE_EXPANSION

#define rand_init 1
#ifndef GABE_FULL_RAND
#define GABE_FULL_RAND 1
#endif
#define field_full_rand GABE_FULL_RAND
#ifdef GABE_SPEC_CUT /* reference :73-74 (commented out there: sqrt(3.)/8., 0.5) */
#define spec_cut_off GABE_SPEC_CUT
#define spec_smooth GABE_SPEC_SMOOTH
#endif

const gNum screentime = 0;
const int slicewait = GABE_SLICEWAIT;
const int slicenumber = 1;
const int field_sliceskip = 2;
const int specnumber = 1;
#define field_outdim GABE_FIELD_OUTDIM
#define spec_output 1
#define var_output GABE_VAR_OUTPUT

const int nflds = num_flds;
const gNum dx = L / ((gNum)N);
const gNum gridsize = N * N * N;

#if parallelize != 1
#undef tot_num_thrds
#define tot_num_thrds 1
#endif
