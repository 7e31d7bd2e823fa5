/*
 * CPU FFT with the FFTW3 double-precision API subset that GABE calls.
 *
 * TEST INFRASTRUCTURE ONLY: this header and fftw_shim.c exist so that the
 * unmodified reference sources and the oracle restatement can be compiled in
 * an image that has no FFTW.  Nothing in the product library links it.
 *
 * Third-party dependency being stood in for: FFTW 3 (double precision,
 * threads/omp variants; the reference's makefile:9 links
 * -lfftw3_threads -lfftw3_omp -lfftw3, no version pinned).  What is restated
 * is FFTW's published convention, not its code:
 *   - forward (r2c) uses exp(-2*pi*i*j*k/n), backward (c2r) exp(+...);
 *   - neither direction is normalised;
 *   - r2c of an n0 x n1 x n2 row-major real array produces an
 *     n0 x n1 x (n2/2+1) complex array (last dimension halved);
 *   - c2r reads that half layout and treats it as Hermitian data: the
 *     imaginary parts of the last-dimension DC and Nyquist entries are
 *     ignored after the transforms along the first two dimensions.
 *
 * Call sites in the reference: g2init.cpp:55-63,174,182,196-200;
 * g2spectra.cpp:47-50,61,237-239; g2evolutionpert.cpp:183-195.
 *
 * Planning never touches the arrays (like FFTW_ESTIMATE).  Real FFTW with
 * FFTW_MEASURE overwrites them while planning; see the oracle header for the
 * one reference call site where that matters (g2evolutionpert.cpp:186).
 */
#ifndef GABE_FFTW_SHIM_H
#define GABE_FFTW_SHIM_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_complex[2];
typedef struct gabe_fft_plan_s *fftw_plan;

#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)

fftw_plan fftw_plan_dft_r2c_3d(int n0, int n1, int n2, double *in,
                               fftw_complex *out, unsigned flags);
fftw_plan fftw_plan_dft_c2r_3d(int n0, int n1, int n2, fftw_complex *in,
                               double *out, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_execute_dft_r2c(const fftw_plan p, double *in, fftw_complex *out);
void fftw_execute_dft_c2r(const fftw_plan p, fftw_complex *in, double *out);
void fftw_destroy_plan(fftw_plan p);
void *fftw_malloc(size_t n);
void fftw_free(void *p);
void fftw_plan_with_nthreads(int nthreads);
int fftw_init_threads(void);
void fftw_cleanup_threads(void);

/* Non-FFTW helpers used by the oracle's tests. */
int gabe_fft_get_nthreads(void);
/* 1-D complex DFT of length n on interleaved (re,im) data, in place.
 * sign = -1 forward, +1 backward, unnormalised. */
void gabe_fft_c2c_1d(int n, double *data, int sign);

#ifdef __cplusplus
}
#endif

#endif
