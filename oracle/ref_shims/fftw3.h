/*
 * TEST INFRASTRUCTURE (oracle build only) -- never linked into the product.
 *
 * The subset of the FFTW3 API that the reference calls (fft_fftw3.cpp:13-46,
 * FormFactorAtomic / KerkerRhoMix through fft_fftw3).  FFTW3 itself is not
 * installed in this image; fft_shim.c implements these entry points with its
 * own mixed-radix FP64 FFT and FFTW's sign and ordering conventions:
 *   plan_dft_3d(n0,n1,n2): row-major, n2 fastest;
 *   FFTW_FORWARD = -1 (exponent -i), FFTW_BACKWARD = +1 (exponent +i);
 *   no normalisation in either direction.
 */
#ifndef PSPW_ORACLE_FFTW3_SHIM_H
#define PSPW_ORACLE_FFTW3_SHIM_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_complex[2];
typedef struct pspw_fftw_plan_s *fftw_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)

fftw_plan fftw_plan_dft_3d(int n0, int n1, int n2, fftw_complex *in, fftw_complex *out,
                           int sign, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);
void *fftw_malloc(size_t n);
void fftw_free(void *p);

#ifdef __cplusplus
}
#endif

#endif
