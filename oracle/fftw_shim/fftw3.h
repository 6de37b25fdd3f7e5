/* A stand-in for the small part of FFTW's single-precision API that the
 * reference's cross-correlator (src/CrossCorr.cpp) calls, so that the
 * reference source compiles and runs unmodified where FFTW is not
 * installed. TEST INFRASTRUCTURE ONLY: it backs the oracle build in
 * oracle/_ref and is never linked into the product library.
 *
 * The declarations follow FFTW 3's documented interface (the names, the
 * argument order and the r2c output convention: bins 0 .. n/2 of the
 * unnormalised forward transform, X[k] = sum_j x[j] e^{-2 pi i j k / n});
 * the implementation in fftw_shim.cpp is this project's own FP64 transform
 * rounded to float. Only what CrossCorr.cpp uses is provided. */
#ifndef CCFJ_FFTW_SHIM_H
#define CCFJ_FFTW_SHIM_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef float fftwf_complex[2];
typedef struct ccfj_fftwf_plan_s *fftwf_plan;

#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)

float *fftwf_alloc_real(size_t n);
fftwf_complex *fftwf_alloc_complex(size_t n);
void fftwf_free(void *p);
fftwf_plan fftwf_plan_dft_r2c_1d(int n, float *in, fftwf_complex *out, unsigned flags);
void fftwf_execute(const fftwf_plan p);
void fftwf_destroy_plan(fftwf_plan p);

#ifdef __cplusplus
}
#endif

#endif /* CCFJ_FFTW_SHIM_H */
