/*
 * Prototype-only stand-in for the FFTW3 header, used solely to compile the
 * reference library as a CPU oracle.  The wave-propagation path never calls
 * FFTW (only the Hilbert transform, the f-x transform and the filter phase
 * do); every function here is defined in fftw_stub.c to abort, so an
 * accidental call fails loudly instead of returning garbage.
 *
 * Test infrastructure only: nothing under fwi3d_b200/ includes this file.
 */
#pragma once
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_complex[2];
typedef float fftwf_complex[2];
typedef struct fftw_plan_s *fftw_plan;
typedef struct fftwf_plan_s *fftwf_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_ESTIMATE (1U << 6)

void *fftw_malloc(size_t n);
void fftw_free(void *p);
void fftw_cleanup(void);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);
fftw_plan fftw_plan_dft_1d(int n, fftw_complex *in, fftw_complex *out, int sign, unsigned flags);
fftw_plan fftw_plan_dft_r2c_1d(int n, double *in, fftw_complex *out, unsigned flags);
fftw_plan fftw_plan_dft_c2r_1d(int n, fftw_complex *in, double *out, unsigned flags);

void *fftwf_malloc(size_t n);
void fftwf_free(void *p);
void fftwf_cleanup(void);
void fftwf_execute(const fftwf_plan p);
void fftwf_destroy_plan(fftwf_plan p);
fftwf_plan fftwf_plan_dft_1d(int n, fftwf_complex *in, fftwf_complex *out, int sign, unsigned flags);
fftwf_plan fftwf_plan_dft_r2c_1d(int n, float *in, fftwf_complex *out, unsigned flags);
fftwf_plan fftwf_plan_dft_c2r_1d(int n, fftwf_complex *in, float *out, unsigned flags);

#ifdef __cplusplus
}
#endif
