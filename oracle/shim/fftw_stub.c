/* Abort-bodies for the FFTW prototypes in fftw3.h (oracle build only). */
#include <stdio.h>
#include <stdlib.h>
#include "fftw3.h"

static void fftw_unavailable(const char *name)
{
    fprintf(stderr, "oracle: %s called, but FFTW is not part of the propagation path\n", name);
    abort();
}

void *fftw_malloc(size_t n) { (void)n; fftw_unavailable("fftw_malloc"); return NULL; }
void fftw_free(void *p) { (void)p; fftw_unavailable("fftw_free"); }
void fftw_cleanup(void) { fftw_unavailable("fftw_cleanup"); }
void fftw_execute(const fftw_plan p) { (void)p; fftw_unavailable("fftw_execute"); }
void fftw_destroy_plan(fftw_plan p) { (void)p; fftw_unavailable("fftw_destroy_plan"); }
fftw_plan fftw_plan_dft_1d(int n, fftw_complex *i, fftw_complex *o, int s, unsigned f)
{ (void)n; (void)i; (void)o; (void)s; (void)f; fftw_unavailable("fftw_plan_dft_1d"); return NULL; }
fftw_plan fftw_plan_dft_r2c_1d(int n, double *i, fftw_complex *o, unsigned f)
{ (void)n; (void)i; (void)o; (void)f; fftw_unavailable("fftw_plan_dft_r2c_1d"); return NULL; }
fftw_plan fftw_plan_dft_c2r_1d(int n, fftw_complex *i, double *o, unsigned f)
{ (void)n; (void)i; (void)o; (void)f; fftw_unavailable("fftw_plan_dft_c2r_1d"); return NULL; }

void *fftwf_malloc(size_t n) { (void)n; fftw_unavailable("fftwf_malloc"); return NULL; }
void fftwf_free(void *p) { (void)p; fftw_unavailable("fftwf_free"); }
void fftwf_cleanup(void) { fftw_unavailable("fftwf_cleanup"); }
void fftwf_execute(const fftwf_plan p) { (void)p; fftw_unavailable("fftwf_execute"); }
void fftwf_destroy_plan(fftwf_plan p) { (void)p; fftw_unavailable("fftwf_destroy_plan"); }
fftwf_plan fftwf_plan_dft_1d(int n, fftwf_complex *i, fftwf_complex *o, int s, unsigned f)
{ (void)n; (void)i; (void)o; (void)s; (void)f; fftw_unavailable("fftwf_plan_dft_1d"); return NULL; }
fftwf_plan fftwf_plan_dft_r2c_1d(int n, float *i, fftwf_complex *o, unsigned f)
{ (void)n; (void)i; (void)o; (void)f; fftw_unavailable("fftwf_plan_dft_r2c_1d"); return NULL; }
fftwf_plan fftwf_plan_dft_c2r_1d(int n, fftwf_complex *i, float *o, unsigned f)
{ (void)n; (void)i; (void)o; (void)f; fftw_unavailable("fftwf_plan_dft_c2r_1d"); return NULL; }
