/*
 * fftw3_shim.c -- forwards the FFTW3 calls used by the reference
 * (libEZmock/EZmock/fftw_def.h:32-64) to the oracle CPU FFT.
 * Test infrastructure only.
 */
#include "fftw3.h"
#include "../cpufft.h"
#include <stdlib.h>

struct ezshim_plan_s {
  int n0, n1, n2;
};

static int shim_nthreads = 0;

static struct ezshim_plan_s *mkplan(int n0, int n1, int n2) {
  struct ezshim_plan_s *p = malloc(sizeof(*p));
  if (p) { p->n0 = n0; p->n1 = n1; p->n2 = n2; }
  return p;
}

void *fftw_malloc(size_t n) {
  void *p = NULL;
  if (posix_memalign(&p, 64, n ? n : 1)) return NULL;
  return p;
}
void fftw_free(void *p) { free(p); }
int fftw_init_threads(void) { return 1; }
void fftw_plan_with_nthreads(int n) { shim_nthreads = n; }
fftw_plan fftw_plan_dft_r2c_3d(int n0, int n1, int n2, double *in,
    fftw_complex *out, unsigned flags) {
  (void) in; (void) out; (void) flags;
  return mkplan(n0, n1, n2);
}
fftw_plan fftw_plan_dft_c2r_3d(int n0, int n1, int n2, fftw_complex *in,
    double *out, unsigned flags) {
  (void) in; (void) out; (void) flags;
  return mkplan(n0, n1, n2);
}
void fftw_execute_dft_r2c(const fftw_plan p, double *in, fftw_complex *out) {
  cpufft_r2c3d(p->n0, p->n1, p->n2, in, (double *) out, shim_nthreads);
}
void fftw_execute_dft_c2r(const fftw_plan p, fftw_complex *in, double *out) {
  cpufft_c2r3d(p->n0, p->n1, p->n2, (const double *) in, out, shim_nthreads);
}
void fftw_destroy_plan(fftw_plan p) { free(p); }
void fftw_cleanup(void) {}
void fftw_cleanup_threads(void) {}

void *fftwf_malloc(size_t n) { return fftw_malloc(n); }
void fftwf_free(void *p) { free(p); }
int fftwf_init_threads(void) { return 1; }
void fftwf_plan_with_nthreads(int n) { shim_nthreads = n; }
fftwf_plan fftwf_plan_dft_r2c_3d(int n0, int n1, int n2, float *in,
    fftwf_complex *out, unsigned flags) {
  (void) in; (void) out; (void) flags;
  return mkplan(n0, n1, n2);
}
fftwf_plan fftwf_plan_dft_c2r_3d(int n0, int n1, int n2, fftwf_complex *in,
    float *out, unsigned flags) {
  (void) in; (void) out; (void) flags;
  return mkplan(n0, n1, n2);
}
void fftwf_execute_dft_r2c(const fftwf_plan p, float *in, fftwf_complex *out) {
  cpufft_r2c3d_f(p->n0, p->n1, p->n2, in, (float *) out, shim_nthreads);
}
void fftwf_execute_dft_c2r(const fftwf_plan p, fftwf_complex *in, float *out) {
  cpufft_c2r3d_f(p->n0, p->n1, p->n2, (const float *) in, out, shim_nthreads);
}
void fftwf_destroy_plan(fftwf_plan p) { free(p); }
void fftwf_cleanup(void) {}
void fftwf_cleanup_threads(void) {}
