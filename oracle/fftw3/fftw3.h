/*
 * fftw3.h -- minimal FFTW3-API shim for building the reference's unmodified
 * libEZmock sources in this environment (test infrastructure: oracle only).
 *
 * It declares exactly the entry points behind the reference's FFT macros
 * (libEZmock/EZmock/fftw_def.h:32-64) and forwards them to the oracle's own
 * CPU FFT (oracle/cpufft.c).  FFTW3 itself is not installed here; every CPU
 * number measured with this shim says so.
 */
#ifndef EZ_ORACLE_FFTW3_SHIM_H
#define EZ_ORACLE_FFTW3_SHIM_H

#include <stddef.h>

#define FFTW_ESTIMATE (1U << 6)
#define FFTW_MEASURE 0U

typedef double fftw_complex[2];
typedef float fftwf_complex[2];
typedef struct ezshim_plan_s *fftw_plan;
typedef struct ezshim_plan_s *fftwf_plan;

void *fftw_malloc(size_t n);
void fftw_free(void *p);
int fftw_init_threads(void);
void fftw_plan_with_nthreads(int nthreads);
fftw_plan fftw_plan_dft_r2c_3d(int n0, int n1, int n2, double *in,
    fftw_complex *out, unsigned flags);
fftw_plan fftw_plan_dft_c2r_3d(int n0, int n1, int n2, fftw_complex *in,
    double *out, unsigned flags);
void fftw_execute_dft_r2c(const fftw_plan p, double *in, fftw_complex *out);
void fftw_execute_dft_c2r(const fftw_plan p, fftw_complex *in, double *out);
void fftw_destroy_plan(fftw_plan p);
void fftw_cleanup(void);
void fftw_cleanup_threads(void);

void *fftwf_malloc(size_t n);
void fftwf_free(void *p);
int fftwf_init_threads(void);
void fftwf_plan_with_nthreads(int nthreads);
fftwf_plan fftwf_plan_dft_r2c_3d(int n0, int n1, int n2, float *in,
    fftwf_complex *out, unsigned flags);
fftwf_plan fftwf_plan_dft_c2r_3d(int n0, int n1, int n2, fftwf_complex *in,
    float *out, unsigned flags);
void fftwf_execute_dft_r2c(const fftwf_plan p, float *in, fftwf_complex *out);
void fftwf_execute_dft_c2r(const fftwf_plan p, fftwf_complex *in, float *out);
void fftwf_destroy_plan(fftwf_plan p);
void fftwf_cleanup(void);
void fftwf_cleanup_threads(void);

#endif
