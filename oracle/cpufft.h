/*
 * cpufft.h -- CPU FFT for the oracle (test infrastructure only).
 *
 * Mixed-radix Stockham FFT in FP64 with twiddles rounded from long double,
 * plus the 3D real transforms with FFTW's conventions (unnormalised; c2r uses
 * sign +1 and r2c sign -1).  The 3D c2r follows FFTW's multi-dimensional
 * real-data algorithm: complex transforms over the leading two axes, then a
 * 1D complex-to-real transform along the last axis, which ignores the
 * imaginary parts of the k=0 and k=n/2 entries.  The reference relies on
 * that behaviour for its non-Hermitian kz=0 / Nyquist planes
 * (libEZmock/EZmock/perturb.c:166-211, fftw_def.h:38-42).
 */
#ifndef EZ_ORACLE_CPUFFT_H
#define EZ_ORACLE_CPUFFT_H

#include <stddef.h>

typedef struct cfft_plan cfft_plan;

cfft_plan *cfft_plan_new(int n, int sign);
void cfft_plan_free(cfft_plan *p);
/* In-place transform of n interleaved (re,im) doubles; `work` holds 2n. */
void cfft_exec(const cfft_plan *p, double *data, double *work);

/* 3D transforms on n0 x n1 x n2 real arrays (C order) and
   n0 x n1 x (n2/2+1) complex arrays.  `nthread` <= 0 uses all threads. */
void cpufft_c2r3d(int n0, int n1, int n2, const double *in, double *out,
    int nthread);
void cpufft_c2r3d_f(int n0, int n1, int n2, const float *in, float *out,
    int nthread);
void cpufft_r2c3d(int n0, int n1, int n2, const double *in, double *out,
    int nthread);
void cpufft_r2c3d_f(int n0, int n1, int n2, const float *in, float *out,
    int nthread);

#endif
