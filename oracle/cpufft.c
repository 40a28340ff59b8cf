/*
 * cpufft.c -- CPU FFT for the oracle (see cpufft.h).  Test infrastructure:
 * it stands in for FFTW3, which the reference links (options.mk:16-20) but
 * which is not installed in this environment.
 */
#include "cpufft.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define MAXFAC 32

struct cfft_plan {
  int n, sign, nfac;
  int fac[MAXFAC];
  double *tw;                /* tw[2e], tw[2e+1] = cos, sin(sign*2*pi*e/n) */
};

cfft_plan *cfft_plan_new(int n, int sign) {
  cfft_plan *p = calloc(1, sizeof(cfft_plan));
  if (!p) return NULL;
  p->n = n;
  p->sign = sign;
  p->tw = malloc(sizeof(double) * 2 * (size_t) (n > 0 ? n : 1));
  if (!p->tw) { free(p); return NULL; }
  const long double tpi = 6.283185307179586476925286766559005768L;
  for (int e = 0; e < n; e++) {
    long double a = tpi * (long double) e / (long double) n;
    p->tw[2 * e] = (double) cosl(a);
    p->tw[2 * e + 1] = (double) (sign * sinl(a));
  }
  int m = n;
  while (m > 1 && p->nfac < MAXFAC) {
    int r;
    if (m % 4 == 0) r = 4;
    else if (m % 2 == 0) r = 2;
    else {
      r = 3;
      while (m % r) r += 2;
    }
    p->fac[p->nfac++] = r;
    m /= r;
  }
  return p;
}

void cfft_plan_free(cfft_plan *p) {
  if (!p) return;
  free(p->tw);
  free(p);
}

/* One Stockham pass: radix r, p = product of previous radices. */
static void stockham_pass(const cfft_plan *pl, int r, int p, const double *x,
    double *y) {
  const int n = pl->n;
  const int T = n / r;
  const double *tw = pl->tw;
  double ur[MAXFAC * 4], ui[MAXFAC * 4];
  double *ure = (r <= MAXFAC * 4) ? ur : malloc(sizeof(double) * r);
  double *uim = (r <= MAXFAC * 4) ? ui : malloc(sizeof(double) * r);
  const int stride_tw = n / (p * r);          /* e = q*k*stride_tw */
  for (int i = 0; i < T; i++) {
    const int k = i % p;
    for (int q = 0; q < r; q++) {
      double a = x[2 * (i + q * T)], b = x[2 * (i + q * T) + 1];
      const long e = ((long) q * k * stride_tw) % n;
      if (e) {
        const double c = tw[2 * e], s = tw[2 * e + 1];
        const double t = a * c - b * s;
        b = a * s + b * c;
        a = t;
      }
      ure[q] = a; uim[q] = b;
    }
    const int j = (i - k) * r + k;
    if (r == 2) {
      y[2 * j] = ure[0] + ure[1];
      y[2 * j + 1] = uim[0] + uim[1];
      y[2 * (j + p)] = ure[0] - ure[1];
      y[2 * (j + p) + 1] = uim[0] - uim[1];
    }
    else if (r == 4) {
      const double s = (double) pl->sign;
      const double a0r = ure[0] + ure[2], a0i = uim[0] + uim[2];
      const double a1r = ure[0] - ure[2], a1i = uim[0] - uim[2];
      const double a2r = ure[1] + ure[3], a2i = uim[1] + uim[3];
      const double a3r = ure[1] - ure[3], a3i = uim[1] - uim[3];
      /* v1 = a1 + s*i*a3 ; v3 = a1 - s*i*a3 */
      y[2 * j] = a0r + a2r;
      y[2 * j + 1] = a0i + a2i;
      y[2 * (j + p)] = a1r - s * a3i;
      y[2 * (j + p) + 1] = a1i + s * a3r;
      y[2 * (j + 2 * p)] = a0r - a2r;
      y[2 * (j + 2 * p) + 1] = a0i - a2i;
      y[2 * (j + 3 * p)] = a1r + s * a3i;
      y[2 * (j + 3 * p) + 1] = a1i - s * a3r;
    }
    else {
      const int nr = n / r;
      for (int sidx = 0; sidx < r; sidx++) {
        double vr = 0, vi = 0;
        for (int q = 0; q < r; q++) {
          const long e = ((long) q * sidx % r) * nr;
          const double c = tw[2 * e], s = tw[2 * e + 1];
          vr += ure[q] * c - uim[q] * s;
          vi += ure[q] * s + uim[q] * c;
        }
        y[2 * (j + sidx * p)] = vr;
        y[2 * (j + sidx * p) + 1] = vi;
      }
    }
  }
  if (ure != ur) free(ure);
  if (uim != ui) free(uim);
}

void cfft_exec(const cfft_plan *pl, double *data, double *work) {
  double *x = data, *y = work;
  int p = 1;
  for (int f = 0; f < pl->nfac; f++) {
    stockham_pass(pl, pl->fac[f], p, x, y);
    p *= pl->fac[f];
    double *t = x; x = y; y = t;
  }
  if (x != data) memcpy(data, x, sizeof(double) * 2 * (size_t) pl->n);
}

/*============================================================================*\
                          3D transforms (FFTW layout)
\*============================================================================*/

#define KBLK 8

static int nthr(int nthread) {
#ifdef _OPENMP
  return nthread > 0 ? nthread : omp_get_max_threads();
#else
  (void) nthread; return 1;
#endif
}

/* Complex transforms along axis 0 and axis 1 of an n0 x n1 x nk array. */
static void c2c_axes01(int n0, int n1, int nk, double *a, int sign,
    int nthread) {
  cfft_plan *p0 = cfft_plan_new(n0, sign);
  cfft_plan *p1 = cfft_plan_new(n1, sign);
  const int nb = (nk + KBLK - 1) / KBLK;
  const int nmax = n0 > n1 ? n0 : n1;
#pragma omp parallel num_threads(nthr(nthread))
  {
    double *line = malloc(sizeof(double) * 2 * (size_t) nmax * KBLK);
    double *buf = malloc(sizeof(double) * 2 * (size_t) nmax);
    double *work = malloc(sizeof(double) * 2 * (size_t) nmax);
    /* axis 0: lines over i for fixed (j, k) */
#pragma omp for schedule(static)
    for (long t = 0; t < (long) n1 * nb; t++) {
      const int j = (int) (t / nb), k0 = (int) (t % nb) * KBLK;
      const int kc = (k0 + KBLK <= nk) ? KBLK : nk - k0;
      for (int i = 0; i < n0; i++) {
        const double *src = a + 2 * (((size_t) i * n1 + j) * nk + k0);
        for (int c = 0; c < kc; c++) {
          line[2 * ((size_t) c * n0 + i)] = src[2 * c];
          line[2 * ((size_t) c * n0 + i) + 1] = src[2 * c + 1];
        }
      }
      for (int c = 0; c < kc; c++) {
        memcpy(buf, line + 2 * (size_t) c * n0, sizeof(double) * 2 * n0);
        cfft_exec(p0, buf, work);
        memcpy(line + 2 * (size_t) c * n0, buf, sizeof(double) * 2 * n0);
      }
      for (int i = 0; i < n0; i++) {
        double *dst = a + 2 * (((size_t) i * n1 + j) * nk + k0);
        for (int c = 0; c < kc; c++) {
          dst[2 * c] = line[2 * ((size_t) c * n0 + i)];
          dst[2 * c + 1] = line[2 * ((size_t) c * n0 + i) + 1];
        }
      }
    }
    /* axis 1: lines over j for fixed (i, k) */
#pragma omp for schedule(static)
    for (long t = 0; t < (long) n0 * nb; t++) {
      const int i = (int) (t / nb), k0 = (int) (t % nb) * KBLK;
      const int kc = (k0 + KBLK <= nk) ? KBLK : nk - k0;
      for (int j = 0; j < n1; j++) {
        const double *src = a + 2 * (((size_t) i * n1 + j) * nk + k0);
        for (int c = 0; c < kc; c++) {
          line[2 * ((size_t) c * n1 + j)] = src[2 * c];
          line[2 * ((size_t) c * n1 + j) + 1] = src[2 * c + 1];
        }
      }
      for (int c = 0; c < kc; c++) {
        memcpy(buf, line + 2 * (size_t) c * n1, sizeof(double) * 2 * n1);
        cfft_exec(p1, buf, work);
        memcpy(line + 2 * (size_t) c * n1, buf, sizeof(double) * 2 * n1);
      }
      for (int j = 0; j < n1; j++) {
        double *dst = a + 2 * (((size_t) i * n1 + j) * nk + k0);
        for (int c = 0; c < kc; c++) {
          dst[2 * c] = line[2 * ((size_t) c * n1 + j)];
          dst[2 * c + 1] = line[2 * ((size_t) c * n1 + j) + 1];
        }
      }
    }
    free(line); free(buf); free(work);
  }
  cfft_plan_free(p0);
  cfft_plan_free(p1);
}

/* 1D complex-to-real along the last axis; X holds nk complex values (the
   imaginary parts of X[0] and, for even n, X[n/2] are ignored). */
static void c2r_row(const cfft_plan *ph, const double *tw_n, int n,
    const double *X, double *out, double *z, double *work) {
  const int nk = n / 2 + 1;
  if ((n & 1) == 0) {
    const int nh = n / 2;
    for (int k = 0; k < nh; k++) {
      double xr = X[2 * k], xi = (k == 0) ? 0 : X[2 * k + 1];
      const int kc = nh - k;
      double yr = X[2 * kc], yi = (kc == nh) ? 0 : -X[2 * kc + 1];
      const double er = xr + yr, ei = xi + yi;
      double orr = xr - yr, oi = xi - yi;
      const double c = tw_n[2 * k], s = tw_n[2 * k + 1];   /* e^{+i 2pi k/n} */
      const double t = orr * c - oi * s;
      oi = orr * s + oi * c;
      orr = t;
      z[2 * k] = er - oi;                  /* E + i*O */
      z[2 * k + 1] = ei + orr;
    }
    cfft_exec(ph, z, work);
    for (int m = 0; m < nh; m++) {
      out[2 * m] = z[2 * m];
      out[2 * m + 1] = z[2 * m + 1];
    }
  }
  else {
    /* Hermitian extension, full complex inverse transform. */
    for (int k = 0; k < nk; k++) {
      z[2 * k] = X[2 * k];
      z[2 * k + 1] = (k == 0) ? 0 : X[2 * k + 1];
    }
    for (int k = 1; k < nk; k++) {
      z[2 * (n - k)] = X[2 * k];
      z[2 * (n - k) + 1] = -X[2 * k + 1];
    }
    cfft_exec(ph, z, work);
    for (int m = 0; m < n; m++) out[m] = z[2 * m];
  }
}

static void c2r3d_core(int n0, int n1, int n2, double *a, double *out,
    int nthread) {
  const int nk = n2 / 2 + 1;
  c2c_axes01(n0, n1, nk, a, +1, nthread);
  const int even = (n2 & 1) == 0;
  cfft_plan *ph = cfft_plan_new(even ? n2 / 2 : n2, +1);
  cfft_plan *pn = cfft_plan_new(n2, +1);
#pragma omp parallel num_threads(nthr(nthread))
  {
    double *z = malloc(sizeof(double) * 2 * (size_t) n2);
    double *work = malloc(sizeof(double) * 2 * (size_t) n2);
#pragma omp for schedule(static)
    for (long r = 0; r < (long) n0 * n1; r++)
      c2r_row(ph, pn->tw, n2, a + 2 * (size_t) r * nk, out + (size_t) r * n2,
          z, work);
    free(z); free(work);
  }
  cfft_plan_free(ph);
  cfft_plan_free(pn);
}

void cpufft_c2r3d(int n0, int n1, int n2, const double *in, double *out,
    int nthread) {
  const size_t nc = (size_t) n0 * n1 * (n2 / 2 + 1);
  double *a = malloc(sizeof(double) * 2 * nc);
  memcpy(a, in, sizeof(double) * 2 * nc);
  c2r3d_core(n0, n1, n2, a, out, nthread);
  free(a);
}

void cpufft_c2r3d_f(int n0, int n1, int n2, const float *in, float *out,
    int nthread) {
  const size_t nc = (size_t) n0 * n1 * (n2 / 2 + 1);
  const size_t nr = (size_t) n0 * n1 * n2;
  double *a = malloc(sizeof(double) * 2 * nc);
  double *o = malloc(sizeof(double) * nr);
#pragma omp parallel for num_threads(nthr(nthread))
  for (size_t i = 0; i < 2 * nc; i++) a[i] = in[i];
  c2r3d_core(n0, n1, n2, a, o, nthread);
#pragma omp parallel for num_threads(nthr(nthread))
  for (size_t i = 0; i < nr; i++) out[i] = (float) o[i];
  free(a); free(o);
}

static void r2c_row(const cfft_plan *ph, const double *tw_n, int n,
    const double *x, double *X, double *z, double *work) {
  const int nk = n / 2 + 1;
  if ((n & 1) == 0) {
    const int nh = n / 2;
    for (int m = 0; m < nh; m++) {
      z[2 * m] = x[2 * m];
      z[2 * m + 1] = x[2 * m + 1];
    }
    cfft_exec(ph, z, work);
    for (int k = 0; k <= nh; k++) {
      const int k1 = k % nh, k2 = (nh - k) % nh;
      const double zr = z[2 * k1], zi = z[2 * k1 + 1];
      const double cr = z[2 * k2], ci = -z[2 * k2 + 1];     /* conj(Z[nh-k]) */
      const double er = 0.5 * (zr + cr), ei = 0.5 * (zi + ci);
      /* O = (Z - conj)/(2i) */
      const double dr = 0.5 * (zr - cr), di = 0.5 * (zi - ci);
      const double orr = di, oi = -dr;
      const double c = tw_n[2 * k], s = tw_n[2 * k + 1];
      /* e^{-i 2 pi k/n} (tw_n has sign -1) */
      X[2 * k] = er + orr * c - oi * s;
      X[2 * k + 1] = ei + orr * s + oi * c;
    }
  }
  else {
    for (int m = 0; m < n; m++) { z[2 * m] = x[m]; z[2 * m + 1] = 0; }
    cfft_exec(ph, z, work);
    for (int k = 0; k < nk; k++) { X[2 * k] = z[2 * k]; X[2 * k + 1] = z[2 * k + 1]; }
  }
}

static void r2c3d_core(int n0, int n1, int n2, const double *x, double *a,
    int nthread) {
  const int nk = n2 / 2 + 1;
  const int even = (n2 & 1) == 0;
  cfft_plan *ph = cfft_plan_new(even ? n2 / 2 : n2, -1);
  cfft_plan *pn = cfft_plan_new(n2, -1);
#pragma omp parallel num_threads(nthr(nthread))
  {
    double *z = malloc(sizeof(double) * 2 * (size_t) n2);
    double *work = malloc(sizeof(double) * 2 * (size_t) n2);
#pragma omp for schedule(static)
    for (long r = 0; r < (long) n0 * n1; r++)
      r2c_row(ph, pn->tw, n2, x + (size_t) r * n2, a + 2 * (size_t) r * nk,
          z, work);
    free(z); free(work);
  }
  cfft_plan_free(ph);
  cfft_plan_free(pn);
  c2c_axes01(n0, n1, nk, a, -1, nthread);
}

void cpufft_r2c3d(int n0, int n1, int n2, const double *in, double *out,
    int nthread) {
  r2c3d_core(n0, n1, n2, in, out, nthread);
}

void cpufft_r2c3d_f(int n0, int n1, int n2, const float *in, float *out,
    int nthread) {
  const size_t nc = (size_t) n0 * n1 * (n2 / 2 + 1);
  const size_t nr = (size_t) n0 * n1 * n2;
  double *x = malloc(sizeof(double) * nr);
  double *a = malloc(sizeof(double) * 2 * nc);
#pragma omp parallel for num_threads(nthr(nthread))
  for (size_t i = 0; i < nr; i++) x[i] = in[i];
  r2c3d_core(n0, n1, n2, x, a, nthread);
#pragma omp parallel for num_threads(nthr(nthread))
  for (size_t i = 0; i < 2 * nc; i++) out[i] = (float) a[i];
  free(x); free(a);
}
