/*
 * ezoracle.c -- CPU restatement of the EZmock hot path (TEST INFRASTRUCTURE;
 * see ezoracle.h).  Serial semantics, written from the reference's behaviour;
 * every function names the reference lines it restates.  Expression order
 * and `real` rounding points follow the reference so that, on the same
 * random streams and FFT, results agree bit for bit with the reference
 * compiled single-threaded.
 */
#include "ezoracle.h"
#include "prand/prand.h"
#include "cpufft.h"
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 0x1.921fb54442d18p+1
#endif

#ifdef SINGLE_PREC
#define REAL_MIN_V FLT_MIN
#define REAL_TOL_V 1e-5
#else
#define REAL_MIN_V DBL_MIN
#define REAL_TOL_V 1e-10
#endif

/* Error codes in the numbering of the default (OpenMP) reference build,
   libEZmock/EZmock/errmsg.h:33-88. */
enum {
  E_OK = 0, E_MEMORY = 1, E_ARG_COSMO = 4, E_ARG_NBIN = 13,
  E_ARG_LOWEXP = 15, E_ARG_HIEXP = 16, E_COS_GROWTH = 20, E_PK_FINITE = 21,
  E_PK_NONPOS = 22, E_PK_NONASC = 23, E_PK_RANGE = 24, E_PK_NBIN = 25,
  E_PK_MODBAO = 26, E_RNG_JUMP = 29, E_PAR_COSMO = 30, E_PAR_RCUT = 31,
  E_PAR_REXP = 32, E_PAR_PBASE = 33, E_PAR_SIGV = 34, E_RHO_LESS = 36,
  E_RHO_PBASE = 37, E_RHO_NPART = 38, E_UNKNOWN = 41
};

#define NLOGB 64          /* config.h:64 */
#define RHO_SAT 100       /* config.h:71 */
#define GAUSS_WIDTH 10    /* config.h:73 */
#define MAX_NT_PER_CELL 1024

int ezo_real_size(void) { return (int) sizeof(real); }

/*============================================================================*\
             Gauss hypergeometric function (math/hypergeom.c:42-194)
\*============================================================================*/

/* Taylor series (hypergeom.c:42-79). */
static int h2f1_series(double a, double b, double c, double z, double tol,
    int maxiter, double *res) {
  if (fabs(a) >= 50 || fabs(b) >= 50 || fabs(c) <= 1 || fabs(z) >= 0.9)
    return 1;
  int hits = 0;
  double term = 1, sum = 1;
  for (int i = 0; i < maxiter; i++) {
    const double j = (double) i;
    term *= (a + j) * (b + j) * z / ((c + j) * (j + 1));
    if (fabs(term) < fabs(sum) * tol) {
      if (++hits >= 3) { *res = sum; return 0; }
    }
    else hits = 0;
    sum += term;
  }
  return 1;
}

/* Single-fraction recurrence (hypergeom.c:98-135). */
static int h2f1_fraction(double a, double b, double c, double z, double tol,
    int maxiter, double *res) {
  if (fabs(a) >= 50 || fabs(b) >= 50 || fabs(c) >= 20 || fabs(z) >= 0.9)
    return 1;
  int hits = 0;
  double al = 0, be = 1, ga = 1, ze = 1;
  for (int i = 0; i < maxiter; i++) {
    const double j = (double) i;
    const double prev = ze;
    const double f = (j + 1) * (c + j);
    al = (al + be) * f;
    be *= (a + j) * (b + j) * z;
    ga *= f;
    ze = (al + be) / ga;
    if (fabs(ze - prev) < fabs(prev) * tol) {
      if (++hits >= 3) { *res = ze; return 0; }
    }
    else hits = 0;
  }
  return 1;
}

/* Transformations for z < 0 (hypergeom.c:151-194). */
static int h2f1(double a, double b, double c, double z, double tol,
    int maxiter, double *res) {
  if (fabs(a) >= 50 || fabs(b) >= 50) return 1;
  if (z < -1) {
    const double w = 1 / (1 - z);
    double f1, f2;
    if (h2f1(a, c - b, a - b + 1, w, tol, maxiter, &f1) ||
        h2f1(b, c - a, b - a + 1, w, tol, maxiter, &f2)) return 1;
    const double gc = lgamma(c);
    const double g1 = gc + lgamma(b - a) - lgamma(b) - lgamma(c - a);
    const double g2 = gc + lgamma(a - b) - lgamma(a) - lgamma(c - b);
    *res = -pow(w, a) * exp(g1) * f1 + pow(w, b) * exp(g2) * f2;
    return 0;
  }
  if (z < 0) {
    const double w = z / (z - 1);
    double f;
    if (h2f1(a, c - b, c, w, tol, maxiter, &f)) return 1;
    *res = pow(1 - z, -a) * f;
    return 0;
  }
  if (z > 0.5) return 1;
  if (fabs(c) > 1) return h2f1_series(a, b, c, z, tol, maxiter, res);
  return h2f1_fraction(a, b, c, z, tol, maxiter, res);
}

/* Growth factor and rate in flat wCDM (cosmology.c:53-95, 121-158). */
int ezo_growth(double z, double z_pk, double Om, double Onu, double w,
    double *growth2, double *vfac) {
  if (z < 0 || z_pk < 0 || Om <= 0 || Om > 1 || Onu < 0 || Onu >= 1 ||
      w >= -1.0 / 3.0) return E_PAR_COSMO;
  const double a = 1 / (1 + z), a0 = 1 / (1 + z_pk);
  const double tol = 1e-12;
  const int maxit = 10000;
  const double iw = 1 / w;
  const double p1 = 0.5 * (1 - iw);
  const double p2 = -0x1.5555555555555p-2 * iw;
  const double p3 = 1 - 0x1.aaaaaaaaaaaabp-1 * iw;
  const double za = (1 - 1 / Om) * pow(a, -3 * w);
  double h1, h2, D, f;
  if (h2f1(p1, p2, p3, za, tol, maxit, &h1) ||
      h2f1(p1 + 1, p2 + 1, p3 + 1, za, tol, maxit, &h2)) return E_COS_GROWTH;
  f = 1 + 3 * (w - 1) * za / (6 * w - 5) * h2 / h1;
  if (a == a0) D = 1;
  else {
    const double z0 = (1 - 1 / Om) * pow(a0, -3 * w);
    if (h2f1(p1, p2, p3, z0, tol, maxit, &h2)) return E_COS_GROWTH;
    D = (a * h1) / (a0 * h2);
  }
  const double Omn = Om + Onu;
  const double H = 100 * sqrt((1 - Omn) * pow(a, -3 * (1 + w)) +
      Omn * pow(a, -3));
  *growth2 = D * D;
  *vfac = f * H * a;
  return E_OK;
}

/*============================================================================*\
                 Linear power spectrum (linear_pk.c, cspline.c)
\*============================================================================*/

/* Natural cubic spline second derivatives (math/cspline.c:35-76). */
static void spline_second_deriv(const double *x, const double *y, int n,
    double *ypp) {
  double *cp = malloc(sizeof(double) * n);
  double nx = x[1], ny = y[1];
  double c = x[1] - x[0];
  double nd = (y[1] - y[0]) / c;
  cp[0] = cp[n - 1] = ypp[0] = ypp[n - 1] = 0;
  int j = 1;
  while (j < n - 1) {
    const double ox = nx, oy = ny, a = c, od = nd;
    nx = x[j + 1];
    ny = y[j + 1];
    c = nx - ox;
    nd = (ny - oy) / c;
    const double b = (c + a) * 2;
    const double inv = 1 / (b - a * cp[j - 1]);
    const double d = (nd - od) * 6;
    ypp[j] = (d - a * ypp[j - 1]) * inv;
    cp[j] = c * inv;
    j++;
  }
  while (j) {
    j--;
    ypp[j] -= cp[j] * ypp[j + 1];
  }
  free(cp);
}

int ezo_pk_setup(ezo_pk *pk, int Ng, double Lbox, double growth2,
    const double *k, int n, const double *P, const double *Pnw, double mBAO,
    int logint) {
  if (n <= 3) return E_ARG_NBIN;
  for (int i = 0; i < n; i++) {
    if (!isfinite(k[i]) || !isfinite(P[i])) return E_PK_FINITE;
    if (k[i] <= 0 || P[i] <= 0) return E_PK_NONPOS;
    if (i && k[i] <= k[i - 1]) return E_PK_NONASC;
  }
  if (mBAO != 0) {
    for (int i = 0; i < n; i++) {
      if (!isfinite(Pnw[i])) return E_PK_FINITE;
      if (Pnw[i] <= 0) return E_PK_NONPOS;
    }
  }
  const double kmin = 2 * M_PI / Lbox;
  const double kmax = M_PI * Ng / Lbox * sqrt(3);
  if (k[0] > kmin - 1e-8 || k[n - 1] < kmax + 1e-8) return E_PK_RANGE;
  int lo = 0, hi;
  while (lo < n && !(k[lo] > kmin)) lo++;
  hi = lo;
  while (hi < n && !(k[hi] > kmax)) hi++;
  lo = (lo < 3) ? 0 : lo - 3;
  hi = (hi + 3 >= n) ? n : hi + 3;
  const int nb = hi - lo;
  if (nb < 3) return E_PK_NBIN;
  if (nb > (int) (sizeof(pk->k) / sizeof(double))) return E_MEMORY;
  for (int i = 0; i < nb; i++) {
    const int j = i + lo;
    double v;
    if (mBAO == 0) v = P[j] * growth2;
    else {
      v = (k[j] <= 0.5) ? (P[j] - Pnw[j]) * exp(k[j] * k[j] * mBAO) + Pnw[j]
          : P[j];
      if (!isfinite(v) || v <= 0) return E_PK_MODBAO;
      v *= growth2;
    }
    pk->P[i] = v;
  }
  for (int i = 0; i < nb; i++) {
    if (logint) { pk->k[i] = log(k[i + lo]); pk->P[i] = log(pk->P[i]); }
    else pk->k[i] = k[i + lo];
  }
  pk->n = nb;
  pk->log = logint;
  pk->kmin = k[lo];
  pk->kmax = k[hi - 1];
  spline_second_deriv(pk->k, pk->P, nb, pk->P2);
  return E_OK;
}

/* Interval search (linear_pk.c:36-51). */
static int interval_of(const double *x, int n, double v) {
  int l = 0, u = n - 1;
  while (l <= u) {
    const int i = (l + u) >> 1;
    if (i >= n - 1) return (x[n - 1] == v) ? n - 1 : -1;
    if (x[i + 1] <= v) l = i + 1;
    else if (x[i] > v) u = i - 1;
    else return i;
  }
  return -1;
}

double ezo_pk_interp(const ezo_pk *pk, double kv) {
  const int i = interval_of(pk->k, pk->n, kv);
  if (i == pk->n - 1) return pk->P[i];
  if (i < 0) {
    if (kv >= pk->k[pk->n - 1]) return pk->P[pk->n - 1];
    if (kv <= pk->k[0]) return pk->P[0];
  }
  /* cspline.c:91-105 */
  const int j = i + 1;
  const double ba = pk->k[j] - pk->k[i];
  const double xa = kv - pk->k[i];
  const double bx = pk->k[j] - kv;
  const double ba2 = ba * ba;
  const double lower = xa * pk->P[j] + bx * pk->P[i];
  const double c = (xa * xa - ba2) * xa * pk->P2[j];
  const double d = (bx * bx - ba2) * bx * pk->P2[i];
  return (lower + 0x1.5555555555555p-3 * (c + d)) / ba;
}

/*============================================================================*\
                     Initial conditions (perturb.c:78-399)
\*============================================================================*/

static void rng_fill(int rng, uint64_t seed, uint64_t start, uint64_t count,
    uint32_t *out) {
  prand_fill_raw(rng, seed, start, count, out);
}

static inline double u_dbl(int rng, uint32_t x) {
  return (rng == PRAND_RNG_MT19937) ? (double) x * (1.0 / 4294967296.0)
      : (double) x * 2.328306549295727688e-10;
}
static inline double u_pos(int rng, uint32_t x) {
  return (rng == PRAND_RNG_MT19937) ? ((double) x + 0.5) * (1.0 / 4294967296.0)
      : (double) x * 2.328306549295727688e-10;
}

void ezo_rng_raw(int rng, uint64_t seed, uint64_t start, uint64_t count,
    uint32_t *out) {
  rng_fill(rng, seed, start, count, out);
}

/* Value of a sampled mode: perturb.c:146-211 (P, phase -> rhok). */
static void mode_value(const ezo_pk *pk, double ksq, double kfac,
    double logkfac, double Pfac, int fixamp, int iphase, double uamp,
    double uphase, real *re, real *im) {
  const double kmod = pk->log ? log(ksq) * 0.5 + logkfac : kfac * sqrt(ksq);
  double P = ezo_pk_interp(pk, kmod);
  double amp = 0;
  if (!fixamp) amp = -log(uamp);
  if (pk->log) P = fixamp ? exp(P * 0.5) : exp(P * 0.5) * sqrt(amp);
  else P = fixamp ? sqrt(P) : sqrt(P * amp);
  P *= Pfac;
  double phase = uphase * 2 * M_PI;
  if (iphase) phase += M_PI;
  P /= (ksq * kfac);
  *re = -P * sin(phase);
  *im = P * cos(phase);
}

int ezo_ic_spectrum(const ezo_pk *pk, int Ng, double Lbox, int rng,
    uint64_t seed, int fixamp, int iphase, real *rhok) {
  const int Ngh = Ng >> 1, Ngk = Ngh + 1;
  const size_t ncell = (size_t) Ng * Ng * Ngk;
  const int per = fixamp ? 1 : 2;
  const size_t ndraw = (ncell - 1) * per;
  uint32_t *u = malloc(sizeof(uint32_t) * (ndraw ? ndraw : 1));
  if (!u) return E_MEMORY;
  rng_fill(rng, seed, 0, ndraw, u);
  const double kfac = M_PI * 2 / Lbox;
  const double logkfac = log(kfac);
  const double Pfac = pow(Lbox, -1.5);

  for (int i = 0; i < Ng; i++) {
    const double ki = (i <= Ngh) ? i : i - Ng;
    const int ni = (i == 0) ? 0 : Ng - i;
    for (int j = 0; j < Ng; j++) {
      const double kj = (j <= Ngh) ? j : j - Ng;
      const int nj = (j == 0) ? 0 : Ng - j;
      const double kij = ki * ki + kj * kj;
      const size_t row = ((size_t) i * Ng + j) * Ngk;
      const size_t prow = ((size_t) ni * Ng + nj) * Ngk;
      const int lower = (i == ni && j <= Ngh) || (i != ni && i <= Ngh);
      for (int k = 0; k < Ngk; k++) {
        const size_t c = row + k;
        real *out = rhok + 2 * c;
        if (c == 0) { out[0] = out[1] = 0; continue; }
        const int plane = (k == 0) || ((Ng & 1) == 0 && k == Ngh);
        /* On the k=0 / Nyquist planes the upper half takes the value of its
           partner (-i,-j) with the real part negated (perturb.c:195-210). */
        const size_t src = (!plane || lower) ? c : prow + k;
        const double ua = fixamp ? 0 : u_pos(rng, u[(src - 1) * per]);
        const double up = u_dbl(rng, u[(src - 1) * per + per - 1]);
        const double ksq = kij + k * k;
        real re, im;
        mode_value(pk, ksq, kfac, logkfac, Pfac, fixamp, iphase, ua, up,
            &re, &im);
        if (plane && (!lower || (i == ni && j == nj))) re = -re;
        out[0] = re;
        out[1] = im;
      }
    }
  }
  /* Real parts zeroed at the self-conjugate corners (perturb.c:344-359). */
  if ((Ng & 1) == 0) {
    const size_t cs[7] = {
      (size_t) Ngh, (size_t) Ngh * Ngk, (size_t) Ngh * (Ngk + 1),
      (size_t) Ngh * Ng * Ngk, (size_t) Ngh * ((size_t) Ng * Ngk + 1),
      (size_t) Ngh * (Ng + 1) * Ngk, ((size_t) Ngh * Ng + Ngh) * Ngk + Ngh};
    for (int t = 0; t < 7; t++) rhok[2 * cs[t]] = 0;
  }
  free(u);
  return E_OK;
}

static void c2r(int Ng, const real *in, real *out, int nthread) {
#ifdef SINGLE_PREC
  cpufft_c2r3d_f(Ng, Ng, Ng, in, out, nthread);
#else
  cpufft_c2r3d(Ng, Ng, Ng, in, out, nthread);
#endif
}

/* perturb.c:361-398: rhok2 = rhok*k_x -> psi0; rhok*k_y -> psi1;
   rhok*k_z -> psi2, each product rounded to `real`. */
void ezo_disp_from_spectrum(int Ng, const real *rhok, real *psi0, real *psi1,
    real *psi2, int nthread) {
  const int Ngh = Ng >> 1, Ngk = Ngh + 1;
  const size_t nc = (size_t) Ng * Ng * Ngk;
  real *t = malloc(sizeof(real) * 2 * nc);
  for (int pass = 0; pass < 3; pass++) {
    for (int i = 0; i < Ng; i++) {
      const double ki = (i <= Ngh) ? i : i - Ng;
      for (int j = 0; j < Ng; j++) {
        const double kj = (j <= Ngh) ? j : j - Ng;
        const size_t row = ((size_t) i * Ng + j) * Ngk;
        for (int k = 0; k < Ngk; k++) {
          const double f = (pass == 0) ? ki : (pass == 1) ? kj : k;
          t[2 * (row + k)] = rhok[2 * (row + k)] * f;
          t[2 * (row + k) + 1] = rhok[2 * (row + k) + 1] * f;
        }
      }
    }
    c2r(Ng, t, (pass == 0) ? psi0 : (pass == 1) ? psi1 : psi2, nthread);
  }
  free(t);
}

/* perturb.c:456-604: white-noise input. */
void ezo_disp_whitenoise(const ezo_pk *pk, int Ng, double Lbox,
    const real *delta, real *psi0, real *psi1, real *psi2, int nthread) {
  const int Ngh = Ng >> 1, Ngk = Ngh + 1;
  const size_t nc = (size_t) Ng * Ng * Ngk;
  real *w = malloc(sizeof(real) * 2 * nc);
  real *rk = malloc(sizeof(real) * 2 * nc);
#ifdef SINGLE_PREC
  cpufft_r2c3d_f(Ng, Ng, Ng, delta, w, nthread);
#else
  cpufft_r2c3d(Ng, Ng, Ng, delta, w, nthread);
#endif
  const double kfac = M_PI * 2 / Lbox;
  const double logkfac = log(kfac);
  const double Pfac = pow(Lbox, -1.5);
  for (int i = 0; i < Ng; i++) {
    const double ki = (i <= Ngh) ? i : i - Ng;
    for (int j = 0; j < Ng; j++) {
      const double kj = (j <= Ngh) ? j : j - Ng;
      const double kij = ki * ki + kj * kj;
      const size_t row = ((size_t) i * Ng + j) * Ngk;
      for (int k = 0; k < Ngk; k++) {
        const size_t c = row + k;
        if (c == 0) { rk[0] = rk[1] = 0; continue; }
        const double ksq = kij + k * k;
        const double kmod = pk->log ? log(ksq) * 0.5 + logkfac
            : kfac * sqrt(ksq);
        double P = ezo_pk_interp(pk, kmod);
        P = pk->log ? exp(P * 0.5) : sqrt(P);
        P *= Pfac / (ksq * kfac);
        rk[2 * c] = -P * w[2 * c + 1];
        rk[2 * c + 1] = P * w[2 * c];
      }
    }
  }
  free(w);
  ezo_disp_from_spectrum(Ng, rk, psi0, psi1, psi2, nthread);
  free(rk);
  const size_t num = (size_t) Ng * Ng * Ng;
  const real norm = 1 / sqrt(num);
  for (size_t i = 0; i < num; i++) {
    psi0[i] *= norm; psi1[i] *= norm; psi2[i] *= norm;
  }
}

/*============================================================================*\
                     Cloud-in-cell density (dens_field.c:233-310)
\*============================================================================*/

#define IDX3(Ng, a, b, c) (((size_t) (a) * (Ng) + (b)) * (Ng) + (c))

static inline void cic_cell(int Ng, real p, real igs, int i, int *c0, int *c1,
    real *w0, real *w1) {
  const real x = p * igs + i;
  int x0 = (int) floor(x);
  *w1 = x - x0;
  *w0 = 1 - *w1;
  if (x0 < 0) x0 += Ng;
  else if (x0 >= Ng) x0 -= Ng;
  *c0 = x0;
  *c1 = (x0 == Ng - 1) ? 0 : x0 + 1;
}

void ezo_cic(int Ng, double Lbox, const real *psi0, const real *psi1,
    const real *psi2, real *rho) {
  const real igs = Ng / Lbox;
  memset(rho, 0, sizeof(real) * (size_t) Ng * Ng * Ng);
  for (int i = 0; i < Ng; i++)
    for (int j = 0; j < Ng; j++)
      for (int k = 0; k < Ng; k++) {
        const size_t id = IDX3(Ng, i, j, k);
        int x0, x1, y0, y1, z0, z1;
        real wx0, wx1, wy0, wy1, wz0, wz1;
        cic_cell(Ng, psi0[id], igs, i, &x0, &x1, &wx0, &wx1);
        cic_cell(Ng, psi1[id], igs, j, &y0, &y1, &wy0, &wy1);
        cic_cell(Ng, psi2[id], igs, k, &z0, &z1, &wz0, &wz1);
        rho[IDX3(Ng, x0, y0, z0)] += wx0 * wy0 * wz0;
        rho[IDX3(Ng, x0, y0, z1)] += wx0 * wy0 * wz1;
        rho[IDX3(Ng, x0, y1, z0)] += wx0 * wy1 * wz0;
        rho[IDX3(Ng, x0, y1, z1)] += wx0 * wy1 * wz1;
        rho[IDX3(Ng, x1, y0, z0)] += wx1 * wy0 * wz0;
        rho[IDX3(Ng, x1, y0, z1)] += wx1 * wy0 * wz1;
        rho[IDX3(Ng, x1, y1, z0)] += wx1 * wy1 * wz0;
        rho[IDX3(Ng, x1, y1, z1)] += wx1 * wy1 * wz1;
      }
}

/*============================================================================*\
                    Effective bias model (pop_tracer.c:70-583)
\*============================================================================*/

int ezo_eval_pdf(int Ng, size_t nexp, real pbase, size_t *pdf, int *nmax,
    size_t *ncell, size_t *ntot) {
  size_t n;
  double A = 0, sum = 0, power = pbase;
  for (n = 1; n <= nexp; n++) {
    sum += power * n;
    A = nexp / sum;
    power *= pbase;
    if (A * power < 0.5) break;
  }
  if (n > MAX_NT_PER_CELL) return E_RHO_PBASE;
  size_t nc = 0, nobj = 0;
  for (size_t i = 0; i < n; i++) {
    pdf[i] = round(A * pow(pbase, n - i));
    nc += pdf[i];
    nobj += pdf[i] * (n - i);
  }
  if (nc > (size_t) Ng * Ng * Ng || nobj == 0) return E_PAR_PBASE;
  *nmax = (int) n;
  *ncell = nc;
  *ntot = nobj;
  return E_OK;
}

/* log2 histogram bin of a tracer density (pop_tracer.c:264-270); a value of
   exactly zero, whose ilogb the reference leaves undefined, is put in the
   last bin. */
static inline int logb_bin(int imax, real v) {
  if (v == 0) return NLOGB - 1;
  int idx = imax - ilogb(v);
  if (idx < 0) idx = 0;
  else if (idx >= NLOGB) idx = NLOGB - 1;
  return idx;
}

int ezo_bias(int Ng, int rng, uint64_t seed, const real *rho, real rho_c,
    real rho_exp, size_t ncell, real *rhot, size_t *hist, size_t *nvalid) {
  const size_t num = (size_t) Ng * Ng * Ng;
  const real rho_sat = RHO_SAT, lambda = GAUSS_WIDTH;
  const real thres = (rho_c == 0) ? REAL_MIN_V : rho_c;
  const double iexp = -1 / rho_exp;
  const real rho_max = 1 + lambda * 5;
  const int imax = ilogb(rho_max);
  memset(hist, 0, sizeof(size_t) * NLOGB);
  size_t nv = 0;
  for (size_t i = 0; i < num; i++) nv += !(rho[i] < thres);
  uint32_t *u = malloc(sizeof(uint32_t) * (nv + 2));
  if (!u) return E_MEMORY;
  rng_fill(rng, seed, num << 1, nv + (nv & 1), u);
  size_t r = 0;              /* rank among valid cells */
  for (size_t i = 0; i < num; i++) {
    if (rho[i] < thres) { rhot[i] = 0; continue; }
    const real v = (rho[i] > rho_sat) ? rho_sat : rho[i];
    const size_t p = r >> 1;
    /* gauss_rand (pop_tracer.c:70-79) with the pair's two draws */
    const double rr = -2 * log(u_pos(rng, u[2 * p]));
    const double th = u_dbl(rng, u[2 * p + 1]) * 2 * M_PI;
    double g = (r & 1) ? lambda * sqrt(rr) * sin(th)
        : lambda * sqrt(rr) * cos(th);
    g = (g >= 0) ? 1 + g : exp(g);
    rhot[i] = (1 - exp(v * iexp)) * g;
    hist[logb_bin(imax, rhot[i])]++;
    r++;
  }
  free(u);
  *nvalid = nv;
  if (nv < ncell) return E_RHO_LESS;
  return E_OK;
}

typedef struct { real v; size_t i; } vcell;

static int cmp_desc(const void *a, const void *b) {
  const real x = ((const vcell *) a)->v, y = ((const vcell *) b)->v;
  if (x > y) return -1;
  if (x < y) return 1;
  const size_t p = ((const vcell *) a)->i, q = ((const vcell *) b)->i;
  return (p < q) ? -1 : (p > q);
}

/* n_tracer_in_cell (pop_tracer.c:359-509).  Cells are ranked by tracer
   density, highest first; PDF bin j takes the next pdf[j] cells and then
   every further cell whose density equals the smallest one it took (the tie
   extension, pop_tracer.c:436-446), which grows pdf[j], ncell and ntot.  A
   bin whose quota is zero takes no cell. */
int ezo_select(int Ng, const real *rhot, const size_t *hist, size_t *pdf,
    int nmax, size_t *ncell, size_t *ntot, int16_t *nt) {
  const size_t num = (size_t) Ng * Ng * Ng;
  const real lambda = GAUSS_WIDTH;
  const int ilogb_max = ilogb((real) (1 + lambda * 5));
  int imax;
  size_t cnt = 0;
  for (imax = 0; imax < NLOGB; imax++) {
    cnt += hist[imax];
    if (cnt >= *ncell) break;
  }
  const real thres = (imax == NLOGB - 1) ? REAL_MIN_V : pow(2, ilogb_max - imax);
  size_t M = 0;
  for (size_t i = 0; i < num; i++) M += !(rhot[i] < thres);
  vcell *c = malloc(sizeof(vcell) * (M ? M : 1));
  if (!c) return E_MEMORY;
  M = 0;
  for (size_t i = 0; i < num; i++)
    if (!(rhot[i] < thres)) { c[M].v = rhot[i]; c[M].i = i; M++; }
  qsort(c, M, sizeof(vcell), cmp_desc);

  memset(nt, 0, sizeof(int16_t) * num);
  size_t P = 0;
  for (int j = 0; j < nmax; j++) {
    if (pdf[j] == 0) continue;
    size_t E = P + pdf[j];
    if (E > M) { free(c); return E_UNKNOWN; }
    while (E < M && c[E].v == c[E - 1].v) {
      E++;
      pdf[j]++;
      (*ncell)++;
      *ntot += (size_t) (nmax - j);
    }
    for (size_t t = P; t < E; t++) nt[c[t].i] = (int16_t) (nmax - j);
    P = E;
  }
  free(c);
  return E_OK;
}

/* generate_tracers without host particles (pop_tracer.c:894-994). */
int ezo_positions(int Ng, double Lbox, int rng, uint64_t seed,
    const int16_t *nt, size_t ntot, real *x, real *y, real *z) {
  const size_t num = (size_t) Ng * Ng * Ng;
  const real gs = Lbox / Ng;
  uint32_t *u = malloc(sizeof(uint32_t) * 3 * (ntot ? ntot : 1));
  if (!u) return E_MEMORY;
  rng_fill(rng, seed, num * 5, 3 * ntot, u);
  size_t t = 0;
  for (int i = 0; i < Ng; i++)
    for (int j = 0; j < Ng; j++)
      for (int k = 0; k < Ng; k++) {
        const int16_t n = nt[IDX3(Ng, i, j, k)];
        for (int m = 0; m < n; m++) {
          if (t >= ntot) { free(u); return E_UNKNOWN; }
          double r = u_dbl(rng, u[3 * t]) - 0.5;
          real xx = (i + r) * gs;
          r = u_dbl(rng, u[3 * t + 1]) - 0.5;
          real yy = (j + r) * gs;
          r = u_dbl(rng, u[3 * t + 2]) - 0.5;
          real zz = (k + r) * gs;
          if (xx < 0) xx += Lbox;
          if (yy < 0) yy += Lbox;
          if (zz < 0) zz += Lbox;
          x[t] = xx; y[t] = yy; z[t] = zz;
          t++;
        }
      }
  free(u);
  return (t == ntot) ? E_OK : E_UNKNOWN;
}

/* disp_cic (pop_tracer.c:593-683). */
void ezo_paint(int Ng, double Lbox, const real *psi0, const real *psi1,
    const real *psi2, const real *rho, int dim, real *out) {
  const real igs = Ng / Lbox;
  const size_t num = (size_t) Ng * Ng * Ng;
  const real *pd = (dim == 0) ? psi0 : (dim == 1) ? psi1 : psi2;
  memset(out, 0, sizeof(real) * num);
  for (int i = 0; i < Ng; i++)
    for (int j = 0; j < Ng; j++)
      for (int k = 0; k < Ng; k++) {
        const size_t id = IDX3(Ng, i, j, k);
        int x0, x1, y0, y1, z0, z1;
        real wx0, wx1, wy0, wy1, wz0, wz1;
        cic_cell(Ng, psi0[id], igs, i, &x0, &x1, &wx0, &wx1);
        cic_cell(Ng, psi1[id], igs, j, &y0, &y1, &wy0, &wy1);
        cic_cell(Ng, psi2[id], igs, k, &z0, &z1, &wz0, &wz1);
        wx0 *= pd[id];
        wx1 *= pd[id];
        out[IDX3(Ng, x0, y0, z0)] += wx0 * wy0 * wz0;
        out[IDX3(Ng, x0, y0, z1)] += wx0 * wy0 * wz1;
        out[IDX3(Ng, x0, y1, z0)] += wx0 * wy1 * wz0;
        out[IDX3(Ng, x0, y1, z1)] += wx0 * wy1 * wz1;
        out[IDX3(Ng, x1, y0, z0)] += wx1 * wy0 * wz0;
        out[IDX3(Ng, x1, y0, z1)] += wx1 * wy0 * wz1;
        out[IDX3(Ng, x1, y1, z0)] += wx1 * wy1 * wz0;
        out[IDX3(Ng, x1, y1, z1)] += wx1 * wy1 * wz1;
      }
  for (size_t i = 0; i < num; i++)
    if (rho[i] > REAL_TOL_V) out[i] /= rho[i];
}

/* assign_vel (pop_tracer.c:697-753). */
void ezo_assign_vel(int Ng, double Lbox, double vfac, const real *painted,
    const real *rho, size_t n, const real *x, const real *y, const real *z,
    real *v) {
  const real igs = Ng / Lbox;
  for (size_t t = 0; t < n; t++) {
    const real xx = x[t] * igs, yy = y[t] * igs, zz = z[t] * igs;
    int x0 = (int) xx, y0 = (int) yy, z0 = (int) zz;
    const real wx1 = xx - x0, wx0 = 1 - wx1;
    const real wy1 = yy - y0, wy0 = 1 - wy1;
    const real wz1 = zz - z0, wz0 = 1 - wz1;
    if (x0 == Ng) x0 = 0;
    if (y0 == Ng) y0 = 0;
    if (z0 == Ng) z0 = 0;
    const int x1 = (x0 == Ng - 1) ? 0 : x0 + 1;
    const int y1 = (y0 == Ng - 1) ? 0 : y0 + 1;
    const int z1 = (z0 == Ng - 1) ? 0 : z0 + 1;
    const real r000 = rho[IDX3(Ng, x0, y0, z0)] * wx0 * wy0 * wz0;
    const real r001 = rho[IDX3(Ng, x0, y0, z1)] * wx0 * wy0 * wz1;
    const real r010 = rho[IDX3(Ng, x0, y1, z0)] * wx0 * wy1 * wz0;
    const real r011 = rho[IDX3(Ng, x0, y1, z1)] * wx0 * wy1 * wz1;
    const real r100 = rho[IDX3(Ng, x1, y0, z0)] * wx1 * wy0 * wz0;
    const real r101 = rho[IDX3(Ng, x1, y0, z1)] * wx1 * wy0 * wz1;
    const real r110 = rho[IDX3(Ng, x1, y1, z0)] * wx1 * wy1 * wz0;
    const real r111 = rho[IDX3(Ng, x1, y1, z1)] * wx1 * wy1 * wz1;
    const real rs = r000 + r001 + r010 + r011 + r100 + r101 + r110 + r111;
    real vv = painted[IDX3(Ng, x0, y0, z0)] * r000
        + painted[IDX3(Ng, x0, y0, z1)] * r001
        + painted[IDX3(Ng, x0, y1, z0)] * r010
        + painted[IDX3(Ng, x0, y1, z1)] * r011
        + painted[IDX3(Ng, x1, y0, z0)] * r100
        + painted[IDX3(Ng, x1, y0, z1)] * r101
        + painted[IDX3(Ng, x1, y1, z0)] * r110
        + painted[IDX3(Ng, x1, y1, z1)] * r111;
    vv *= vfac / rs;
    v[t] = vv;
  }
}

/* add_vel_scatter (pop_tracer.c:1043-1113): tracer pair m uses draws
   8N+6m .. 8N+6m+5 as three Box-Muller pairs. */
void ezo_vel_scatter(int Ng, int rng, uint64_t seed, size_t n, real sigma_v,
    real *vx, real *vy, real *vz) {
  const size_t num = (size_t) Ng * Ng * Ng;
  const size_t ndraw = 6 * ((n + 1) / 2);
  uint32_t *u = malloc(sizeof(uint32_t) * (ndraw ? ndraw : 1));
  rng_fill(rng, seed, num << 3, ndraw, u);
  size_t q = 0;
  const double s = sigma_v;
#define GPAIR(g1, g2) do {                                              \
    const double rr_ = -2 * log(u_pos(rng, u[q]));                      \
    const double th_ = u_dbl(rng, u[q + 1]) * 2 * M_PI;                 \
    q += 2;                                                             \
    g1 = s * sqrt(rr_) * cos(th_);                                      \
    g2 = s * sqrt(rr_) * sin(th_);                                      \
  } while (0)
  for (size_t i = 0; i < n; i++) {
    double g1, g2;
    GPAIR(g1, g2);
    vx[i] += g1;
    vy[i] += g2;
    GPAIR(g1, g2);
    vz[i++] += g1;
    if (i == n) break;
    vx[i] += g2;
    GPAIR(g1, g2);
    vy[i] += g1;
    vz[i] += g2;
  }
#undef GPAIR
  free(u);
}

void ezo_rsd(size_t n, const real *z, const real *vz, double rsd_fac,
    double Lbox, double *zout) {
  for (size_t i = 0; i < n; i++) {
    double zr = z[i] + rsd_fac * vz[i];
    if (zr >= Lbox) zr -= Lbox;
    if (zr < 0) zr += Lbox;
    zout[i] = zr;
  }
}

/* Eulerian position of particle (i,j,k) in grid units, wrapped into
   [0, Ng), and its nearest grid cell (pop_tracer.c:541-561, :819-835). */
static size_t ngp_cell(int Ng, real igs, const real *psi0, const real *psi1,
    const real *psi2, int i, int j, int k, real *p) {
  const size_t idx = IDX3(Ng, i, j, k);
  real px = psi0[idx] * igs + i;
  real py = psi1[idx] * igs + j;
  real pz = psi2[idx] * igs + k;
  if (px < 0) px += Ng;
  else if (px >= Ng) px -= Ng;
  if (py < 0) py += Ng;
  else if (py >= Ng) py -= Ng;
  if (pz < 0) pz += Ng;
  else if (pz >= Ng) pz -= Ng;
  int ix = (int) (px + 0.5);
  int iy = (int) (py + 0.5);
  int iz = (int) (pz + 0.5);
  if (ix >= Ng) ix = 0;
  if (iy >= Ng) iy = 0;
  if (iz >= Ng) iz = 0;
  p[0] = px; p[1] = py; p[2] = pz;
  return IDX3(Ng, ix, iy, iz);
}

/* Particles per tracer-hosting cell (pop_tracer.c:517-582). */
int ezo_count_particles(int Ng, double Lbox, const real *psi0, const real *psi1,
    const real *psi2, const int16_t *nt, uint16_t *np) {
  const real igs = Ng / Lbox;
  memset(np, 0, sizeof(uint16_t) * (size_t) Ng * Ng * Ng);
  real p[3];
  for (int i = 0; i < Ng; i++)
    for (int j = 0; j < Ng; j++)
      for (int k = 0; k < Ng; k++) {
        const size_t c = ngp_cell(Ng, igs, psi0, psi1, psi2, i, j, k, p);
        if (nt[c] == 0) continue;
        if (np[c] == UINT16_MAX) return E_RHO_NPART;
        np[c]++;
      }
  return E_OK;
}

/* Tracers attached to particles (pop_tracer.c:804-879): particles in index
   order; in a cell with fewer tracers than particles each particle takes one
   draw of the stream from 4N and is kept if u np < nt (selection sampling).
   nt and np are consumed; *iv = number of attached tracers. */
int ezo_attach(int Ng, double Lbox, int rng, uint64_t seed, double vfac,
    const real *psi0, const real *psi1, const real *psi2, int16_t *nt,
    uint16_t *np, size_t ntot, real *x, real *y, real *z, real *vx, real *vy,
    real *vz, size_t *iv) {
  const size_t num = (size_t) Ng * Ng * Ng;
  const real igs = Ng / Lbox, gs = Lbox / Ng;
  uint32_t *u = malloc(sizeof(uint32_t) * num);
  if (!u) return E_MEMORY;
  rng_fill(rng, seed, num << 2, num, u);
  size_t cnt = 0, d = 0;
  real p[3];
  for (int i = 0; i < Ng; i++)
    for (int j = 0; j < Ng; j++)
      for (int k = 0; k < Ng; k++) {
        const size_t c = ngp_cell(Ng, igs, psi0, psi1, psi2, i, j, k, p);
        if (nt[c] == 0) continue;
        if (nt[c] < np[c]) {
          const double ran = u_dbl(rng, u[d++]);
          if (ran * np[c] >= nt[c]) {
            np[c]--;
            continue;
          }
        }
        nt[c]--;
        np[c]--;
        if (cnt >= ntot) { free(u); return E_UNKNOWN; }
        const size_t id = IDX3(Ng, i, j, k);
        x[cnt] = p[0] * gs;
        y[cnt] = p[1] * gs;
        z[cnt] = p[2] * gs;
        vx[cnt] = psi0[id] * vfac;
        vy[cnt] = psi1[id] * vfac;
        vz[cnt] = psi2[id] * vfac;
        cnt++;
      }
  free(u);
  *iv = cnt;
  return E_OK;
}

/* EZmock_populate_tracer (pop_tracer.c:1140-1219).  With att_part the
   attached tracers come first, the others follow in cell order (the OpenMP
   build's layout, pop_tracer.c:916-931). */
int ezo_populate(int Ng, double Lbox, int rng, uint64_t seed, double vfac,
    const real *psi0, const real *psi1, const real *psi2, const real *rho,
    const real *params, size_t nexp, int att_part, size_t cap, size_t *ntracer,
    real *x, real *y, real *z, real *vx, real *vy, real *vz) {
  const size_t num = (size_t) Ng * Ng * Ng;
  if (nexp < 128) return E_ARG_LOWEXP;
  if (nexp >= num) return E_ARG_HIEXP;
  const real rho_c = params[0], rho_exp = params[1], pbase = params[2],
      sigma_v = params[3];
  if (!isfinite(rho_c) || rho_c < 0) return E_PAR_RCUT;
  if (!isfinite(rho_exp) || rho_exp <= 0) return E_PAR_REXP;
  if (!isfinite(pbase) || pbase <= 0 || pbase >= 1) return E_PAR_PBASE;
  if (!isfinite(sigma_v) || sigma_v < 0) return E_PAR_SIGV;

  size_t pdf[MAX_NT_PER_CELL + 1], hist[NLOGB], ncell, ntot, nvalid;
  int nmax, e;
  if ((e = ezo_eval_pdf(Ng, nexp, pbase, pdf, &nmax, &ncell, &ntot))) return e;
  real *rhot = malloc(sizeof(real) * num);
  int16_t *nt = malloc(sizeof(int16_t) * num);
  real *paint = malloc(sizeof(real) * num);
  if (!rhot || !nt || !paint) { free(rhot); free(nt); free(paint); return E_MEMORY; }
  if ((e = ezo_bias(Ng, rng, seed, rho, rho_c, rho_exp, ncell, rhot, hist,
      &nvalid)) ||
      (e = ezo_select(Ng, rhot, hist, pdf, nmax, &ncell, &ntot, nt))) {
    free(rhot); free(nt); free(paint); return e;
  }
  free(rhot);
  if (ntot > cap) { free(nt); free(paint); *ntracer = ntot; return E_MEMORY; }
  size_t iv = 0;
  if (att_part) {
    uint16_t *np = malloc(sizeof(uint16_t) * num);
    if (!np) { free(nt); free(paint); return E_MEMORY; }
    if ((e = ezo_count_particles(Ng, Lbox, psi0, psi1, psi2, nt, np)) ||
        (e = ezo_attach(Ng, Lbox, rng, seed, vfac, psi0, psi1, psi2, nt, np, ntot,
            x, y, z, vx, vy, vz, &iv))) {
      free(np); free(nt); free(paint); return e;
    }
    free(np);
  }
  if ((e = ezo_positions(Ng, Lbox, rng, seed, nt, ntot - iv, x + iv, y + iv, z + iv))) {
    free(nt); free(paint); return e;
  }
  free(nt);
  for (int d = 0; d < 3; d++) {
    ezo_paint(Ng, Lbox, psi0, psi1, psi2, rho, d, paint);
    ezo_assign_vel(Ng, Lbox, vfac, paint, rho, ntot - iv, x + iv, y + iv, z + iv,
        ((d == 0) ? vx : (d == 1) ? vy : vz) + iv);
  }
  free(paint);
  ezo_vel_scatter(Ng, rng, seed, ntot, sigma_v, vx, vy, vz);
  *ntracer = ntot;
  return E_OK;
}
