// ez_host.cu -- C-ABI entry points of the B200 EZmock engine.
//
// Each function keeps the reference's argument validation order, error codes
// and sticky `*err` convention (libEZmock/EZmock/EZmock.c, cosmology.c,
// linear_pk.c, dens_field.c, pop_tracer.c, save_res.c); the work is done on
// the GPU on one CUDA stream per instance.  Host-side scalars (growth factor,
// P(k) spline setup, PDF evaluation) are computed in FP64 on the host.
#include "ez_internal.cuh"
#include "ezmock_b200.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <thread>

#include <omp.h>
#include <sys/mman.h>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <vector>

int ez_fft_tile_k(int Ng);
bool ez_fft_supported(int Ng);
int ez_fft_r2c_delta(EzMesh *m, const real *d_delta);
int ez_wn_scale(EzMesh *m, const EzPk *pk, double Lbox);
int ez_scale_psi(EzMesh *m, real f);

// ============================================================================
//                         host math (FP64, restated)
// ============================================================================
namespace {

// Gauss hypergeometric function: Taylor series, single-fraction recurrence
// and the z < 0 transformations (libEZmock/math/hypergeom.c:42-194).
int hg_series(double a, double b, double c, double z, double tol, int maxit,
    double *res) {
  if (fabs(a) >= 50 || fabs(b) >= 50 || fabs(c) <= 1 || fabs(z) >= 0.9) return 1;
  int hits = 0;
  double term = 1, sum = 1;
  for (int i = 0; i < maxit; i++) {
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

int hg_fraction(double a, double b, double c, double z, double tol, int maxit,
    double *res) {
  if (fabs(a) >= 50 || fabs(b) >= 50 || fabs(c) >= 20 || fabs(z) >= 0.9) return 1;
  int hits = 0;
  double al = 0, be = 1, ga = 1, ze = 1;
  for (int i = 0; i < maxit; i++) {
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

int hg(double a, double b, double c, double z, double tol, int maxit,
    double *res) {
  if (fabs(a) >= 50 || fabs(b) >= 50) return 1;
  if (z < -1) {
    const double w = 1 / (1 - z);
    double f1, f2;
    if (hg(a, c - b, a - b + 1, w, tol, maxit, &f1) ||
        hg(b, c - a, b - a + 1, w, tol, maxit, &f2)) return 1;
    const double gc = lgamma(c);
    const double g1 = gc + lgamma(b - a) - lgamma(b) - lgamma(c - a);
    const double g2 = gc + lgamma(a - b) - lgamma(a) - lgamma(c - b);
    *res = -pow(w, a) * exp(g1) * f1 + pow(w, b) * exp(g2) * f2;
    return 0;
  }
  if (z < 0) {
    const double w = z / (z - 1);
    double f;
    if (hg(a, c - b, c, w, tol, maxit, &f)) return 1;
    *res = pow(1 - z, -a) * f;
    return 0;
  }
  if (z > 0.5) return 1;
  if (fabs(c) > 1) return hg_series(a, b, c, z, tol, maxit, res);
  return hg_fraction(a, b, c, z, tol, maxit, res);
}

// Natural cubic spline second derivatives (libEZmock/math/cspline.c:35-76).
void spline_ypp(const double *x, const double *y, int n, double *ypp) {
  std::vector<double> cp(n);
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
}

// ============================================================================
//                              instance helpers
// ============================================================================
EzConf *CONF(EZMOCK *ez) { return (EzConf *) ez->conf; }
EzRng *RNG(EZMOCK *ez) { return (EzRng *) ez->rng; }
EzCosmo *COSMO(EZMOCK *ez) { return (EzCosmo *) ez->cosmo; }
EzPk *PK(EZMOCK *ez) { return (EzPk *) ez->pk; }
EzPar *PAR(EZMOCK *ez) { return (EzPar *) ez->par; }
EzMesh *MESH(EZMOCK *ez) { return (EzMesh *) ez->mesh; }

void pk_free(EzPk *p) {
  if (!p) return;
  free(p->k); free(p->P); free(p->P2);
  if (p->d_tab) cudaFree(p->d_tab);
  free(p);
}

void mesh_free_device(EzMesh *m) {
  if (m->side) cudaStreamSynchronize(m->side);
  if (m->spec[0]) cudaFree(m->spec[0]);
  if (m->psi[0]) cudaFree(m->psi[0]);
  if (m->rho) cudaFree(m->rho);
  if (m->paint[0]) cudaFree(m->paint[0]);
  if (m->draws) cudaFree(m->draws);
  if (m->scratch) cudaFree(m->scratch);
  if (m->rng_scratch) cudaFree(m->rng_scratch);
  if (m->fixacc) cudaFree(m->fixacc);
  if (m->pkq) cudaFree(m->pkq);
  if (m->est) cudaFree(m->est);
  if (m->att) cudaFree(m->att);
  if (m->stats) cudaFree(m->stats);
  if (m->cat) cudaFree(m->cat);
  if (m->h_stage) cudaFreeHost(m->h_stage);
  if (m->h_small) cudaFreeHost(m->h_small);
  if (m->h_cic) cudaFreeHost(m->h_cic);
  if (m->ev_cic) cudaEventDestroy(m->ev_cic);
  for (int i = 0; i < 4; i++) if (m->d2h_ev[i]) cudaEventDestroy(m->d2h_ev[i]);
  if (m->cpy) cudaStreamDestroy(m->cpy);
  if (m->ev_pos) cudaEventDestroy(m->ev_pos);
  if (m->ev_cat) cudaEventDestroy(m->ev_cat);
  if (m->stream) cudaStreamDestroy(m->stream);
  if (m->side) cudaStreamDestroy(m->side);
  if (m->ev_main) cudaEventDestroy(m->ev_main);
  if (m->ev_side) cudaEventDestroy(m->ev_side);
  if (m->ev_pop) cudaEventDestroy(m->ev_pop);
  if (m->rng_side) cudaFree(m->rng_side);
  if (m->draws_bias) cudaFree(m->draws_bias);
  if (m->draws_pop) cudaFree(m->draws_pop);
  for (int i = 0; i < 2 * ST_NSTAGE; i++) if (m->ev[i]) cudaEventDestroy(m->ev[i]);
  for (int i = 0; i < 8; i++) if (m->mark[i]) cudaEventDestroy(m->mark[i]);
}

// The population stages' random streams for the instance seed (bias draws
// 2N.., positions 5N.., dispersion 8N..; pop_tracer.c:233-237, :919, :1071),
// prepared on the side stream while the field is created.  The position and
// dispersion capacities are the largest of the previous field's populations.
void side_streams(EZMOCK *ez) {
  EzMesh *m = MESH(ez);
  const uint64_t N = m->N, h = m->pop_hint;
  const uint64_t starts[3] = {N << 1, N * 5, N << 3};
  const uint64_t caps[3] = {N + 2, 3 * h, 6 * ((h + 1) / 2)};
  ez_rng_side_prepare(m, RNG(ez)->ran, RNG(ez)->seed, starts, caps, h ? 3 : 1, N + 2);
  m->pop_hint_reset = true;
}

void side_streams_cb(void *ez) { side_streams((EZMOCK *) ez); }

int set_device(EzMesh *m) {
  return EZ_CUDA_OK(cudaSetDevice(m->device)) ? 0 : EZMOCK_ERR_UNKNOWN;
}

// Uploads the P(k) spline table to the device (k, P, P2 back to back).
int pk_upload(EzPk *pk) {
  if (pk->d_tab) return 0;
  std::vector<double> t(3 * (size_t) pk->n);
  memcpy(t.data(), pk->k, pk->n * sizeof(double));
  memcpy(t.data() + pk->n, pk->P, pk->n * sizeof(double));
  memcpy(t.data() + 2 * pk->n, pk->P2, pk->n * sizeof(double));
  if (!EZ_CUDA_OK(cudaMalloc(&pk->d_tab, t.size() * sizeof(double)))) {
    pk->d_tab = nullptr;
    return EZMOCK_ERR_MEMORY;
  }
  if (!EZ_CUDA_OK(cudaMemcpy(pk->d_tab, t.data(), t.size() * sizeof(double),
          cudaMemcpyHostToDevice)))
    return EZMOCK_ERR_UNKNOWN;
  return 0;
}

// eval_pdf (libEZmock/EZmock/pop_tracer.c:94-133)
int eval_pdf(int Ng, size_t nexp, real pbase, std::vector<size_t> &pdf,
    int *nmax, size_t *ncell, size_t *ntot) {
  size_t n;
  double A = 0, sum = 0, power = pbase;
  for (n = 1; n <= nexp; n++) {
    sum += power * n;
    A = nexp / sum;
    power *= pbase;
    if (A * power < 0.5) break;
  }
  if (n > EZ_MAX_NT) return EZMOCK_ERR_RHO_PBASE;
  pdf.assign(n, 0);
  size_t nc = 0, nobj = 0;
  for (size_t i = 0; i < n; i++) {
    pdf[i] = (size_t) round(A * pow(pbase, (double) (n - i)));
    nc += pdf[i];
    nobj += pdf[i] * (n - i);
  }
  if (nc > (size_t) Ng * Ng * Ng || nobj == 0) return EZMOCK_ERR_PAR_PBASE;
  *nmax = (int) n;
  *ncell = nc;
  *ntot = nobj;
  return 0;
}

int run_populate(EZMOCK *ez, const real *params, size_t nexp, bool att_part,
    size_t *ntracer, int *err) {
  EzConf *conf = CONF(ez);
  if (nexp < EZ_MIN_TRACER) return (*err = EZMOCK_ERR_ARG_LOWEXP);
  if (!ntracer) return (*err = EZMOCK_ERR_ARG_NDATA);
  if (nexp >= (size_t) conf->Ng * conf->Ng * conf->Ng)
    return (*err = EZMOCK_ERR_ARG_HIEXP);
  EzMesh *m = MESH(ez);
  if (!m->have_field) return (*err = EZMOCK_ERR_ARG_MESH);
  if (m->rho_replaced) return (*err = EZMOCK_ERR_RHO_USED);
  if (COSMO(ez)->vfac == HUGE_VAL) return (*err = EZMOCK_ERR_ARG_COSMO);
  const real rho_c = params[0], rho_exp = params[1], pbase = params[2],
      sigma_v = params[3];
  if (!std::isfinite(rho_c) || rho_c < 0) return (*err = EZMOCK_ERR_PAR_RCUT);
  if (!std::isfinite(rho_exp) || rho_exp <= 0) return (*err = EZMOCK_ERR_PAR_REXP);
  if (!std::isfinite(pbase) || pbase <= 0 || pbase >= 1) return (*err = EZMOCK_ERR_PAR_PBASE);
  if (!std::isfinite(sigma_v) || sigma_v < 0) return (*err = EZMOCK_ERR_PAR_SIGV);

  std::vector<size_t> pdf;
  int nmax;
  size_t ncell, ntot;
  int e = eval_pdf(conf->Ng, nexp, pbase, pdf, &nmax, &ncell, &ntot);
  if (e) return (*err = e);
  if ((e = set_device(m))) return (*err = e);
  EzPopResult res;
  e = ez_populate(m, conf->Ng, conf->Lbox, RNG(ez)->ran, RNG(ez)->seed,
      COSMO(ez)->vfac, params, pdf.data(), nmax, ncell, ntot, att_part, &res);
  if (e) return (*err = e);
  if (res.err) return (*err = res.err);
  *ntracer = res.ntot;
  EzPar *par = PAR(ez);
  par->rho_c = rho_c;
  par->rho_exp = rho_exp;
  par->pdf_base = pbase;
  par->sigma_v = sigma_v;
  return 0;
}

}  // namespace

static std::atomic<long long> g_launches(0);
void ez_count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

// ============================================================================
//                       memory management (used by stages)
// ============================================================================
int ez_scratch(EzMesh *m, size_t bytes) {
  if (bytes <= m->scratch_cap) return 0;
  if (m->scratch) cudaFree(m->scratch);
  m->scratch = nullptr;
  m->scratch_cap = 0;
  bytes = (bytes + 4095) / 4096 * 4096;
  if (!EZ_CUDA_OK(cudaMalloc(&m->scratch, bytes))) return EZMOCK_ERR_MEMORY;
  m->scratch_cap = bytes;
  return 0;
}

// Grows the RNG scratch, keeping its contents (prepared stream states).
int ez_rng_scratch(EzMesh *m, size_t bytes) {
  if (bytes <= m->rng_scratch_cap) return 0;
  bytes = (bytes + 4095) / 4096 * 4096;
  void *p = nullptr;
  if (!EZ_CUDA_OK(cudaMalloc(&p, bytes))) return EZMOCK_ERR_MEMORY;
  if (m->rng_scratch) {
    cudaMemcpyAsync(p, m->rng_scratch, m->rng_scratch_cap, cudaMemcpyDeviceToDevice, m->stream);
    cudaStreamSynchronize(m->stream);
    cudaFree(m->rng_scratch);
  }
  m->rng_scratch = p;
  m->rng_scratch_cap = bytes;
  return 0;
}

void ez_stage_begin(EzMesh *m, int st) {
  if (!m->timing) return;
  cudaEventRecord(m->ev[2 * st], m->stream);
}

void ez_stage_end(EzMesh *m, int st) {
  if (!m->timing) return;
  cudaEventRecord(m->ev[2 * st + 1], m->stream);
  m->ev_used[st] = true;
}

int ez_mesh_alloc(EzMesh *m, int Ng) {
  if (m->spec[0]) return 0;
  if (!EZ_CUDA_OK(cudaSetDevice(m->device))) return EZMOCK_ERR_UNKNOWN;
  if (!m->stream) {
    // highest priority: the side stream's preparations yield to it
    int lo = 0, hi = 0;
    cudaDeviceGetStreamPriorityRange(&lo, &hi);
    if (!EZ_CUDA_OK(cudaStreamCreateWithPriority(&m->stream, cudaStreamNonBlocking, hi)))
      return EZMOCK_ERR_UNKNOWN;
  }
  for (int i = 0; i < 2 * ST_NSTAGE; i++)
    if (!m->ev[i] && !EZ_CUDA_OK(cudaEventCreate(&m->ev[i]))) return EZMOCK_ERR_UNKNOWN;
  m->Ng = Ng;
  m->N = (size_t) Ng * Ng * Ng;
  m->Nk = Ng / 2 + 1;
  m->Nkp = (m->Nk + EZ_KPAD - 1) / EZ_KPAD * EZ_KPAD;
  m->Nspec = (size_t) Ng * Ng * m->Nkp;
  cplx *spec = nullptr;
  real *psi = nullptr, *paint = nullptr;
  const size_t ndraw = 2 * ((size_t) Ng * Ng * m->Nk) + 16;
  if (!EZ_CUDA_OK(cudaMalloc(&spec, 3 * m->Nspec * sizeof(cplx))) ||
      !EZ_CUDA_OK(cudaMalloc(&psi, 3 * m->N * sizeof(real))) ||
      !EZ_CUDA_OK(cudaMalloc(&m->rho, m->N * sizeof(real))) ||
      !EZ_CUDA_OK(cudaMalloc(&paint, (sizeof(real) == 4 ? 4 : 3) * m->N * sizeof(real))) ||
      !EZ_CUDA_OK(cudaMalloc(&m->draws, ndraw * sizeof(uint32_t)))) {
    if (spec) cudaFree(spec);
    if (psi) cudaFree(psi);
    if (paint) cudaFree(paint);
    if (m->rho) cudaFree(m->rho);
    if (m->draws) cudaFree(m->draws);
    m->rho = nullptr;
    m->draws = nullptr;
    cudaGetLastError();
    return EZMOCK_ERR_MEMORY;
  }
  m->draws_cap = ndraw;
  if (!EZ_CUDA_OK(cudaMalloc(&m->stats, sizeof(EzCicStats)))) return EZMOCK_ERR_MEMORY;
  cudaMemset(m->stats, 0, sizeof(EzCicStats));
  for (int d = 0; d < 3; d++) {
    m->spec[d] = spec + d * m->Nspec;
    m->psi[d] = psi + d * m->N;
    m->paint[d] = paint + d * m->N;
  }
  m->pq = paint;
  return 0;
}

// ============================================================================
//                                 C interface
// ============================================================================
extern "C" {

EZMOCK *EZmock_init(const double Lbox, const int Ngrid, const int randgen,
    const uint64_t seed, const int nthread, int *err) {
  if (!err || *err != EZMOCK_SUCCESS) return NULL;
  if (Lbox <= 0) { *err = EZMOCK_ERR_ARG_LBOX; return NULL; }
  if (Ngrid <= 0 || Ngrid > EZ_MAX_GRID || !ez_fft_supported(Ngrid)) {
    *err = EZMOCK_ERR_ARG_NGRID; return NULL;
  }
  if (randgen != EZMOCK_RNG_MRG32K3A && randgen != EZMOCK_RNG_MT19937) {
    *err = EZMOCK_ERR_ARG_RNG; return NULL;
  }
  if (seed == 0) { *err = EZMOCK_ERR_ARG_SEED; return NULL; }
  if (nthread < 0) { *err = EZMOCK_ERR_ARG_THREAD; return NULL; }

  EZMOCK *ez = (EZMOCK *) calloc(1, sizeof(EZMOCK));
  if (!ez) { *err = EZMOCK_ERR_MEMORY; return NULL; }
  ez->conf = calloc(1, sizeof(EzConf));
  ez->rng = calloc(1, sizeof(EzRng));
  ez->cosmo = calloc(1, sizeof(EzCosmo));
  ez->par = calloc(1, sizeof(EzPar));
  ez->mesh = calloc(1, sizeof(EzMesh));
  if (!ez->conf || !ez->rng || !ez->cosmo || !ez->par || !ez->mesh) {
    EZmock_destroy(ez);
    *err = EZMOCK_ERR_MEMORY;
    return NULL;
  }
  EzConf *conf = CONF(ez);
  conf->nthread = nthread;
  conf->Ng = Ngrid;
  conf->Lbox = Lbox;
  RNG(ez)->ran = randgen;
  RNG(ez)->seed = seed;
  COSMO(ez)->growth2 = COSMO(ez)->vfac = HUGE_VAL;
  EzPar *par = PAR(ez);
  par->bao_enhance = par->rho_c = par->rho_exp = HUGE_VAL;
  par->pdf_base = par->sigma_v = HUGE_VAL;
  EzMesh *m = MESH(ez);
  m->device = -1;
  m->fft_tma = true;
  m->fft_tma_i = true;
  m->sel_path = -1;
  return ez;
}

int EZmock_set_cosmology(EZMOCK *ez, const double pk_norm, const double fHa,
    const bool eval, const double z, const double z_pk, const double Omega_m,
    const double Omega_nu, const double w, int *err) {
  if (!err) return EZMOCK_ERR_ARG_ECODE;
  if (*err != EZMOCK_SUCCESS) return *err;
  if (!ez) return EZMOCK_ERR_ARG_EZ;        // the reference leaves *err unset
  EzCosmo *cosmo = COSMO(ez);
  if (!eval) {
    if (pk_norm <= 0 || fHa <= 0) return (*err = EZMOCK_ERR_PAR_COSMO);
    cosmo->growth2 = pk_norm;
    cosmo->vfac = fHa;
    return EZMOCK_SUCCESS;
  }
  if (z < 0 || z_pk < 0 || Omega_m <= 0 || Omega_m > 1 || Omega_nu < 0 ||
      Omega_nu >= 1 || w >= -1.0 / 3.0)
    return (*err = EZMOCK_ERR_PAR_COSMO);
  const double a = 1 / (1 + z), a0 = 1 / (1 + z_pk);
  // cosmo_growth (cosmology.c:53-95)
  if (a <= 0 || a > 1 || a0 <= 0 || a0 > 1 || Omega_m <= 0 || Omega_m > 1 ||
      w >= -1.0 / 3.0)
    return (*err = EZMOCK_ERR_PAR_COSMO);
  const double tol = 1e-12;
  const int maxit = 10000;
  const double iw = 1 / w;
  const double f1 = 0.5 * (1 - iw);
  const double f2 = -0x1.5555555555555p-2 * iw;
  const double f3 = 1 - 0x1.aaaaaaaaaaaabp-1 * iw;
  const double f4 = (1 - 1 / Omega_m) * pow(a, -3 * w);
  double h1, h2, D, f;
  if (hg(f1, f2, f3, f4, tol, maxit, &h1) ||
      hg(f1 + 1, f2 + 1, f3 + 1, f4, tol, maxit, &h2))
    return (*err = EZMOCK_ERR_COS_GROWTH);
  f = 1 + 3 * (w - 1) * f4 / (6 * w - 5) * h2 / h1;
  if (a == a0) D = 1;
  else {
    const double f5 = (1 - 1 / Omega_m) * pow(a0, -3 * w);
    if (hg(f1, f2, f3, f5, tol, maxit, &h2)) return (*err = EZMOCK_ERR_COS_GROWTH);
    D = (a * h1) / (a0 * h2);
  }
  const double Omn = Omega_m + Omega_nu;
  const double H = 100 * sqrt((1 - Omn) * pow(a, -3 * (1 + w)) + Omn * pow(a, -3));
  cosmo->growth2 = D * D;
  cosmo->vfac = f * H * a;
  return EZMOCK_SUCCESS;
}

int EZmock_setup_linear_pk(EZMOCK *ez, const double *k, const int n,
    const double *Pk, const double *Pnw, const double mBAO, const bool logint,
    int *err) {
  if (!err) return EZMOCK_ERR_ARG_ECODE;
  if (*err != EZMOCK_SUCCESS) return *err;
  if (!ez) return (*err = EZMOCK_ERR_ARG_EZ);
  if (!k || !Pk || (mBAO != 0 && !Pnw)) return (*err = EZMOCK_ERR_ARG_NULL);
  if (n <= 3 || n > EZ_MAX_PK_N) return (*err = EZMOCK_ERR_ARG_NBIN);
  EzCosmo *cosmo = COSMO(ez);
  if (cosmo->growth2 == HUGE_VAL) return (*err = EZMOCK_ERR_ARG_COSMO);
  for (int i = 0; i < n; i++) {
    if (!std::isfinite(k[i]) || !std::isfinite(Pk[i])) return (*err = EZMOCK_ERR_PK_FINITE);
    if (k[i] <= 0 || Pk[i] <= 0) return (*err = EZMOCK_ERR_PK_NONPOS);
    if (i && k[i] <= k[i - 1]) return (*err = EZMOCK_ERR_PK_NONASC);
  }
  if (mBAO != 0) {
    for (int i = 0; i < n; i++) {
      if (!std::isfinite(Pnw[i])) return (*err = EZMOCK_ERR_PK_FINITE);
      if (Pnw[i] <= 0) return (*err = EZMOCK_ERR_PK_NONPOS);
    }
  }
  EzConf *conf = CONF(ez);
  const double kmin = 2 * EZ_PI / conf->Lbox;
  const double kmax = EZ_PI * conf->Ng / conf->Lbox * sqrt(3);
  if (k[0] > kmin - EZ_DOUBLE_TOL || k[n - 1] < kmax + EZ_DOUBLE_TOL)
    return (*err = EZMOCK_ERR_PK_RANGE);
  int imin, imax;
  for (imin = 0; imin < n; imin++) if (k[imin] > kmin) break;
  for (imax = imin; imax < n; imax++) if (k[imax] > kmax) break;
  imin = (imin < 3) ? 0 : imin - 3;
  imax = (imax + 3 >= n) ? n : imax + 3;
  const int nbin = imax - imin;
  if (nbin < 3) return (*err = EZMOCK_ERR_PK_NBIN);
  EzPk *pk = (EzPk *) calloc(1, sizeof(EzPk));
  if (!pk) return (*err = EZMOCK_ERR_MEMORY);
  pk->k = (double *) malloc(nbin * sizeof(double));
  pk->P = (double *) malloc(nbin * sizeof(double));
  pk->P2 = (double *) malloc(nbin * sizeof(double));
  if (!pk->k || !pk->P || !pk->P2) { pk_free(pk); return (*err = EZMOCK_ERR_MEMORY); }
  for (int i = 0; i < nbin; i++) {
    const int j = i + imin;
    double v;
    if (mBAO == 0) v = Pk[j] * cosmo->growth2;
    else {
      v = (k[j] <= EZ_KMAX_BAO) ? (Pk[j] - Pnw[j]) * exp(k[j] * k[j] * mBAO) + Pnw[j] : Pk[j];
      if (!std::isfinite(v) || v <= 0) { pk_free(pk); return (*err = EZMOCK_ERR_PK_MODBAO); }
      v *= cosmo->growth2;
    }
    pk->P[i] = v;
  }
  for (int i = 0; i < nbin; i++) {
    if (logint) { pk->k[i] = log(k[i + imin]); pk->P[i] = log(pk->P[i]); }
    else pk->k[i] = k[i + imin];
  }
  pk->n = nbin;
  pk->log = logint;
  pk->kmin = k[imin];
  pk->kmax = k[imax - 1];
  spline_ypp(pk->k, pk->P, nbin, pk->P2);
  if (ez->pk) pk_free(PK(ez));
  ez->pk = pk;
  PAR(ez)->bao_enhance = mBAO;
  return EZMOCK_SUCCESS;
}

int EZmock_create_dens_field(EZMOCK *ez, real *psi[3], bool deepcopy,
    real *delta, const bool fixamp, const bool iphase, int *err) {
  if (!err) return EZMOCK_ERR_ARG_ECODE;
  if (*err != EZMOCK_SUCCESS) return *err;
  if (!ez) return (*err = EZMOCK_ERR_ARG_EZ);
  EzConf *conf = CONF(ez);
  EzMesh *m = MESH(ez);
  const bool user_psi = psi && psi[0] && psi[1] && psi[2];
  EzPk *pk = PK(ez);
  if (!user_psi) {
    if (!pk) return (*err = EZMOCK_ERR_ARG_PK);
    const double kmin = 2 * EZ_PI / conf->Lbox;
    const double kmax = EZ_PI * conf->Ng / conf->Lbox * sqrt(3);
    if (pk->kmin > kmin - EZ_DOUBLE_TOL || pk->kmax < kmax + EZ_DOUBLE_TOL)
      return (*err = EZMOCK_ERR_PK_RANGE);
  }
  if (m->device < 0 && !EZ_CUDA_OK(cudaGetDevice(&m->device))) {
    cudaGetLastError();
    m->device = -1;
    return (*err = EZMOCK_ERR_UNKNOWN);
  }
  int e;
  if ((e = ez_mesh_alloc(m, conf->Ng))) return (*err = e);
  if ((e = set_device(m))) return (*err = e);
  for (int s = 0; s < ST_NSTAGE; s++) m->ev_used[s] = false;
  m->have_field = false;
  m->psimax_valid = false;
  const size_t bytes = m->N * sizeof(real);
  if (user_psi) {
    // dens_field.c:351-374: the displacements are taken as given
    for (int d = 0; d < 3; d++)
      if (!EZ_CUDA_OK(cudaMemcpyAsync(m->psi[d], psi[d], bytes, cudaMemcpyHostToDevice, m->stream)))
        return (*err = EZMOCK_ERR_UNKNOWN);
    m->psi_ref = !deepcopy;
  }
  else {
    if ((e = pk_upload(pk))) return (*err = e);
    if (delta) {
      // dens_field.c:188-220, perturb.c:456-604
      real *d_delta = m->psi[2];                // staging; overwritten later
      if (!EZ_CUDA_OK(cudaMemcpyAsync(d_delta, delta, bytes, cudaMemcpyHostToDevice, m->stream)))
        return (*err = EZMOCK_ERR_UNKNOWN);
      if ((e = ez_fft_r2c_delta(m, d_delta)) || (e = ez_wn_scale(m, pk, conf->Lbox)) ||
          (e = ez_fft_c2r_psi(m)))
        return (*err = e);
      const real norm = 1 / sqrt((double) m->N);
      if ((e = ez_scale_psi(m, norm))) return (*err = e);
      m->psimax_valid = false;
    }
    else {
      const size_t ndraw = ((size_t) conf->Ng * conf->Ng * m->Nk - 1) * (fixamp ? 1 : 2);
      ez_stage_begin(m, ST_RNG_IC);
      if ((e = ez_rng_fill_around(m, RNG(ez)->ran, RNG(ez)->seed, 0, ndraw, m->draws,
              side_streams_cb, ez)))
        return (*err = e);
      ez_stage_end(m, ST_RNG_IC);
      if ((e = ez_ic_spectrum(m, pk, conf->Lbox, RNG(ez)->ran, fixamp, iphase, m->draws)) ||
          (e = ez_fft_c2r_psi(m)))
        return (*err = e);
    }
    m->psi_ref = false;
  }
  if (user_psi || delta) side_streams(ez);
  if ((e = ez_cic(m, conf->Lbox))) return (*err = e);
  // A field made from the initial conditions returns with its kernels still
  // queued: every later call of the instance is ordered after them on the
  // instance stream.  With caller arrays (psi, delta) the call waits, since
  // a copy from page-locked host memory may still be reading them.
  if ((user_psi || delta) && !EZ_CUDA_OK(cudaStreamSynchronize(m->stream)))
    return (*err = EZMOCK_ERR_UNKNOWN);
  m->fixamp = fixamp;
  m->iphase = iphase;
  m->have_field = true;
  return EZMOCK_SUCCESS;
}

// Pre-faulted host blocks for the catalogue arrays handed to the caller.
// First-touch faults of fresh malloc() memory ran at 3-4 GB/s on one host
// thread (20 ms for the 75 MB catalogue of a 512^3 mock, against 1.5 ms for
// its DMA), so after each copy-out a worker thread mallocs and faults in the
// blocks of the next catalogue of that size while the GPU computes it.  The
// blocks are plain malloc() memory: the caller frees them as before.
void touch_pages(void *p, size_t bytes, int nthr) {
  const size_t pg = 4096, npg = (bytes + pg - 1) / pg;
#pragma omp parallel for num_threads(nthr) schedule(static)
  for (long i = 0; i < (long) npg; i++) ((volatile char *) p)[(size_t) i * pg] = 0;
}

class HostPool {
 public:
  explicit HostPool(int nthr) : nthr_(nthr), worker_([this] { run(); }) {}
  // While a copy-out holds the pool, the worker faults no pages: its threads
  // would compete with the copy-out's for the cores and the memory bus (a
  // 1024^3 mock's second population took 18 ms to copy out its 300 MB while
  // the worker faulted the first population's 619 MB; paused, 4.8 ms, and
  // the three copy-outs 37 -> 16 ms).
  void hold() { held_out_.fetch_add(1); }
  void release() { held_out_.fetch_sub(1); }
  ~HostPool() {
    stop_flag_.store(true);
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_ = true;
      queue_.clear();
    }
    cv_.notify_all();
    worker_.join();
    for (const Block &b : ready_) free(b.p);
  }
  // A faulted block of need .. 2 need bytes, or nullptr; waits for a queued
  // or running fill of such a block.
  void *take(size_t need) {
    std::unique_lock<std::mutex> lk(mu_);
    for (;;) {
      int best = -1;
      for (int i = 0; i < (int) ready_.size(); i++)
        if (fits(ready_[i].cap, need) && (best < 0 || ready_[i].cap < ready_[best].cap)) best = i;
      if (best >= 0) {
        void *p = ready_[best].p;
        held_ -= ready_[best].cap;
        ready_.erase(ready_.begin() + best);
        return p;
      }
      bool pending = fits(busy_, need);
      for (size_t c : queue_) pending = pending || fits(c, need);
      if (!pending) return nullptr;
      cv_.wait(lk);
    }
  }
  // Queues `count` blocks of `cap` bytes, dropping the oldest held blocks
  // so that the pool stays within `limit` bytes.
  void request(size_t cap, int count, size_t limit) {
    {
      std::lock_guard<std::mutex> lk(mu_);
      size_t queued = busy_;
      for (size_t c : queue_) queued += c;
      const size_t add = cap * (size_t) count;
      while (!ready_.empty() && held_ + queued + add > limit) {
        held_ -= ready_.front().cap;
        free(ready_.front().p);
        ready_.erase(ready_.begin());
      }
      if (held_ + queued + add > limit) return;
      for (int i = 0; i < count; i++) queue_.push_back(cap);
    }
    cv_.notify_all();
  }

 private:
  struct Block { void *p; size_t cap; };
  static bool fits(size_t cap, size_t need) { return cap >= need && cap <= 2 * need; }
  void run() {
    std::unique_lock<std::mutex> lk(mu_);
    for (;;) {
      cv_.wait(lk, [this] { return stop_ || !queue_.empty(); });
      if (stop_) return;
      busy_ = queue_.front();
      queue_.pop_front();
      const size_t cap = busy_;
      lk.unlock();
      void *p = malloc(cap);
      // faulted in 8 MB pieces, between copy-outs
      constexpr size_t PIECE = (size_t) 8 << 20;
      for (size_t o = 0; p && o < cap; o += PIECE) {
        while (held_out_.load() > 0 && !stop_flag_.load())
          std::this_thread::sleep_for(std::chrono::microseconds(50));
        if (stop_flag_.load()) break;
        touch_pages((char *) p + o, std::min(PIECE, cap - o), nthr_);
      }
      lk.lock();
      busy_ = 0;
      if (p) {
        ready_.push_back({p, cap});
        held_ += cap;
      }
      cv_.notify_all();
    }
  }
  int nthr_;
  std::mutex mu_;
  std::condition_variable cv_;
  std::deque<size_t> queue_;
  std::vector<Block> ready_;
  size_t held_ = 0, busy_ = 0;
  bool stop_ = false;
  std::atomic<int> held_out_{0};             // copy-outs in progress
  std::atomic<bool> stop_flag_{false};
  std::thread worker_;                       // last: starts after the rest
};

int EZmock_populate_tracer(EZMOCK *ez, const real *params, const size_t nexp,
    const bool att_part, size_t *ntracer, real **x, real **y, real **z,
    real **vx, real **vy, real **vz, int *err) {
  if (!err) return EZMOCK_ERR_ARG_ECODE;
  if (*err != EZMOCK_SUCCESS) return *err;
  if (!ez) return (*err = EZMOCK_ERR_ARG_EZ);
  if (!params) return (*err = EZMOCK_ERR_ARG_PARAMS);
  size_t n = 0;
  EzMesh *m = MESH(ez);
  // the copy-out's stream and events (the device is set by the first field)
  if (m->device >= 0 && !m->cpy) {
    if (!EZ_CUDA_OK(cudaSetDevice(m->device)) ||
        !EZ_CUDA_OK(cudaStreamCreateWithFlags(&m->cpy, cudaStreamNonBlocking)) ||
        !EZ_CUDA_OK(cudaEventCreateWithFlags(&m->ev_pos, cudaEventDisableTiming)) ||
        !EZ_CUDA_OK(cudaEventCreateWithFlags(&m->ev_cat, cudaEventDisableTiming)))
      return (*err = EZMOCK_ERR_UNKNOWN);
  }
  if (run_populate(ez, params, nexp, att_part, &n, err)) return *err;
  if (!m->cpy || !EZ_CUDA_OK(cudaEventRecord(m->ev_cat, m->stream)))
    return (*err = EZMOCK_ERR_UNKNOWN);
  // host threads of the copy-out: on the GPU boxes (16 cores) a 75 MB
  // pinned-to-malloc copy took 1.86 ms with 8 threads (slower than its
  // 1.40 ms DMA) and 1.08 ms with 16; more threads than cores were slower
  int nthr = CONF(ez)->nthread > 0 ? CONF(ez)->nthread : omp_get_num_procs();
  nthr = std::max(1, std::min(nthr, 16));
  const size_t bytes_arr = n * sizeof(real);
  const bool pooled = m->hpool_mib >= 0 && bytes_arr >= ((size_t) 4 << 20);
  if (pooled && !m->hpool) m->hpool = new HostPool(nthr);
  HostPool *pool = pooled ? (HostPool *) m->hpool : nullptr;
  real *cat[6];
  bool fresh[6];
  for (int i = 0; i < 6; i++) {
    cat[i] = pool ? (real *) pool->take(bytes_arr) : nullptr;
    fresh[i] = !cat[i];
    if (!cat[i] && !(cat[i] = (real *) malloc((n ? n : 1) * sizeof(real)))) {
      for (int j = 0; j < i; j++) free(cat[j]);
      return (*err = EZMOCK_ERR_MEMORY);
    }
  }
  // Fresh malloc() memory is faulted in with several threads while the GPU
  // finishes the catalogue, so the copy-out below runs at memcpy speed.  (No
  // huge-page advice: where the kernel compacts memory synchronously for
  // advised regions, a fault stalled for up to a second.)
  if (bytes_arr >= ((size_t) 4 << 20)) {
    const size_t pg = 4096, npg = (bytes_arr + pg - 1) / pg;
#pragma omp parallel for num_threads(nthr) schedule(static)
    for (long p = 0; p < (long) (6 * npg); p++)
      if (fresh[p / npg]) ((volatile char *) cat[p / npg])[(p % npg) * pg] = 0;
  }
  // device -> pinned staging (a ring of three 16 MB buffers: the DMA of the
  // next pieces overlaps the copy-out of this one) -> the caller's malloc()
  // arrays, copied out by up to eight host threads.  The copies run on their
  // own stream: the positions once they are final, while the GPU computes
  // the velocities.  (512^3, 75 MB: the copy-out after the GPU work took
  // 2.26 ms with two 8 MB buffers and four threads, 1.85 with three, 1.49
  // with three and six threads, 1.18 with three 16 MB buffers and eight
  // threads; 32 MB pieces or four buffers no better; 1.08 with sixteen
  // threads, against 1.1-1.6 for 4 or 8 MB pieces in four to eight buffers.)
  ez_stage_begin(m, ST_D2H);
  // the pool's worker pauses its page faulting until the copies are done
  struct PoolHold {
    HostPool *p;
    explicit PoolHold(HostPool *q) : p(q) { if (p) p->hold(); }
    ~PoolHold() { if (p) p->release(); }
  } pool_hold(pool);
  const size_t piece = (size_t) 16 << 20;
  constexpr int NB = 3;
  if (m->h_stage_cap < NB * piece) {
    if (m->h_stage) cudaFreeHost(m->h_stage);
    m->h_stage = nullptr;
    m->h_stage_cap = 0;
    if (!EZ_CUDA_OK(cudaMallocHost(&m->h_stage, NB * piece))) {
      for (int j = 0; j < 6; j++) free(cat[j]);
      return (*err = EZMOCK_ERR_MEMORY);
    }
    m->h_stage_cap = NB * piece;
  }
  for (int i = 0; i < NB; i++)
    if (!m->d2h_ev[i]) cudaEventCreateWithFlags(&m->d2h_ev[i], cudaEventDisableTiming);
  const size_t per = piece / sizeof(real);              // reals per piece
  struct Piece { int arr; size_t off, len; };
  std::vector<Piece> pieces;
  for (int a = 0; a < 6; a++)
    for (size_t o = 0; o < n; o += per) pieces.push_back({a, o, std::min(per, n - o)});
  bool ok = true;
  auto issue = [&](size_t k) {
    const Piece &pc = pieces[k];
    real *stage = (real *) ((char *) m->h_stage + (k % NB) * piece);
    if (k == 0 || pc.arr != pieces[k - 1].arr) {
      // each array waits for the kernel that completes it
      ok = ok && EZ_CUDA_OK(cudaStreamWaitEvent(m->cpy, pc.arr < 3 ? m->ev_pos : m->ev_cat, 0));
    }
    ok = ok && EZ_CUDA_OK(cudaMemcpyAsync(stage, m->cat + (size_t) pc.arr * n + pc.off,
        pc.len * sizeof(real), cudaMemcpyDeviceToHost, m->cpy));
    ok = ok && EZ_CUDA_OK(cudaEventRecord(m->d2h_ev[k % NB], m->cpy));
  };
  for (size_t k = 0; k < pieces.size() && k < (size_t) NB; k++) issue(k);
  for (size_t k = 0; k < pieces.size() && ok; k++) {
    ok = ok && EZ_CUDA_OK(cudaEventSynchronize(m->d2h_ev[k % NB]));
    const Piece &pc = pieces[k];
    const char *src = (const char *) m->h_stage + (k % NB) * piece;
    char *dst = (char *) (cat[pc.arr] + pc.off);
    const size_t nb = pc.len * sizeof(real);
    const int nt = (nb >= ((size_t) 1 << 20)) ? nthr : 1;
    if (nt == 1) memcpy(dst, src, nb);
    else {
      const size_t step = (nb + nt - 1) / nt;
#pragma omp parallel for num_threads(nt) schedule(static)
      for (int t = 0; t < nt; t++) {
        const size_t b0 = std::min(nb, t * step), b1 = std::min(nb, b0 + step);
        if (b1 > b0) memcpy(dst + b0, src + b0, b1 - b0);
      }
    }
    // this buffer is free again
    if (k + NB < pieces.size()) issue(k + NB);
  }
  // later work of the instance stream (the next catalogue) follows the copies
  if (ok && !pieces.empty())
    ok = EZ_CUDA_OK(cudaStreamWaitEvent(m->stream, m->d2h_ev[(pieces.size() - 1) % NB], 0));
  if (!ok) {
    for (int j = 0; j < 6; j++) free(cat[j]);
    return (*err = EZMOCK_ERR_UNKNOWN);
  }
  ez_stage_end(m, ST_D2H);
  // blocks for the next catalogue of this size (the tie extension varies
  // the count by a few tracers)
  if (pool)
    pool->request(bytes_arr + bytes_arr / 32 + 65536, 6,
        (size_t) (m->hpool_mib ? m->hpool_mib : 2048) << 20);
  *ntracer = n;
  *x = cat[0]; *y = cat[1]; *z = cat[2];
  *vx = cat[3]; *vy = cat[4]; *vz = cat[5];
  return EZMOCK_SUCCESS;
}

// save_res.c:95-178, same formats and chunked buffering.
#define EZ_FILE_CHUNK 1048576
#ifdef SINGLE_PREC
#define EZ_REAL_OFMT "%.6g"
#else
#define EZ_REAL_OFMT "%.10g"
#endif

static int put_line(FILE *fp, char *chunk, size_t *size, const char *fmt, ...) {
  va_list args;
  va_start(args, fmt);
  int n = vsnprintf(chunk + *size, EZ_FILE_CHUNK - *size, fmt, args);
  va_end(args);
  if (n < 0 || n >= EZ_FILE_CHUNK) return EZMOCK_ERR_FILE;
  if (*size + n >= EZ_FILE_CHUNK) {
    if (fwrite(chunk, *size, 1, fp) != 1) return EZMOCK_ERR_FILE;
    *size = 0;
    va_start(args, fmt);
    n = vsnprintf(chunk, EZ_FILE_CHUNK, fmt, args);
    va_end(args);
    if (n >= EZ_FILE_CHUNK) return EZMOCK_ERR_FILE;
  }
  *size += n;
  return 0;
}

int EZmock_write_ascii(EZMOCK *ez, const real *x, const real *y, const real *z,
    const real *vx, const real *vy, const real *vz, const size_t ntracer,
    const double rsd_fac, const bool header, const char *fname, int *err) {
  if (!err) return EZMOCK_ERR_ARG_ECODE;
  if (*err != EZMOCK_SUCCESS) return *err;
  if (!ez) return (*err = EZMOCK_ERR_ARG_EZ);
  // the reference also rejects arrays whose first element is zero
  if (!x || !(*x) || !y || !(*y) || !z || !(*z) || !vx || !(*vx) || !vy ||
      !(*vy) || !vz || !(*vz))
    return (*err = EZMOCK_ERR_ARG_NULL);
  if (!ntracer) return (*err = EZMOCK_ERR_ARG_NDATA);
  EzConf *conf = CONF(ez);
  if (rsd_fac > conf->Lbox) return (*err = EZMOCK_ERR_ARG_RSD);
  if (!fname || !(*fname)) return (*err = EZMOCK_ERR_ARG_NULL);
  char *chunk = (char *) calloc(EZ_FILE_CHUNK, 1);
  if (!chunk) return (*err = EZMOCK_ERR_MEMORY);
  FILE *fp = fopen(fname, "w");
  if (!fp) { free(chunk); return (*err = EZMOCK_ERR_FILE); }
  size_t size = 0;
  int e = 0;
#define PUT(...) do { if ((e = put_line(fp, chunk, &size, __VA_ARGS__))) goto fail; } while (0)
  if (header) {
    EzCosmo *cosmo = COSMO(ez);
    EzPar *par = PAR(ez);
    EzMesh *m = MESH(ez);
    const char *rng_name[2] = {"MRG32K3A", "MT19937"};
    PUT("%c BOX_SIZE=%.10lg , NUM_GRID=%d , FIX_AMPLITUDE=%c , INVERT_PHASE=%c\n",
        '#', conf->Lbox, conf->Ng, m->fixamp ? 'T' : 'F', m->iphase ? 'T' : 'F');
    PUT("%c GROWTH_PK=%.10lg , VELOCITY_FAC=%.10lg\n", '#', cosmo->growth2, cosmo->vfac);
    PUT("%c BAO_ENHANCE=%.10lg , RHO_CRITICAL=%.10lg , RHO_EXP=%.10lg , PDF_BASE=%.10lg , "
        "SIGMA_VELOCITY=%.10lg\n%c RAND_GENERATOR=%s , RAND_SEED=%ld\n",
        '#', par->bao_enhance, par->rho_c, par->rho_exp, par->pdf_base, par->sigma_v,
        '#', rng_name[RNG(ez)->ran], (long) RNG(ez)->seed);
  }
  if (rsd_fac > 0) {
    PUT("%c x(1) y(2) z_rsd(3)\n", '#');
    for (size_t i = 0; i < ntracer; i++) {
      double zr = z[i] + rsd_fac * vz[i];
      if (zr >= conf->Lbox) zr -= conf->Lbox;
      if (zr < 0) zr += conf->Lbox;
      PUT(EZ_REAL_OFMT " " EZ_REAL_OFMT " " EZ_REAL_OFMT "\n", x[i], y[i], zr);
    }
  }
  else {
    PUT("%c x(1) y(2) z(3) vx(4) vy(5) vz(6)\n", '#');
    for (size_t i = 0; i < ntracer; i++)
      PUT(EZ_REAL_OFMT " " EZ_REAL_OFMT " " EZ_REAL_OFMT " " EZ_REAL_OFMT " "
          EZ_REAL_OFMT " " EZ_REAL_OFMT "\n", x[i], y[i], z[i], vx[i], vy[i], vz[i]);
  }
#undef PUT
  if (fwrite(chunk, size, 1, fp) != 1) { e = EZMOCK_ERR_FILE; goto fail; }
  free(chunk);
  fclose(fp);
  return (*err = EZMOCK_SUCCESS);
fail:
  free(chunk);
  fclose(fp);
  return (*err = e);
}

void EZmock_destroy(EZMOCK *ez) {
  if (!ez) return;
  EzMesh *m = MESH(ez);
  if (m) {
    delete (HostPool *) m->hpool;
    if (m->device >= 0) {
      cudaSetDevice(m->device);
      mesh_free_device(m);
    }
    free(m);
  }
  pk_free(PK(ez));
  free(ez->conf);
  free(ez->rng);
  free(ez->cosmo);
  free(ez->par);
  free(ez);
}

const char *EZmock_errmsg(const int err) {
  switch (err) {
    case EZMOCK_SUCCESS:        return "no error";
    case EZMOCK_ERR_MEMORY:     return "failed to allocate memory";
    case EZMOCK_ERR_ARG_ECODE:  return "error code is not set";
    case EZMOCK_ERR_ARG_EZ:     return "EZmock interface uninitialized";
    case EZMOCK_ERR_ARG_COSMO:  return "EZmock cosmology uninitialized";
    case EZMOCK_ERR_ARG_PK:     return "EZmock power spectrum uninitialized";
    case EZMOCK_ERR_ARG_MESH:   return "EZmock density fields uninitialized";
    case EZMOCK_ERR_ARG_LBOX:   return "invalid box size";
    case EZMOCK_ERR_ARG_NGRID:  return "invalid grid size";
    case EZMOCK_ERR_ARG_RNG:    return "invalid random number generator";
    case EZMOCK_ERR_ARG_SEED:   return "invalid random seed";
    case EZMOCK_ERR_ARG_THREAD: return "invalid number of threads";
    case EZMOCK_ERR_ARG_NULL:   return "null input array";
    case EZMOCK_ERR_ARG_NBIN:   return "invalid number of bins";
    case EZMOCK_ERR_ARG_PARAMS: return "EZmock calibration parameters not set";
    case EZMOCK_ERR_ARG_LOWEXP: return "too few expected number of tracers";
    case EZMOCK_ERR_ARG_HIEXP:  return "too many expected number of tracers";
    case EZMOCK_ERR_ARG_NDATA:  return "cannot return the number of tracers";
    case EZMOCK_ERR_ARG_FNAME:  return "invalid file name";
    case EZMOCK_ERR_ARG_RSD:    return "invalid RSD factor";
    case EZMOCK_ERR_COS_GROWTH: return "cannot obtain cosmic growth parameters";
    case EZMOCK_ERR_PK_FINITE:  return "infinite value detected";
    case EZMOCK_ERR_PK_NONPOS:  return "non-positive value detected";
    case EZMOCK_ERR_PK_NONASC:  return "non-ascending k array detected";
    case EZMOCK_ERR_PK_RANGE:   return "k range insufficient for density field";
    case EZMOCK_ERR_PK_NBIN:    return "too few k bins available for the field";
    case EZMOCK_ERR_PK_MODBAO:  return "invalid P(k) after BAO modification";
    case EZMOCK_ERR_RNG_SET:    return "failed to setup the random generator";
    case EZMOCK_ERR_RNG_RESET:  return "random generator reseting failed";
    case EZMOCK_ERR_RNG_JUMP:   return "random generator jumping ahead failed";
    case EZMOCK_ERR_PAR_COSMO:  return "invalid cosmological parameters";
    case EZMOCK_ERR_PAR_RCUT:   return "invalid density threshold parameter";
    case EZMOCK_ERR_PAR_REXP:   return "invalid exponential bias parameter";
    case EZMOCK_ERR_PAR_PBASE:  return "invalid base number for PDF mapping";
    case EZMOCK_ERR_PAR_SIGV:   return "invalid parameter for random motions";
    case EZMOCK_ERR_RHO_USED:   return "the density field has been overwritten";
    case EZMOCK_ERR_RHO_LESS:   return "not enough cells to host all tracers";
    case EZMOCK_ERR_RHO_PBASE:  return "PDF implies too many tracers per cell";
    case EZMOCK_ERR_RHO_NPART:  return "too many particles per cell";
    case EZMOCK_ERR_FFT_INIT:   return "failed to initialise FFTW with OpenMP";
    case EZMOCK_ERR_FILE:       return "failed to write to the output file";
    case EZMOCK_ERR_UNKNOWN:    return "unknown error";
    case EZMOCKB200_ERR_SCRATCH_SIZE:
      return "draw count exceeds the static scratch of the no-allocation fill";
    default:                    return "unregistered error code";
  }
}

// ---------------------------------------------------------------- extensions
int EZmockB200_set_option(EZMOCK *ez, const int option, const long value,
    int *err) {
  if (!err) return EZMOCK_ERR_ARG_ECODE;
  if (*err != EZMOCK_SUCCESS) return *err;
  if (!ez) return (*err = EZMOCK_ERR_ARG_EZ);
  EzMesh *m = MESH(ez);
  switch (option) {
    case EZMOCKB200_OPT_CIC_MODE: m->cic_mode = value ? 1 : 0; return 0;
    case EZMOCKB200_OPT_TIMING: m->timing = value ? 1 : 0; return 0;
    case EZMOCKB200_OPT_DEVICE:
      if (m->spec[0] || value < 0) return (*err = EZMOCK_ERR_ARG_PARAMS);
      m->device = (int) value;
      return 0;
    case EZMOCKB200_OPT_SEED:
      if (value <= 0) return (*err = EZMOCK_ERR_ARG_SEED);
      RNG(ez)->seed = (uint64_t) value;
      return 0;
    case EZMOCKB200_OPT_HOST_POOL:
      if (value < 0) return (*err = EZMOCK_ERR_ARG_PARAMS);
      m->hpool_mib = value ? value : -1;
      if (!value) {
        delete (HostPool *) m->hpool;
        m->hpool = nullptr;
      }
      return 0;
    case EZMOCKB200_OPT_CIC_HALO:
      if (value != 2 && value != 3) return (*err = EZMOCK_ERR_ARG_PARAMS);
      m->cic_oh = (int) value;
      m->cic_oh_set = true;               // not replaced by the last field's count
      return 0;
    case EZMOCKB200_OPT_CIC_TILE:
      if (value != 16 && value != 32) return (*err = EZMOCK_ERR_ARG_PARAMS);
      m->cic_legacy = value == 16;
      return 0;
    case EZMOCKB200_OPT_FFT_TMA:
      if (value != 0 && value != 1) return (*err = EZMOCK_ERR_ARG_PARAMS);
      m->fft_tma = value == 1;
      return 0;
    case EZMOCKB200_OPT_FFT_TMA_I:
      if (value != 0 && value != 1) return (*err = EZMOCK_ERR_ARG_PARAMS);
      m->fft_tma_i = value == 1;
      return 0;
    case EZMOCKB200_OPT_SELECT_SORT:
      if (value != 0 && value != 1) return (*err = EZMOCK_ERR_ARG_PARAMS);
      m->sel_sort = value == 1;
      return 0;
    default: return (*err = EZMOCK_ERR_ARG_PARAMS);
  }
}

int EZmockB200_stage_times(EZMOCK *ez, double *ms, const int n) {
  if (!ez || !ms) return 0;
  EzMesh *m = MESH(ez);
  if (!m->timing || m->device < 0) return 0;
  cudaSetDevice(m->device);
  cudaStreamSynchronize(m->stream);
  int k = 0;
  for (int s = 0; s < ST_NSTAGE && k < n; s++, k++) {
    float t = 0;
    if (m->ev_used[s] && EZ_CUDA_OK(cudaEventElapsedTime(&t, m->ev[2 * s], m->ev[2 * s + 1])))
      ms[k] = t;
    else {
      cudaGetLastError();
      ms[k] = -1;
    }
  }
  return k;
}

int EZmockB200_copy_field(EZMOCK *ez, const int which, real *out, int *err) {
  if (!err) return EZMOCK_ERR_ARG_ECODE;
  if (*err != EZMOCK_SUCCESS) return *err;
  if (!ez) return (*err = EZMOCK_ERR_ARG_EZ);
  if (!out) return (*err = EZMOCK_ERR_ARG_NULL);
  EzMesh *m = MESH(ez);
  if (!m->have_field) return (*err = EZMOCK_ERR_ARG_MESH);
  const real *src = nullptr;
  if (which >= 0 && which < 3) src = m->psi[which];
  else if (which == 3) src = m->rho;
  else if (which >= 4 && which < 7) src = m->paint[which - 4];
  else return (*err = EZMOCK_ERR_ARG_PARAMS);
  cudaSetDevice(m->device);
  if (which >= 4 && m->paint_il) {
    // the interleaved grids: component which - 4 of each cell's four values
    // (a strided copy; this accessor is for tests and inspection)
    if (!EZ_CUDA_OK(cudaMemcpy2DAsync(out, sizeof(real), m->pq + (which - 4), 4 * sizeof(real),
            sizeof(real), m->N, cudaMemcpyDeviceToHost, m->stream)) ||
        !EZ_CUDA_OK(cudaStreamSynchronize(m->stream)))
      return (*err = EZMOCK_ERR_UNKNOWN);
    return 0;
  }
  if (!EZ_CUDA_OK(cudaMemcpyAsync(out, src, m->N * sizeof(real), cudaMemcpyDeviceToHost, m->stream)) ||
      !EZ_CUDA_OK(cudaStreamSynchronize(m->stream)))
    return (*err = EZMOCK_ERR_UNKNOWN);
  return 0;
}

int EZmockB200_populate_device(EZMOCK *ez, const real *params,
    const size_t nexp, size_t *ntracer, int *err) {
  if (!err) return EZMOCK_ERR_ARG_ECODE;
  if (*err != EZMOCK_SUCCESS) return *err;
  if (!ez) return (*err = EZMOCK_ERR_ARG_EZ);
  if (!params) return (*err = EZMOCK_ERR_ARG_PARAMS);
  return run_populate(ez, params, nexp, false, ntracer, err);
}

int EZmockB200_copy_catalog(EZMOCK *ez, real *x, real *y, real *z, real *vx,
    real *vy, real *vz, const size_t n, int *err) {
  if (!err) return EZMOCK_ERR_ARG_ECODE;
  if (*err != EZMOCK_SUCCESS) return *err;
  if (!ez) return (*err = EZMOCK_ERR_ARG_EZ);
  EzMesh *m = MESH(ez);
  if (!m->cat || n != m->cat_n) return (*err = EZMOCK_ERR_ARG_NDATA);
  real *dst[6] = {x, y, z, vx, vy, vz};
  cudaSetDevice(m->device);
  for (int i = 0; i < 6; i++) {
    if (!dst[i]) return (*err = EZMOCK_ERR_ARG_NULL);
    if (!EZ_CUDA_OK(cudaMemcpyAsync(dst[i], m->cat + (size_t) i * n, n * sizeof(real),
            cudaMemcpyDeviceToHost, m->stream)))
      return (*err = EZMOCK_ERR_UNKNOWN);
  }
  if (!EZ_CUDA_OK(cudaStreamSynchronize(m->stream))) return (*err = EZMOCK_ERR_UNKNOWN);
  return 0;
}

int EZmockB200_select_counts(EZMOCK *ez, const real *rhot,
    const size_t *hist, size_t *pdf, const int nmax, size_t *ncell,
    size_t *ntot, int16_t *nt, int *err) {
  if (!err) return EZMOCK_ERR_ARG_ECODE;
  if (*err != EZMOCK_SUCCESS) return *err;
  if (!ez) return (*err = EZMOCK_ERR_ARG_EZ);
  if (!rhot || !hist || !pdf || !ncell || !ntot || !nt) return (*err = EZMOCK_ERR_ARG_NULL);
  if (nmax <= 0 || nmax > EZ_MAX_NT) return (*err = EZMOCK_ERR_ARG_PARAMS);
  EzMesh *m = MESH(ez);
  if (!m->have_field) return (*err = EZMOCK_ERR_ARG_MESH);
  cudaSetDevice(m->device);
  unsigned long long h[EZ_NLOGB];
  for (int i = 0; i < EZ_NLOGB; i++) h[i] = hist[i];
  // staging for the counts: the draw buffer holds >= Ngrid^3 32-bit words
  int16_t *d_nt = (int16_t *) m->draws;
  if (!EZ_CUDA_OK(cudaMemcpyAsync(m->spec[0], rhot, m->N * sizeof(real), cudaMemcpyHostToDevice, m->stream)))
    return (*err = EZMOCK_ERR_UNKNOWN);
  int e = ez_select_counts(m, h, pdf, nmax, ncell, ntot, d_nt);
  if (e) return (*err = e);
  if (!EZ_CUDA_OK(cudaMemcpyAsync(nt, d_nt, m->N * sizeof(int16_t), cudaMemcpyDeviceToHost, m->stream)) ||
      !EZ_CUDA_OK(cudaStreamSynchronize(m->stream)))
    return (*err = EZMOCK_ERR_UNKNOWN);
  return 0;
}

int EZmockB200_rng_raw(const int randgen, const uint64_t seed,
    const uint64_t start, const uint64_t count, uint32_t *out) {
  if (!out) return EZMOCK_ERR_ARG_NULL;
  if (randgen != EZMOCK_RNG_MRG32K3A && randgen != EZMOCK_RNG_MT19937) return EZMOCK_ERR_ARG_RNG;
  EzMesh m;
  memset(&m, 0, sizeof(m));
  if (!EZ_CUDA_OK(cudaGetDevice(&m.device))) { cudaGetLastError(); return EZMOCK_ERR_UNKNOWN; }
  if (!EZ_CUDA_OK(cudaStreamCreateWithFlags(&m.stream, cudaStreamNonBlocking))) return EZMOCK_ERR_UNKNOWN;
  uint32_t *d = nullptr;
  int e = 0;
  if (!EZ_CUDA_OK(cudaMalloc(&d, (count ? count : 1) * sizeof(uint32_t)))) e = EZMOCK_ERR_MEMORY;
  if (!e) e = ez_rng_fill(&m, randgen, seed, start, count, d);
  if (!e && (!EZ_CUDA_OK(cudaMemcpyAsync(out, d, count * sizeof(uint32_t), cudaMemcpyDeviceToHost, m.stream)) ||
             !EZ_CUDA_OK(cudaStreamSynchronize(m.stream))))
    e = EZMOCK_ERR_UNKNOWN;
  if (d) cudaFree(d);
  if (m.scratch) cudaFree(m.scratch);
  if (m.rng_scratch) cudaFree(m.rng_scratch);
  cudaStreamDestroy(m.stream);
  return e;
}

// Device and stream of an instance that has no field yet.
int ensure_stream(EzMesh *m) {
  if (m->device < 0 && !EZ_CUDA_OK(cudaGetDevice(&m->device))) {
    cudaGetLastError();
    m->device = -1;
    return EZMOCK_ERR_UNKNOWN;
  }
  if (set_device(m)) return EZMOCK_ERR_UNKNOWN;
  if (!m->stream) {
    int lo = 0, hi = 0;
    cudaDeviceGetStreamPriorityRange(&lo, &hi);
    if (!EZ_CUDA_OK(cudaStreamCreateWithPriority(&m->stream, cudaStreamNonBlocking, hi)))
      return EZMOCK_ERR_UNKNOWN;
  }
  return 0;
}

int EZmockB200_powspec(EZMOCK *ez, const real *x, const real *y, const real *z,
    const real *vz, const size_t n, const double rsd_fac, const int ngrid,
    const int interlace, const double kmin, const double kmax, const int nbin,
    double *kavg, double *nmodes, double *pk0, double *pk2, int *err) {
  if (!err) return EZMOCK_ERR_ARG_ECODE;
  if (*err != EZMOCK_SUCCESS) return *err;
  if (!ez) return (*err = EZMOCK_ERR_ARG_EZ);
  if (!kavg || !nmodes || !pk0 || !pk2) return (*err = EZMOCK_ERR_ARG_NULL);
  if (x && !n) return (*err = EZMOCK_ERR_ARG_NDATA);
  EzMesh *m = MESH(ez);
  int e = ensure_stream(m);
  if (!e) e = ez_powspec(m, CONF(ez)->Lbox, x, y, z, vz, n, rsd_fac, ngrid, interlace ? 1 : 0,
      kmin, kmax, nbin, kavg, nmodes, pk0, pk2);
  return (*err = e);
}

int EZmockB200_cic_pdf(EZMOCK *ez, const real *x, const real *y, const real *z,
    const real *vz, const size_t n, const double rsd_fac, const int ngrid,
    const int nbin, double *pdf, int *err) {
  if (!err) return EZMOCK_ERR_ARG_ECODE;
  if (*err != EZMOCK_SUCCESS) return *err;
  if (!ez) return (*err = EZMOCK_ERR_ARG_EZ);
  if (!pdf) return (*err = EZMOCK_ERR_ARG_NULL);
  EzMesh *m = MESH(ez);
  int e = ensure_stream(m);
  if (!e) e = ez_cic_pdf(m, CONF(ez)->Lbox, x, y, z, vz, n, rsd_fac, ngrid, nbin, pdf);
  return (*err = e);
}

int EZmockB200_sync(EZMOCK *ez) {
  if (!ez) return EZMOCK_ERR_ARG_EZ;
  EzMesh *m = MESH(ez);
  if (m->device < 0 || !m->stream) return 0;
  cudaSetDevice(m->device);
  return EZ_CUDA_OK(cudaStreamSynchronize(m->stream)) ? 0 : EZMOCK_ERR_UNKNOWN;
}

int EZmockB200_real_size(void) { return (int) sizeof(real); }

long long EZmockB200_launch_count(void) { return g_launches.load(); }

int EZmockB200_select_path(EZMOCK *ez) { return ez ? MESH(ez)->sel_path : -1; }

int EZmockB200_mark(EZMOCK *ez, const int slot) {
  if (!ez || slot < 0 || slot >= 8) return EZMOCK_ERR_ARG_PARAMS;
  EzMesh *m = MESH(ez);
  if (m->device < 0 || !m->stream) return EZMOCK_ERR_ARG_MESH;
  cudaSetDevice(m->device);
  if (!m->mark[slot] && !EZ_CUDA_OK(cudaEventCreate(&m->mark[slot]))) return EZMOCK_ERR_UNKNOWN;
  return EZ_CUDA_OK(cudaEventRecord(m->mark[slot], m->stream)) ? 0 : EZMOCK_ERR_UNKNOWN;
}

int EZmockB200_elapsed(EZMOCK *ez, const int a, const int b, double *ms) {
  if (!ez || !ms || a < 0 || a >= 8 || b < 0 || b >= 8) return EZMOCK_ERR_ARG_PARAMS;
  EzMesh *m = MESH(ez);
  if (!m->mark[a] || !m->mark[b]) return EZMOCK_ERR_ARG_PARAMS;
  cudaSetDevice(m->device);
  float t = 0;
  if (!EZ_CUDA_OK(cudaEventSynchronize(m->mark[b])) ||
      !EZ_CUDA_OK(cudaEventElapsedTime(&t, m->mark[a], m->mark[b])))
    return EZMOCK_ERR_UNKNOWN;
  *ms = t;
  return 0;
}

}  // extern "C"
