/*
 * ezref_access.c -- stage-level access to the reference's own libEZmock
 * (TEST INFRASTRUCTURE).  oracle/Makefile builds this translation unit in
 * place of the reference's pop_tracer.c: it includes that file unchanged from
 * the reference tree, so the static stages it defines (eval_pdf, bias_model,
 * n_tracer_in_cell) can be run one at a time and their intermediate fields
 * compared with the oracle restatement and with the GPU library.
 */
#include "pop_tracer.c"
#include <string.h>

int ezref_real_size(void) { return (int) sizeof(real); }

/* 0..2: psi[d], 3: rho (dens_field.c:401-406). */
const void *ezref_mesh_ptr(EZMOCK *ez, int which) {
  if (!ez || !ez->mesh) return NULL;
  EZMOCK_MESH *m = (EZMOCK_MESH *) ez->mesh;
  switch (which) {
    case 0: case 1: case 2: return m->psi[which];
    case 3: return m->rho;
    default: return NULL;
  }
}

double ezref_growth2(EZMOCK *ez) { return ((EZMOCK_COSMO *) ez->cosmo)->growth2; }
double ezref_vfac(EZMOCK *ez) { return ((EZMOCK_COSMO *) ez->cosmo)->vfac; }

/* eval_pdf + bias_model + n_tracer_in_cell of the reference
   (pop_tracer.c:1175-1194) on the current density field. */
int ezref_bias_select(EZMOCK *ez, const real *params, size_t nexp,
    real *rhot_out, int16_t *nt_out, size_t *hist_out, size_t *pdf_out,
    int *nmax, size_t *ncell, size_t *ntot, int *err) {
  EZMOCK_CONF *conf = (EZMOCK_CONF *) ez->conf;
  EZMOCK_MESH *mesh = (EZMOCK_MESH *) ez->mesh;
  const size_t num = (size_t) conf->Ng * conf->Ng * conf->Ng;
  EZMOCK_PDF *pdf = EZmock_pdf_init();
  if (!pdf) return (*err = EZMOCK_ERR_MEMORY);
  eval_pdf(ez, nexp, params[2], pdf, err);
  if (*err) { EZmock_pdf_destroy(pdf); return *err; }
  bias_model(ez, pdf, params[0], EZMOCK_MODEL_RHO_SATURATION, params[1],
      EZMOCK_MODEL_GAUSS_WIDTH, err);
  if (*err) { EZmock_pdf_destroy(pdf); return *err; }
  memcpy(rhot_out, mesh->rhot, num * sizeof(real));
  memcpy(hist_out, pdf->hist, EZMOCK_TRACER_DENSITY_NUM_LOGB_BIN * sizeof(size_t));
  n_tracer_in_cell(ez, pdf, false, err);
  if (*err) { EZmock_pdf_destroy(pdf); return *err; }
  memcpy(nt_out, mesh->nt, num * sizeof(int16_t));
  memcpy(pdf_out, pdf->pdf, pdf->nmax * sizeof(size_t));
  *nmax = pdf->nmax;
  *ncell = pdf->ncell;
  *ntot = pdf->ntot;
  EZmock_pdf_destroy(pdf);
  return 0;
}

/* n_tracer_in_cell (pop_tracer.c:359-509) of the reference on a given tracer
   density field, for exercising the selection with ties.  Needs a density
   field created first (so that the mesh owns the buffer it reuses). */
int ezref_select_from(EZMOCK *ez, const real *rhot_in, const size_t *hist_in,
    const size_t *pdf_in, int nmax, size_t ncell, size_t ntot,
    int16_t *nt_out, size_t *pdf_out, size_t *ncell_out, size_t *ntot_out,
    int *err) {
  EZMOCK_CONF *conf = (EZMOCK_CONF *) ez->conf;
  EZMOCK_MESH *mesh = (EZMOCK_MESH *) ez->mesh;
  const size_t num = (size_t) conf->Ng * conf->Ng * conf->Ng;
  if (!mesh->rhot) {
    if (mesh->rhok2) mesh->rhot = (FFT_REAL *) mesh->rhok2;
    else return (*err = EZMOCK_ERR_ARG_MESH);
  }
  EZMOCK_PDF *pdf = EZmock_pdf_init();
  if (!pdf) return (*err = EZMOCK_ERR_MEMORY);
  pdf->pdf = malloc(nmax * sizeof(size_t));
  memcpy(pdf->pdf, pdf_in, nmax * sizeof(size_t));
  memcpy(pdf->hist, hist_in, EZMOCK_TRACER_DENSITY_NUM_LOGB_BIN * sizeof(size_t));
  pdf->nmax = nmax;
  pdf->ncell = ncell;
  pdf->ntot = ntot;
  pdf->ilogb_max = ilogb((real) (1 + EZMOCK_MODEL_GAUSS_WIDTH * 5));
  memcpy(mesh->rhot, rhot_in, num * sizeof(real));
  n_tracer_in_cell(ez, pdf, false, err);
  if (!*err) {
    memcpy(nt_out, mesh->nt, num * sizeof(int16_t));
    memcpy(pdf_out, pdf->pdf, nmax * sizeof(size_t));
    *ncell_out = pdf->ncell;
    *ntot_out = pdf->ntot;
  }
  EZmock_pdf_destroy(pdf);
  return *err;
}

/* Wall time (seconds) of the three complex-to-real FFTs that
   EZmock_create_dens_field runs on an Ng^3 grid (perturb.c:361,397-398),
   through the same FFTW interface and thread count, on a zeroed spectrum:
   the FFT's share of the reference's CPU time. */
#include <time.h>
double ezref_fft_c2r_seconds(int Ng, int nthread) {
  const size_t nk = (size_t) Ng * Ng * (Ng / 2 + 1);
  FFT_CMPLX *in = FFT_MALLOC(sizeof(FFT_CMPLX) * nk);
  FFT_REAL *out = FFT_MALLOC(sizeof(FFT_REAL) * (size_t) Ng * Ng * Ng);
  if (!in || !out) { FFT_FREE(in); FFT_FREE(out); return -1; }
  memset(in, 0, sizeof(FFT_CMPLX) * nk);
  FFT_PLAN_OMP(nthread > 0 ? nthread : omp_get_max_threads());
  FFT_PLAN p = FFT_PLAN_C2R(Ng, Ng, Ng, in, out, FFT_FLAG);
  struct timespec t0, t1;
  clock_gettime(CLOCK_MONOTONIC, &t0);
  for (int d = 0; d < 3; d++) FFT_EXEC_C2R(p, in, out);
  clock_gettime(CLOCK_MONOTONIC, &t1);
  FFT_DESTROY(p);
  FFT_FREE(in);
  FFT_FREE(out);
  return (t1.tv_sec - t0.tv_sec) + 1e-9 * (t1.tv_nsec - t0.tv_nsec);
}
