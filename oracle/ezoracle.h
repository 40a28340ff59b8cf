/*
 * ezoracle.h -- CPU restatement of the EZmock hot path (TEST INFRASTRUCTURE).
 *
 * This is the checker the GPU library is compared against.  It restates, in
 * serial order, the algorithm of the reference's libEZmock (each function
 * cites the reference file:line it follows) on top of the oracle prand and
 * the oracle CPU FFT.  It is pinned against the reference's own sources,
 * built by oracle/Makefile into oracle/_ref/, by the CPU tests.
 *
 * Nothing in the product (ezmock_b200/, include/) may call into this file.
 *
 * `real` follows the reference (libEZmock/EZmock/EZmock.h:38-42): float when
 * compiled with -DSINGLE_PREC, double otherwise.
 */
#ifndef EZ_ORACLE_H
#define EZ_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef SINGLE_PREC
typedef float real;
#else
typedef double real;
#endif

/* Linear P(k) spline table (libEZmock/EZmock/structs.h:63-71). */
typedef struct {
  int n, log;
  double kmin, kmax;
  double k[8192], P[8192], P2[8192];
} ezo_pk;

int ezo_real_size(void);

/* cosmology.c:121-158 (eval = true) */
int ezo_growth(double z, double z_pk, double Om, double Onu, double w,
    double *growth2, double *vfac);

/* linear_pk.c:75-183 */
int ezo_pk_setup(ezo_pk *pk, int Ng, double Lbox, double growth2,
    const double *k, int n, const double *P, const double *Pnw, double mBAO,
    int logint);
/* linear_pk.c:194-202 */
double ezo_pk_interp(const ezo_pk *pk, double k);

/* perturb.c:78-359: Fourier-space field before the k_i multiplications,
   Ng x Ng x (Ng/2+1) complex values (interleaved). */
int ezo_ic_spectrum(const ezo_pk *pk, int Ng, double Lbox, int rng,
    uint64_t seed, int fixamp, int iphase, real *rhok);
/* perturb.c:361-398: psi_d = c2r(rhok * k_d) */
void ezo_disp_from_spectrum(int Ng, const real *rhok, real *psi0, real *psi1,
    real *psi2, int nthread);
/* perturb.c:456-604 (white-noise input) */
void ezo_disp_whitenoise(const ezo_pk *pk, int Ng, double Lbox,
    const real *delta, real *psi0, real *psi1, real *psi2, int nthread);
/* dens_field.c:233-310 */
void ezo_cic(int Ng, double Lbox, const real *psi0, const real *psi1,
    const real *psi2, real *rho);

/* pop_tracer.c:94-133; pdf has room for 1025 entries. */
int ezo_eval_pdf(int Ng, size_t nexp, real pbase, size_t *pdf, int *nmax,
    size_t *ncell, size_t *ntot);
/* pop_tracer.c:149-348 (serial semantics, :291-347) */
int ezo_bias(int Ng, int rng, uint64_t seed, const real *rho, real rho_c,
    real rho_exp, size_t ncell, real *rhot, size_t *hist, size_t *nvalid);
/* pop_tracer.c:359-509: per-cell tracer numbers; pdf/ncell/ntot updated
   with the tie extension. */
int ezo_select(int Ng, const real *rhot, const size_t *hist, size_t *pdf,
    int nmax, size_t *ncell, size_t *ntot, int16_t *nt);
/* pop_tracer.c:894-994 (tracers without host particles) */
int ezo_positions(int Ng, double Lbox, int rng, uint64_t seed,
    const int16_t *nt, size_t ntot, real *x, real *y, real *z);
/* pop_tracer.c:593-683 */
void ezo_paint(int Ng, double Lbox, const real *psi0, const real *psi1,
    const real *psi2, const real *rho, int dim, real *out);
/* pop_tracer.c:697-753 */
void ezo_assign_vel(int Ng, double Lbox, double vfac, const real *painted,
    const real *rho, size_t n, const real *x, const real *y, const real *z,
    real *v);
/* pop_tracer.c:1043-1113 (serial semantics, :1093-1112) */
void ezo_vel_scatter(int Ng, int rng, uint64_t seed, size_t n, real sigma_v,
    real *vx, real *vy, real *vz);
/* save_res.c:147-151 */
void ezo_rsd(size_t n, const real *z, const real *vz, double rsd_fac,
    double Lbox, double *zout);

/* pop_tracer.c:517-582: particles per tracer-hosting cell (nearest cell). */
int ezo_count_particles(int Ng, double Lbox, const real *psi0, const real *psi1,
    const real *psi2, const int16_t *nt, uint16_t *np);
/* pop_tracer.c:804-879: tracers attached to particles (serial selection
   sampling, draws from 4N); consumes nt and np. */
int ezo_attach(int Ng, double Lbox, int rng, uint64_t seed, double vfac,
    const real *psi0, const real *psi1, const real *psi2, int16_t *nt,
    uint16_t *np, size_t ntot, real *x, real *y, real *z, real *vx, real *vy,
    real *vz, size_t *iv);

/* Whole EZmock_populate_tracer (pop_tracer.c:1140-1219).
   Arrays x..vz must hold `cap` entries; returns 0 or an EZmock error code. */
int ezo_populate(int Ng, double Lbox, int rng, uint64_t seed, double vfac,
    const real *psi0, const real *psi1, const real *psi2, const real *rho,
    const real *params, size_t nexp, int att_part, size_t cap, size_t *ntracer,
    real *x, real *y, real *z, real *vx, real *vy, real *vz);

/* Raw 32-bit draws of a stream (for RNG parity tests). */
void ezo_rng_raw(int rng, uint64_t seed, uint64_t start, uint64_t count,
    uint32_t *out);

#endif
