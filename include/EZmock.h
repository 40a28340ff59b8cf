/*
 * EZmock.h -- public C interface of the B200 EZmock engine.
 *
 * Drop-in for the reference's libEZmock interface
 * (libEZmock/EZmock/EZmock.h:38-216): the same eight functions, the same
 * argument meaning, the same sticky `int *err` convention and the same error
 * codes (libEZmock/EZmock/errmsg.h:33-88, numbered as in the default OpenMP
 * build, so EZMOCK_ERR_FFT_INIT is present).  `real` is float when the
 * including code defines SINGLE_PREC (link libEZmock_f32.so) and double
 * otherwise (link libEZmock_f64.so), as in the reference.
 *
 * The library keeps all fields in GPU memory and computes every stage on the
 * GPU; catalogue arrays returned by EZmock_populate_tracer are plain
 * malloc() memory that the caller releases with free(), as in the reference.
 */
#ifndef EZMOCK_B200_H
#define EZMOCK_B200_H

#include <stdint.h>
#include <stdbool.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#ifdef SINGLE_PREC
typedef float real;
#else
typedef double real;
#endif

/* Opaque instance: six sub-structures (libEZmock/EZmock/EZmock.h:49-56).
   `cosmo` points to {double growth2; double vfac;} as in the reference
   (libEZmock/EZmock/structs.h:56-59), which the reference CLI reads
   (src/main/run_mock.c:119-121). */
typedef struct {
  void *conf;
  void *rng;
  void *cosmo;
  void *pk;
  void *par;
  void *mesh;
} EZMOCK;

/* Random number generators (libEZmock/EZmock/save_res.c:138). */
#define EZMOCK_RNG_MRG32K3A 0
#define EZMOCK_RNG_MT19937  1

/* Error codes (libEZmock/EZmock/errmsg.h:33-88). */
enum {
  EZMOCK_SUCCESS = 0,
  EZMOCK_ERR_MEMORY,
  EZMOCK_ERR_ARG_ECODE,
  EZMOCK_ERR_ARG_EZ,
  EZMOCK_ERR_ARG_COSMO,
  EZMOCK_ERR_ARG_PK,
  EZMOCK_ERR_ARG_MESH,
  EZMOCK_ERR_ARG_LBOX,
  EZMOCK_ERR_ARG_NGRID,
  EZMOCK_ERR_ARG_RNG,
  EZMOCK_ERR_ARG_SEED,
  EZMOCK_ERR_ARG_THREAD,
  EZMOCK_ERR_ARG_NULL,
  EZMOCK_ERR_ARG_NBIN,
  EZMOCK_ERR_ARG_PARAMS,
  EZMOCK_ERR_ARG_LOWEXP,
  EZMOCK_ERR_ARG_HIEXP,
  EZMOCK_ERR_ARG_NDATA,
  EZMOCK_ERR_ARG_FNAME,
  EZMOCK_ERR_ARG_RSD,
  EZMOCK_ERR_COS_GROWTH,
  EZMOCK_ERR_PK_FINITE,
  EZMOCK_ERR_PK_NONPOS,
  EZMOCK_ERR_PK_NONASC,
  EZMOCK_ERR_PK_RANGE,
  EZMOCK_ERR_PK_NBIN,
  EZMOCK_ERR_PK_MODBAO,
  EZMOCK_ERR_RNG_SET,
  EZMOCK_ERR_RNG_RESET,
  EZMOCK_ERR_RNG_JUMP,
  EZMOCK_ERR_PAR_COSMO,
  EZMOCK_ERR_PAR_RCUT,
  EZMOCK_ERR_PAR_REXP,
  EZMOCK_ERR_PAR_PBASE,
  EZMOCK_ERR_PAR_SIGV,
  EZMOCK_ERR_RHO_USED,
  EZMOCK_ERR_RHO_LESS,
  EZMOCK_ERR_RHO_PBASE,
  EZMOCK_ERR_RHO_NPART,
  EZMOCK_ERR_FFT_INIT,
  EZMOCK_ERR_FILE,
  EZMOCK_ERR_UNKNOWN
};

/* Replaces EZmock_init (libEZmock/EZmock/EZmock.h:76-77,
   libEZmock/EZmock/EZmock.c:41-124).  Validation and error codes as in the
   reference; `nthread` (0 = all) sizes host-side work only.  No GPU memory
   is touched until the first field is created. */
EZMOCK *EZmock_init(const double Lbox, const int Ngrid, const int randgen,
    const uint64_t seed, const int nthread, int *err);

/* Replaces EZmock_set_cosmology (libEZmock/EZmock/EZmock.h:98-100,
   libEZmock/EZmock/cosmology.c:121-158), FP64 on the host. */
int EZmock_set_cosmology(EZMOCK *ez, const double pk_norm, const double fHa,
    const bool eval, const double z, const double z_pk, const double Omega_m,
    const double Omega_nu, const double w, int *err);

/* Replaces EZmock_setup_linear_pk (libEZmock/EZmock/EZmock.h:119-121,
   libEZmock/EZmock/linear_pk.c:75-183); the spline table is uploaded to the
   GPU in FP64. */
int EZmock_setup_linear_pk(EZMOCK *ez, const double *k, const int n,
    const double *Pk, const double *Pnw, const double mBAO, const bool logint,
    int *err);

/* Replaces EZmock_create_dens_field (libEZmock/EZmock/EZmock.h:144-145,
   libEZmock/EZmock/dens_field.c:337-432): initial field, three Zel'dovich
   displacement fields and the CIC density, all on the GPU.  `psi` / `delta`
   are host arrays of Ngrid^3 `real` values; they are copied to the GPU during
   the call (with deepcopy == false the library keeps no reference to them). */
int EZmock_create_dens_field(EZMOCK *ez, real *psi[3], bool deepcopy,
    real *delta, const bool fixamp, const bool iphase, int *err);

/* Replaces EZmock_populate_tracer (libEZmock/EZmock/EZmock.h:170-172,
   libEZmock/EZmock/pop_tracer.c:1140-1219).  The six arrays are malloc()'d
   host memory owned by the caller. */
int EZmock_populate_tracer(EZMOCK *ez, const real *params, const size_t nexp,
    const bool att_part, size_t *ntracer, real **x, real **y, real **z,
    real **vx, real **vy, real **vz, int *err);

/* Replaces EZmock_write_ascii (libEZmock/EZmock/EZmock.h:196-198,
   libEZmock/EZmock/save_res.c:95-178). */
int EZmock_write_ascii(EZMOCK *ez, const real *x, const real *y, const real *z,
    const real *vx, const real *vy, const real *vz, const size_t ntracer,
    const double rsd_fac, const bool header, const char *fname, int *err);

/* Replaces EZmock_destroy (libEZmock/EZmock/EZmock.h:206,
   libEZmock/EZmock/EZmock.c:132-142); also releases the GPU buffers. */
void EZmock_destroy(EZMOCK *ez);

/* Replaces EZmock_errmsg (libEZmock/EZmock/EZmock.h:216,
   libEZmock/EZmock/errmsg.c:33-72). */
const char *EZmock_errmsg(const int err);

#ifdef __cplusplus
}
#endif

#endif
