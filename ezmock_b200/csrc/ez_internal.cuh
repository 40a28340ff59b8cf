// ez_internal.cuh -- shared declarations of the B200 EZmock engine.
//
// One library per precision: libEZmock_f32.so is built with -DSINGLE_PREC
// (real = float), libEZmock_f64.so without (real = double), as the reference
// selects `real` at compile time (libEZmock/EZmock/EZmock.h:38-42).
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "EZmock.h"

#ifdef SINGLE_PREC
typedef float2 cplx;
#define EZ_REAL_MIN 1.175494350822287508e-38f   // FLT_MIN
#define EZ_REAL_TOL 1e-5                        // config.h:45-50
#else
typedef double2 cplx;
#define EZ_REAL_MIN 2.2250738585072014e-308     // DBL_MIN
#define EZ_REAL_TOL 1e-10
#endif

#define EZ_PI 0x1.921fb54442d18p+1
#define EZ_NLOGB 64                 // config.h:64
#define EZ_RHO_SAT 100              // config.h:71
#define EZ_GAUSS_WIDTH 10           // config.h:73
#define EZ_MAX_NT 1024              // config.h:59
#define EZ_MAX_GRID 65536           // config.h:56
#define EZ_MIN_TRACER 128           // config.h:58
#define EZ_MAX_PK_N 1073741824      // config.h:57
#define EZ_KMAX_BAO 0.5             // config.h:60
#define EZ_DOUBLE_TOL 1e-8          // config.h:39

// Spectral rows are padded to a multiple of this many complex values so that
// every row starts on a 128-byte boundary and FFT column tiles are uniform.
#define EZ_KPAD 16

// ---- sub-structures of EZMOCK (layouts of the first members follow
//      libEZmock/EZmock/structs.h:43-105 where callers may read them) ----
struct EzConf {
  int nthread;
  int Ng;
  double Lbox;
};

struct EzRng {
  void *unused;            // the reference keeps its prand_t* here
  int ran;                 // EZMOCK_RNG_MRG32K3A / EZMOCK_RNG_MT19937
  uint64_t seed;
};

struct EzCosmo {
  double growth2;
  double vfac;
};

struct EzPk {
  int n;
  bool log;
  double kmin, kmax;
  double *k, *P, *P2;      // host copies
  double *d_tab;           // device: k[n], P[n], P2[n]
};

struct EzPar {
  double bao_enhance, rho_c, rho_exp, pdf_base, sigma_v;
};

// Per-stage device timings of the last calls (milliseconds).
enum EzStage {
  ST_RNG_IC = 0, ST_IC, ST_FFT_I, ST_FFT_J, ST_FFT_K, ST_CIC,
  ST_BIAS, ST_SELECT, ST_EMIT, ST_VEL, ST_D2H, ST_NSTAGE
};

struct EzMesh {
  bool rho_replaced, psi_ref, fixamp, iphase;
  bool have_field;         // psi and rho on the device are valid
  int device;
  cudaStream_t stream;
  cudaEvent_t ev[2 * ST_NSTAGE];
  bool ev_used[ST_NSTAGE];
  int timing;              // record per-stage events
  cudaEvent_t mark[8];     // caller-placed events on the instance stream
  int cic_mode;            // 0: float atomics, 1: deterministic fixed-point
  int cic_oh;              // halo of the owner-computes CIC (2; otherwise 3)
  bool cic_oh_set;         // cic_oh set by the caller for the next field
  bool cic_legacy;         // FP32 CIC on 16 x 16 tiles instead of 16 x 32
  bool fft_tma;            // FP32 FFT passes I and J through TMA-staged tiles
  bool fft_tma_i;           // FP32 FFT pass I through TMA-staged tiles (with fft_tma)
  bool sel_sort;           // selection boundaries from a full radix sort
  int sel_path;            // last selection: 0 buckets, 1 sort, 2 buckets then sort

  int Ng;
  size_t N;                // Ng^3
  int Nk, Nkp;             // Ng/2+1 and its padded length
  size_t Nspec;            // Ng*Ng*Nkp
  real *psi[3];
  real *rho;
  real *paint[3];          // CIC of psi_d (un-normalised momenta)
  // (FP32) the same grids interleaved with the density, (q0, q1, q2, rho) per
  // cell in 4 N reals (the block that holds paint[]), written instead of
  // paint[] by the 16 x 32 tile assignment when paint_il is set
  real *pq;
  bool paint_il;
  cplx *spec[3];
  uint32_t *draws;
  size_t draws_cap;
  void *scratch;           // general scratch (block sums, histograms, ...)
  size_t scratch_cap;
  void *rng_scratch;       // skip-ahead states of the MT19937 streams
  size_t rng_scratch_cap;
  struct EzRange { uint64_t start, cap; int l, P; size_t first; bool side; };
  EzRange rng_prep[4];     // P chunks of 2^l; states in rng_side when `side`
  int rng_nprep;           // prepared stream ranges (ez_rng_prepare)
  size_t rng_prep_end;     // first free state slot after them
  // side stream: the population stages' random streams for the current seed,
  // prepared while the field is being created (ez_rng_side_prepare)
  cudaStream_t side;
  cudaEvent_t ev_main, ev_side, ev_pop;
  uint32_t *rng_side;      // chunk states of the side ranges
  size_t rng_side_cap;     // bytes
  uint32_t *draws_bias;    // draws of side range 0 (the bias stage)
  size_t draws_bias_cap;   // uint32 values
  uint32_t *draws_pop;     // draws of side ranges 1 and 2 (positions, dispersion)
  size_t draws_pop_cap;    // uint32 values
  bool pre_valid;
  int pre_ran, pre_n;
  uint64_t pre_seed, pre_bias_n;
  uint64_t pre_pop_n[2];   // draws of ranges 1, 2 generated into draws_pop (ez_rng_side_pop)
  bool pop_pending;        // that generation may still read prepared states
  EzRange pre[3];
  size_t pop_hint;         // largest tracer capacity of the last field's populations
  bool pop_hint_reset;     // the next population starts a new field's maximum
  void *est;               // clustering-estimator buffer (ez_pk.cu)
  size_t est_cap;
  void *att;               // attach-to-particle stage buffer (ez_pop.cu)
  size_t att_cap;
  unsigned long long *fixacc;   // deterministic CIC accumulators (4 x N)
  double *pkq;             // interpolated P(k) by integer k^2 (3 (Ng/2)^2 + 1)
  void *stats;             // EzCicStats on the device
  bool psimax_valid;       // stats->psimax_bits holds max |psi| of the fields
  real *cat;               // device catalogue (6 x cap)
  size_t cat_cap;
  size_t cat_n;            // length of the last catalogue (array stride)
  real *h_stage;           // pinned host staging for the catalogue
  unsigned long long *h_small;  // pinned host staging for small uploads (EZ_MAX_NT words)
  unsigned int *h_cic;     // pinned: the last CIC's nfar2, read without waiting
  cudaEvent_t ev_cic;      // h_cic written
  size_t h_stage_cap;
  cudaEvent_t d2h_ev[4];   // staging buffers ready
  cudaStream_t cpy;        // catalogue copy-out
  cudaEvent_t ev_pos;      // positions of the catalogue final (ez_populate)
  cudaEvent_t ev_cat;      // whole catalogue final
  void *hpool;             // pre-faulted host blocks for catalogues (ez_host.cu)
  long hpool_mib;          // bytes the pool may hold, MiB (0: default; < 0: off)
};

// Device-side statistics of the displacement/density assignment.
struct EzCicStats {
  unsigned int psimax_bits;   // max |psi| over the three fields (float bits)
  unsigned int nlist;         // far-displaced particles listed for fixup
  unsigned int nfar2;         // particles displaced by more than 2 cells on some axis
  unsigned int tma_err;       // a TMA-staged FFT pass gave up waiting (never expected)
};

// ---- error helpers ----
#define EZ_CUDA_OK(call) (cudaSuccess == (call))

// ---- FFT (ez_fft.cu) ----
// Forward (sign -1, unnormalised) r2c of an Ng^3 real grid into half-complex
// rows padded to Nkp values; Ng as accepted by ez_fft_supported.
int ez_fft_r2c(int dev, cudaStream_t st, const real *in, cplx *out, int Ng, int Nkp);
bool ez_fft_supported(int Ng);

// ---- clustering estimators (ez_pk.cu) ----
// Catalogue: the instance's last catalogue on the device (x == NULL) or host
// arrays of n tracers (vz may be NULL: no redshift-space shift).
int ez_powspec(EzMesh *m, double L, const real *x, const real *y, const real *z,
    const real *vz, size_t n, double rsd, int Ng, int interlace, double kmin,
    double kmax, int nbin, double *kavg, double *nmodes, double *p0, double *p2);
int ez_cic_pdf(EzMesh *m, double L, const real *x, const real *y, const real *z,
    const real *vz, size_t n, double rsd, int Ng, int nbin, double *pdf);

// ---- RNG (ez_rng.cu) ----
// Raw 32-bit draws [start, start+count) of the stream seeded by `seed`.
int ez_rng_fill(EzMesh *m, int ran, uint64_t seed, uint64_t start,
    uint64_t count, uint32_t *out);
// ez_rng_fill that calls between(arg) once the work generating the draws no
// longer needs the whole GPU (MT19937: after the chunk jumps, before the
// generation), so that work launched there can share the SMs with it.
int ez_rng_fill_around(EzMesh *m, int ran, uint64_t seed, uint64_t start,
    uint64_t count, uint32_t *out, void (*between)(void *), void *arg);
// ez_rng_fill that keeps the prepared ranges (their states stay valid).
int ez_rng_fill_free(EzMesh *m, int ran, uint64_t seed, uint64_t start,
    uint64_t count, uint32_t *out);
// Prepares the ranges [starts[i], starts[i] + caps[i]) of one stream so that
// later fills of them skip the jump (MT19937 chunk states computed together).
#define EZ_RNG_MAXPREP 4
int ez_rng_prepare(EzMesh *m, int ran, uint64_t seed, const uint64_t *starts,
    const uint64_t *caps, int n);
// Draws [starts[i], starts[i] + count) of prepared range i: *res points to
// them, either in `out` (generated on the instance stream) or in the side
// stream's buffer.
int ez_rng_draws(EzMesh *m, int ran, uint64_t seed, int i, uint64_t count,
    uint32_t *out, const uint32_t **res);
// On the instance's low-priority side stream, after the instance stream's
// work so far: chunk states of the ranges [starts[i], starts[i] + caps[i])
// (MT19937) and the first `nbias` draws of range 0.  Failures only leave
// the side results unused.
void ez_rng_side_pop(EzMesh *m, int ran, uint64_t seed);
void ez_rng_side_prepare(EzMesh *m, int ran, uint64_t seed,
    const uint64_t *starts, const uint64_t *caps, int n, uint64_t nbias);
// Conversions shared by all kernels (prand definitions of the oracle):
//   MT19937  : u = x 2^-32 in [0,1); u_pos = (x + 0.5) 2^-32 in (0,1)
//   MRG32k3a : u = u_pos = x * 2.328306549295727688e-10 in (0,1)
__device__ __forceinline__ double ez_u(int ran, uint32_t x) {
  return ran ? (double) x * (1.0 / 4294967296.0)
             : (double) x * 2.328306549295727688e-10;
}
__device__ __forceinline__ double ez_upos(int ran, uint32_t x) {
  return ran ? ((double) x + 0.5) * (1.0 / 4294967296.0)
             : (double) x * 2.328306549295727688e-10;
}

// ---- stages ----
int ez_ic_spectrum(EzMesh *m, const EzPk *pk, double Lbox, int ran,
    int fixamp, int iphase, const uint32_t *draws);
int ez_whitenoise_spectrum(EzMesh *m, const EzPk *pk, double Lbox,
    const real *d_delta);
int ez_fft_c2r_psi(EzMesh *m);
int ez_cic(EzMesh *m, double Lbox);

struct EzPopResult {
  size_t ntot, ncell, nvalid;
  int err;
};
int ez_populate(EzMesh *m, int Ng, double Lbox, int ran, uint64_t seed,
    double vfac, const real *params, const size_t *pdf, int nmax,
    size_t ncell, size_t ntot, bool att_part, EzPopResult *res);

// Counts kernel launches made by the library (reported to benchmarks).
void ez_count_launch();

// ---- memory ----
int ez_mesh_alloc(EzMesh *m, int Ng);
int ez_scratch(EzMesh *m, size_t bytes);
int ez_rng_scratch(EzMesh *m, size_t bytes);
int ez_select_counts(EzMesh *m, const unsigned long long *h, size_t *pdf,
    int nmax, size_t *ncell, size_t *ntot, int16_t *d_nt);
void ez_stage_begin(EzMesh *m, int st);
void ez_stage_end(EzMesh *m, int st);
