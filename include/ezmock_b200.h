/*
 * ezmock_b200.h -- extensions of the B200 EZmock engine.
 *
 * These entry points have no counterpart in the reference's libEZmock; they
 * expose GPU-side controls and data for tests, benchmarks and callers that
 * keep the catalogue on the GPU.  All follow the sticky-error convention of
 * EZmock.h and return an EZmock error code.
 */
#ifndef EZMOCK_B200_EXT_H
#define EZMOCK_B200_EXT_H

#include "EZmock.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Options for EZmockB200_set_option. */
/* 0: the default assignment; 1: deterministic, bit-identical between runs
   (64-bit fixed point, 2^-50 units for the density and 2^-40 for the painted
   displacements, added with integer atomics): exact while no cell's density
   reaches 8192 and no cell's summed displacement reaches 2^23 Mpc/h, far
   above what a Zel'dovich field produces; beyond that the sums wrap. */
#define EZMOCKB200_OPT_CIC_MODE 1
#define EZMOCKB200_OPT_TIMING   2   /* 1: record per-stage CUDA-event timings */
#define EZMOCKB200_OPT_DEVICE   3   /* CUDA device ordinal (before the first field) */
#define EZMOCKB200_OPT_SEED     4   /* new random seed (> 0) for the next field */
/* Halo (2 or 3 cells) of the FP32 density assignment for the next field.
   Particles displaced farther go through a slower global-atomic pass; after
   each field the engine picks 2 when fewer than 1/4096 of the particles
   moved beyond 2 cells, else 3.  Results agree either way (FP32 rounding). */
#define EZMOCKB200_OPT_CIC_HALO 5
/* Host memory (MiB) that EZmock_populate_tracer may keep in pre-faulted
   malloc() blocks for the next catalogues (a worker thread faults them in
   while the GPU computes); 0 turns the pool off.  Default 2048. */
#define EZMOCKB200_OPT_HOST_POOL 6
/* Column tile of the FP32 density assignment: 32 (16 x 32 cells, the
   default, for grids that are multiples of 32) or 16 (16 x 16 cells).  Both
   give the same field. */
#define EZMOCKB200_OPT_CIC_TILE 7
/* FP32 transforms of the initial field along x and y: 1 (default) moves the
   tiles with the Tensor Memory Accelerator on grids of 256^3 and 512^3, 0
   with per-thread asynchronous copies.  Both give the same field. */
#define EZMOCKB200_OPT_FFT_TMA 8
/* Boundaries of the PDF bins in the tracer selection: 0 (default) from the
   candidates' value buckets, sorting only the few buckets that can hold a
   boundary; 1 from a radix sort of every candidate.  Both give the same
   counts; the first falls back to the second by itself when the buckets at
   the boundaries hold too many candidates. */
#define EZMOCKB200_OPT_SELECT_SORT 9
/* FP32 transform of the initial field along x, while EZMOCKB200_OPT_FFT_TMA
   is 1: 1 (default) moves its tiles with the Tensor Memory Accelerator on
   grids of 512^3 and 1024^3, 0 with per-thread asynchronous copies.
   Both give the same field bit for bit. */
#define EZMOCKB200_OPT_FFT_TMA_I 10

int EZmockB200_set_option(EZMOCK *ez, const int option, const long value,
    int *err);

/* Stage timings (milliseconds, CUDA events on the instance stream) of the
   most recent create/populate calls, in the order: rng, ic, fft_i, fft_j,
   fft_k, cic, bias, select, emit, vel, d2h.  Returns the number written. */
int EZmockB200_stage_times(EZMOCK *ez, double *ms, const int n);

/* Copies a device field to host memory (Ngrid^3 `real` values):
   0..2 psi_x,y,z; 3 rho; 4..6 CIC-painted displacements (un-normalised). */
int EZmockB200_copy_field(EZMOCK *ez, const int which, real *out, int *err);

/* EZmock_populate_tracer without the device-to-host copy: the catalogue
   stays in GPU memory (read it with EZmockB200_copy_catalog). */
int EZmockB200_populate_device(EZMOCK *ez, const real *params,
    const size_t nexp, size_t *ntracer, int *err);

/* Copies the last device catalogue (n = its length) into six host arrays. */
int EZmockB200_copy_catalog(EZMOCK *ez, real *x, real *y, real *z, real *vx,
    real *vy, real *vz, const size_t n, int *err);

/* The GPU selection of cells (PDF bins with the tie extension,
   libEZmock/EZmock/pop_tracer.c:359-509) applied to a given tracer-density
   field `rhot` (Ngrid^3 host values) with its log2 histogram `hist` (64
   counts) and PDF `pdf` (nmax counts, updated in place with the tie
   extension, as are *ncell and *ntot).  Writes the number of tracers of every
   cell to `nt` (Ngrid^3 values).  Needs a density field created first. */
int EZmockB200_select_counts(EZMOCK *ez, const real *rhot,
    const size_t *hist, size_t *pdf, const int nmax, size_t *ncell,
    size_t *ntot, int16_t *nt, int *err);

/* Raw 32-bit draws [start, start+count) of stream `seed` generated on the
   GPU (0: MRG32k3a, 1: MT19937). */
int EZmockB200_rng_raw(const int randgen, const uint64_t seed,
    const uint64_t start, const uint64_t count, uint32_t *out);

/* MT19937 draws [start, start+count) of stream `seed` (the stream of
   EZmockB200_rng_raw with randgen 1) written to the DEVICE buffer `d_out`
   (count uint32 values) on CUDA stream `stream` (a cudaStream_t; NULL for
   the legacy default stream), without allocating memory.  No counterpart in
   the reference: it is for callers that cannot allocate device memory on
   this path (a framework that owns the device memory through its own pool,
   or a pipeline that must not take the implicit synchronisation of
   cudaMalloc/cudaFree).  Scratch is a static device array of 324,320 bytes
   per device (129 generator states of 624 words, 128 jump descriptors, 72
   polynomial indices), which bounds one call to count <=
   EZMOCKB200_NOALLOC_MAX_DRAWS; larger counts (or start + count beyond
   2^64) return EZMOCKB200_ERR_SCRATCH_SIZE without launching anything.
   The scratch needs no zeroing.  The first call on a device (the device
   current at the call) does a synchronous set-up: the host jump tables
   (built once per process), the device addresses of the static arrays, a
   copy of the 159,744-byte jump table; make that first call before any
   stream capture.  Later calls only launch kernels on `stream` and return
   without waiting.  The set-up is kept for the life of the process: a
   device reset (cudaDeviceReset) while the library is loaded is not
   supported, since the static arrays would come back zeroed.  There is one scratch per device: calls that overlap on
   the same device race on it, so the caller serialises them (one stream,
   one host thread at a time). */
#define EZMOCKB200_NOALLOC_MAX_DRAWS ((uint64_t) 1 << 47)
#define EZMOCKB200_ERR_SCRATCH_SIZE 64
int EZmockB200_mt19937_fill_noalloc(const uint64_t seed, const uint64_t start,
    const uint64_t count, uint32_t *d_out, void *stream);

/* Clustering of a catalogue in the instance's periodic box (no counterpart
   in libEZmock: the reference calls external programs,
   example/fit/pyclustering.py:173-186, with example/fit/conf/powspec.conf).
   Catalogue: x == NULL selects the instance's last catalogue, kept on the
   GPU; otherwise x, y, z (and vz, may be NULL) are host arrays of n tracers.
   With vz and rsd_fac != 0 the z coordinate is moved to redshift space,
   z + rsd_fac vz wrapped into [0, Lbox).

   EZmockB200_powspec: power-spectrum multipoles l = 0, 2 with CIC assignment
   on ngrid^3 (even, 5-smooth), optional interlacing, window compensation,
   line of sight z, nbin linear bins of |k| in [kmin, kmax) h/Mpc; per bin the
   mean |k|, the number of modes, P0 (shot noise Lbox^3/N subtracted) and P2
   in (Mpc/h)^3.

   EZmockB200_cic_pdf: fraction of the ngrid^3 cells holding c tracers,
   c = 0 .. nbin-2, and c >= nbin-1 in the last bin (nbin <= 1024). */
int EZmockB200_powspec(EZMOCK *ez, const real *x, const real *y, const real *z,
    const real *vz, const size_t n, const double rsd_fac, const int ngrid,
    const int interlace, const double kmin, const double kmax, const int nbin,
    double *kavg, double *nmodes, double *pk0, double *pk2, int *err);
int EZmockB200_cic_pdf(EZMOCK *ez, const real *x, const real *y, const real *z,
    const real *vz, const size_t n, const double rsd_fac, const int ngrid,
    const int nbin, double *pdf, int *err);

/* Waits for all work of the instance. */
int EZmockB200_sync(EZMOCK *ez);

/* Size in bytes of `real` in this build (4 or 8). */
int EZmockB200_real_size(void);

/* Number of GPU kernels launched by the library in this process. */
long long EZmockB200_launch_count(void);

/* How the last selection of this instance found the PDF-bin boundaries:
   0 from the value buckets, 1 from the full sort (requested, or the cut in
   the last histogram bin), 2 from the full sort after the buckets at the
   boundaries held too many candidates; -1 before any selection. */
int EZmockB200_select_path(EZMOCK *ez);

/* Records CUDA event `slot` (0..7) on the instance stream, and the device
   time between two recorded slots (waits for the later one). */
int EZmockB200_mark(EZMOCK *ez, const int slot);
int EZmockB200_elapsed(EZMOCK *ez, const int a, const int b, double *ms);

#ifdef __cplusplus
}
#endif

#endif
