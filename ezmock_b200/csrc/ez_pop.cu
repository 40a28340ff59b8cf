// ez_pop.cu -- tracer population on the GPU
// (libEZmock/EZmock/pop_tracer.c:149-1113, serial semantics).
//
//  1. valid cells (rho >= rho_c) counted per 4096-cell chunk, scanned, so each
//     valid cell knows its rank r in index order;
//  2. bias: pair p = r/2 takes draws 2N+2p (radius) and 2N+2p+1 (angle);
//     even r uses cos, odd r sin (gauss_rand, :70-79); rho_t = (1 -
//     exp(-min(rho,100)/rho_exp)) G with G = 1+g or exp(g); log2 histogram
//     of rho_t (:170-172, :264-270);
//  3. selection (:359-509): cells with rho_t above the histogram cut are
//     compacted, their keys sorted (LSD radix sort), and PDF bin j takes the
//     next pdf[j] cells in descending order plus every further cell equal to
//     the smallest one taken (tie extension, :436-446).  Bin j is then the
//     value interval [lo_j, lo_{j-1}), so per-cell counts follow from rho_t
//     alone;
//  4. emission (:894-994): tracer t (cell-index order) takes draws
//     5N+3t..5N+3t+2 for its position in the cell;
//  5. velocities (:593-753): mass-weighted CIC gather of the momentum grids
//     painted during the density assignment, times vfac;
//  6. dispersion (:1043-1113): tracer pair m takes draws 8N+6m..8N+6m+5 as
//     three Box-Muller pairs.
#include "ez_internal.cuh"

#include <algorithm>
#include <cstring>
#include <vector>

namespace {

constexpr int NT = 256;
constexpr int ROWS = 16;
constexpr int CH = NT * ROWS;           // cells per chunk

#ifdef SINGLE_PREC
typedef uint32_t skey_t;
__device__ __forceinline__ skey_t to_key(real v) { return ~__float_as_uint(v); }
__device__ __forceinline__ real from_key(skey_t k) { return __uint_as_float(~k); }
#else
typedef unsigned long long skey_t;
__device__ __forceinline__ skey_t to_key(real v) { return ~(skey_t) __double_as_longlong(v); }
__device__ __forceinline__ real from_key(skey_t k) { return __longlong_as_double((long long) ~k); }
#endif

// exclusive block scan over NT threads; returns the prefix, writes the total
template <typename T>
__device__ __forceinline__ T block_scan(T v, T *total, T *sw) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  T x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const T y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) sw[w] = x;
  __syncthreads();
  if (w == 0) {
    T s = (lane < (int) (blockDim.x >> 5)) ? sw[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const T y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    sw[lane] = s;                       // inclusive warp-total prefix
  }
  __syncthreads();
  const T before = (w ? sw[w - 1] : 0) + x - v;
  *total = sw[(blockDim.x >> 5) - 1];
  __syncthreads();
  return before;
}

__global__ void __launch_bounds__(NT)
valid_count_kernel(const real *__restrict__ rho, size_t N, real thres,
    unsigned long long *cnt) {
  __shared__ unsigned long long sw[32];
  unsigned long long c = 0;
  const size_t b0 = (size_t) blockIdx.x * CH;
  for (int q = 0; q < ROWS; q++) {
    const size_t id = b0 + (size_t) q * NT + threadIdx.x;
    if (id < N && !(rho[id] < thres)) c++;
  }
  unsigned long long tot;
  block_scan<unsigned long long>(c, &tot, sw);
  if (threadIdx.x == 0) cnt[blockIdx.x] = tot;
}

// single-block exclusive scan of n values (in place allowed); out[n] =
// total.  Warp w owns the w-th of 32 contiguous segments: it sums its
// segment with coalesced loads (eight in flight per lane), the warp totals
// are scanned, and each warp rescans its segment 32 values at a time.
__global__ void __launch_bounds__(1024)
scan_kernel(const unsigned long long *in, unsigned long long *out, size_t n) {
  __shared__ unsigned long long sw[32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const size_t seg = ((n + 31) / 32 + 31) & ~(size_t) 31;
  const size_t s0 = min(n, (size_t) w * seg), s1 = min(n, s0 + seg);
  unsigned long long loc = 0;
  for (size_t b = s0; b < s1; b += 8 * 32) {
    unsigned long long v[8];
#pragma unroll
    for (int u = 0; u < 8; u++) {
      const size_t g = b + (size_t) u * 32 + lane;
      v[u] = (g < s1) ? in[g] : 0ull;
    }
#pragma unroll
    for (int u = 0; u < 8; u++) loc += v[u];
  }
#pragma unroll
  for (int o = 16; o; o >>= 1) loc += __shfl_xor_sync(0xffffffffu, loc, o);
  if (lane == 0) sw[w] = loc;
  __syncthreads();
  unsigned long long run = 0, tot = 0;
  for (int k = 0; k < 32; k++) {
    const unsigned long long t = sw[k];
    run += (k < w) ? t : 0ull;
    tot += t;
  }
  __syncthreads();                               // all reads of `in` done before
  for (size_t b = s0; b < s1; b += 32) {         // in-place writes
    const size_t g = b + lane;
    const unsigned long long v = (g < s1) ? in[g] : 0ull;
    unsigned long long x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned long long y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (g < s1) out[g] = run + x - v;
    run += __shfl_sync(0xffffffffu, x, 31);
  }
  if (threadIdx.x == 0) out[n] = tot;
}

// Bin of the log2 histogram (pop_tracer.c:264-270): 5 - ilogb(v) clamped to
// [0, 63]; exactly zero goes to the last bin.
#ifdef SINGLE_PREC
// From the float's exponent field: 5 - ilogb(v) = 132 - e for a normal v;
// zero and subnormals (e = 0) give 132, clamped to the last bin, as the
// double-precision ilogb of their values does.
__device__ __forceinline__ int logb_bin(float v) {
  const int e = (int) ((__float_as_uint(v) >> 23) & 0xffu);
  return min(max(132 - e, 0), EZ_NLOGB - 1);
}
#else
__device__ __forceinline__ int logb_bin(double v) {
  if (v == 0) return EZ_NLOGB - 1;
  const int idx = 5 - ilogb(v);
  return idx < 0 ? 0 : (idx >= EZ_NLOGB ? EZ_NLOGB - 1 : idx);
}
#endif

// rho_t of the valid cells of a 4096-cell chunk (pop_tracer.c:233-300).  A
// cell's valid rank is the chunk offset plus the valid cells before it,
// found from per-warp ballots.  The valid cells are then compacted in
// shared memory (their chunk places in rank order), so the double-precision
// Box-Muller pairs (gauss_rand, pop_tracer.c:70-79: pair p takes draws 2p
// (radius) and 2p+1 (angle) of the bias range; rank 2p uses the cosine,
// 2p+1 the sine) and exps run on full warps: about half of the cells are
// valid, and a warp of mixed cells would run them for all 32 lanes.  rho_t
// goes back to cell order through the same shared array, so the stores stay
// coalesced.
__global__ void __launch_bounds__(NT)
bias_kernel(const real *__restrict__ rho, real *__restrict__ rhot, size_t N,
    real thres, double iexp, const unsigned long long *off,
    const uint32_t *__restrict__ draws, int ran, double lambda,
    unsigned long long *hist) {
  constexpr int NW = NT / 32;
  __shared__ unsigned int pre[ROWS * NW];    // valid counts, then prefixes
  __shared__ unsigned int wsum[ROWS * NW / 32];
  __shared__ unsigned int sh[EZ_NLOGB];
  __shared__ unsigned int snloc;             // valid cells of the chunk
  __shared__ real st[CH];                    // clamped rho, then rho_t (cell order)
  __shared__ uint16_t spos[CH];              // chunk place of each valid rank
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (threadIdx.x < EZ_NLOGB) sh[threadIdx.x] = 0;
  const size_t b0 = (size_t) blockIdx.x * CH;
  real r[ROWS];
  unsigned int bal[ROWS];
  // (loads interleaved with the ballots: issuing all loads first measured
  // slower here, 0.83 vs 0.64 ms at 512^3)
#pragma unroll
  for (int q = 0; q < ROWS; q++) {
    const size_t id = b0 + (size_t) q * NT + threadIdx.x;
    r[q] = (id < N) ? rho[id] : (real) 0;
    bal[q] = __ballot_sync(0xffffffffu, id < N && !(r[q] < thres));
    if (lane == 0) pre[q * NW + w] = __popc(bal[q]);
  }
  __syncthreads();
  // exclusive scan of the ROWS * NW counts (row-major: index order)
  static_assert(ROWS * NW <= 32 * 32, "scan width");
  unsigned int c = 0, incl = 0;
  if (threadIdx.x < ROWS * NW) {
    c = pre[threadIdx.x];
    incl = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned int v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += v;
    }
    if (lane == 31) wsum[w] = incl;
  }
  __syncthreads();
  if (threadIdx.x < ROWS * NW) {
    unsigned int base = 0;
    for (int k = 0; k < w; k++) base += wsum[k];
    pre[threadIdx.x] = base + incl - c;
    if (threadIdx.x == ROWS * NW - 1) snloc = base + incl;
  }
  __syncthreads();
  // cell order: clamped rho of valid cells, 0 elsewhere; rank order: places
  const unsigned int lt = (1u << lane) - 1;
#pragma unroll
  for (int q = 0; q < ROWS; q++) {
    const int pos = q * NT + threadIdx.x;
    const bool valid = (bal[q] >> lane) & 1;
    st[pos] = valid ? ((r[q] > (real) EZ_RHO_SAT) ? (real) EZ_RHO_SAT : r[q]) : (real) 0;
    if (valid) spos[pre[q * NW + w] + __popc(bal[q] & lt)] = (uint16_t) pos;
  }
  __syncthreads();
  // one Box-Muller pair per thread and step: pair p gives ranks 2p (cos)
  // and 2p+1 (sin); a rank outside the chunk's [run, run + nloc) belongs to
  // the neighbouring chunk, which computes the same pair for it.  Each place
  // is read and rewritten by the thread holding its rank only.
  const unsigned int nloc = snloc;
  if (nloc) {
    const unsigned long long run = off[blockIdx.x];
    const unsigned long long plo = run >> 1, phi = (run + nloc - 1) >> 1;
    const unsigned int npl = (unsigned int) (phi - plo + 1);
    for (unsigned int k0 = 0; k0 < npl; k0 += NT) {
      const unsigned int k = k0 + threadIdx.x;
      const bool act = k < npl;
      const unsigned long long p = plo + k;
      double g[2] = {0.0, 0.0};
      if (act) {                             // gauss_rand (pop_tracer.c:70-79)
        const double rr = -2 * log(ez_upos(ran, draws[2 * p]));
        const double th = ez_u(ran, draws[2 * p + 1]) * 2 * EZ_PI;
        const double s = lambda * sqrt(rr);
        double sn, cs;
        sincos(th, &sn, &cs);                // one argument reduction for both
        g[0] = s * cs;
        g[1] = s * sn;
      }
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const unsigned long long rank = 2 * p + h;
        const bool mine = act && rank >= run && rank < run + nloc;
        int bin = -1;
        if (mine) {
          const int pos = spos[rank - run];
          const double G = (g[h] >= 0) ? 1 + g[h] : exp(g[h]);   // pop_tracer.c:288-300
          const real t = (1 - exp((double) st[pos] * iexp)) * G;
          st[pos] = t;
          bin = logb_bin(t);
        }
        // one shared atomic per rank (at 512^3: 1.18 -> 1.11 ms for the stage
        // against one per distinct bin of the warp through __match_any_sync,
        // and 2.06 ms with a ballot per bin between the warp's extremes)
        if (mine) atomicAdd(&sh[bin], 1u);
      }
    }
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < ROWS; q++) {
    const size_t id = b0 + (size_t) q * NT + threadIdx.x;
    if (id < N) rhot[id] = st[q * NT + threadIdx.x];
  }
  if (threadIdx.x < EZ_NLOGB && sh[threadIdx.x])
    atomicAdd(hist + threadIdx.x, (unsigned long long) sh[threadIdx.x]);
}

// Candidates (rho_t >= cut) of a 4096-cell chunk are counted, one atomic per
// block reserves their slots, and their keys are written (the order of the
// candidate list is irrelevant: it is sorted next).
// Value buckets of the candidates for the boundary search below: a monotone
// map of a candidate's bits (v >= cut > 0, so its bits order as its value),
// SEL_NB buckets from the cut up; larger values share the last bucket.
constexpr int SEL_NB = 32768;

#ifdef SINGLE_PREC
typedef uint32_t ubits_t;
__device__ __forceinline__ ubits_t val_bits(real v) { return __float_as_uint(v); }
#else
typedef unsigned long long ubits_t;
__device__ __forceinline__ ubits_t val_bits(real v) { return (ubits_t) __double_as_longlong(v); }
#endif

struct SelBucket {
  ubits_t base;              // bits of the cut
  int shift;
};

__device__ __forceinline__ int sel_bucket(real v, SelBucket sb) {
  const ubits_t d = (val_bits(v) - sb.base) >> sb.shift;
  return d < (ubits_t) SEL_NB ? (int) d : SEL_NB - 1;
}

__global__ void __launch_bounds__(NT)
compact_kernel(const real *__restrict__ rhot, size_t N, real thres,
    skey_t *__restrict__ keys, unsigned long long *counter, skey_t *__restrict__ cand,
    uint16_t *__restrict__ cidx, size_t ccap, unsigned long long *__restrict__ cstart,
    unsigned int *__restrict__ ccnt) {
  // candidates are written in cell order within the chunk's range (an
  // exclusive scan of the (row, warp) ballot counts), so that emission can
  // walk them in the order of the tracers
  constexpr int NW = NT / 32;
  __shared__ unsigned int pre[ROWS * NW];
  __shared__ unsigned int wsum[ROWS * NW / 32];
  __shared__ unsigned long long sbase;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const size_t b0 = (size_t) blockIdx.x * CH;
  real v[ROWS];
  unsigned int bal[ROWS];
#pragma unroll
  for (int q = 0; q < ROWS; q++) {               // all loads first
    const size_t id = b0 + (size_t) q * NT + threadIdx.x;
    v[q] = (id < N) ? rhot[id] : (real) 0;
  }
#pragma unroll
  for (int q = 0; q < ROWS; q++) {
    const size_t id = b0 + (size_t) q * NT + threadIdx.x;
    bal[q] = __ballot_sync(0xffffffffu, id < N && !(v[q] < thres));
    if (lane == 0) pre[q * NW + w] = __popc(bal[q]);
  }
  __syncthreads();
  static_assert(ROWS * NW <= 32 * 32, "scan width");
  unsigned int c = 0, incl = 0;
  if (threadIdx.x < ROWS * NW) {
    c = pre[threadIdx.x];
    incl = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned int y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    if (lane == 31) wsum[w] = incl;
  }
  __syncthreads();
  if (threadIdx.x < ROWS * NW) {
    unsigned int base = 0;
    for (int k = 0; k < w; k++) base += wsum[k];
    pre[threadIdx.x] = base + incl - c;
    if (threadIdx.x == ROWS * NW - 1) {
      const unsigned long long tot = base + incl;
      sbase = tot ? atomicAdd(counter, tot) : 0;
      cstart[blockIdx.x] = sbase;
      ccnt[blockIdx.x] = (unsigned int) tot;
    }
  }
  __syncthreads();
  const unsigned long long off = sbase;
  const unsigned int lt = (1u << lane) - 1;
#pragma unroll
  for (int q = 0; q < ROWS; q++) {
    if ((bal[q] >> lane) & 1) {
      const unsigned long long pos = off + pre[q * NW + w] + __popc(bal[q] & lt);
      const skey_t k = to_key(v[q]);
      keys[pos] = k;
      // a second copy with the cell's place in the chunk, kept for emission
      if (pos < ccap) { cand[pos] = k; cidx[pos] = (uint16_t) (q * NT + threadIdx.x); }
    }
  }
}

// Multi-block exclusive scan for long arrays: chunk sums, a scan of the sums,
// then each chunk rescanned with its offset.  out[n] = total.
constexpr int SCAN_CHUNK = 8192;

__global__ void __launch_bounds__(1024)
chunk_sum_kernel(const unsigned long long *__restrict__ in, size_t n,
    unsigned long long *sums) {
  __shared__ unsigned long long sw[32];
  const size_t c0 = (size_t) blockIdx.x * SCAN_CHUNK;
  unsigned long long s = 0;
  for (int e = threadIdx.x; e < SCAN_CHUNK; e += 1024) {
    const size_t g = c0 + e;
    if (g < n) s += in[g];
  }
  unsigned long long tot;
  block_scan<unsigned long long>(s, &tot, sw);
  if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(1024)
chunk_scan_kernel(const unsigned long long *__restrict__ in, size_t n,
    const unsigned long long *__restrict__ offs, unsigned long long *out) {
  __shared__ unsigned long long sw[32];
  const size_t c0 = (size_t) blockIdx.x * SCAN_CHUNK;
  constexpr int PER = SCAN_CHUNK / 1024;
  unsigned long long v[PER], loc = 0;
#pragma unroll
  for (int j = 0; j < PER; j++) {
    const size_t g = c0 + (size_t) threadIdx.x * PER + j;
    v[j] = (g < n) ? in[g] : 0;
    loc += v[j];
  }
  unsigned long long tot;
  unsigned long long run = offs[blockIdx.x] + block_scan<unsigned long long>(loc, &tot, sw);
#pragma unroll
  for (int j = 0; j < PER; j++) {
    const size_t g = c0 + (size_t) threadIdx.x * PER + j;
    if (g < n) out[g] = run;
    run += v[j];
  }
}

// ---- LSD radix sort of keys (ascending), 8-bit digits ----
constexpr int SORT_NT = 256;
constexpr int SORT_PER = 8;
constexpr int TILE = SORT_NT * SORT_PER;

__global__ void __launch_bounds__(SORT_NT)
digit_hist_kernel(const skey_t *__restrict__ keys, size_t M, int shift,
    unsigned long long *counts, size_t ntiles) {
  __shared__ unsigned int h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  const size_t t0 = (size_t) blockIdx.x * TILE;
  for (int e = threadIdx.x; e < TILE; e += SORT_NT) {
    const size_t g = t0 + e;
    if (g < M) atomicAdd(&h[(keys[g] >> shift) & 255], 1u);
  }
  __syncthreads();
  counts[(size_t) threadIdx.x * ntiles + blockIdx.x] = h[threadIdx.x];
}

// Scatter of one tile by the digit at `shift`, stable: key i of the tile
// goes to the tile's start of its digit (offs, from the digit counts of all
// tiles) plus the number of keys with the same digit before it in the tile.
// Warp w takes tile positions w*32*PER + j*32 + lane (j = 0 .. PER-1, in
// order); a key's rank among equal digits comes from __match_any_sync, the
// warp's running count per digit and, after the loop, the counts of the
// warps before it.
__global__ void __launch_bounds__(SORT_NT)
digit_scatter_kernel(const skey_t *__restrict__ in, skey_t *__restrict__ out,
    size_t M, int shift, const unsigned long long *__restrict__ offs,
    size_t ntiles) {
  constexpr int NW = SORT_NT / 32;
  static_assert(SORT_NT == 256, "one thread per digit");
  __shared__ unsigned int cnt[NW][256];
  __shared__ unsigned long long base[256];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int e = threadIdx.x; e < NW * 256; e += SORT_NT) (&cnt[0][0])[e] = 0;
  base[threadIdx.x] = offs[(size_t) threadIdx.x * ntiles + blockIdx.x];
  __syncthreads();
  const size_t t0 = (size_t) blockIdx.x * TILE;
  const unsigned int lt = (1u << lane) - 1;
  skey_t k[SORT_PER];
  unsigned int r[SORT_PER];
  int dg[SORT_PER];
#pragma unroll
  for (int j = 0; j < SORT_PER; j++) {
    const size_t g = t0 + (size_t) (w * 32 * SORT_PER + j * 32 + lane);
    const bool valid = g < M;
    k[j] = valid ? in[g] : (skey_t) 0;
    const int d = valid ? (int) ((k[j] >> shift) & 255) : 256;   // 256: no key
    const unsigned int mask = __match_any_sync(0xffffffffu, d);
    r[j] = valid ? cnt[w][d] + __popc(mask & lt) : 0;
    __syncwarp();
    if (valid && !(mask & lt)) cnt[w][d] += __popc(mask);          // lowest lane
    __syncwarp();
    dg[j] = d;
  }
  __syncthreads();
  {                                      // counts of the warps before each warp
    const int d = threadIdx.x;
    unsigned int run = 0;
#pragma unroll
    for (int v = 0; v < NW; v++) {
      const unsigned int c = cnt[v][d];
      cnt[v][d] = run;
      run += c;
    }
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < SORT_PER; j++)
    if (dg[j] < 256) out[base[dg[j]] + cnt[w][dg[j]] + r[j]] = k[j];
}

// ---- boundaries of the PDF bins (one thread; pop_tracer.c:405-461) ----
struct BoundOut {
  unsigned long long ncell, ntot;
  int err;
  int nbins;                 // number of non-empty bins
  real lo[EZ_MAX_NT];        // lowest rho_t of each non-empty bin
  int ntr[EZ_MAX_NT];        // tracers per cell of that bin
  unsigned long long pdf[EZ_MAX_NT];
};

// First index in [lo, hi) of the ascending keys with a[i] > v.  The bins'
// boundaries rarely fall inside a run of ties, so the search gallops from
// lo (one load when a[lo] > v already) before bisecting: a chain of
// dependent global loads is the cost of this single-thread kernel.
__device__ size_t upper_bound_key(const skey_t *a, size_t lo, size_t hi, skey_t v) {
  size_t step = 1, base = lo;
  while (base < hi && a[base] <= v) {
    lo = base + 1;
    base = lo + step - 1 < hi ? lo + step - 1 : hi;
    step <<= 1;
  }
  hi = base;                                 // a[hi] > v, or hi is the end
  while (lo < hi) {
    const size_t mid = (lo + hi) >> 1;
    if (a[mid] <= v) lo = mid + 1; else hi = mid;
  }
  return lo;
}

__global__ void bounds_kernel(const skey_t *__restrict__ keys, size_t M,
    const unsigned long long *__restrict__ pdf, int nmax,
    unsigned long long ncell, unsigned long long ntot, BoundOut *o) {
  size_t P = 0;
  int nb = 0;
  o->err = 0;
  for (int j = 0; j < nmax; j++) {
    unsigned long long q = pdf[j];
    if (!q) { o->pdf[j] = 0; continue; }
    size_t E = P + q;
    if (E > M) { o->err = EZMOCK_ERR_UNKNOWN; return; }
    const size_t E2 = upper_bound_key(keys, E, M, keys[E - 1]);
    const unsigned long long extra = E2 - E;
    q += extra;
    ncell += extra;
    ntot += extra * (unsigned long long) (nmax - j);
    E = E2;
    o->pdf[j] = q;
    o->lo[nb] = from_key(keys[E - 1]);
    o->ntr[nb] = nmax - j;
    nb++;
    P = E;
  }
  o->nbins = nb;
  o->ncell = ncell;
  o->ntot = ntot;
}

// ---- boundaries of the PDF bins from the value buckets ----
//
// Bin j ends at rank E_j = P_j + pdf[j] (ranks in descending value order)
// and the next starts at E2_j, the rank after the ties of rank E_j - 1.  A
// run of equal values lies in one bucket, so E2_j is at most the end of the
// bucket holding rank E_j - 1.  sel_plan_kernel follows the chain with these
// bounds (P_j in [Plo, Phi]) and marks every bucket that can hold rank
// E_j - 1 for some admissible P_j; sel_gather_kernel copies the candidates of
// the marked buckets (a few thousand of millions); sel_resolve_kernel sorts
// them and runs bounds_kernel's exact chain on their ranks.  Results equal
// bounds_kernel's on the fully sorted keys; when the marked buckets hold more
// than SEL_GCAP candidates, sel_resolve_kernel asks for the full sort.
constexpr int SEL_NT = 1024;
constexpr int SEL_HB = 148;                               // bucket histogram blocks at most
constexpr int SEL_GCAP = 65536 / (int) sizeof(skey_t);   // gathered keys (64 KB)
constexpr int SEL_FALLBACK = -2;                          // BoundOut.err: sort all
constexpr size_t SEL_PLAN_SMEM = SEL_NB * sizeof(unsigned int);
constexpr size_t SEL_RESOLVE_SMEM = SEL_PLAN_SMEM + SEL_GCAP * sizeof(skey_t);

// cum[b] = candidates in buckets above b (exclusive prefix in descending
// bucket order); returns the total.  Warp w scans the 1024 buckets of places
// w*1024 .. w*1024+1023 in descending order (coalesced reads), then adds the
// counts of the warps before it.  All threads; ends with a barrier.
__device__ unsigned int sel_cum(const unsigned int *__restrict__ bh, unsigned int *cum,
    unsigned int *sw) {
  constexpr int SEG = SEL_NB / (SEL_NT / 32);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  unsigned int run = 0;
#pragma unroll 8
  for (int i = 0; i < SEG / 32; i++) {
    const int b = SEL_NB - 1 - (w * SEG + i * 32 + lane);
    const unsigned int c = bh[b];
    unsigned int x = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    cum[b] = run + x - c;
    run += __shfl_sync(0xffffffffu, x, 31);
  }
  if (lane == 0) sw[w] = run;
  __syncthreads();
  unsigned int off = 0, tot = 0;
  for (int k = 0; k < SEL_NT / 32; k++) {
    const unsigned int v = sw[k];
    off += (k < w) ? v : 0u;
    tot += v;
  }
  if (off)
    for (int i = 0; i < SEG / 32; i++) cum[SEL_NB - 1 - (w * SEG + i * 32 + lane)] += off;
  __syncthreads();
  return tot;
}

// First i in [0, n) with pred(i) (pred false then true), n if none: a
// 32-way search by one warp; every lane returns the answer.
template <class Pred>
__device__ __forceinline__ int warp_first(int n, Pred pred, int lane) {
  int lo = 0, hi = n;            // pred false below lo; true at hi (or hi = n)
  while (lo < hi) {
    const int step = (hi - lo + 31) >> 5;
    const int idx = lo + (lane + 1) * step - 1;
    const unsigned int bal = __ballot_sync(0xffffffffu, idx >= hi || pred(idx));
    if (!bal) { lo = hi; break; }
    const int f = __ffs(bal) - 1;
    const int nhi = lo + (f + 1) * step - 1;
    lo += f * step;
    hi = nhi < hi ? nhi : hi;
  }
  return lo;
}

// Bucket of rank r: the lowest b with cum[b] <= r (cum does not increase
// with b; that b is non-empty).
__device__ __forceinline__ int sel_rank_bucket(const unsigned int *cum, unsigned long long r,
    int lane) {
  return warp_first(SEL_NB, [&](int b) { return cum[b] <= r; }, lane);
}

__device__ __forceinline__ unsigned long long sel_bucket_end(const unsigned int *cum, int b,
    unsigned long long M) {
  return b > 0 ? cum[b - 1] : M;
}

// Per-block histograms of the candidates' buckets (shared-memory atomics),
// then their sum: SEL_NB counts.
__global__ void __launch_bounds__(SEL_NT)
sel_hist_kernel(const skey_t *__restrict__ keys, size_t M, SelBucket sb, unsigned int *part) {
  extern __shared__ unsigned int hb[];              // SEL_NB
  for (int e = threadIdx.x; e < SEL_NB; e += SEL_NT) hb[e] = 0;
  __syncthreads();
  const size_t per = (M + gridDim.x - 1) / gridDim.x;
  const size_t a = (size_t) blockIdx.x * per, b = min(M, a + per);
#pragma unroll 4
  for (size_t i = a + threadIdx.x; i < b; i += SEL_NT)
    atomicAdd(&hb[sel_bucket(from_key(keys[i]), sb)], 1u);
  __syncthreads();
  unsigned int *o = part + (size_t) blockIdx.x * SEL_NB;
  for (int e = threadIdx.x; e < SEL_NB; e += SEL_NT) o[e] = hb[e];
}

__global__ void __launch_bounds__(NT)
sel_reduce_kernel(const unsigned int *__restrict__ part, int nparts, unsigned int *bh) {
  const int e = blockIdx.x * NT + threadIdx.x;
  if (e >= SEL_NB) return;
  unsigned int s = 0;
#pragma unroll 8
  for (int p = 0; p < nparts; p++) s += part[(size_t) p * SEL_NB + e];
  bh[e] = s;
}

__global__ void __launch_bounds__(SEL_NT)
sel_plan_kernel(const unsigned int *__restrict__ bh, unsigned long long M,
    const unsigned long long *__restrict__ pdf, int nmax, unsigned int *mask_out) {
  extern __shared__ unsigned int cum[];             // SEL_NB
  __shared__ unsigned int sw[32];
  __shared__ unsigned int mask[SEL_NB / 32];
  __shared__ unsigned long long spdf[EZ_MAX_NT];
  for (int w = threadIdx.x; w < SEL_NB / 32; w += SEL_NT) mask[w] = 0;
  for (int j = threadIdx.x; j < nmax; j += SEL_NT) spdf[j] = pdf[j];
  sel_cum(bh, cum, sw);
  if (threadIdx.x < 32) {                           // one warp follows the chain
    const int lane = threadIdx.x;
    unsigned long long plo = 0, phi = 0;
    for (int j = 0; j < nmax; j++) {
      const unsigned long long q = spdf[j];
      if (!q) continue;
      const unsigned long long elo = plo + q;
      if (elo > M) break;                            // the exact chain fails here
      const unsigned long long ehi = min(phi + q, M);
      const int bhi = sel_rank_bucket(cum, elo - 1, lane);   // higher values, higher bucket
      const int blo = sel_rank_bucket(cum, ehi - 1, lane);
      for (int w = (blo >> 5) + lane; w <= (bhi >> 5); w += 32) {
        const int a = max(blo - 32 * w, 0), b = min(bhi - 32 * w, 31);
        mask[w] |= (b == 31 ? 0xffffffffu : ((2u << b) - 1)) & ~((1u << a) - 1);
      }
      __syncwarp();
      plo = elo;
      phi = sel_bucket_end(cum, blo, M);
    }
  }
  __syncthreads();
  for (int w = threadIdx.x; w < SEL_NB / 32; w += SEL_NT) mask_out[w] = mask[w];
}

__global__ void __launch_bounds__(NT)
sel_gather_kernel(const skey_t *__restrict__ keys, size_t M, SelBucket sb,
    const unsigned int *__restrict__ mask_g, unsigned int *gcount, skey_t *gbuf) {
  __shared__ unsigned int mask[SEL_NB / 32];
  for (int w = threadIdx.x; w < SEL_NB / 32; w += NT) mask[w] = mask_g[w];
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const size_t stride = (size_t) gridDim.x * NT;
  for (size_t b0 = (size_t) blockIdx.x * NT; b0 < M; b0 += stride) {   // block-uniform trips
    const size_t i = b0 + threadIdx.x;
    skey_t k = 0;
    bool take = false;
    if (i < M) {
      k = keys[i];
      const int b = sel_bucket(from_key(k), sb);
      take = (mask[b >> 5] >> (b & 31)) & 1u;
    }
    const unsigned int bal = __ballot_sync(0xffffffffu, take);
    if (bal) {
      unsigned int p0 = 0;
      if (lane == 0) p0 = atomicAdd(gcount, (unsigned int) __popc(bal));
      p0 = __shfl_sync(0xffffffffu, p0, 0);
      const unsigned int p = p0 + __popc(bal & ((1u << lane) - 1));
      if (take && p < (unsigned int) SEL_GCAP) gbuf[p] = k;
    }
  }
}

__global__ void __launch_bounds__(SEL_NT)
sel_resolve_kernel(const unsigned int *__restrict__ bh, unsigned long long M, SelBucket sb,
    const unsigned int *__restrict__ gcount, const skey_t *__restrict__ gbuf,
    const unsigned long long *__restrict__ pdf, int nmax, unsigned long long ncell,
    unsigned long long ntot, BoundOut *o) {
  extern __shared__ unsigned int cum[];             // SEL_NB, then the keys
  skey_t *g = reinterpret_cast<skey_t *>(cum + SEL_NB);
  __shared__ unsigned int sw[32];
  __shared__ unsigned long long spdf[EZ_MAX_NT];
  for (int j = threadIdx.x; j < nmax; j += SEL_NT) spdf[j] = pdf[j];
  const unsigned int tot = sel_cum(bh, cum, sw);
  const unsigned int G = *gcount;
  if (tot != M || G > (unsigned int) SEL_GCAP) {     // uniform over the block
    if (threadIdx.x == 0) o->err = SEL_FALLBACK;
    return;
  }
  int n2 = 1;
  while (n2 < (int) G) n2 <<= 1;
  for (int i = threadIdx.x; i < n2; i += SEL_NT) g[i] = (i < (int) G) ? gbuf[i] : ~(skey_t) 0;
  __syncthreads();
  // bitonic sort, ascending keys (descending values)
  for (int k = 2; k <= n2; k <<= 1)
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = threadIdx.x; i < n2; i += SEL_NT) {
        const int ixj = i ^ j;
        if (ixj > i) {
          const skey_t a = g[i], b = g[ixj];
          if ((a > b) == ((i & k) == 0)) { g[i] = b; g[ixj] = a; }
        }
      }
      __syncthreads();
    }
  if (threadIdx.x >= 32) return;
  // bounds_kernel's chain, one warp; the key of rank r is found in the sorted
  // gathered keys: its bucket b's keys start at the first key with bucket <= b
  const int lane = threadIdx.x;
  unsigned long long P = 0;
  int nb = 0;
  for (int j = 0; j < nmax; j++) {
    unsigned long long q = spdf[j];
    if (!q) { if (!lane) o->pdf[j] = 0; continue; }
    unsigned long long E = P + q;
    if (E > M) { if (!lane) o->err = EZMOCK_ERR_UNKNOWN; return; }
    const int b = sel_rank_bucket(cum, E - 1, lane);
    const int lo = warp_first((int) G, [&](int i) { return sel_bucket(from_key(g[i]), sb) <= b; },
        lane);
    const unsigned long long i = lo + (E - 1 - cum[b]);
    if (i >= G || sel_bucket(from_key(g[i]), sb) != b) {
      if (!lane) o->err = SEL_FALLBACK;
      return;
    }
    const skey_t kv = g[i];
    unsigned long long ie = i;                     // last key equal to kv
    for (;;) {
      const unsigned long long t = ie + 1 + lane;
      const unsigned int eq = __ballot_sync(0xffffffffu, t < G && g[t] == kv);
      if (eq == 0xffffffffu) { ie += 32; continue; }
      ie += __ffs(~eq) - 1;
      break;
    }
    const unsigned long long E2 = cum[b] + (ie - lo) + 1;
    const unsigned long long extra = E2 - E;
    q += extra;
    ncell += extra;
    ntot += extra * (unsigned long long) (nmax - j);
    E = E2;
    if (!lane) {
      o->pdf[j] = q;
      o->lo[nb] = from_key(kv);
      o->ntr[nb] = nmax - j;
    }
    nb++;
    P = E;
  }
  if (!lane) {
    o->nbins = nb;
    o->ncell = ncell;
    o->ntot = ntot;
    o->err = 0;
  }
}

__device__ __forceinline__ int cell_count(real v, const real *lo, const int *ntr,
    int nb) {
  // first non-empty bin (descending thresholds) with v >= lo
  if (!nb || v < lo[nb - 1] || !(v == v)) return 0;
  int a = 0, b = nb - 1;
  while (a < b) {
    const int mid = (a + b) >> 1;
    if (v >= lo[mid]) b = mid; else a = mid + 1;
  }
  return ntr[a];
}

// Tracers of a chunk from its candidates (the cells at or above the
// selection's cut, listed by compact_kernel): only they can hold tracers.
// One warp per chunk, eight chunks per block.
constexpr int CW = NT / 32;                      // chunks per block (emission)

__global__ void __launch_bounds__(NT)
cand_count_kernel(const skey_t *__restrict__ cand,
    const unsigned long long *__restrict__ cstart, const unsigned int *__restrict__ ccnt,
    const BoundOut *__restrict__ bo, unsigned long long *cnt, size_t nblk) {
  __shared__ real slo[EZ_MAX_NT];
  __shared__ int sntr[EZ_MAX_NT];
  const int nb = bo->nbins;
  for (int e = threadIdx.x; e < nb; e += NT) { slo[e] = bo->lo[e]; sntr[e] = bo->ntr[e]; }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const size_t ch = (size_t) blockIdx.x * CW + (threadIdx.x >> 5);
  if (ch >= nblk) return;
  const unsigned int n = ccnt[ch];
  const skey_t *c = cand + cstart[ch];
  unsigned long long t = 0;
  for (unsigned int i = lane; i < n; i += 32) t += cell_count(from_key(c[i]), slo, sntr, nb);
#pragma unroll
  for (int o = 16; o; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
  if (lane == 0) cnt[ch] = t;
}

__global__ void __launch_bounds__(NT)
tracer_count_kernel(const real *__restrict__ rhot, size_t N,
    const BoundOut *__restrict__ bo, unsigned long long *cnt,
    const int16_t *__restrict__ nt16) {
  __shared__ real slo[EZ_MAX_NT];
  __shared__ int sntr[EZ_MAX_NT];
  __shared__ unsigned long long sw[32];
  const int nb = bo->nbins;
  for (int e = threadIdx.x; e < nb; e += NT) { slo[e] = bo->lo[e]; sntr[e] = bo->ntr[e]; }
  __syncthreads();
  unsigned long long c = 0;
  const size_t b0 = (size_t) blockIdx.x * CH;
  real v[ROWS];
#pragma unroll
  for (int q = 0; q < ROWS; q++) {               // all loads first
    const size_t id = b0 + (size_t) q * NT + threadIdx.x;
    v[q] = (id < N && !nt16) ? rhot[id] : (real) 0;
  }
#pragma unroll
  for (int q = 0; q < ROWS; q++) {
    const size_t id = b0 + (size_t) q * NT + threadIdx.x;
    if (id < N) c += nt16 ? nt16[id] : cell_count(v[q], slo, sntr, nb);
  }
  unsigned long long tot;
  block_scan<unsigned long long>(c, &tot, sw);
  if (threadIdx.x == 0) cnt[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(NT)
nt_kernel(const real *__restrict__ rhot, size_t N,
    const BoundOut *__restrict__ bo, int16_t *nt) {
  __shared__ real slo[EZ_MAX_NT];
  __shared__ int sntr[EZ_MAX_NT];
  const int nb = bo->nbins;
  for (int e = threadIdx.x; e < nb; e += NT) { slo[e] = bo->lo[e]; sntr[e] = bo->ntr[e]; }
  __syncthreads();
  for (size_t id = (size_t) blockIdx.x * blockDim.x + threadIdx.x; id < N;
       id += (size_t) gridDim.x * blockDim.x)
    nt[id] = (int16_t) cell_count(rhot[id], slo, sntr, nb);
}

// Tracer cells (pop_tracer.c:894-967): the tracers of a cell follow, in
// cell-index order, those of all earlier cells.  The first index of each
// cell comes from the chunk offset, per-(row, warp) prefixes and a warp scan
// (skipped for the many warp rows without tracers); each tracer's cell index
// is written to `cid`, and place_kernel computes the positions one thread per
// tracer.  (With the selection's candidates at hand, tracer_cell_cand_kernel
// visits only them.)
template <typename cid_t>
__global__ void __launch_bounds__(NT)
tracer_cell_kernel(const real *__restrict__ rhot, size_t N,
    const BoundOut *__restrict__ bo, const unsigned long long *__restrict__ off,
    unsigned long long ntr, cid_t *__restrict__ cid, const int16_t *__restrict__ nt16) {
  constexpr int NW = NT / 32;
  __shared__ real slo[EZ_MAX_NT];
  __shared__ int sntr[EZ_MAX_NT];
  __shared__ unsigned int pre[ROWS * NW];
  __shared__ unsigned int wsum[ROWS * NW / 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int nb = bo->nbins;
  for (int e = threadIdx.x; e < nb; e += NT) { slo[e] = bo->lo[e]; sntr[e] = bo->ntr[e]; }
  __syncthreads();
  const size_t b0 = (size_t) blockIdx.x * CH;
  int n[ROWS];
  unsigned int ex[ROWS];                       // exclusive prefix within the warp row
  real v[ROWS];
#pragma unroll
  for (int q = 0; q < ROWS; q++) {               // all loads first
    const size_t id = b0 + (size_t) q * NT + threadIdx.x;
    v[q] = (id < N && !nt16) ? rhot[id] : (real) 0;
  }
#pragma unroll
  for (int q = 0; q < ROWS; q++) {
    const size_t id = b0 + (size_t) q * NT + threadIdx.x;
    n[q] = (id >= N) ? 0 : (nt16 ? (int) nt16[id] : cell_count(v[q], slo, sntr, nb));
    unsigned int incl = (unsigned int) n[q];
    if (__ballot_sync(0xffffffffu, n[q] != 0)) {
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const unsigned int v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
      }
    }
    ex[q] = incl - (unsigned int) n[q];
    if (lane == 31) pre[q * NW + w] = incl;
  }
  __syncthreads();
  unsigned int c = 0, incl = 0;
  if (threadIdx.x < ROWS * NW) {
    c = pre[threadIdx.x];
    incl = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned int v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += v;
    }
    if (lane == 31) wsum[w] = incl;
  }
  __syncthreads();
  if (threadIdx.x < ROWS * NW) {
    unsigned int base = 0;
    for (int k = 0; k < w; k++) base += wsum[k];
    pre[threadIdx.x] = base + incl - c;
  }
  __syncthreads();
  const unsigned long long run = off[blockIdx.x];
#pragma unroll
  for (int q = 0; q < ROWS; q++) {
    if (!n[q]) continue;
    const cid_t id = (cid_t) (b0 + (size_t) q * NT + threadIdx.x);
    const unsigned long long t0 = run + pre[q * NW + w] + ex[q];
    for (int m = 0; m < n[q] && t0 + m < ntr; m++) cid[t0 + m] = id;
  }
}

// Tracer cells from the selection's candidates only: compact_kernel lists a
// chunk's candidates in cell order, so one warp per chunk walks them 32 at a
// time, and a warp scan of their counts gives each candidate's first tracer
// (the same order and offsets as tracer_cell_kernel, which walks every cell
// of the chunk).
template <typename cid_t>
__global__ void __launch_bounds__(NT)
tracer_cell_cand_kernel(const BoundOut *__restrict__ bo, const unsigned long long *__restrict__ off,
    unsigned long long ntr, cid_t *__restrict__ cid, const skey_t *__restrict__ cand,
    const uint16_t *__restrict__ cidx, const unsigned long long *__restrict__ cstart,
    const unsigned int *__restrict__ ccnt, size_t nblk) {
  __shared__ real slo[EZ_MAX_NT];
  __shared__ int sntr[EZ_MAX_NT];
  const int nb = bo->nbins;
  for (int e = threadIdx.x; e < nb; e += NT) { slo[e] = bo->lo[e]; sntr[e] = bo->ntr[e]; }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const size_t ch = (size_t) blockIdx.x * CW + (threadIdx.x >> 5);
  if (ch >= nblk) return;
  const unsigned int n = ccnt[ch];
  const unsigned long long c0 = cstart[ch];
  const size_t b0 = ch * CH;
  unsigned long long tt = off[ch];
  for (unsigned int i0 = 0; i0 < n; i0 += 32) {
    const unsigned int i = i0 + lane;
    const int k = (i < n) ? cell_count(from_key(cand[c0 + i]), slo, sntr, nb) : 0;
    unsigned int incl = (unsigned int) k;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned int y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    if (k) {
      const cid_t id = (cid_t) (b0 + cidx[c0 + i]);
      unsigned long long t = tt + incl - (unsigned int) k;
      for (int m = 0; m < k && t < ntr; m++, t++) cid[t] = id;
    }
    tt += __shfl_sync(0xffffffffu, incl, 31);
  }
}

// Position of tracer t in its cell (pop_tracer.c:946-967): draws
// 3t .. 3t+2 of the position range.
template <typename cid_t>
__global__ void __launch_bounds__(NT)
place_kernel(const cid_t *__restrict__ cid, unsigned long long ntr, int Ng,
    const uint32_t *__restrict__ draws, int ran, real gs, double Lbox,
    real *x, real *y, real *z) {
  for (unsigned long long t = (unsigned long long) blockIdx.x * NT + threadIdx.x; t < ntr;
       t += (unsigned long long) gridDim.x * NT) {
    const cid_t id = cid[t];
    const cid_t ij = id / (cid_t) Ng;
    const int kk = (int) (id - ij * (cid_t) Ng);
    const cid_t ii = ij / (cid_t) Ng;
    const int jj = (int) (ij - ii * (cid_t) Ng);
    double r = ez_u(ran, draws[3 * t]) - 0.5;
    real xx = ((int) ii + r) * (double) gs;
    r = ez_u(ran, draws[3 * t + 1]) - 0.5;
    real yy = (jj + r) * (double) gs;
    r = ez_u(ran, draws[3 * t + 2]) - 0.5;
    real zz = (kk + r) * (double) gs;
    if (xx < 0) xx = (double) xx + Lbox;
    if (yy < 0) yy = (double) yy + Lbox;
    if (zz < 0) zz = (double) zz + Lbox;
    x[t] = xx; y[t] = yy; z[t] = zz;
  }
}

// ============================================================================
//     tracers attached to particles (att_part; pop_tracer.c:517-582, :804-879)
// ============================================================================
// Particle ids are 32-bit here (Ng^3 < 2^32).

// Eulerian position (grid units, wrapped into [0, Ng)) and nearest cell of
// particle id, in the reference's `real` arithmetic (pop_tracer.c:541-561).
__device__ __forceinline__ uint32_t ngp_of(const real *__restrict__ p0,
    const real *__restrict__ p1, const real *__restrict__ p2, uint32_t id,
    int Ng, real igs, real *pos) {
  const uint32_t ij = id / (uint32_t) Ng, i = ij / (uint32_t) Ng;
  const int k = (int) (id - ij * Ng), j = (int) (ij - i * Ng);
  real px = p0[id] * igs + (int) i;
  real py = p1[id] * igs + j;
  real pz = p2[id] * igs + k;
  if (px < 0) px += Ng;
  else if (px >= Ng) px -= Ng;
  if (py < 0) py += Ng;
  else if (py >= Ng) py -= Ng;
  if (pz < 0) pz += Ng;
  else if (pz >= Ng) pz -= Ng;
  int ix = (int) ((double) px + 0.5), iy = (int) ((double) py + 0.5),
      iz = (int) ((double) pz + 0.5);
  if (ix >= Ng) ix = 0;
  if (iy >= Ng) iy = 0;
  if (iz >= Ng) iz = 0;
  pos[0] = px; pos[1] = py; pos[2] = pz;
  return ((uint32_t) ix * Ng + iy) * Ng + iz;
}

// Particles per tracer-hosting cell.
__global__ void __launch_bounds__(NT)
np_kernel(const real *__restrict__ p0, const real *__restrict__ p1,
    const real *__restrict__ p2, uint32_t N, int Ng, real igs,
    const int16_t *__restrict__ nt, unsigned int *np) {
  real pos[3];
  for (uint32_t id = blockIdx.x * NT + threadIdx.x; id < N; id += gridDim.x * NT) {
    const uint32_t c = ngp_of(p0, p1, p2, id, Ng, igs, pos);
    if (nt[c] > 0) atomicAdd(np + c, 1u);
  }
}

// Exclusive ranks, in index order, of the flagged cells of a chunk of ROWS x
// NT cells (row q, thread t: cell q NT + t), and the chunk total.
constexpr int NWP = NT / 32;
__device__ __forceinline__ unsigned int chunk_ranks(const bool *f, unsigned int *rk,
    unsigned int *pre, unsigned int *wsum) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const unsigned int lt = (1u << lane) - 1;
  unsigned int bal[ROWS];
#pragma unroll
  for (int q = 0; q < ROWS; q++) {
    bal[q] = __ballot_sync(0xffffffffu, f[q]);
    if (lane == 0) pre[q * NWP + w] = __popc(bal[q]);
  }
  __syncthreads();
  unsigned int c = 0, incl = 0;
  if (threadIdx.x < ROWS * NWP) {
    c = pre[threadIdx.x];
    incl = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned int v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += v;
    }
    if (lane == 31) wsum[w] = incl;
  }
  __syncthreads();
  unsigned int total = 0;
  for (int k = 0; k < ROWS * NWP / 32; k++) total += wsum[k];
  if (threadIdx.x < ROWS * NWP) {
    unsigned int base = 0;
    for (int k = 0; k < w; k++) base += wsum[k];
    pre[threadIdx.x] = base + incl - c;
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < ROWS; q++) rk[q] = pre[q * NWP + w] + __popc(bal[q] & lt);
  __syncthreads();                       // pre and wsum may be reused
  return total;
}

// Class of each particle: 0 its cell hosts no tracer, 1 every particle of the
// cell takes a tracer (nt >= np), 2 contested (0 < nt < np: selection
// sampling).  Counts the contested particles of each chunk; flags cells
// with more than 65535 particles (the reference's uint16 counter).
__global__ void __launch_bounds__(NT)
class_kernel(const real *__restrict__ p0, const real *__restrict__ p1,
    const real *__restrict__ p2, uint32_t N, int Ng, real igs,
    const int16_t *__restrict__ nt, const unsigned int *__restrict__ np,
    uint8_t *__restrict__ cls, unsigned long long *cnt, int *ovf) {
  __shared__ unsigned int pre[ROWS * NWP], wsum[ROWS * NWP / 32];
  bool f[ROWS];
  unsigned int rk[ROWS];
  real pos[3];
  const size_t b0 = (size_t) blockIdx.x * CH;
#pragma unroll
  for (int q = 0; q < ROWS; q++) {
    const size_t id = b0 + (size_t) q * NT + threadIdx.x;
    uint8_t k = 0;
    if (id < N) {
      const uint32_t c = ngp_of(p0, p1, p2, (uint32_t) id, Ng, igs, pos);
      const int t = nt[c];
      const unsigned int n = np[c];
      if (n > 65535u) *ovf = 1;
      k = (t <= 0) ? 0 : ((unsigned) t >= n ? 1 : 2);
      cls[id] = k;
    }
    f[q] = k == 2;
  }
  const unsigned int tot = chunk_ranks(f, rk, pre, wsum);
  if (threadIdx.x == 0) cnt[blockIdx.x] = tot;
}

// Cell of each contested particle, in particle order.
__global__ void __launch_bounds__(NT)
entry_kernel(const real *__restrict__ p0, const real *__restrict__ p1,
    const real *__restrict__ p2, uint32_t N, int Ng, real igs,
    const uint8_t *__restrict__ cls, const unsigned long long *__restrict__ off,
    uint32_t *__restrict__ ecell) {
  __shared__ unsigned int pre[ROWS * NWP], wsum[ROWS * NWP / 32];
  bool f[ROWS];
  unsigned int rk[ROWS];
  real pos[3];
  const size_t b0 = (size_t) blockIdx.x * CH;
#pragma unroll
  for (int q = 0; q < ROWS; q++) {
    const size_t id = b0 + (size_t) q * NT + threadIdx.x;
    f[q] = id < N && cls[id] == 2;
  }
  chunk_ranks(f, rk, pre, wsum);
  const unsigned long long o = off[blockIdx.x];
#pragma unroll
  for (int q = 0; q < ROWS; q++)
    if (f[q]) {
      const uint32_t id = (uint32_t) (b0 + (size_t) q * NT + threadIdx.x);
      ecell[o + rk[q]] = ngp_of(p0, p1, p2, id, Ng, igs, pos);
    }
}

// The selection-sampling chain (pop_tracer.c:838-849) over the contested
// particles in particle order, one warp, 32 particles per step.  A particle
// whose cell still has 0 < nt < np takes the next draw u and is kept if not
// u np >= nt; every particle of a cell with nt > 0 decrements np, a kept one
// nt.  When the 32 particles of a step lie in 32 different cells they are
// decided together (each knows its draw from a ballot of the earlier ones);
// otherwise they are decided one after another, lanes of the same cell
// updating their copy of its counters.  Contested cells end with nt = np = 0.
// The next step's cells, counters and 64 draws (it starts within 32 draws of
// the current one) are loaded before the current step is decided; counters
// of cells the current step changes are then taken from its lanes.
__global__ void __launch_bounds__(32)
chain_kernel(const uint32_t *__restrict__ ecell, unsigned long long E,
    int16_t *nt, unsigned int *np, const uint32_t *__restrict__ draws, int ran,
    uint8_t *__restrict__ att) {
  const int lane = threadIdx.x;
  const unsigned int full = 0xffffffffu, lt = (1u << lane) - 1;
  unsigned long long d = 0;                  // draws used before this step
  // step 0
  bool valid = (unsigned long long) lane < E;
  uint32_t c = valid ? ecell[lane] : 0xffffffffu;
  int tn = valid ? nt[c] : 0;
  int pn = valid ? (int) np[c] : 0;
  uint32_t w0 = ((unsigned long long) lane < E) ? draws[lane] : 0u;
  uint32_t w1 = (32ull + lane < E) ? draws[32 + lane] : 0u;
  for (unsigned long long b = 0; b < E; b += 32) {
    // prefetch of the next step
    const unsigned long long e1 = b + 32 + lane;
    const bool valid1 = e1 < E;
    const uint32_t c1 = valid1 ? ecell[e1] : 0xffffffffu;
    int tn1 = valid1 ? nt[c1] : 0;
    int pn1 = valid1 ? (int) np[c1] : 0;
    const uint32_t nx = (d + 64 + lane < E) ? draws[d + 64 + lane] : 0u;   // draw d+64+lane
    // this step; its draws are w0 (d .. d+31)
    const unsigned int same = __match_any_sync(full, c);
    const bool dup = __any_sync(full, valid && __popc(same) > 1);
    bool kept = false;
    int used;
    if (!dup) {
      const bool cons = valid && tn > 0 && tn < pn;
      const unsigned int cm = __ballot_sync(full, cons);
      const uint32_t uk = __shfl_sync(full, w0, __popc(cm & lt));
      if (valid && tn > 0) {
        kept = !cons || !(ez_u(ran, uk) * pn >= tn);
        pn -= 1;
        tn -= kept ? 1 : 0;
      }
      used = __popc(cm);
    }
    else {
      used = 0;
      for (int i = 0; i < 32; i++) {
        const uint32_t ci = __shfl_sync(full, c, i);
        const int ti = __shfl_sync(full, tn, i), pi = __shfl_sync(full, pn, i);
        const int vi = __shfl_sync(full, (int) valid, i);
        const uint32_t ui = __shfl_sync(full, w0, used);
        bool ki = false, cons = false;
        if (vi && ti > 0) {
          cons = ti < pi;
          ki = !cons || !(ez_u(ran, ui) * pi >= ti);
        }
        if (lane == i) kept = ki;
        if (vi && ti > 0 && valid && c == ci) {
          pn = pi - 1;
          tn = ti - (ki ? 1 : 0);
        }
        used += cons ? 1 : 0;
      }
    }
    if (valid) {
      nt[c] = (int16_t) tn;
      np[c] = (unsigned int) pn;
      att[b + lane] = kept ? 1 : 0;
    }
    // counters of the next step that this step changed
    for (int i = 0; i < 32; i++) {
      const uint32_t ci = __shfl_sync(full, c, i);
      const int ti = __shfl_sync(full, tn, i), pi = __shfl_sync(full, pn, i);
      const int vi = __shfl_sync(full, (int) valid, i);
      if (vi && valid1 && c1 == ci) { tn1 = ti; pn1 = pi; }
    }
    __syncwarp();
    // window of the next step, draws d + used + (0 .. 63), out of the draws
    // d .. d+95 held in w0 | w1 | nx (used <= 32)
    const int s0 = lane + used, src = s0 & 31;
    const uint32_t a0 = __shfl_sync(full, w0, src), a1 = __shfl_sync(full, w1, src),
                   a2 = __shfl_sync(full, nx, src);
    w0 = (s0 < 32) ? a0 : a1;                 // draw d + s0
    w1 = (s0 < 32) ? a1 : a2;                 // draw d + 32 + s0
    d += (unsigned long long) used;
    c = c1; tn = tn1; pn = pn1; valid = valid1;
  }
}

// Attached particles of each chunk (class 1, or class 2 and kept).
__global__ void __launch_bounds__(NT)
att_count_kernel(uint32_t N, const uint8_t *__restrict__ cls,
    const unsigned long long *__restrict__ eoff, const uint8_t *__restrict__ att,
    unsigned long long *cnt) {
  __shared__ unsigned int pre[ROWS * NWP], wsum[ROWS * NWP / 32];
  bool f[ROWS];
  unsigned int rk[ROWS];
  uint8_t k[ROWS];
  const size_t b0 = (size_t) blockIdx.x * CH;
#pragma unroll
  for (int q = 0; q < ROWS; q++) {
    const size_t id = b0 + (size_t) q * NT + threadIdx.x;
    k[q] = (id < N) ? cls[id] : 0;
    f[q] = k[q] == 2;
  }
  chunk_ranks(f, rk, pre, wsum);
  const unsigned long long o = eoff[blockIdx.x];
  unsigned int n = 0;
#pragma unroll
  for (int q = 0; q < ROWS; q++)
    n += (k[q] == 1 || (k[q] == 2 && att[o + rk[q]])) ? 1 : 0;
#pragma unroll
  for (int m = 16; m; m >>= 1) n += __shfl_xor_sync(0xffffffffu, n, m);
  if (threadIdx.x == 0) pre[0] = 0;
  __syncthreads();
  if ((threadIdx.x & 31) == 0) atomicAdd(&pre[0], n);
  __syncthreads();
  if (threadIdx.x == 0) cnt[blockIdx.x] = pre[0];
}

// Attached tracers in particle order: position = particle position, velocity
// = psi vfac (pop_tracer.c:855-871).
__global__ void __launch_bounds__(NT)
att_write_kernel(const real *__restrict__ p0, const real *__restrict__ p1,
    const real *__restrict__ p2, uint32_t N, int Ng, real igs, real gs,
    double vfac, const uint8_t *__restrict__ cls,
    const unsigned long long *__restrict__ eoff, const uint8_t *__restrict__ att,
    const unsigned long long *__restrict__ aoff, real *x, real *y, real *z,
    real *vx, real *vy, real *vz) {
  __shared__ unsigned int pre[ROWS * NWP], wsum[ROWS * NWP / 32];
  bool f[ROWS], a[ROWS];
  unsigned int rk[ROWS], ra[ROWS];
  uint8_t k[ROWS];
  const size_t b0 = (size_t) blockIdx.x * CH;
#pragma unroll
  for (int q = 0; q < ROWS; q++) {
    const size_t id = b0 + (size_t) q * NT + threadIdx.x;
    k[q] = (id < N) ? cls[id] : 0;
    f[q] = k[q] == 2;
  }
  chunk_ranks(f, rk, pre, wsum);
  const unsigned long long oe = eoff[blockIdx.x];
#pragma unroll
  for (int q = 0; q < ROWS; q++) a[q] = k[q] == 1 || (k[q] == 2 && att[oe + rk[q]]);
  chunk_ranks(a, ra, pre, wsum);
  const unsigned long long oa = aoff[blockIdx.x];
  real pos[3];
#pragma unroll
  for (int q = 0; q < ROWS; q++)
    if (a[q]) {
      const uint32_t id = (uint32_t) (b0 + (size_t) q * NT + threadIdx.x);
      ngp_of(p0, p1, p2, id, Ng, igs, pos);
      const unsigned long long t = oa + ra[q];
      x[t] = pos[0] * gs;
      y[t] = pos[1] * gs;
      z[t] = pos[2] * gs;
      vx[t] = p0[id] * vfac;
      vy[t] = p1[id] * vfac;
      vz[t] = p2[id] * vfac;
    }
}

// Tracers left per cell once the particles are taken: nt - np where every
// particle was attached; contested cells are already at nt = 0.
__global__ void __launch_bounds__(NT)
leftover_kernel(int16_t *nt, const unsigned int *__restrict__ np, uint32_t N) {
  for (uint32_t c = blockIdx.x * NT + threadIdx.x; c < N; c += gridDim.x * NT) {
    const int t = nt[c];
    if (t > 0) nt[c] = (int16_t) max(t - (int) np[c], 0);
  }
}

__device__ __forceinline__ size_t idx3(int Ng, int a, int b, int c) {
  return ((size_t) a * Ng + b) * Ng + c;
}

// Velocity of each tracer from the painted grids at its eight CIC cells
// (pop_tracer.c:593-683 painting, :697-753 interpolation).  IL: the grids interleaved with the density,
// (q0, q1, q2, rho) per cell, one 16-byte load per cell instead of four
// 4-byte loads from four grids (a tracer's eight cells touch 4 to 8 sectors
// instead of 16 to 32).
template <bool IL>
__global__ void __launch_bounds__(NT)
vel_kernel(const real *__restrict__ rho, const real *__restrict__ q0,
    const real *__restrict__ q1, const real *__restrict__ q2, const real *__restrict__ pq,
    int Ng, real igs,
    double vfac, size_t n, const real *__restrict__ x, const real *__restrict__ y,
    const real *__restrict__ z, real *vx, real *vy, real *vz) {
  for (size_t t = (size_t) blockIdx.x * blockDim.x + threadIdx.x; t < n;
       t += (size_t) gridDim.x * blockDim.x) {
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
    const size_t cs[8] = {idx3(Ng, x0, y0, z0), idx3(Ng, x0, y0, z1),
                          idx3(Ng, x0, y1, z0), idx3(Ng, x0, y1, z1),
                          idx3(Ng, x1, y0, z0), idx3(Ng, x1, y0, z1),
                          idx3(Ng, x1, y1, z0), idx3(Ng, x1, y1, z1)};
    const real wa[8] = {wx0, wx0, wx0, wx0, wx1, wx1, wx1, wx1};
    const real wb[8] = {wy0, wy0, wy1, wy1, wy0, wy0, wy1, wy1};
    const real wc[8] = {wz0, wz1, wz0, wz1, wz0, wz1, wz0, wz1};
    // all 32 gathers issued before any of them is used
    const real *qs[3] = {q0, q1, q2};
    real rv[8], qv[3][8];
    if constexpr (IL) {
#ifdef SINGLE_PREC
#pragma unroll
      for (int c = 0; c < 8; c++) {
        const float4 a = reinterpret_cast<const float4 *>(pq)[cs[c]];
        qv[0][c] = a.x;
        qv[1][c] = a.y;
        qv[2][c] = a.z;
        rv[c] = a.w;
      }
#endif
    } else {
#pragma unroll
      for (int c = 0; c < 8; c++) rv[c] = rho[cs[c]];
#pragma unroll
      for (int d = 0; d < 3; d++)
#pragma unroll
        for (int c = 0; c < 8; c++) qv[d][c] = qs[d][cs[c]];
    }
    real rw[8];
    real rs = 0;
#pragma unroll
    for (int c = 0; c < 8; c++) {
      rw[c] = rv[c] * wa[c] * wb[c] * wc[c];
      rs = (c == 0) ? rw[0] : rs + rw[c];
    }
    const double fac = vfac / rs;
    real *outs[3] = {vx, vy, vz};
#pragma unroll
    for (int d = 0; d < 3; d++) {
      real v = 0;
#pragma unroll
      for (int c = 0; c < 8; c++) {
        // the painted momentum per unit density (pop_tracer.c:681)
        const real np = (rv[c] > (real) EZ_REAL_TOL) ? qv[d][c] / rv[c] : qv[d][c];
        const real pr = np * rw[c];
        v = (c == 0) ? pr : v + pr;
      }
      outs[d][t] = v * fac;
    }
  }
}

__global__ void __launch_bounds__(NT)
disp_kernel(size_t n, const uint32_t *__restrict__ draws, int ran,
    double sigma, real *vx, real *vy, real *vz) {
  const size_t npair = (n + 1) / 2;
  for (size_t m = (size_t) blockIdx.x * blockDim.x + threadIdx.x; m < npair;
       m += (size_t) gridDim.x * blockDim.x) {
    double g[6];
#pragma unroll
    for (int p = 0; p < 3; p++) {
      const double rr = -2 * log(ez_upos(ran, draws[6 * m + 2 * p]));
      const double th = ez_u(ran, draws[6 * m + 2 * p + 1]) * 2 * EZ_PI;
      g[2 * p] = sigma * sqrt(rr) * cos(th);
      g[2 * p + 1] = sigma * sqrt(rr) * sin(th);
    }
    const size_t a = 2 * m;
    vx[a] = vx[a] + g[0];
    vy[a] = vy[a] + g[1];
    vz[a] = vz[a] + g[2];
    if (a + 1 < n) {
      vx[a + 1] = vx[a + 1] + g[3];
      vy[a + 1] = vy[a + 1] + g[4];
      vz[a + 1] = vz[a + 1] + g[5];
    }
  }
}

unsigned grid_for(size_t n, int nt) {
  const size_t b = (n + nt - 1) / nt;
  return (unsigned) (b < 148 * 32 ? (b ? b : 1) : 148 * 32);
}

// Buffer of the attach-to-particle stage, grown on demand.
int att_buffer(EzMesh *m, size_t bytes) {
  if (bytes <= m->att_cap) return 0;
  if (m->att) {
    cudaStreamSynchronize(m->stream);
    cudaFree(m->att);
  }
  m->att = nullptr;
  m->att_cap = 0;
  bytes = (bytes + 4095) / 4096 * 4096;
  if (!EZ_CUDA_OK(cudaMalloc(&m->att, bytes))) { cudaGetLastError(); return EZMOCK_ERR_MEMORY; }
  m->att_cap = bytes;
  return 0;
}

int ensure_draws(EzMesh *m, size_t count) {
  if (count <= m->draws_cap) return 0;
  if (m->draws) cudaFree(m->draws);
  m->draws = nullptr;
  if (!EZ_CUDA_OK(cudaMalloc(&m->draws, count * sizeof(uint32_t)))) {
    m->draws_cap = 0;
    return EZMOCK_ERR_MEMORY;
  }
  m->draws_cap = count;
  return 0;
}


// Exclusive scan of n values into out[0..n], out[n] = total.  `tmp` holds
// ceil(n / SCAN_CHUNK) + 1 values.
void scan_u64(const unsigned long long *in, unsigned long long *out, size_t n,
    unsigned long long *tmp, cudaStream_t st) {
  if (n <= 4 * SCAN_CHUNK) {
    scan_kernel<<<1, 1024, 0, st>>>(in, out, n); ez_count_launch();
    return;
  }
  const size_t nc = (n + SCAN_CHUNK - 1) / SCAN_CHUNK;
  chunk_sum_kernel<<<(unsigned) nc, 1024, 0, st>>>(in, n, tmp); ez_count_launch();
  scan_kernel<<<1, 1024, 0, st>>>(tmp, tmp, nc); ez_count_launch();
  chunk_scan_kernel<<<(unsigned) nc, 1024, 0, st>>>(in, n, tmp, out); ez_count_launch();
  cudaMemcpyAsync(out + n, tmp + nc, 8, cudaMemcpyDeviceToDevice, st);
}

struct PopScratch {
  unsigned long long *bcnt, *bscan, *hist, *dpdf, *dcount, *dcscan, *counter, *tmp;
  BoundOut *bo;
  unsigned long long *cstart;   // per chunk: first candidate (compact_kernel)
  unsigned int *ccnt;           // per chunk: candidates
  unsigned int *bhist;          // SEL_NB candidate counts per value bucket
  unsigned int *bmask;          // SEL_NB bits: buckets that can hold a boundary
  unsigned int *gcount;         // candidates of the marked buckets
  skey_t *gbuf;                 // their keys (SEL_GCAP)
  unsigned int *bpart;          // per-block bucket histograms (SEL_HB x SEL_NB)
};

// Candidate copies for emission, in the draws buffer (free between the bias
// draws and the position draws): keys, then their places in the chunk.
struct CandBuf {
  skey_t *key;
  uint16_t *idx;
  size_t cap;                   // entries
  bool ok;                      // every candidate was copied
};

CandBuf cand_buf(EzMesh *m) {
  CandBuf c;
  c.cap = m->draws ? m->draws_cap * sizeof(uint32_t) / (sizeof(skey_t) + sizeof(uint16_t)) : 0;
  c.key = (skey_t *) m->draws;
  c.idx = (uint16_t *) ((char *) m->draws + c.cap * sizeof(skey_t));
  c.ok = false;
  return c;
}

int pop_scratch(EzMesh *m, PopScratch *ps) {
  const size_t N = m->N;
  const size_t nblk = (N + CH - 1) / CH;
  const size_t ntile_max = (N + TILE - 1) / TILE;
  const size_t off_cnt = 0;
  const size_t off_scan = off_cnt + (nblk + 1) * 8;
  const size_t off_hist = off_scan + (nblk + 1) * 8;
  const size_t off_bo = (off_hist + EZ_NLOGB * 8 + 255) / 256 * 256;
  const size_t off_pdf = (off_bo + sizeof(BoundOut) + 255) / 256 * 256;
  const size_t off_dc = (off_pdf + EZ_MAX_NT * 8 + 255) / 256 * 256;
  const size_t off_dcs = off_dc + (256 * ntile_max + 1) * 8;
  const size_t off_ctr = off_dcs + (256 * ntile_max + 1) * 8;
  const size_t off_tmp = off_ctr + 64;
  const size_t ntmp = (256 * ntile_max + nblk) / SCAN_CHUNK + 8;
  const size_t off_cst = off_tmp + ntmp * 8;
  const size_t off_ccn = off_cst + nblk * 8;
  const size_t off_bh = (off_ccn + nblk * 4 + 255) / 256 * 256;
  const size_t off_bm = off_bh + SEL_NB * 4;
  const size_t off_gc = off_bm + SEL_NB / 8;
  const size_t off_gb = off_gc + 256;
  const size_t off_bp = (off_gb + SEL_GCAP * sizeof(skey_t) + 255) / 256 * 256;
  int e = ez_scratch(m, off_bp + (size_t) SEL_HB * SEL_NB * sizeof(unsigned int));
  if (e) return e;
  char *sc = (char *) m->scratch;
  ps->bcnt = (unsigned long long *) (sc + off_cnt);
  ps->bscan = (unsigned long long *) (sc + off_scan);
  ps->hist = (unsigned long long *) (sc + off_hist);
  ps->bo = (BoundOut *) (sc + off_bo);
  ps->dpdf = (unsigned long long *) (sc + off_pdf);
  ps->dcount = (unsigned long long *) (sc + off_dc);
  ps->dcscan = (unsigned long long *) (sc + off_dcs);
  ps->counter = (unsigned long long *) (sc + off_ctr);
  ps->tmp = (unsigned long long *) (sc + off_tmp);
  ps->cstart = (unsigned long long *) (sc + off_cst);
  ps->ccnt = (unsigned int *) (sc + off_ccn);
  ps->bhist = (unsigned int *) (sc + off_bh);
  ps->bmask = (unsigned int *) (sc + off_bm);
  ps->gcount = (unsigned int *) (sc + off_gc);
  ps->gbuf = (skey_t *) (sc + off_gb);
  ps->bpart = (unsigned int *) (sc + off_bp);
  return 0;
}

struct HostBounds {
  unsigned long long ncell, ntot;
  int err;
  int nbins;
};

// Full LSD radix sort of the M candidate keys in keys_a (keys_b: scratch);
// returns the sorted copy.
skey_t *sort_keys(const PopScratch &ps, skey_t *keys_a, skey_t *keys_b, size_t M,
    cudaStream_t st) {
  if (M <= 1) return keys_a;
  const size_t ntiles = (M + TILE - 1) / TILE;
  skey_t *src = keys_a, *dst = keys_b;
  for (int shift = 0; shift < (int) (8 * sizeof(skey_t)); shift += 8) {
    digit_hist_kernel<<<(unsigned) ntiles, SORT_NT, 0, st>>>(src, M, shift, ps.dcount, ntiles); ez_count_launch();
    scan_u64(ps.dcount, ps.dcscan, 256 * ntiles, ps.tmp, st);
    digit_scatter_kernel<<<(unsigned) ntiles, SORT_NT, 0, st>>>(src, dst, M, shift, ps.dcscan, ntiles); ez_count_launch();
    skey_t *t = src; src = dst; dst = t;
  }
  return src;
}

ubits_t host_bits(real v) {
  ubits_t b;
  memcpy(&b, &v, sizeof(b));
  return b;
}

// Selection (pop_tracer.c:359-461): cut from the log2 histogram, compaction
// of the candidates, PDF-bin boundaries with the tie extension (from the
// value buckets, or from a full sort).  Leaves the boundaries in ps.bo on
// the device.
int select_stage(EzMesh *m, const PopScratch &ps, const real *rhot,
    const unsigned long long *h, const size_t *pdf, int nmax, size_t ncell,
    size_t ntot, HostBounds *hb, CandBuf *cb = nullptr) {
  const size_t N = m->N;
  cudaStream_t st = m->stream;
  skey_t *keys_a = (skey_t *) m->spec[1];
  skey_t *keys_b = (skey_t *) m->spec[2];
  int imax, i0 = -1;
  size_t cnt = 0;
  for (imax = 0; imax < EZ_NLOGB; imax++) {
    if (i0 < 0 && h[imax]) i0 = imax;
    cnt += h[imax];
    if (cnt >= ncell) break;
  }
  const real ilogb_max = 5;
  const real cut = (imax == EZ_NLOGB - 1) ? (real) EZ_REAL_MIN
      : (real) pow(2.0, (double) ilogb_max - imax);
  // The candidate count is known without waiting for the compaction: a
  // cell's histogram bin is 5 - ilogb(rho_t) (clamped), so for a cut below
  // the last bin, bin <= imax exactly when rho_t >= 2^(5 - imax) = cut, and
  // the candidates are the cells counted in bins 0..imax (cells that are not
  // valid have rho_t = 0 and are in no bin).  The device counter is checked
  // against it at the boundaries' read-back below.  With the cut in the last
  // bin (zero and subnormal rho_t) the count is read back and the keys are
  // sorted.
  const bool buckets = !m->sel_sort && imax < EZ_NLOGB - 1 && cnt > 0 &&
      cnt < (1ull << 32) && i0 >= 0;
  SelBucket sb = {0, 0};
  if (buckets) {
    // bucket range: the cut up to the top of bin i0 (2^(6 - i0)); values of
    // bin 0 above 64 share the last bucket
    const real upper = (real) pow(2.0, (double) (i0 >= 1 ? 6 - i0 : 6));
    const ubits_t range = host_bits(upper) - host_bits(cut);
    sb.base = host_bits(cut);
    while (((range - 1) >> sb.shift) >= (ubits_t) SEL_NB) sb.shift++;
  }
  cudaMemsetAsync(ps.counter, 0, 8, st);
  CandBuf none = {nullptr, nullptr, 0, false};
  CandBuf &c = cb ? *cb : none;
  compact_kernel<<<(unsigned) ((N + CH - 1) / CH), NT, 0, st>>>(rhot, N, cut, keys_a,
      ps.counter, c.key, c.idx, c.cap, ps.cstart, ps.ccnt); ez_count_launch();
  unsigned long long M = cnt;
  if (imax == EZ_NLOGB - 1 &&
      (!EZ_CUDA_OK(cudaMemcpyAsync(&M, ps.counter, 8, cudaMemcpyDeviceToHost, st)) ||
       !EZ_CUDA_OK(cudaStreamSynchronize(st))))
    return EZMOCK_ERR_UNKNOWN;
  c.ok = c.key && M <= c.cap;
  // the PDF goes through pinned memory: a pageable upload would wait for
  // the stream (the buffer is reused only after this stage's final wait)
  if (!m->h_small && !EZ_CUDA_OK(cudaMallocHost(&m->h_small, EZ_MAX_NT * sizeof(unsigned long long)))) {
    m->h_small = nullptr;
    return EZMOCK_ERR_MEMORY;
  }
  for (int j = 0; j < nmax; j++) m->h_small[j] = pdf[j];
  cudaMemcpyAsync(ps.dpdf, m->h_small, nmax * 8, cudaMemcpyHostToDevice, st);
  if (buckets) {
    // attributes per call: the kernels may run on several devices
    cudaFuncSetAttribute(sel_hist_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
        (int) SEL_PLAN_SMEM);
    cudaFuncSetAttribute(sel_plan_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
        (int) SEL_PLAN_SMEM);
    cudaFuncSetAttribute(sel_resolve_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
        (int) SEL_RESOLVE_SMEM);
    const int nh = (int) std::min<size_t>((M + 8191) / 8192, SEL_HB);
    sel_hist_kernel<<<nh, SEL_NT, SEL_PLAN_SMEM, st>>>(keys_a, M, sb, ps.bpart); ez_count_launch();
    sel_reduce_kernel<<<SEL_NB / NT, NT, 0, st>>>(ps.bpart, nh, ps.bhist); ez_count_launch();
    sel_plan_kernel<<<1, SEL_NT, SEL_PLAN_SMEM, st>>>(ps.bhist, M, ps.dpdf, nmax, ps.bmask); ez_count_launch();
    cudaMemsetAsync(ps.gcount, 0, sizeof(unsigned int), st);
    const size_t gb = std::min<size_t>((M + NT - 1) / NT, 148 * 8);
    sel_gather_kernel<<<(unsigned) std::max<size_t>(gb, 1), NT, 0, st>>>(keys_a, M, sb,
        ps.bmask, ps.gcount, ps.gbuf); ez_count_launch();
    sel_resolve_kernel<<<1, SEL_NT, SEL_RESOLVE_SMEM, st>>>(ps.bhist, M, sb, ps.gcount,
        ps.gbuf, ps.dpdf, nmax, ncell, ntot, ps.bo); ez_count_launch();
  } else {
    const skey_t *sorted = sort_keys(ps, keys_a, keys_b, M, st);
    bounds_kernel<<<1, 1, 0, st>>>(sorted, M, ps.dpdf, nmax, ncell, ntot, ps.bo); ez_count_launch();
  }
  unsigned long long Mdev = 0;
  if (!EZ_CUDA_OK(cudaMemcpyAsync(hb, ps.bo, sizeof(*hb), cudaMemcpyDeviceToHost, st)) ||
      !EZ_CUDA_OK(cudaMemcpyAsync(&Mdev, ps.counter, 8, cudaMemcpyDeviceToHost, st)) ||
      !EZ_CUDA_OK(cudaStreamSynchronize(st)))
    return EZMOCK_ERR_UNKNOWN;
  if (Mdev != M) return EZMOCK_ERR_UNKNOWN;
  m->sel_path = buckets ? 0 : 1;
  if (buckets && hb->err == SEL_FALLBACK) {
    m->sel_path = 2;
    // the marked buckets held more candidates than the gather buffer
    const skey_t *sorted = sort_keys(ps, keys_a, keys_b, M, st);
    bounds_kernel<<<1, 1, 0, st>>>(sorted, M, ps.dpdf, nmax, ncell, ntot, ps.bo); ez_count_launch();
    if (!EZ_CUDA_OK(cudaMemcpyAsync(hb, ps.bo, sizeof(*hb), cudaMemcpyDeviceToHost, st)) ||
        !EZ_CUDA_OK(cudaStreamSynchronize(st)))
      return EZMOCK_ERR_UNKNOWN;
  }
  return 0;
}

}  // namespace

// Selection on a tracer-density field already in spec[0] (test entry):
// per-cell counts into nt (device), updated pdf/ncell/ntot.
int ez_select_counts(EzMesh *m, const unsigned long long *h, size_t *pdf,
    int nmax, size_t *ncell, size_t *ntot, int16_t *d_nt) {
  PopScratch ps;
  int e = pop_scratch(m, &ps);
  if (e) return e;
  HostBounds hb;
  const real *rhot = (const real *) m->spec[0];
  if ((e = select_stage(m, ps, rhot, h, pdf, nmax, *ncell, *ntot, &hb))) return e;
  if (hb.err) return hb.err;
  nt_kernel<<<grid_for(m->N, NT), NT, 0, m->stream>>>(rhot, m->N, ps.bo, d_nt); ez_count_launch();
  std::vector<unsigned long long> po(nmax);
  if (!EZ_CUDA_OK(cudaMemcpyAsync(po.data(), ps.bo->pdf, nmax * 8, cudaMemcpyDeviceToHost, m->stream)) ||
      !EZ_CUDA_OK(cudaStreamSynchronize(m->stream)))
    return EZMOCK_ERR_UNKNOWN;
  for (int j = 0; j < nmax; j++) pdf[j] = po[j];
  *ncell = hb.ncell;
  *ntot = hb.ntot;
  return 0;
}

int ez_populate(EzMesh *m, int Ng, double Lbox, int ran, uint64_t seed,
    double vfac, const real *params, const size_t *pdf, int nmax,
    size_t ncell, size_t ntot, bool att_part, EzPopResult *res) {
  const size_t N = m->N;
  const real rho_c = params[0], rho_exp = params[1], sigma_v = params[3];
  const real thres = (rho_c == 0) ? (real) EZ_REAL_MIN : rho_c;
  const double iexp = -1 / rho_exp;
  const size_t nblk = (N + CH - 1) / CH;
  int e;
  res->err = 0;

  PopScratch ps;
  if ((e = pop_scratch(m, &ps))) return e;
  unsigned long long *bcnt = ps.bcnt, *bscan = ps.bscan, *hist = ps.hist;
  BoundOut *bo = ps.bo;
  real *rhot = (real *) m->spec[0];
  cudaStream_t st = m->stream;

  // random streams of the three stages, prepared together (MT19937 jumps)
  ez_stage_begin(m, ST_BIAS);
  {
    const uint64_t nt_cap = ntot + ntot / 32 + 1024;
    // capacity for the next field's side streams: the largest population
    m->pop_hint = m->pop_hint_reset ? nt_cap : std::max<size_t>(m->pop_hint, nt_cap);
    m->pop_hint_reset = false;
    const uint64_t starts[3] = {(uint64_t) N << 1, (uint64_t) N * 5, (uint64_t) N << 3};
    const uint64_t caps[3] = {(uint64_t) N + 2, 3 * nt_cap, 6 * ((nt_cap + 1) / 2)};
    if ((e = ez_rng_prepare(m, ran, seed, starts, caps, 3))) return e;
    ez_rng_side_pop(m, ran, seed);
  }

  // ---- 1. valid ranks ----
  valid_count_kernel<<<(unsigned) nblk, NT, 0, st>>>(m->rho, N, thres, bcnt); ez_count_launch();
  scan_u64(bcnt, bscan, nblk, ps.tmp, st);

  // ---- 2. bias ----
  // The valid count stays on the device until the histogram is read: the
  // draws cover every cell (the side stream prepared N + 2 of them), the
  // Box-Muller pairs stop at the count.
  const size_t nd_max = N + (N & 1);
  if ((e = ensure_draws(m, std::max(nd_max, (size_t) 1)))) return e;
  const uint32_t *dbias = nullptr;
  if ((e = ez_rng_draws(m, ran, seed, 0, nd_max, m->draws, &dbias))) return e;
  cudaMemsetAsync(hist, 0, EZ_NLOGB * 8, st);
  bias_kernel<<<(unsigned) nblk, NT, 0, st>>>(m->rho, rhot, N, thres, iexp,
      bscan, dbias, ran, (double) (real) EZ_GAUSS_WIDTH, hist); ez_count_launch();
  unsigned long long h[EZ_NLOGB], nvalid = 0;
  unsigned int tma_err = 0;        // the field's TMA-staged FFT passes gave up
  if (!EZ_CUDA_OK(cudaMemcpyAsync(h, hist, sizeof(h), cudaMemcpyDeviceToHost, st)) ||
      !EZ_CUDA_OK(cudaMemcpyAsync(&nvalid, bscan + nblk, 8, cudaMemcpyDeviceToHost, st)) ||
      !EZ_CUDA_OK(cudaMemcpyAsync(&tma_err, &((EzCicStats *) m->stats)->tma_err, sizeof(tma_err),
          cudaMemcpyDeviceToHost, st)) ||
      !EZ_CUDA_OK(cudaStreamSynchronize(st)) || tma_err)
    return EZMOCK_ERR_UNKNOWN;
  res->nvalid = nvalid;
  if (nvalid < ncell) { res->err = EZMOCK_ERR_RHO_LESS; return 0; }
  ez_stage_end(m, ST_BIAS);

  // ---- 3. selection ----
  ez_stage_begin(m, ST_SELECT);
  HostBounds hb;
  CandBuf cb = cand_buf(m);
  if ((e = select_stage(m, ps, rhot, h, pdf, nmax, ncell, ntot, &hb, &cb))) return e;
  ez_stage_end(m, ST_SELECT);
  if (hb.err) { res->err = hb.err; return 0; }
  res->ncell = hb.ncell;
  res->ntot = hb.ntot;
  const size_t nt_all = hb.ntot;

  // ---- 4. emission ----
  ez_stage_begin(m, ST_EMIT);
  if (nt_all > m->cat_cap) {
    // with slack: the tie extension varies the count by a few tracers from
    // one field to the next, and a reallocation (cudaFree synchronises the
    // device) cost 45-500 ms
    const size_t cap = nt_all + nt_all / 32 + 4096;
    if (m->cat) cudaFree(m->cat);
    m->cat = nullptr;
    m->cat_cap = 0;
    if (!EZ_CUDA_OK(cudaMalloc(&m->cat, 6 * cap * sizeof(real)))) return EZMOCK_ERR_MEMORY;
    m->cat_cap = cap;
  }
  m->cat_n = nt_all;
  real *cx = m->cat, *cy = cx + nt_all, *cz = cy + nt_all;
  real *cvx = cz + nt_all, *cvy = cvx + nt_all, *cvz = cvy + nt_all;
  const real gs = Lbox / Ng;
  const real igs = Ng / Lbox;

  // tracers attached to particles first (att_part)
  size_t iv = 0;
  int16_t *nt16 = nullptr;
  if (att_part) {
    if (N > 0xffffffffULL) return EZMOCK_ERR_UNKNOWN;
    nt16 = (int16_t *) m->spec[2];
    unsigned int *np32 = (unsigned int *) m->spec[1];
    uint8_t *cls = (uint8_t *) m->spec[0];       // after rho_t is read below
    const uint32_t N32 = (uint32_t) N;
    nt_kernel<<<grid_for(N, NT), NT, 0, st>>>(rhot, N, bo, nt16); ez_count_launch();
    if (!EZ_CUDA_OK(cudaMemsetAsync(np32, 0, N * sizeof(unsigned int), st)))
      return EZMOCK_ERR_UNKNOWN;
    np_kernel<<<grid_for(N, NT), NT, 0, st>>>(m->psi[0], m->psi[1], m->psi[2], N32, Ng,
        igs, nt16, np32); ez_count_launch();
    // chunk offsets of the attached particles and an overflow flag
    const size_t aoff_b = (nblk + 1) * sizeof(unsigned long long);
    if ((e = att_buffer(m, 2 * aoff_b + 256))) return e;
    unsigned long long *acnt = (unsigned long long *) m->att;
    unsigned long long *aoff = acnt + (nblk + 1);
    int *ovf = (int *) (aoff + (nblk + 1));
    if (!EZ_CUDA_OK(cudaMemsetAsync(ovf, 0, sizeof(int), st))) return EZMOCK_ERR_UNKNOWN;
    class_kernel<<<(unsigned) nblk, NT, 0, st>>>(m->psi[0], m->psi[1], m->psi[2], N32, Ng,
        igs, nt16, np32, cls, bcnt, ovf); ez_count_launch();
    scan_u64(bcnt, bscan, nblk, ps.tmp, st);
    unsigned long long E = 0;
    int hovf = 0;
    if (!EZ_CUDA_OK(cudaMemcpyAsync(&E, bscan + nblk, 8, cudaMemcpyDeviceToHost, st)) ||
        !EZ_CUDA_OK(cudaMemcpyAsync(&hovf, ovf, sizeof(int), cudaMemcpyDeviceToHost, st)) ||
        !EZ_CUDA_OK(cudaStreamSynchronize(st)))
      return EZMOCK_ERR_UNKNOWN;
    if (hovf) { res->err = EZMOCK_ERR_RHO_NPART; return 0; }
    // contested particles: their cells, the draws of the chain (from 4N), the
    // kept flags
    if ((e = att_buffer(m, 2 * aoff_b + 256 + E * (sizeof(uint32_t) + 1)))) return e;
    acnt = (unsigned long long *) m->att;
    aoff = acnt + (nblk + 1);
    uint32_t *ecell = (uint32_t *) ((char *) m->att + 2 * aoff_b + 256);
    uint8_t *kept = (uint8_t *) (ecell + E);
    if (E) {
      entry_kernel<<<(unsigned) nblk, NT, 0, st>>>(m->psi[0], m->psi[1], m->psi[2], N32, Ng,
          igs, cls, bscan, ecell); ez_count_launch();
      if ((e = ensure_draws(m, E))) return e;
      if ((e = ez_rng_fill_free(m, ran, seed, (uint64_t) N << 2, E, m->draws))) return e;
      chain_kernel<<<1, 32, 0, st>>>(ecell, E, nt16, np32, m->draws, ran, kept);
      ez_count_launch();
    }
    att_count_kernel<<<(unsigned) nblk, NT, 0, st>>>(N32, cls, bscan, kept, acnt); ez_count_launch();
    scan_u64(acnt, aoff, nblk, ps.tmp, st);
    unsigned long long na = 0;
    if (!EZ_CUDA_OK(cudaMemcpyAsync(&na, aoff + nblk, 8, cudaMemcpyDeviceToHost, st)) ||
        !EZ_CUDA_OK(cudaStreamSynchronize(st)))
      return EZMOCK_ERR_UNKNOWN;
    if (na > nt_all) { res->err = EZMOCK_ERR_UNKNOWN; return 0; }
    iv = (size_t) na;
    if (iv) {
      att_write_kernel<<<(unsigned) nblk, NT, 0, st>>>(m->psi[0], m->psi[1], m->psi[2], N32,
          Ng, igs, gs, vfac, cls, bscan, kept, aoff, cx, cy, cz, cvx, cvy, cvz);
      ez_count_launch();
    }
    leftover_kernel<<<grid_for(N, NT), NT, 0, st>>>(nt16, np32, N32); ez_count_launch();
  }
  const size_t nrand = nt_all - iv;              // tracers at random cell positions

  // per-cell counts from the selection's candidates, unless attached tracers
  // changed them (then the remaining counts are in nt16)
  const bool usecand = !nt16 && cb.ok;
  if (usecand)
    cand_count_kernel<<<(unsigned) ((nblk + CW - 1) / CW), NT, 0, st>>>(cb.key, ps.cstart,
        ps.ccnt, bo, bcnt, nblk);
  else
    tracer_count_kernel<<<(unsigned) nblk, NT, 0, st>>>(rhot, N, bo, bcnt, nt16);
  ez_count_launch();
  scan_u64(bcnt, bscan, nblk, ps.tmp, st);
  unsigned long long ncount = 0;
  if (!EZ_CUDA_OK(cudaMemcpyAsync(&ncount, bscan + nblk, 8, cudaMemcpyDeviceToHost, st)) ||
      !EZ_CUDA_OK(cudaStreamSynchronize(st)))
    return EZMOCK_ERR_UNKNOWN;
  // the per-cell counts must add up to the selected total (pop_tracer.c:989-993)
  if (ncount != nrand) { res->err = EZMOCK_ERR_UNKNOWN; return 0; }
  // tracer cell indices in the velocity arrays (written later); before the
  // position draws, which may reuse the draws buffer holding the candidates
  void *cidv = (N <= 0xffffffffULL) ? (void *) (cvx + iv) : (void *) cvx;
  if (N <= 0xffffffffULL) {
    if (usecand)
      tracer_cell_cand_kernel<uint32_t><<<(unsigned) ((nblk + CW - 1) / CW), NT, 0, st>>>(bo,
          bscan, (unsigned long long) nrand, (uint32_t *) cidv, cb.key, cb.idx, ps.cstart,
          ps.ccnt, nblk);
    else
      tracer_cell_kernel<uint32_t><<<(unsigned) nblk, NT, 0, st>>>(rhot, N, bo, bscan,
          (unsigned long long) nrand, (uint32_t *) cidv, nt16);
  }
  else {                                            // vx and vy (iv = 0)
    if (usecand)
      tracer_cell_cand_kernel<unsigned long long><<<(unsigned) ((nblk + CW - 1) / CW), NT, 0,
          st>>>(bo, bscan, (unsigned long long) nrand, (unsigned long long *) cidv, cb.key,
          cb.idx, ps.cstart, ps.ccnt, nblk);
    else
      tracer_cell_kernel<unsigned long long><<<(unsigned) nblk, NT, 0, st>>>(rhot, N,
          bo, bscan, (unsigned long long) nrand, (unsigned long long *) cidv, nt16);
  }
  ez_count_launch();
  if ((e = ensure_draws(m, std::max((size_t) 3 * nrand, (size_t) 1)))) return e;
  const uint32_t *dpos = nullptr;
  if ((e = ez_rng_draws(m, ran, seed, 1, 3 * nrand, m->draws, &dpos))) return e;
  if (nrand) {
    if (N <= 0xffffffffULL)
      place_kernel<uint32_t><<<grid_for(nrand, NT), NT, 0, st>>>((const uint32_t *) cidv,
          nrand, Ng, dpos, ran, gs, Lbox, cx + iv, cy + iv, cz + iv);
    else
      place_kernel<unsigned long long><<<grid_for(nrand, NT), NT, 0, st>>>(
          (const unsigned long long *) cidv, nrand, Ng, dpos, ran, gs, Lbox, cx, cy, cz);
    ez_count_launch();
  }
  ez_stage_end(m, ST_EMIT);
  // the positions are final: their copy-out may overlap the velocities
  if (m->ev_pos && !EZ_CUDA_OK(cudaEventRecord(m->ev_pos, st))) return EZMOCK_ERR_UNKNOWN;

  // ---- 5./6. velocities and dispersion ----
  ez_stage_begin(m, ST_VEL);
  if (nrand) {
    if (m->paint_il)
      vel_kernel<true><<<grid_for(nrand, NT), NT, 0, st>>>(m->rho, m->paint[0],
          m->paint[1], m->paint[2], m->pq, Ng, igs, vfac, nrand, cx + iv, cy + iv, cz + iv,
          cvx + iv, cvy + iv, cvz + iv);
    else
      vel_kernel<false><<<grid_for(nrand, NT), NT, 0, st>>>(m->rho, m->paint[0],
          m->paint[1], m->paint[2], m->pq, Ng, igs, vfac, nrand, cx + iv, cy + iv, cz + iv,
          cvx + iv, cvy + iv, cvz + iv);
    ez_count_launch();
  }
  const size_t nd_disp = 6 * ((nt_all + 1) / 2);
  if ((e = ensure_draws(m, std::max(nd_disp, (size_t) 1)))) return e;
  const uint32_t *ddisp = nullptr;
  if ((e = ez_rng_draws(m, ran, seed, 2, nd_disp, m->draws, &ddisp))) return e;
  disp_kernel<<<grid_for((nt_all + 1) / 2, NT), NT, 0, st>>>(nt_all, ddisp,
      ran, (double) sigma_v, cvx, cvy, cvz); ez_count_launch();
  ez_stage_end(m, ST_VEL);
  return EZ_CUDA_OK(cudaGetLastError()) ? 0 : EZMOCK_ERR_UNKNOWN;
}
