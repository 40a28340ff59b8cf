// ez_rng.cu -- GPU random streams with absolute skip-ahead.
//
// EZmock addresses every random draw by an absolute index of one stream per
// seed: `reset(state, seed, s)` then sequential draws
// (libEZmock/EZmock/perturb.c:112-118, pop_tracer.c:233-237, :919, :1071).
// The generator library (`prand`) is not part of the reference tree; the
// definitions here are the published algorithms, with the seeding and draw
// conversions documented in ez_internal.cuh:
//
//  * MRG32k3a (L'Ecuyer 1999): every block jumps to its first draw with
//    precomputed powers A^(2^k) of the 3x3 transition matrices, every thread
//    then jumps to its sub-chunk with A^(t*G) and generates G draws, which
//    are transposed through shared memory so global stores are coalesced.
//
//  * MT19937 (Matsumoto & Nishimura 1998): the 624-word window of the stream
//    at any offset J is p(T) applied to the seed window, p = x^J mod phi
//    (Haramoto et al. 2008).  phi is found once on the host by
//    Berlekamp-Massey and the table x^(2^k) mod phi by repeated squaring.
//    Chunk c of a range [start, start + P*L) is reached directly from the
//    seed window with x^(start + c L) mod phi; the host computes these
//    polynomials once per (start, L) with carry-less products (ez_gf2.cpp)
//    and keeps them on the device.  Since T^b s is the stream's window at b,
//    p(T) s is a convolution of p's bits with the first 20k words of the
//    stream: all chunk states of a launch come from one barrier-free pass
//    over 4-bit tables (mt_jumpd_kernel).  Each chunk is then generated by
//    one block through a ring buffer, 227 words per barrier.  (Without the
//    host arithmetic the states are built with Horner's rule over 16-bit
//    windows, by one jump to `start` and log2(P) doubling levels, the scheme
//    the allocation-free entry point uses.)
#include "ez_internal.cuh"
#include "ezmock_b200.h"
#include "ez_gf2.h"

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

namespace {

// ============================================================================
//                                 MRG32k3a
// ============================================================================

constexpr uint64_t M1 = 4294967087ULL, M2 = 4294944443ULL;
constexpr uint32_t C1 = 209, C2 = 22853;          // m = 2^32 - c
constexpr uint64_t A12 = 1403580, A13N = 810728, A21 = 527612, A23N = 1370589;

constexpr int MRG_THREADS = 128;
constexpr int MRG_G = 64;                          // draws per thread
constexpr int MRG_BLOCK = MRG_THREADS * MRG_G;     // draws per block

__constant__ uint32_t c_mrg_pow1[64][9];
__constant__ uint32_t c_mrg_pow2[64][9];

__device__ __forceinline__ uint32_t mod_special(uint64_t x, uint32_t c) {
  const uint64_t m = (1ULL << 32) - c;
  uint64_t y = (x >> 32) * c + (x & 0xffffffffULL);
  y = (y >> 32) * c + (y & 0xffffffffULL);
  if (y >= m) y -= m;
  if (y >= m) y -= m;
  return (uint32_t) y;
}

__device__ __forceinline__ void matvec(const uint32_t *a, uint32_t *v,
    uint32_t c) {
  const uint64_t m = (1ULL << 32) - c;
  uint32_t t[3];
#pragma unroll
  for (int i = 0; i < 3; i++) {
    uint64_t s = 0;
#pragma unroll
    for (int k = 0; k < 3; k++)
      s += mod_special((uint64_t) a[3 * i + k] * v[k], c);
    while (s >= m) s -= m;
    t[i] = (uint32_t) s;
  }
  v[0] = t[0]; v[1] = t[1]; v[2] = t[2];
}

__device__ __forceinline__ uint32_t mrg_step(uint32_t *s1, uint32_t *s2) {
  uint64_t p1 = (uint64_t) mod_special(A12 * s1[1], C1) +
                mod_special((M1 - A13N) * s1[0], C1);
  if (p1 >= M1) p1 -= M1;
  uint64_t p2 = (uint64_t) mod_special(A21 * s2[2], C2) +
                mod_special((M2 - A23N) * s2[0], C2);
  if (p2 >= M2) p2 -= M2;
  s1[0] = s1[1]; s1[1] = s1[2]; s1[2] = (uint32_t) p1;
  s2[0] = s2[1]; s2[1] = s2[2]; s2[2] = (uint32_t) p2;
  return (uint32_t) ((p1 > p2) ? p1 - p2 : p1 + M1 - p2);
}

__global__ void __launch_bounds__(MRG_THREADS)
mrg_fill_kernel(uint32_t s10, uint32_t s11, uint32_t s12, uint32_t s20,
    uint32_t s21, uint32_t s22, uint64_t start, uint64_t count,
    const uint32_t *__restrict__ thread_jump, uint32_t *__restrict__ out) {
  __shared__ uint32_t sbuf[MRG_THREADS * (MRG_G + 1)];
  __shared__ uint32_t bstate[6];
  const uint64_t b0 = (uint64_t) blockIdx.x * MRG_BLOCK;
  if (threadIdx.x == 0) {
    uint32_t v1[3] = {s10, s11, s12}, v2[3] = {s20, s21, s22};
    uint64_t J = start + b0;
    for (int k = 0; J; k++, J >>= 1) {
      if (J & 1) {
        matvec(c_mrg_pow1[k], v1, C1);
        matvec(c_mrg_pow2[k], v2, C2);
      }
    }
    for (int i = 0; i < 3; i++) { bstate[i] = v1[i]; bstate[3 + i] = v2[i]; }
  }
  __syncthreads();
  uint32_t v1[3] = {bstate[0], bstate[1], bstate[2]};
  uint32_t v2[3] = {bstate[3], bstate[4], bstate[5]};
  const int t = threadIdx.x;
  if (t) {
    matvec(thread_jump + 18 * t, v1, C1);
    matvec(thread_jump + 18 * t + 9, v2, C2);
  }
#pragma unroll 4
  for (int i = 0; i < MRG_G; i++) sbuf[t * (MRG_G + 1) + i] = mrg_step(v1, v2);
  __syncthreads();
  for (int e = t; e < MRG_BLOCK; e += MRG_THREADS) {
    const uint64_t g = b0 + e;
    if (g < count) out[g] = sbuf[(e / MRG_G) * (MRG_G + 1) + (e % MRG_G)];
  }
}

// host-side 3x3 arithmetic modulo m
void hmat_mul(const uint64_t *a, const uint64_t *b, uint64_t *c, uint64_t m) {
  uint64_t t[9];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      unsigned __int128 s = 0;
      for (int k = 0; k < 3; k++) s += (unsigned __int128) a[3 * i + k] * b[3 * k + j];
      t[3 * i + j] = (uint64_t) (s % m);
    }
  memcpy(c, t, sizeof(t));
}

uint64_t splitmix64(uint64_t *z) {
  uint64_t r = (*z += 0x9e3779b97f4a7c15ULL);
  r = (r ^ (r >> 30)) * 0xbf58476d1ce4e5b9ULL;
  r = (r ^ (r >> 27)) * 0x94d049bb133111ebULL;
  return r ^ (r >> 31);
}

std::mutex g_mrg_mu;
// per device (constant-memory tables and a global copy of the thread jumps
// live in each device's context): tables set, thread jumps
constexpr int EZ_MAX_DEV = 64;
bool g_mrg_dev_ready[EZ_MAX_DEV];
uint32_t *g_mrg_thread_jump[EZ_MAX_DEV];  // device, MRG_THREADS x 18

int mrg_prepare(int dev) {
  std::lock_guard<std::mutex> lk(g_mrg_mu);
  if (dev < 0 || dev >= EZ_MAX_DEV) return EZMOCK_ERR_UNKNOWN;
  if (g_mrg_dev_ready[dev]) return 0;
  uint64_t p1[64][9], p2[64][9];
  const uint64_t a1[9] = {0, 1, 0, 0, 0, 1, M1 - A13N, A12, 0};
  const uint64_t a2[9] = {0, 1, 0, 0, 0, 1, M2 - A23N, 0, A21};
  memcpy(p1[0], a1, sizeof(a1));
  memcpy(p2[0], a2, sizeof(a2));
  for (int k = 1; k < 64; k++) {
    hmat_mul(p1[k - 1], p1[k - 1], p1[k], M1);
    hmat_mul(p2[k - 1], p2[k - 1], p2[k], M2);
  }
  uint32_t q1[64][9], q2[64][9];
  for (int k = 0; k < 64; k++)
    for (int i = 0; i < 9; i++) { q1[k][i] = (uint32_t) p1[k][i]; q2[k][i] = (uint32_t) p2[k][i]; }
  if (!EZ_CUDA_OK(cudaMemcpyToSymbol(c_mrg_pow1, q1, sizeof(q1))) ||
      !EZ_CUDA_OK(cudaMemcpyToSymbol(c_mrg_pow2, q2, sizeof(q2))))
    return EZMOCK_ERR_UNKNOWN;
  // A^(t*G) for t < MRG_THREADS
  std::vector<uint32_t> tj(18 * MRG_THREADS);
  uint64_t g1[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1}, g2[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  uint64_t s1[9], s2[9];          // A^G
  memcpy(s1, g1, sizeof(s1));
  memcpy(s2, g2, sizeof(s2));
  for (int k = 0; (1 << k) <= MRG_G; k++)
    if (MRG_G & (1 << k)) { hmat_mul(p1[k], s1, s1, M1); hmat_mul(p2[k], s2, s2, M2); }
  for (int t = 0; t < MRG_THREADS; t++) {
    for (int i = 0; i < 9; i++) { tj[18 * t + i] = (uint32_t) g1[i]; tj[18 * t + 9 + i] = (uint32_t) g2[i]; }
    hmat_mul(s1, g1, g1, M1);
    hmat_mul(s2, g2, g2, M2);
  }
  uint32_t *&tjd = g_mrg_thread_jump[dev];
  if (!tjd && !EZ_CUDA_OK(cudaMalloc(&tjd, tj.size() * 4))) {
    tjd = nullptr;
    return EZMOCK_ERR_MEMORY;
  }
  if (!EZ_CUDA_OK(cudaMemcpy(tjd, tj.data(), tj.size() * 4, cudaMemcpyHostToDevice)))
    return EZMOCK_ERR_MEMORY;
  g_mrg_dev_ready[dev] = true;
  return 0;
}

int mrg_fill_st(int dev, cudaStream_t st, uint64_t seed, uint64_t start,
    uint64_t count, uint32_t *out) {
  int e = mrg_prepare(dev);
  if (e) return e;
  uint64_t z = seed, s1[3], s2[3];
  for (int j = 0; j < 3; j++) s1[j] = splitmix64(&z) % M1;
  for (int j = 0; j < 3; j++) s2[j] = splitmix64(&z) % M2;
  if (!s1[0] && !s1[1] && !s1[2]) s1[0] = 1;
  if (!s2[0] && !s2[1] && !s2[2]) s2[0] = 1;
  const uint64_t nblk = (count + MRG_BLOCK - 1) / MRG_BLOCK;
  if (!nblk) return 0;
  mrg_fill_kernel<<<(unsigned) nblk, MRG_THREADS, 0, st>>>(
      (uint32_t) s1[0], (uint32_t) s1[1], (uint32_t) s1[2], (uint32_t) s2[0],
      (uint32_t) s2[1], (uint32_t) s2[2], start, count, g_mrg_thread_jump[dev], out); ez_count_launch();
  return EZ_CUDA_OK(cudaGetLastError()) ? 0 : EZMOCK_ERR_UNKNOWN;
}

int mrg_fill(EzMesh *m, uint64_t seed, uint64_t start, uint64_t count,
    uint32_t *out) {
  return mrg_fill_st(m->device, m->stream, seed, start, count, out);
}

// ============================================================================
//                                  MT19937
// ============================================================================

constexpr int MT_N = 624, MT_M = 397, MT_DEG = 19937, MT_PW = 312;
constexpr uint32_t MT_A = 0x9908b0dfU, MT_UP = 0x80000000U, MT_LO = 0x7fffffffU;
constexpr int HW = 16;                                  // Horner window bits
constexpr int HSUB = 4;                                 // bits per sub-table
constexpr int HG = HW / HSUB;                           // sub-tables
constexpr int HTAB = 1 << HSUB;                         // entries per sub-table
constexpr int H_THREADS = 640;
constexpr int G_THREADS = 640;

__host__ __device__ __forceinline__ uint32_t mt_f(uint32_t a, uint32_t b,
    uint32_t c) {   // x_{m+624} from x_m (a), x_{m+1} (b), x_{m+397} (c)
  const uint32_t y = (a & MT_UP) | (b & MT_LO);
  return c ^ (y >> 1) ^ ((y & 1U) ? MT_A : 0U);
}

__device__ __forceinline__ uint32_t mt_temper(uint32_t y) {
  y ^= y >> 11;
  y ^= (y << 7) & 0x9d2c5680U;
  y ^= (y << 15) & 0xefc60000U;
  y ^= y >> 18;
  return y;
}

// Shared-memory layout of a Horner block: HG x HTAB x MT_N table words, the
// window extended by HW words, two MT_N result buffers, one polynomial.
constexpr size_t H_SMEM_WORDS = (size_t) HG * HTAB * MT_N + 3 * MT_N + HW;
constexpr size_t H_SMEM = H_SMEM_WORDS * sizeof(uint32_t);

// Applies p(T) to the window held in ext[0, MT_N) (logical order), in place.
// Horner's rule runs over 16-bit windows of p: r <- T^16 r + sum_g
// tab_g[c_g], where tab_g[c] = sum_{j<4} c_j T^(4g+j) s are four 16-entry
// tables of combinations of the source state, so each window costs one
// barrier.  All threads of the block take part.
__device__ __forceinline__ void horner_apply(uint32_t *ext, uint32_t *tab,
    uint32_t *ra, uint32_t *rb, const uint64_t *p) {
  const int t = threadIdx.x;
  if (t < HW) ext[MT_N + t] = mt_f(ext[t], ext[t + 1], ext[MT_M + t]);
  __syncthreads();
  for (int e = t; e < HG * HTAB * MT_N; e += blockDim.x) {
    const int gc = e / MT_N, k = e - gc * MT_N;
    const int g = gc / HTAB, c = gc - g * HTAB;
    uint32_t v = 0;
#pragma unroll
    for (int j = 0; j < HSUB; j++)
      if (c & (1 << j)) v ^= ext[k + HSUB * g + j];
    tab[e] = v;
  }
  for (int k = t; k < MT_N; k += blockDim.x) ra[k] = 0;
  __syncthreads();
  uint32_t *r0 = ra, *r1 = rb;
  const int nwin = (MT_DEG + HW - 1) / HW;
  for (int q = nwin - 1; q >= 0; q--) {
    const int b = q * HW;                      // HW = 16 divides 64
    const uint32_t bits = (uint32_t) (p[b >> 6] >> (b & 63)) & 0xffffu;
    if (t < MT_N) {
      uint32_t v;
      if (t < MT_N - HW) v = r0[t + HW];
      else {
        const int s = t - (MT_N - HW);
        v = mt_f(r0[s], r0[s + 1], r0[MT_M + s]);
      }
#pragma unroll
      for (int g = 0; g < HG; g++)
        v ^= tab[(g * HTAB + ((bits >> (HSUB * g)) & (HTAB - 1))) * MT_N + t];
      r1[t] = v;
    }
    __syncthreads();
    uint32_t *tmp = r0; r0 = r1; r1 = tmp;
  }
  for (int k = t; k < MT_N; k += blockDim.x) ext[k] = r0[k];
  __syncthreads();
}

// Apply p(T) for each polynomial in `plist` (npoly entries, each MT_PW words
// in `polys`) to state in[in_base + blockIdx.x]; result to out[out_base + b].
// States are 624-word windows in logical order.  Block b applies desc[b] =
// {in state, out state, first poly, npoly}.
__global__ void __launch_bounds__(H_THREADS)
mt_horner_kernel(uint32_t *states, const int4 *__restrict__ desc,
    const uint64_t *__restrict__ polys, const int *__restrict__ plist_all) {
  extern __shared__ uint32_t sm[];
  const int4 dsc = desc[blockIdx.x];
  const int *plist = plist_all + dsc.z;
  uint32_t *tab = sm;                        // HG x HTAB x MT_N
  uint32_t *ext = tab + HG * HTAB * MT_N;    // MT_N + HW
  uint32_t *ra = ext + MT_N + HW;            // MT_N
  uint32_t *rb = ra + MT_N;                  // MT_N
  const int t = threadIdx.x;
  const uint32_t *src = states + (size_t) dsc.x * MT_N;
  for (int k = t; k < MT_N; k += blockDim.x) ext[k] = src[k];
  __syncthreads();
  for (int ip = 0; ip < dsc.w; ip++)
    horner_apply(ext, tab, ra, rb, polys + (size_t) plist[ip] * MT_PW);
  uint32_t *dst = states + (size_t) dsc.y * MT_N;
  for (int k = t; k < MT_N; k += blockDim.x) dst[k] = ext[k];
}

// Direct jumps of up to four ranges from one seed window, passed by value
// (no host-to-device copy, hence no stream synchronisation): chunk g of the
// launch (range i, chunk c = g - chunks of earlier ranges) is written to
// states[first[i] + c] = (poly[i] + c MT_PW)(T) seed.
constexpr int MT_MAXR = 4;
struct MtJumpArgs {
  uint32_t w[MT_N];                          // seed window
  int nr;
  int P[MT_MAXR];                            // chunks per range
  uint32_t first[MT_MAXR];                   // state index of chunk 0
  const uint64_t *poly[MT_MAXR];             // P polynomials each
};

// Direct jumps as one convolution.  With x_0, x_1, ... the raw stream from
// the seed window (x_0 .. x_623 the window, x_n = f(x_{n-624}, x_{n-623},
// x_{n-227})), the window T^b s is x_b .. x_{b+623}, so word w of p(T) s is
// the XOR of x_{b+w} over the set bits b of p.  Every (chunk, word) is
// independent: no barrier chain, unlike Horner's rule.  The bits of p are
// taken four at a time through 16-row tables tab[v][o] = XOR of x_{o+j} over
// the set bits j of v (built per slice of 64 nibbles from the stream in
// global memory).  In a warp the lanes are 32 chunks and every lane adds
// the same 48 words w, so a lane's nibble selects its row and the row stride
// 897 = 1 (mod 32) keeps the lanes on distinct banks (equal nibbles read
// the same word).  A block covers all 624 words for 32 chunks and one
// segment of the polynomial; the segments' partial windows are combined by
// atomic XOR into zeroed states, through shared memory so that the atomics
// are coalesced.
constexpr int JD_QB = 64;                          // nibbles per table slice
constexpr int JD_OSV = 4 * JD_QB + MT_N;           // table columns used
constexpr int JD_OS = 897;                         // row stride, 1 (mod 32)
constexpr int JD_WT = 48;                          // words per thread
constexpr int JD_THREADS = 32 * (MT_N / JD_WT);    // 13 warps
constexpr int JD_NQ = (MT_DEG + 3) / 4;            // nibbles of p
constexpr int JD_N8 = (JD_NQ + 7) / 8;             // 32-bit words of p read
constexpr int JD_XL = 20832;                       // stream words read
constexpr int JD_TP = 337;                         // transpose row stride
constexpr int JD_HALF = 7 * JD_WT;                 // words of the first half
constexpr size_t JD_SMEM = (size_t) 16 * JD_OS * sizeof(uint32_t);
static_assert(JD_OS >= JD_OSV && JD_OS % 32 == 1, "table stride");
static_assert(JD_XL >= 4 * (JD_N8 * 8 - 8) + JD_OSV + 3, "stream length");
static_assert(32 * JD_TP <= 16 * JD_OS && JD_TP >= JD_HALF && JD_TP % 2 == 1, "transpose");
static_assert(JD_HALF < MT_N && MT_N - JD_HALF <= JD_TP && MT_N % JD_WT == 0, "halves");
static_assert(JD_N8 <= 2 * MT_PW, "polynomial words");

// x_0 .. x_{JD_XL-1} of the stream from the seed window a.w.
constexpr int JD_SEQ_THREADS = 256;
__global__ void __launch_bounds__(JD_SEQ_THREADS)
mt_seq_kernel(const MtJumpArgs a, uint32_t *__restrict__ xs) {
  extern __shared__ uint32_t sx[];                 // JD_XL words
  const int t = threadIdx.x;
  for (int k = t; k < MT_N; k += JD_SEQ_THREADS) sx[k] = a.w[k];
  __syncthreads();
  constexpr int S = MT_N - MT_M;                   // 227 words per step
  for (int n0 = MT_N; n0 < JD_XL; n0 += S) {
    const int n = n0 + t;
    if (t < S && n < JD_XL) sx[n] = mt_f(sx[n - MT_N], sx[n - MT_N + 1], sx[n - S]);
    __syncthreads();
  }
  for (int k = t; k < JD_XL; k += JD_SEQ_THREADS) xs[k] = sx[k];
}

// Block (segment, group): chunks 32 group + lane of the launch, polynomial
// words [8 seg JD_N8 / nseg, ...) (a multiple of 8 nibbles each).  The
// states of the launch's chunks must be zero.
__global__ void __launch_bounds__(JD_THREADS, 2)
mt_jumpd_kernel(uint32_t *states, const MtJumpArgs a, int nst, int nseg,
    const uint32_t *__restrict__ xs) {
  extern __shared__ uint32_t tab[];                // 16 x JD_OS
  __shared__ uint32_t pws[(JD_QB / 8) * 32];       // slice words, [k][lane]
  __shared__ uint32_t *sdst[32];
  const int lane = threadIdx.x & 31, w0 = (threadIdx.x >> 5) * JD_WT;
  const int seg = blockIdx.x, grp = blockIdx.y;
  const int qa = 8 * (int) ((long) seg * JD_N8 / nseg);
  const int qb = 8 * (int) ((long) (seg + 1) * JD_N8 / nseg);
  const uint32_t *poly = nullptr;
  if (threadIdx.x < 32) {
    uint32_t *dst = nullptr;
    const int g = grp * 32 + lane;
    if (g < nst) {
      int i = 0, c = g;
      while (i < a.nr - 1 && c >= a.P[i]) { c -= a.P[i]; i++; }
      poly = (const uint32_t *) (a.poly[i] + (size_t) c * MT_PW);
      dst = states + (size_t) (a.first[i] + c) * MT_N;
    }
    sdst[lane] = dst;
  }
  uint32_t acc[JD_WT];
#pragma unroll
  for (int i = 0; i < JD_WT; i++) acc[i] = 0;
  for (int qs = qa; qs < qb; qs += JD_QB) {
    const int nk = min(JD_QB, qb - qs) >> 3;       // words of p in the slice
    __syncthreads();                               // the previous slice is read
    if (threadIdx.x < 32)
      for (int k = 0; k < JD_QB / 8; k++)
        pws[k * 32 + lane] = (poly && k < nk) ? poly[(qs >> 3) + k] : 0u;
    for (int o = threadIdx.x; o < JD_OSV; o += JD_THREADS) {
      const uint32_t *xp = xs + 4 * qs + o;
      const uint32_t x0 = xp[0], x1 = xp[1], x2 = xp[2], x3 = xp[3];
      const uint32_t t01 = x0 ^ x1, t23 = x2 ^ x3;
      uint32_t *col = tab + o;
      col[0 * JD_OS] = 0;               col[1 * JD_OS] = x0;
      col[2 * JD_OS] = x1;              col[3 * JD_OS] = t01;
      col[4 * JD_OS] = x2;              col[5 * JD_OS] = x0 ^ x2;
      col[6 * JD_OS] = x1 ^ x2;         col[7 * JD_OS] = t01 ^ x2;
      col[8 * JD_OS] = x3;              col[9 * JD_OS] = x0 ^ x3;
      col[10 * JD_OS] = x1 ^ x3;        col[11 * JD_OS] = t01 ^ x3;
      col[12 * JD_OS] = t23;            col[13 * JD_OS] = x0 ^ t23;
      col[14 * JD_OS] = x1 ^ t23;       col[15 * JD_OS] = t01 ^ t23;
    }
    __syncthreads();
    for (int k = 0; k < nk; k++) {
      const uint32_t p = pws[k * 32 + lane];
#pragma unroll
      for (int j = 0; j < 8; j++) {
        const uint32_t *tp = tab + ((p >> (4 * j)) & 15u) * JD_OS + 4 * (8 * k + j) + w0;
#pragma unroll
        for (int i = 0; i < JD_WT; i++) acc[i] ^= tp[i];
      }
    }
  }
  // partial windows to the states, half the words at a time
#pragma unroll
  for (int h = 0; h < 2; h++) {
    const int wlo = h ? JD_HALF : 0, whi = h ? MT_N : JD_HALF;
    __syncthreads();
    if (w0 >= wlo && w0 < whi) {
#pragma unroll
      for (int i = 0; i < JD_WT; i++) tab[lane * JD_TP + (w0 - wlo) + i] = acc[i];
    }
    __syncthreads();
    const int nw = whi - wlo;
    const int nc = min(32, nst - grp * 32);
    for (int e = threadIdx.x; e < nc * nw; e += JD_THREADS) {
      const int c = e / nw, w = e - c * nw;
      const uint32_t v = tab[c * JD_TP + w];
      if (v) atomicXor(sdst[c] + wlo + w, v);
    }
  }
}

// Block c generates draws [c*L, min((c+1)*L, count)) from window states[c]
// through a 2048-word ring: a round computes the 454 words 624+g .. 1077+g,
// which depend only on words g .. 623+g, as two steps of 227 (see the loop
// below).  Reads wrap with a mask (storing every word twice instead, so that
// no read wraps, costs two shared stores per word where the mask costs one
// AND, and the kernel is bound by its shared-memory traffic).
constexpr int R_THREADS = 256;
__global__ void __launch_bounds__(R_THREADS)
mt_ring_kernel(const uint32_t *__restrict__ states, uint64_t L, uint64_t count,
    uint32_t *__restrict__ out) {
  __shared__ uint32_t ring[2048];
  const int t = threadIdx.x;
  const uint64_t c0 = (uint64_t) blockIdx.x * L;
  if (c0 >= count) return;
  const uint64_t n = (count - c0 < L) ? count - c0 : L;
  for (int k = t; k < MT_N; k += R_THREADS) ring[k] = states[(size_t) blockIdx.x * MT_N + k];
  __syncthreads();
  // Step one of a round: x[b + 624] from x[b], x[b + 1], x[b + 397] for
  // b = g + t; step two: x[b + 851] from x[b + 227], x[b + 228] and
  // x[b + 624], step one's result in the same thread.  A round reads words
  // [g, g + 624) and writes [g + 624, g + 1078); the words it overwrites,
  // [g - 1424, g - 970) mod 2048, are no longer needed.
  constexpr int S = MT_N - MT_M;
  constexpr uint32_t W = 2047;
  uint32_t *o = out + c0 + t;
  uint32_t p = (uint32_t) t;                     // (g + t) mod 2048
  const uint64_t nfull = n / (2 * S);
  for (uint64_t r = 0; r < nfull; r++) {
    if (t < S) {
      const uint32_t y = mt_f(ring[p], ring[(p + 1) & W], ring[(p + MT_M) & W]);
      const uint32_t y2 = mt_f(ring[(p + S) & W], ring[(p + S + 1) & W], y);
      ring[(p + MT_N) & W] = y;
      ring[(p + MT_N + S) & W] = y2;
      o[0] = mt_temper(y);
      o[S] = mt_temper(y2);
    }
    o += 2 * S;
    p = (p + 2 * S) & W;
    __syncthreads();
  }
  const uint64_t rem = n - nfull * (2 * S);      // the last, partial round
  if (rem && t < S) {
    const uint32_t y = mt_f(ring[p], ring[(p + 1) & W], ring[(p + MT_M) & W]);
    const uint32_t y2 = mt_f(ring[(p + S) & W], ring[(p + S + 1) & W], y);
    if ((uint64_t) t < rem) o[0] = mt_temper(y);
    if ((uint64_t) (S + t) < rem) o[S] = mt_temper(y2);
  }
}

// Block c generates draws [c*L, min((c+1)*L, count)) from window states[c].
__global__ void __launch_bounds__(G_THREADS)
mt_gen_kernel(const uint32_t *__restrict__ states, uint64_t L, uint64_t count,
    uint32_t *__restrict__ out) {
  __shared__ uint32_t wa[MT_N], wb[MT_N];
  const int t = threadIdx.x;
  const uint64_t c0 = (uint64_t) blockIdx.x * L;
  if (c0 >= count) return;
  const uint64_t c1 = (c0 + L < count) ? c0 + L : count;
  for (int k = t; k < MT_N; k += blockDim.x) wa[k] = states[(size_t) blockIdx.x * MT_N + k];
  __syncthreads();
  uint32_t *o = wa, *n = wb;
  for (uint64_t g = c0; g < c1; g += MT_N) {
    // x_{m+624+t} = x_{m+397+t} ^ f(x_{m+t}, x_{m+t+1}), in three phases
    if (t < 227) n[t] = mt_f(o[t], o[t + 1], o[MT_M + t]);
    __syncthreads();
    if (t >= 227 && t < 454) n[t] = mt_f(o[t], o[t + 1], n[t - 227]);
    __syncthreads();
    if (t >= 454 && t < MT_N)
      n[t] = mt_f(o[t], (t + 1 < MT_N) ? o[t + 1] : n[0], n[t - 227]);
    __syncthreads();
    if (t < MT_N && g + t < c1) out[g + t] = mt_temper(n[t]);
    uint32_t *tmp = o; o = n; n = tmp;
    __syncthreads();
  }
}

// ---- host: characteristic polynomial and x^(2^k) table ----
inline int hbit(const uint64_t *a, long b) { return (int) ((a[b >> 6] >> (b & 63)) & 1ULL); }

struct MtTables {
  bool ok = false;
  std::vector<uint64_t> phi;                 // MT_PW + 1 words
  std::vector<uint64_t> xpow;                // 64 x MT_PW
};

void mt_seed_window(uint64_t seed, uint32_t *w) {
  if (seed <= 0xffffffffULL) {
    w[0] = (uint32_t) seed;
    for (int i = 1; i < MT_N; i++) w[i] = 1812433253U * (w[i - 1] ^ (w[i - 1] >> 30)) + (uint32_t) i;
    return;
  }
  const uint32_t key[2] = {(uint32_t) seed, (uint32_t) (seed >> 32)};
  w[0] = 19650218U;
  for (int i = 1; i < MT_N; i++) w[i] = 1812433253U * (w[i - 1] ^ (w[i - 1] >> 30)) + (uint32_t) i;
  int i = 1, j = 0;
  for (int k = MT_N; k; k--) {
    w[i] = (w[i] ^ ((w[i - 1] ^ (w[i - 1] >> 30)) * 1664525U)) + key[j] + (uint32_t) j;
    i++; j++;
    if (i >= MT_N) { w[0] = w[MT_N - 1]; i = 1; }
    if (j >= 2) j = 0;
  }
  for (int k = MT_N - 1; k; k--) {
    w[i] = (w[i] ^ ((w[i - 1] ^ (w[i - 1] >> 30)) * 1566083941U)) - (uint32_t) i;
    i++;
    if (i >= MT_N) { w[0] = w[MT_N - 1]; i = 1; }
  }
  w[0] = 0x80000000U;
}

void build_mt_tables(MtTables &T) {
  // Berlekamp-Massey on the top bit of the raw words of one stream.
  const long len = 2L * MT_DEG + 128;
  const long nw = (len + 63) / 64 + 2;
  std::vector<uint64_t> rev(nw, 0), C(nw, 0), B(nw, 0), Tt(nw, 0);
  {
    std::vector<uint32_t> w(MT_N);
    mt_seed_window(5489U, w.data());
    int pos = 0;
    for (long n = 0; n < len; n++) {
      const int p1 = (pos + 1) % MT_N, pm = (pos + MT_M) % MT_N;
      const uint32_t x = mt_f(w[pos], w[p1], w[pm]);
      w[pos] = x;
      pos = p1;
      const long tpos = len - 1 - n;
      if (x >> 31) rev[tpos >> 6] |= 1ULL << (tpos & 63);
    }
  }
  C[0] = B[0] = 1;
  long L = 0, m = 1;
  auto add_shift = [&](std::vector<uint64_t> &dst, const std::vector<uint64_t> &src, long sh) {
    const long ws = sh >> 6, bs = sh & 63;
    for (long w = nw - 1; w >= 0; w--) {
      uint64_t v = 0;
      if (w - ws >= 0) v = src[w - ws] << bs;
      if (bs && w - ws - 1 >= 0) v |= src[w - ws - 1] >> (64 - bs);
      dst[w] ^= v;
    }
  };
  for (long n = 0; n < len; n++) {
    const long o = len - 1 - n;
    const long lw = L / 64 + 1;
    uint64_t acc = 0;
    for (long w = 0; w < lw; w++) {
      const long b = o + 64 * w, bw = b >> 6, bs = b & 63;
      uint64_t v = rev[bw] >> bs;
      if (bs && bw + 1 < nw) v |= rev[bw + 1] << (64 - bs);
      acc ^= C[w] & v;
    }
    if (!__builtin_parityll(acc)) { m++; continue; }
    if (2 * L <= n) {
      Tt = C;
      add_shift(C, B, m);
      L = n + 1 - L;
      B = Tt;
      m = 1;
    }
    else { add_shift(C, B, m); m++; }
  }
  if (L != MT_DEG) return;
  T.phi.assign(MT_PW + 1, 0);
  for (long j = 0; j <= L; j++)
    if (hbit(C.data(), L - j)) T.phi[j >> 6] |= 1ULL << (j & 63);
  // phi << s for s < 64
  std::vector<uint64_t> sh(64 * (MT_PW + 2), 0);
  for (int s = 0; s < 64; s++)
    for (int w = 0; w <= MT_PW; w++) {
      sh[s * (MT_PW + 2) + w] ^= T.phi[w] << s;
      if (s) sh[s * (MT_PW + 2) + w + 1] ^= T.phi[w] >> (64 - s);
    }
  auto spread = [](uint32_t v) {
    uint64_t x = v;
    x = (x | (x << 16)) & 0x0000ffff0000ffffULL;
    x = (x | (x << 8)) & 0x00ff00ff00ff00ffULL;
    x = (x | (x << 4)) & 0x0f0f0f0f0f0f0f0fULL;
    x = (x | (x << 2)) & 0x3333333333333333ULL;
    x = (x | (x << 1)) & 0x5555555555555555ULL;
    return x;
  };
  T.xpow.assign(64 * MT_PW, 0);
  T.xpow[0] = 2;                                         // x
  std::vector<uint64_t> r(2 * MT_PW + 4);
  for (int k = 1; k < 64; k++) {
    std::fill(r.begin(), r.end(), 0);
    const uint64_t *prev = &T.xpow[(k - 1) * MT_PW];
    for (int w = 0; w < MT_PW; w++) {
      r[2 * w] = spread((uint32_t) prev[w]);
      r[2 * w + 1] = spread((uint32_t) (prev[w] >> 32));
    }
    for (long b = 2L * MT_DEG; b >= MT_DEG; b--) {
      if (!hbit(r.data(), b)) continue;
      const long t = b - MT_DEG, ws = t >> 6;
      const uint64_t *ph = &sh[(t & 63) * (MT_PW + 2)];
      for (long w = 0; w < MT_PW + 2 && ws + w < (long) r.size(); w++) r[ws + w] ^= ph[w];
    }
    memcpy(&T.xpow[k * MT_PW], r.data(), MT_PW * sizeof(uint64_t));
  }
  T.ok = true;
}

std::mutex g_mt_mu;
MtTables g_mt;
bool g_mt_built = false;
// per device: set up, SM count, device copy of the x^(2^k) table
bool g_mt_dev_ready[EZ_MAX_DEV];
int g_mt_nsm[EZ_MAX_DEV];
uint64_t *g_mt_xpow_dev[EZ_MAX_DEV];

int mt_prepare(int dev) {
  std::lock_guard<std::mutex> lk(g_mt_mu);
  if (!g_mt_built) { build_mt_tables(g_mt); g_mt_built = true; }
  if (!g_mt.ok) return EZMOCK_ERR_RNG_SET;
  if (dev < 0 || dev >= EZ_MAX_DEV) return EZMOCK_ERR_UNKNOWN;
  if (g_mt_dev_ready[dev]) return 0;
  uint64_t *&xp = g_mt_xpow_dev[dev];
  if (!xp && !EZ_CUDA_OK(cudaMalloc(&xp, g_mt.xpow.size() * 8))) {
    xp = nullptr;
    return EZMOCK_ERR_MEMORY;
  }
  if (!EZ_CUDA_OK(cudaMemcpy(xp, g_mt.xpow.data(), g_mt.xpow.size() * 8,
          cudaMemcpyHostToDevice)))
    return EZMOCK_ERR_MEMORY;
  if (!EZ_CUDA_OK(cudaFuncSetAttribute(mt_horner_kernel,
          cudaFuncAttributeMaxDynamicSharedMemorySize,
          (int) H_SMEM)) ||
      !EZ_CUDA_OK(cudaFuncSetAttribute(mt_seq_kernel,
          cudaFuncAttributeMaxDynamicSharedMemorySize, (int) (JD_XL * sizeof(uint32_t)))) ||
      !EZ_CUDA_OK(cudaFuncSetAttribute(mt_jumpd_kernel,
          cudaFuncAttributeMaxDynamicSharedMemorySize, (int) JD_SMEM)) ||
      !EZ_CUDA_OK(cudaDeviceGetAttribute(&g_mt_nsm[dev], cudaDevAttrMultiProcessorCount, dev)))
    return EZMOCK_ERR_UNKNOWN;
  g_mt_dev_ready[dev] = true;
  return 0;
}

// A range of one stream: chunk c starts at draw `start + c L` (L = 2^l,
// c < P = 2^p); its window is states[first + c].
struct MtRange {
  uint64_t start, cap;
  int l, p;                // chunk length 2^l; doubling plans: 2^p chunks
  int P;                   // chunks
  size_t first;
};

MtRange mt_plan(uint64_t start, uint64_t cap) {
  // at most 128 chunks per range, so a doubling level over three ranges
  // stays within a few waves of blocks
  MtRange r;
  r.start = start;
  r.cap = cap;
  r.l = 12;
  r.p = 0;
  while ((1ULL << r.l) * 128ULL < cap && r.l < 40) r.l++;
  while (((uint64_t) 1 << (r.l + r.p)) < cap) r.p++;
  r.P = 1 << r.p;
  r.first = 0;
  return r;
}

// Chunk states of `nr` ranges of the stream seeded by `seed`, computed
// together: one launch for the jumps to the range starts, then one launch per
// doubling level covering all ranges.  State 0 is the seed window; the
// states live at `base` in the RNG scratch.
int mt_prepare_ranges(EzMesh *m, uint64_t seed, MtRange *r, int nr,
    size_t base) {
  int e = mt_prepare(m->device);
  if (e) return e;
  size_t nst = 1;
  int pmax = 0;
  for (int i = 0; i < nr; i++) {
    r[i].first = base + nst;
    nst += (size_t) 1 << r[i].p;
    pmax = std::max(pmax, r[i].p);
  }
  std::vector<int> plist;
  std::vector<int4> desc;
  std::vector<int> lev_off(pmax + 2), lev_n(pmax + 2);
  lev_off[0] = 0;
  for (int i = 0; i < nr; i++) {          // level "base": seed -> range start
    int4 d;
    d.x = (int) base;
    d.y = (int) r[i].first;
    d.z = (int) plist.size();
    for (int k = 0; k < 64; k++)
      if ((r[i].start >> k) & 1ULL) plist.push_back(k);
    d.w = (int) plist.size() - d.z;
    desc.push_back(d);
  }
  lev_n[0] = nr;
  for (int lev = 0; lev < pmax; lev++) {
    lev_off[lev + 1] = (int) desc.size();
    for (int i = 0; i < nr; i++) {
      if (lev >= r[i].p) continue;
      const int pk = (int) plist.size();
      plist.push_back(r[i].l + lev);
      for (int t = 0; t < (1 << lev); t++) {
        int4 d;
        d.x = (int) (r[i].first + t);
        d.y = (int) (r[i].first + t + (1 << lev));
        d.z = pk;
        d.w = 1;
        desc.push_back(d);
      }
    }
    lev_n[lev + 1] = (int) desc.size() - lev_off[lev + 1];
  }
  const size_t st_bytes = (base + nst) * MT_N * sizeof(uint32_t);
  const size_t d_bytes = desc.size() * sizeof(int4);
  const size_t need = st_bytes + d_bytes + plist.size() * sizeof(int) + 512;
  if ((e = ez_rng_scratch(m, need))) return e;
  uint32_t *states = (uint32_t *) m->rng_scratch;
  int4 *d_desc = (int4 *) ((char *) m->rng_scratch + (st_bytes + 15) / 16 * 16);
  int *d_plist = (int *) ((char *) d_desc + d_bytes);
  std::vector<uint32_t> w(MT_N);
  mt_seed_window(seed, w.data());
  if (!EZ_CUDA_OK(cudaMemcpyAsync(states + base * MT_N, w.data(), MT_N * 4,
          cudaMemcpyHostToDevice, m->stream)) ||
      !EZ_CUDA_OK(cudaMemcpyAsync(d_desc, desc.data(), d_bytes, cudaMemcpyHostToDevice, m->stream)) ||
      (plist.size() && !EZ_CUDA_OK(cudaMemcpyAsync(d_plist, plist.data(),
          plist.size() * sizeof(int), cudaMemcpyHostToDevice, m->stream))))
    return EZMOCK_ERR_UNKNOWN;
  const size_t smem = (HG * HTAB * MT_N + 3 * MT_N + HW) * sizeof(uint32_t);
  for (int lev = 0; lev <= pmax; lev++) {
    if (!lev_n[lev]) continue;
    mt_horner_kernel<<<lev_n[lev], H_THREADS, smem, m->stream>>>(states,
        d_desc + lev_off[lev], g_mt_xpow_dev[m->device], d_plist); ez_count_launch();
  }
  // (copies from pageable host memory are staged before cudaMemcpyAsync
  // returns, so the host vectors may be released here)
  return EZ_CUDA_OK(cudaGetLastError()) ? 0 : EZMOCK_ERR_UNKNOWN;
}

// ---- direct jumps ----
// Chunk c of a range starts at draw start + c L; its window is
// (x^(start + c L) mod phi)(T) applied to the seed window.  The polynomials
// depend only on (start, L), so the host computes them once (carry-less
// products reduced modulo phi, ez_gf2.cpp) and keeps them on the device;
// every fill then needs one Horner pass per chunk, all chunks in one launch,
// instead of a jump followed by log2(chunks) dependent doubling levels.
// Chunks per fill: two per SM.  (Measured at 512^3: 592 or 1184 chunks
// cost more in jumps than the shorter chunks save in generation.)
constexpr int MT_CHUNKS = 296;

bool g_gf2_tried = false, g_gf2_ok = false;

// Under g_mt_mu with the tables built: set up the modular arithmetic and
// check it against the squaring table (x^(2^(k+1)) = (x^(2^k))^2 mod phi).
bool gf2_ready() {
  if (g_gf2_tried) return g_gf2_ok;
  g_gf2_tried = true;
  if (!g_mt.ok || !ez_gf2_init(g_mt.phi.data(), MT_DEG, MT_PW)) return false;
  std::vector<uint64_t> sq(MT_PW);
  for (int k : {14, 15, 21, 40, 62}) {
    ez_gf2_mulmod(&g_mt.xpow[(size_t) k * MT_PW], &g_mt.xpow[(size_t) k * MT_PW], sq.data());
    if (memcmp(sq.data(), &g_mt.xpow[(size_t) (k + 1) * MT_PW], MT_PW * sizeof(uint64_t)))
      return false;
  }
  g_gf2_ok = true;
  return true;
}

struct JumpSeq {
  std::vector<uint64_t> host;               // polynomials c = 0, 1, ...
  uint64_t *dev = nullptr;                  // device copy of the first ndev
  size_t ndev = 0;
};
std::map<std::tuple<int, uint64_t, int>, JumpSeq> g_jumps;   // (device, start, l)
// replaced device copies: queued kernels may still read them, so they are
// kept for the life of the process
std::vector<uint64_t *> g_jumps_retired;

// Under g_mt_mu, with device `dev` current: device polynomials
// x^(start + c 2^l) mod phi for c < P.
const uint64_t *jump_polys(int dev, uint64_t start, int l, size_t P) {
  JumpSeq &js = g_jumps[std::make_tuple(dev, start, l)];
  size_t nh = js.host.size() / MT_PW;
  if (nh < P) {
    js.host.resize(P * MT_PW);
    uint64_t *h = js.host.data();
    if (nh == 0) {
      std::vector<uint64_t> t(MT_PW);
      std::fill(h, h + MT_PW, 0);
      h[0] = 1;                               // x^0
      for (int k = 0; k < 64; k++)
        if ((start >> k) & 1ULL) {
          ez_gf2_mulmod(h, &g_mt.xpow[(size_t) k * MT_PW], t.data());
          memcpy(h, t.data(), MT_PW * sizeof(uint64_t));
        }
      nh = 1;
    }
    for (size_t c = nh; c < P; c++)
      ez_gf2_mulmod(h + (c - 1) * MT_PW, &g_mt.xpow[(size_t) l * MT_PW], h + c * MT_PW);
  }
  if (js.ndev < P) {
    uint64_t *d = nullptr;
    if (!EZ_CUDA_OK(cudaMalloc(&d, P * MT_PW * sizeof(uint64_t)))) { cudaGetLastError(); return nullptr; }
    if (!EZ_CUDA_OK(cudaMemcpy(d, js.host.data(), P * MT_PW * sizeof(uint64_t),
            cudaMemcpyHostToDevice))) {
      cudaFree(d);
      return nullptr;
    }
    if (js.dev) g_jumps_retired.push_back(js.dev);
    js.dev = d;
    js.ndev = P;
  }
  return js.dev;
}

// Chunk length 2^l >= 4096 so that at most `target` chunks cover `cap`.
void plan_direct(MtRange &r, int target) {
  if (target < 1) target = 1;
  r.l = 12;
  while (((r.cap + (1ULL << r.l) - 1) >> r.l) > (uint64_t) target && r.l < 62) r.l++;
  r.P = (int) std::max<uint64_t>(1, (r.cap + (1ULL << r.l) - 1) >> r.l);
  r.p = -1;
  r.first = 0;
}

// Direct jumps available (tables built, modular arithmetic checked).
bool mt_direct(int dev) {
  if (mt_prepare(dev)) return false;
  std::lock_guard<std::mutex> lk(g_mt_mu);
  return gf2_ready();
}

// Chunk states of `nr` <= MT_MAXR planned ranges; the chunks of range i are
// stored from state index r[i].first = base + (chunks of earlier ranges) of
// `states`, which holds at least base + sum P states.  One launch on `st`,
// one block per chunk.
int mt_jump_launch(int dev, cudaStream_t st, uint32_t *states, uint64_t seed,
    MtRange *r, int nr, size_t base) {
  if (nr > MT_MAXR) return EZMOCK_ERR_UNKNOWN;
  MtJumpArgs a;
  a.nr = nr;
  size_t nst = 0;
  {
    std::lock_guard<std::mutex> lk(g_mt_mu);
    for (int i = 0; i < nr; i++) {
      r[i].first = base + nst;
      const uint64_t *d = jump_polys(dev, r[i].start, r[i].l, (size_t) r[i].P);
      if (!d) return EZMOCK_ERR_MEMORY;
      a.P[i] = r[i].P;
      a.first[i] = (uint32_t) r[i].first;
      a.poly[i] = d;
      nst += (size_t) r[i].P;
    }
  }
  if (!nst) return 0;
  mt_seed_window(seed, a.w);
  // the stream words after the states; two blocks per SM in one wave
  uint32_t *xs = states + (base + nst) * MT_N;
  const int ncg = (int) ((nst + 31) / 32);
  const int nseg = std::max(1, std::min(JD_N8, 2 * g_mt_nsm[dev] / ncg));
  if (!EZ_CUDA_OK(cudaMemsetAsync(states + base * MT_N, 0, nst * MT_N * sizeof(uint32_t), st)))
    return EZMOCK_ERR_UNKNOWN;
  mt_seq_kernel<<<1, JD_SEQ_THREADS, JD_XL * sizeof(uint32_t), st>>>(a, xs);
  ez_count_launch();
  mt_jumpd_kernel<<<dim3((unsigned) nseg, (unsigned) ncg), JD_THREADS, JD_SMEM, st>>>(
      states, a, (int) nst, nseg, xs);
  ez_count_launch();
  return EZ_CUDA_OK(cudaGetLastError()) ? 0 : EZMOCK_ERR_UNKNOWN;
}

// States (624 words each) a launch of `nr` ranges needs from `base`, with
// the stream words of the direct jumps after them.
size_t mt_states_needed(const MtRange *r, int nr, size_t base) {
  size_t n = base;
  for (int i = 0; i < nr; i++) n += (size_t) r[i].P;
  return n + (JD_XL + MT_N - 1) / MT_N;
}

int mt_prepare_direct(EzMesh *m, uint64_t seed, MtRange *r, int nr, size_t base) {
  int e = ez_rng_scratch(m, mt_states_needed(r, nr, base) * MT_N * sizeof(uint32_t));
  if (e) return e;
  return mt_jump_launch(m->device, m->stream, (uint32_t *) m->rng_scratch, seed, r, nr, base);
}

// Draws [r.start, r.start + count) from the chunk states of r in `states`.
int mt_gen_launch(cudaStream_t st, const uint32_t *states, const MtRange &r,
    uint64_t count, uint32_t *out) {
  if (!count) return 0;
  const uint64_t L = 1ULL << r.l;
  const uint64_t nb = (count + L - 1) / L;
  if (nb > (uint64_t) r.P) return EZMOCK_ERR_UNKNOWN;
  mt_ring_kernel<<<(unsigned) nb, R_THREADS, 0, st>>>(states + r.first * MT_N, L, count, out);
  ez_count_launch();
  return EZ_CUDA_OK(cudaGetLastError()) ? 0 : EZMOCK_ERR_UNKNOWN;
}

int mt_generate(EzMesh *m, const MtRange &r, uint64_t count, uint32_t *out) {
  return mt_gen_launch(m->stream, (const uint32_t *) m->rng_scratch, r, count, out);
}

// One chunk length for all ranges (generation time is set by the longest
// chunk): the shortest whose chunks fit the block budget.
void plan_common(MtRange *r, const uint64_t *starts, const uint64_t *caps, int n) {
  int l = 12;
  for (;; l++) {
    uint64_t tot = 0;
    for (int i = 0; i < n; i++)
      tot += (std::max<uint64_t>(caps[i], 1) + (1ULL << l) - 1) >> l;
    if (tot <= (uint64_t) MT_CHUNKS || l >= 62) break;
  }
  for (int i = 0; i < n; i++) {
    r[i].start = starts[i];
    r[i].cap = std::max<uint64_t>(caps[i], 1);
    r[i].l = l;
    r[i].P = (int) ((r[i].cap + (1ULL << l) - 1) >> l);
    r[i].p = -1;
    r[i].first = 0;
  }
}

int mt_fill(EzMesh *m, uint64_t seed, uint64_t start, uint64_t count,
    uint32_t *out, size_t base) {
  if (!count) return 0;
  MtRange r;
  int e;
  if (mt_direct(m->device)) {
    r.start = start;
    r.cap = count;
    plan_direct(r, MT_CHUNKS);
    e = mt_prepare_direct(m, seed, &r, 1, base);
  }
  else {
    r = mt_plan(start, count);
    e = mt_prepare_ranges(m, seed, &r, 1, base);
  }
  if (e) return e;
  return mt_generate(m, r, count, out);
}

}  // namespace

int ez_rng_fill_around(EzMesh *m, int ran, uint64_t seed, uint64_t start,
    uint64_t count, uint32_t *out, void (*between)(void *), void *arg) {
  m->rng_nprep = 0;
  if (ran == EZMOCK_RNG_MT19937 && count && mt_direct(m->device)) {
    MtRange r;
    r.start = start;
    r.cap = count;
    plan_direct(r, MT_CHUNKS);
    int e = mt_prepare_direct(m, seed, &r, 1, 0);
    if (e) return e;
    between(arg);
    return mt_generate(m, r, count, out);
  }
  const int e = ez_rng_fill(m, ran, seed, start, count, out);
  if (!e) between(arg);
  return e;
}

int ez_rng_fill_free(EzMesh *m, int ran, uint64_t seed, uint64_t start,
    uint64_t count, uint32_t *out) {
  if (ran == EZMOCK_RNG_MT19937)
    return mt_fill(m, seed, start, count, out, m->rng_nprep ? m->rng_prep_end : 0);
  return mrg_fill(m, seed, start, count, out);
}

int ez_rng_fill(EzMesh *m, int ran, uint64_t seed, uint64_t start,
    uint64_t count, uint32_t *out) {
  m->rng_nprep = 0;                         // the scratch is reused
  if (ran == EZMOCK_RNG_MT19937) return mt_fill(m, seed, start, count, out, 0);
  return mrg_fill(m, seed, start, count, out);
}

int ez_rng_prepare(EzMesh *m, int ran, uint64_t seed, const uint64_t *starts,
    const uint64_t *caps, int n) {
  m->rng_nprep = 0;
  // the side stream's position/dispersion generation reads the states about
  // to be replaced
  if (m->pop_pending) {
    if (!EZ_CUDA_OK(cudaStreamWaitEvent(m->stream, m->ev_pop, 0))) return EZMOCK_ERR_UNKNOWN;
    m->pop_pending = false;
  }
  if (n > EZ_RNG_MAXPREP) return EZMOCK_ERR_UNKNOWN;
  // ranges the side stream prepared for this seed and generator
  bool side[EZ_RNG_MAXPREP] = {false, false, false, false};
  if (m->pre_valid && m->pre_seed == seed && m->pre_ran == ran) {
    for (int i = 0; i < n && i < m->pre_n; i++)
      side[i] = m->pre[i].start == starts[i] && m->pre[i].cap >= caps[i];
    if (side[0] || side[1] || side[2]) {
      if (!EZ_CUDA_OK(cudaStreamWaitEvent(m->stream, m->ev_side, 0))) return EZMOCK_ERR_UNKNOWN;
    }
  }
  for (int i = 0; i < n; i++) {
    m->rng_prep[i].start = starts[i];
    m->rng_prep[i].cap = caps[i];
    m->rng_prep[i].side = side[i];
    if (side[i]) {
      m->rng_prep[i].l = m->pre[i].l;
      m->rng_prep[i].P = m->pre[i].P;
      m->rng_prep[i].first = m->pre[i].first;
    }
  }
  if (ran == EZMOCK_RNG_MT19937) {
    // the remaining ranges, prepared together on the instance stream
    MtRange r[EZ_RNG_MAXPREP];
    uint64_t st2[EZ_RNG_MAXPREP], cp2[EZ_RNG_MAXPREP];
    int idx[EZ_RNG_MAXPREP], k = 0;
    for (int i = 0; i < n; i++)
      if (!side[i]) { idx[k] = i; st2[k] = starts[i]; cp2[k] = caps[i] ? caps[i] : 1; k++; }
    size_t end = 0;
    if (k) {
      int e;
      if (mt_direct(m->device)) {
        plan_common(r, st2, cp2, k);
        e = mt_prepare_direct(m, seed, r, k, 0);
      }
      else {
        for (int j = 0; j < k; j++) r[j] = mt_plan(st2[j], cp2[j]);
        e = mt_prepare_ranges(m, seed, r, k, 0);
      }
      if (e) return e;
      for (int j = 0; j < k; j++) {
        const int i = idx[j];
        m->rng_prep[i].l = r[j].l;
        m->rng_prep[i].P = r[j].P;
        m->rng_prep[i].first = r[j].first;
        end = std::max(end, r[j].first + (size_t) r[j].P);
      }
    }
    m->rng_prep_end = end;
  }
  m->rng_nprep = n;
  return 0;
}

int ez_rng_draws(EzMesh *m, int ran, uint64_t seed, int i, uint64_t count,
    uint32_t *out, const uint32_t **res) {
  *res = out;
  const bool prepared = i < m->rng_nprep && count <= m->rng_prep[i].cap;
  if (prepared && i == 0 && m->rng_prep[0].side && count <= m->pre_bias_n) {
    *res = m->draws_bias;                   // generated on the side stream
    return 0;
  }
  if (prepared && (i == 1 || i == 2) && count <= m->pre_pop_n[i - 1]) {
    // generated on the side stream at the start of the population
    if (!EZ_CUDA_OK(cudaStreamWaitEvent(m->stream, m->ev_pop, 0))) return EZMOCK_ERR_UNKNOWN;
    *res = m->draws_pop + (i == 2 ? m->pre_pop_n[0] : 0);
    return 0;
  }
  const uint64_t start = m->rng_prep[i < m->rng_nprep ? i : 0].start;
  if (ran != EZMOCK_RNG_MT19937) return mrg_fill(m, seed, start, count, out);
  if (!prepared)
    // beyond the prepared capacity: states after the prepared ones
    return mt_fill(m, seed, start, count, out, m->rng_nprep ? m->rng_prep_end : 0);
  MtRange r;
  r.start = m->rng_prep[i].start;
  r.cap = m->rng_prep[i].cap;
  r.l = m->rng_prep[i].l;
  r.P = m->rng_prep[i].P;
  r.p = -1;
  r.first = m->rng_prep[i].first;
  return mt_gen_launch(m->stream,
      (const uint32_t *) (m->rng_prep[i].side ? m->rng_side : m->rng_scratch), r, count, out);
}

// Side buffer for the position and dispersion draws (false: none).
bool side_pop_buffer(EzMesh *m, uint64_t words) {
  if (!words) return false;
  if (words > m->draws_pop_cap) {
    if (m->draws_pop) cudaFree(m->draws_pop);
    m->draws_pop = nullptr;
    m->draws_pop_cap = 0;
    if (!EZ_CUDA_OK(cudaMalloc(&m->draws_pop, words * sizeof(uint32_t)))) {
      cudaGetLastError();
      return false;
    }
    m->draws_pop_cap = words;
  }
  return true;
}

// The position and dispersion ranges (prepared ranges 1 and 2 of the
// population, at their prepared capacities) generated on the side stream while
// the instance stream runs the bias and selection stages; ez_rng_draws makes
// the instance stream wait for them.  Their chunks are few and long (the
// chunk length is shared with the bias range), so on the instance stream their
// generation would be latency on the critical path.
void ez_rng_side_pop(EzMesh *m, int ran, uint64_t seed) {
  m->pre_pop_n[0] = m->pre_pop_n[1] = 0;
  if (m->rng_nprep < 3 || !m->side || !m->ev_pop) return;
  const uint64_t c1 = m->rng_prep[1].cap, c2 = m->rng_prep[2].cap;
  if (!side_pop_buffer(m, c1 + c2)) return;
  if (!EZ_CUDA_OK(cudaEventRecord(m->ev_main, m->stream)) ||
      !EZ_CUDA_OK(cudaStreamWaitEvent(m->side, m->ev_main, 0)))
    return;
  uint32_t *out[2] = {m->draws_pop, m->draws_pop + c1};
  for (int i = 1; i <= 2; i++) {
    const EzMesh::EzRange &p = m->rng_prep[i];
    int e;
    if (ran == EZMOCK_RNG_MT19937) {
      MtRange r;
      r.start = p.start;
      r.cap = p.cap;
      r.l = p.l;
      r.P = p.P;
      r.p = -1;
      r.first = p.first;
      e = mt_gen_launch(m->side, (const uint32_t *) (p.side ? m->rng_side : m->rng_scratch),
          r, p.cap, out[i - 1]);
    }
    else e = mrg_fill_st(m->device, m->side, seed, p.start, p.cap, out[i - 1]);
    if (e) return;
  }
  if (!EZ_CUDA_OK(cudaEventRecord(m->ev_pop, m->side))) return;
  m->pop_pending = true;
  m->pre_pop_n[0] = c1;
  m->pre_pop_n[1] = c2;
}

void ez_rng_side_prepare(EzMesh *m, int ran, uint64_t seed,
    const uint64_t *starts, const uint64_t *caps, int n, uint64_t nbias) {
  m->pre_valid = false;
  if (n < 1 || n > 3 || !nbias) return;
  if (ran == EZMOCK_RNG_MT19937 && !mt_direct(m->device)) return;
  if (!m->side) {
    int lo = 0, hi = 0;
    cudaDeviceGetStreamPriorityRange(&lo, &hi);       // lo: lowest priority
    if (!EZ_CUDA_OK(cudaStreamCreateWithPriority(&m->side, cudaStreamNonBlocking, lo)) ||
        !EZ_CUDA_OK(cudaEventCreateWithFlags(&m->ev_main, cudaEventDisableTiming)) ||
        !EZ_CUDA_OK(cudaEventCreateWithFlags(&m->ev_side, cudaEventDisableTiming)) ||
        !EZ_CUDA_OK(cudaEventCreateWithFlags(&m->ev_pop, cudaEventDisableTiming))) {
      cudaGetLastError();
      return;
    }
  }
  if (nbias > m->draws_bias_cap) {
    if (m->draws_bias) cudaFree(m->draws_bias);
    m->draws_bias = nullptr;
    m->draws_bias_cap = 0;
    if (!EZ_CUDA_OK(cudaMalloc(&m->draws_bias, nbias * sizeof(uint32_t)))) { cudaGetLastError(); return; }
    m->draws_bias_cap = nbias;
  }
  // the side buffers may still be read by earlier work of the instance stream
  if (!EZ_CUDA_OK(cudaEventRecord(m->ev_main, m->stream)) ||
      !EZ_CUDA_OK(cudaStreamWaitEvent(m->side, m->ev_main, 0)))
    return;
  MtRange r[3];
  if (ran == EZMOCK_RNG_MT19937) {
    plan_common(r, starts, caps, n);
    const size_t need = mt_states_needed(r, n, 0) * MT_N * sizeof(uint32_t);
    if (need > m->rng_side_cap) {
      if (m->rng_side) cudaFree(m->rng_side);
      m->rng_side = nullptr;
      m->rng_side_cap = 0;
      if (!EZ_CUDA_OK(cudaMalloc(&m->rng_side, need))) { cudaGetLastError(); return; }
      m->rng_side_cap = need;
    }
    if (mt_jump_launch(m->device, m->side, m->rng_side, seed, r, n, 0) ||
        mt_gen_launch(m->side, m->rng_side, r[0], std::min<uint64_t>(nbias, r[0].cap),
            m->draws_bias))
      return;
  }
  else {
    for (int i = 0; i < n; i++) {
      r[i].start = starts[i];
      r[i].cap = caps[i];
      r[i].l = 0;
      r[i].P = 0;
      r[i].first = 0;
    }
    n = 1;                                  // MRG32k3a needs no preparation
    if (mrg_fill_st(m->device, m->side, seed, starts[0], nbias, m->draws_bias)) return;
  }
  if (!EZ_CUDA_OK(cudaEventRecord(m->ev_side, m->side))) return;
  for (int i = 0; i < n; i++) {
    m->pre[i].start = r[i].start;
    m->pre[i].cap = r[i].cap;
    m->pre[i].l = r[i].l;
    m->pre[i].P = r[i].P;
    m->pre[i].first = r[i].first;
    m->pre[i].side = true;
  }
  m->pre_n = n;
  m->pre_ran = ran;
  m->pre_seed = seed;
  m->pre_bias_n = std::min<uint64_t>(nbias, r[0].cap);
  m->pre_valid = true;
}

// ============================================================================
//            MT19937 fill with static device scratch (no allocation)
// ============================================================================
//
// Same kernels and stream as ez_rng_fill (MT19937), but the chunk states, the
// jump descriptors and the jump polynomials live in file-scope device arrays
// instead of memory obtained from cudaMalloc.  It serves callers that must
// not allocate device memory on this path: a host framework that owns the
// whole device memory through its own pool (a caching allocator that a
// cudaMalloc would fight for memory), and pipelines where a cudaMalloc/
// cudaFree pair would add an implicit device synchronisation between
// otherwise asynchronous launches.
//
// Limits: one fill has at most NA_MAXCHUNK = 128 chunks of at most 2^40 draws,
// so count <= 2^47; each chunk needs one 624-word state, plus the seed state.
// Scratch: 129 x 624 words of states, 128 jump descriptors, 72 polynomial
// indices (324,320 bytes).  Nothing in it has to start at zero: every word a
// kernel reads was written earlier in the same call.  The jump table
// x^(2^k) mod phi (64 x 312 words, 159,744 bytes) is copied into its own
// static array by the first call on each device.
//
// The scratch is one per device: calls that overlap on the same device (two
// streams, or two host threads) race on it and must be serialised by the
// caller.
namespace {

constexpr int NA_MAXCHUNK = 128;
constexpr int NA_STATES = 1 + NA_MAXCHUNK;
constexpr int NA_MAXDESC = NA_MAXCHUNK;          // 1 + (1 + 2 + ... + 64)
constexpr int NA_MAXPOLY = 64 + 8;               // bits of start + doublings
constexpr size_t NA_DESC_OFF = (size_t) NA_STATES * MT_N;        // words
constexpr size_t NA_PLIST_OFF = NA_DESC_OFF + 4 * NA_MAXDESC;
constexpr size_t NA_WORDS = NA_PLIST_OFF + NA_MAXPOLY;
static_assert(NA_DESC_OFF % 4 == 0, "descriptors must be 16-byte aligned");

__device__ __align__(256) uint32_t na_scratch[NA_WORDS];
__device__ __align__(256) uint64_t na_xpow[64 * MT_PW];

struct NaSeed {
  uint32_t w[MT_N];                              // seed window (2,496 bytes)
  uint64_t start;
  int l, p;
};

// Writes the seed window into state 0 and builds the descriptors of the
// jump to `start` (level 0, polynomials = set bits of start) and of the
// doubling levels (level m + 1: 2^m jumps by 2^(l + m) draws), in the
// layout mt_prepare_ranges uses for a single range.
__global__ void na_plan_kernel(uint32_t *scratch, NaSeed s) {
  uint32_t *states = scratch;
  int4 *desc = (int4 *) (scratch + NA_DESC_OFF);
  int *plist = (int *) (scratch + NA_PLIST_OFF);
  for (int k = threadIdx.x; k < MT_N; k += blockDim.x) states[k] = s.w[k];
  if (threadIdx.x == 0) {
    int np = 0;
    for (int k = 0; k < 64; k++)
      if ((s.start >> k) & 1ULL) plist[np++] = k;
    desc[0] = make_int4(0, 1, 0, np);
    for (int lev = 0; lev < s.p; lev++) {
      plist[np] = s.l + lev;
      for (int t = 0; t < (1 << lev); t++)
        desc[(1 << lev) + t] = make_int4(1 + t, 1 + t + (1 << lev), np, 1);
      np++;
    }
  }
}

struct NaDevice {
  bool ready = false;
  uint32_t *scratch = nullptr;
  uint64_t *xpow = nullptr;
};
std::mutex g_na_mu;
NaDevice g_na[64];

// One-time set-up for the current device: host jump tables (shared with the
// allocating path), device addresses of the static arrays, the table copy,
// and the Horner kernel's shared-memory limit.  Synchronous.
int na_setup(int dev, NaDevice **out) {
  std::lock_guard<std::mutex> lk(g_na_mu);
  if (dev < 0 || dev >= 64) return EZMOCK_ERR_UNKNOWN;
  NaDevice &d = g_na[dev];
  if (!d.ready) {
    {
      std::lock_guard<std::mutex> lt(g_mt_mu);
      if (!g_mt_built) { build_mt_tables(g_mt); g_mt_built = true; }
    }
    if (!g_mt.ok || g_mt.xpow.size() != (size_t) 64 * MT_PW) return EZMOCK_ERR_RNG_SET;
    void *ps = nullptr, *px = nullptr;
    if (!EZ_CUDA_OK(cudaGetSymbolAddress(&ps, na_scratch)) ||
        !EZ_CUDA_OK(cudaGetSymbolAddress(&px, na_xpow)) || !ps || !px) {
      cudaGetLastError();
      return EZMOCK_ERR_UNKNOWN;
    }
    if (!EZ_CUDA_OK(cudaMemcpy(px, g_mt.xpow.data(), g_mt.xpow.size() * sizeof(uint64_t),
            cudaMemcpyHostToDevice)) ||
        !EZ_CUDA_OK(cudaFuncSetAttribute(mt_horner_kernel,
            cudaFuncAttributeMaxDynamicSharedMemorySize,
            (int) ((HG * HTAB * MT_N + 3 * MT_N + HW) * sizeof(uint32_t)))))
      return EZMOCK_ERR_UNKNOWN;
    d.scratch = (uint32_t *) ps;
    d.xpow = (uint64_t *) px;
    d.ready = true;
  }
  *out = &d;
  return 0;
}

}  // namespace

extern "C" int EZmockB200_mt19937_fill_noalloc(const uint64_t seed,
    const uint64_t start, const uint64_t count, uint32_t *d_out, void *stream) {
  if (!count) return 0;
  if (!d_out) return EZMOCK_ERR_ARG_NULL;
  if (count > EZMOCKB200_NOALLOC_MAX_DRAWS || start > UINT64_MAX - count)
    return EZMOCKB200_ERR_SCRATCH_SIZE;
  const MtRange r = mt_plan(start, count);
  if (r.p > 7 || ((uint64_t) 1 << (r.l + r.p)) < count) return EZMOCKB200_ERR_SCRATCH_SIZE;
  int dev = -1;
  if (!EZ_CUDA_OK(cudaGetDevice(&dev))) { cudaGetLastError(); return EZMOCK_ERR_UNKNOWN; }
  NaDevice *d = nullptr;
  int e = na_setup(dev, &d);
  if (e) return e;
  cudaStream_t st = (cudaStream_t) stream;
  NaSeed s;
  mt_seed_window(seed, s.w);
  s.start = start;
  s.l = r.l;
  s.p = r.p;
  na_plan_kernel<<<1, 256, 0, st>>>(d->scratch, s); ez_count_launch();
  const int4 *desc = (const int4 *) (d->scratch + NA_DESC_OFF);
  const int *plist = (const int *) (d->scratch + NA_PLIST_OFF);
  const size_t smem = (HG * HTAB * MT_N + 3 * MT_N + HW) * sizeof(uint32_t);
  mt_horner_kernel<<<1, H_THREADS, smem, st>>>(d->scratch, desc, d->xpow, plist);
  ez_count_launch();
  for (int lev = 0; lev < r.p; lev++) {
    mt_horner_kernel<<<1 << lev, H_THREADS, smem, st>>>(d->scratch, desc + (1 << lev),
        d->xpow, plist); ez_count_launch();
  }
  const uint64_t L = 1ULL << r.l;
  mt_gen_kernel<<<(unsigned) ((count + L - 1) / L), G_THREADS, 0, st>>>(
      d->scratch + MT_N, L, count, d_out); ez_count_launch();
  return EZ_CUDA_OK(cudaGetLastError()) ? 0 : EZMOCK_ERR_UNKNOWN;
}
