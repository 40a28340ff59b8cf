// ez_fft.cu -- the three Zel'dovich displacement fields by 3D complex-to-real
// FFTs (libEZmock/EZmock/perturb.c:361-398, FFTW plans at dens_field.c:141).
//
// psi_d = c2r(S * k_d) for d = x, y, z, with S the initial Fourier field and
// k_x = freq(i), k_y = freq(j), k_z = k.  The transform follows FFTW's
// multi-dimensional real-data convention: complex (backward, unnormalised)
// transforms over the i and j axes, then a 1D complex-to-real transform
// along k that ignores the imaginary parts of the k = 0 and k = Ng/2 terms.
// The reference's kz = 0 / Nyquist planes are not Hermitian, so the order
// matters and is kept.
//
// Three HBM passes, each a batch of 1D transforms staged through shared
// memory.  Grids with Ng = 32 * 2^p (64 <= Ng <= 1024) use warp-shuffle
// transforms (one line per warp, in registers); every other 5-smooth even
// grid uses a block-wide Stockham autosort (radices 8/4/2/3/5).  Twiddles
// are rounded from long double on the host.
//   pass I : tiles [all i] x [K columns of k] for one j.  Because k_y and k_z
//            are constant along i, only two transforms are needed:
//            A_x = FFT_i(S k_x), A_0 = FFT_i(S).
//   pass J : tiles [all j] x [K columns] for one x.
//            B_x = FFT_j(A_x), B_y = FFT_j(A_0 k_y), B_0 = FFT_j(A_0).
//   pass K : per (x, y) row, c2r of B_x, B_y and k B_0 through a half-length
//            complex FFT (even/odd packing), written as psi rows.
// Traffic: S read once; 2 + 3 spectra written, 5 read; 3 real fields written.
#include "ez_internal.cuh"
#include "ez_tma.cuh"

#include <cuda_pipeline.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include <vector>

typedef decltype(cplx::x) rt;

namespace {

constexpr int FFT_NT = 512;       // threads per block
constexpr int MAXF = 12;

struct FftPlanDev {
  int n, nfac;
  int fac[MAXF];
  const cplx *tw;                  // tw[e] = exp(+2 pi i e / n)
};

__device__ __forceinline__ cplx cmul(cplx a, cplx b) {
  cplx c;
  c.x = a.x * b.x - a.y * b.y;
  c.y = a.x * b.y + a.y * b.x;
  return c;
}
__device__ __forceinline__ cplx cadd(cplx a, cplx b) { cplx c; c.x = a.x + b.x; c.y = a.y + b.y; return c; }
__device__ __forceinline__ cplx csub(cplx a, cplx b) { cplx c; c.x = a.x - b.x; c.y = a.y - b.y; return c; }
// multiply by s*i
__device__ __forceinline__ cplx cmuli(cplx a, int s) { cplx c; c.x = -s * a.y; c.y = s * a.x; return c; }

template <int S>
__device__ __forceinline__ void dft2(cplx *u) {
  const cplx a = u[0], b = u[1];
  u[0] = cadd(a, b); u[1] = csub(a, b);
}

template <int S>
__device__ __forceinline__ void dft4(cplx *u) {
  const cplx t0 = cadd(u[0], u[2]), t1 = csub(u[0], u[2]);
  const cplx t2 = cadd(u[1], u[3]), t3 = cmuli(csub(u[1], u[3]), S);
  u[0] = cadd(t0, t2); u[2] = csub(t0, t2);
  u[1] = cadd(t1, t3); u[3] = csub(t1, t3);
}

template <int S>
__device__ __forceinline__ void dft8(cplx *u) {
  cplx a[4] = {u[0], u[2], u[4], u[6]}, b[4] = {u[1], u[3], u[5], u[7]};
  dft4<S>(a);
  dft4<S>(b);
  const rt h = (rt) 0.70710678118654752440084436210484904;
  // w8^k = exp(S i pi k / 4)
  cplx w1; w1.x = h; w1.y = S * h;
  cplx w3; w3.x = -h; w3.y = S * h;
  b[1] = cmul(b[1], w1);
  b[2] = cmuli(b[2], S);
  b[3] = cmul(b[3], w3);
#pragma unroll
  for (int k = 0; k < 4; k++) { u[k] = cadd(a[k], b[k]); u[k + 4] = csub(a[k], b[k]); }
}

template <int S>
__device__ __forceinline__ void dft3(cplx *u) {
  const rt c = (rt) -0.5, sn = (rt) (S * 0.86602540378443864676372317075293618);
  const cplx s12 = cadd(u[1], u[2]), d12 = csub(u[1], u[2]);
  cplx t; t.x = u[0].x + c * s12.x; t.y = u[0].y + c * s12.y;
  cplx v; v.x = -sn * d12.y; v.y = sn * d12.x;        // i * sn * d12
  u[0] = cadd(u[0], s12);
  u[1] = cadd(t, v);
  u[2] = csub(t, v);
}

template <int S>
__device__ __forceinline__ void dft5(cplx *u) {
  const rt c1 = (rt) 0.30901699437494742410229341718281906;
  const rt c2 = (rt) -0.80901699437494742410229341718281906;
  const rt s1 = (rt) (S * 0.95105651629515357211643933337938214);
  const rt s2 = (rt) (S * 0.58778525229247312916870595463907277);
  const cplx a14 = cadd(u[1], u[4]), d14 = csub(u[1], u[4]);
  const cplx a23 = cadd(u[2], u[3]), d23 = csub(u[2], u[3]);
  cplx t1, t2, v1, v2;
  t1.x = u[0].x + c1 * a14.x + c2 * a23.x; t1.y = u[0].y + c1 * a14.y + c2 * a23.y;
  t2.x = u[0].x + c2 * a14.x + c1 * a23.x; t2.y = u[0].y + c2 * a14.y + c1 * a23.y;
  // v1 = i (s1 d14 + s2 d23), v2 = i (s2 d14 - s1 d23)
  const rt w1r = s1 * d14.x + s2 * d23.x, w1i = s1 * d14.y + s2 * d23.y;
  const rt w2r = s2 * d14.x - s1 * d23.x, w2i = s2 * d14.y - s1 * d23.y;
  v1.x = -w1i; v1.y = w1r;
  v2.x = -w2i; v2.y = w2r;
  u[0] = cadd(u[0], cadd(a14, a23));
  u[1] = cadd(t1, v1);
  u[4] = csub(t1, v1);
  u[2] = cadd(t2, v2);
  u[3] = csub(t2, v2);
}

// One Stockham pass of radix R over `nlines` lines of length n:
// element e of line L is at buf[e*es + L].  Out of place (src -> dst).
template <int R, int S>
__device__ __forceinline__ void stockham_pass(const cplx *src, cplx *dst,
    int n, int nlines, int es, int p, const cplx *tw) {
  const int T = n / R;
  const int nb = T * nlines;
  const int stw = n / (p * R);
  for (int b = threadIdx.x; b < nb; b += blockDim.x) {
    const int L = b % nlines, i = b / nlines;
    const int k = i % p;
    cplx u[R];
#pragma unroll
    for (int q = 0; q < R; q++) {
      cplx v = src[(i + q * T) * es + L];
      if (q && k) {
        const int e = (q * k * stw) % n;
        cplx w = tw[e];
        if (S < 0) w.y = -w.y;
        v = cmul(v, w);
      }
      u[q] = v;
    }
    if (R == 2) dft2<S>(u);
    else if (R == 3) dft3<S>(u);
    else if (R == 4) dft4<S>(u);
    else if (R == 5) dft5<S>(u);
    else dft8<S>(u);
    const int j = (i - k) * R + k;
#pragma unroll
    for (int s = 0; s < R; s++) dst[(j + s * p) * es + L] = u[s];
  }
}

// Batched FFT of `nlines` lines held in a (element-major, line-minor) layout;
// ping-pongs between a and b, returns the buffer holding the result.
template <int S>
__device__ cplx *smem_fft(cplx *a, cplx *b, int nlines, const FftPlanDev &pl,
    const cplx *tw) {
  int p = 1;
  cplx *src = a, *dst = b;
  for (int f = 0; f < pl.nfac; f++) {
    const int r = pl.fac[f];
    switch (r) {
      case 8: stockham_pass<8, S>(src, dst, pl.n, nlines, nlines, p, tw); break;
      case 4: stockham_pass<4, S>(src, dst, pl.n, nlines, nlines, p, tw); break;
      case 2: stockham_pass<2, S>(src, dst, pl.n, nlines, nlines, p, tw); break;
      case 3: stockham_pass<3, S>(src, dst, pl.n, nlines, nlines, p, tw); break;
      default: stockham_pass<5, S>(src, dst, pl.n, nlines, nlines, p, tw); break;
    }
    __syncthreads();
    p *= r;
    cplx *t = src; src = dst; dst = t;
  }
  return src;
}

__device__ __forceinline__ rt freq_of(int i, int Ng) {
  return (rt) ((i <= (Ng >> 1)) ? i : i - Ng);
}

// ---------------------------------------------------------------- pass I --
__global__ void __launch_bounds__(FFT_NT)
fft_pass_i(const cplx *__restrict__ S, cplx *__restrict__ Ax,
    cplx *__restrict__ A0, int Ng, int Nkp, int K, FftPlanDev pl) {
  extern __shared__ unsigned char smraw[];
  cplx *tw = (cplx *) smraw;
  const int nl = 2 * K;
  cplx *ba = tw + Ng;
  cplx *bb = ba + (size_t) Ng * nl;
  const int j = blockIdx.x, k0 = blockIdx.y * K;
  for (int e = threadIdx.x; e < Ng; e += blockDim.x) tw[e] = pl.tw[e];
  const size_t pstride = (size_t) Ng * Nkp;           // stride between i planes
  for (int e = threadIdx.x; e < Ng * K; e += blockDim.x) {
    const int i = e / K, c = e - i * K;
    const cplx v = S[i * pstride + (size_t) j * Nkp + k0 + c];
    const rt f = freq_of(i, Ng);
    cplx w; w.x = v.x * f; w.y = v.y * f;
    ba[i * nl + c] = w;
    ba[i * nl + K + c] = v;
  }
  __syncthreads();
  cplx *res = smem_fft<1>(ba, bb, nl, pl, tw);
  for (int e = threadIdx.x; e < Ng * K; e += blockDim.x) {
    const int i = e / K, c = e - i * K;
    const size_t g = i * pstride + (size_t) j * Nkp + k0 + c;
    Ax[g] = res[i * nl + c];
    A0[g] = res[i * nl + K + c];
  }
}

// ---------------------------------------------------------------- pass J --
// In: Ax (spec1), A0 (spec2).  Out: Bx -> spec1, By -> spec0, B0 -> spec2.
__global__ void __launch_bounds__(FFT_NT)
fft_pass_j(cplx *__restrict__ s0, cplx *__restrict__ s1, cplx *__restrict__ s2,
    int Ng, int Nkp, int K, FftPlanDev pl) {
  extern __shared__ unsigned char smraw[];
  cplx *tw = (cplx *) smraw;
  const int nl = 3 * K;
  cplx *ba = tw + Ng;
  cplx *bb = ba + (size_t) Ng * nl;
  const int x = blockIdx.x, k0 = blockIdx.y * K;
  for (int e = threadIdx.x; e < Ng; e += blockDim.x) tw[e] = pl.tw[e];
  const size_t base = (size_t) x * Ng * Nkp + k0;
  for (int e = threadIdx.x; e < Ng * K; e += blockDim.x) {
    const int j = e / K, c = e - j * K;
    const size_t g = base + (size_t) j * Nkp + c;
    const cplx ax = s1[g], a0 = s2[g];
    const rt f = freq_of(j, Ng);
    cplx w; w.x = a0.x * f; w.y = a0.y * f;
    ba[j * nl + c] = ax;
    ba[j * nl + K + c] = w;
    ba[j * nl + 2 * K + c] = a0;
  }
  __syncthreads();
  cplx *res = smem_fft<1>(ba, bb, nl, pl, tw);
  for (int e = threadIdx.x; e < Ng * K; e += blockDim.x) {
    const int j = e / K, c = e - j * K;
    const size_t g = base + (size_t) j * Nkp + c;
    s1[g] = res[j * nl + c];
    s0[g] = res[j * nl + K + c];
    s2[g] = res[j * nl + 2 * K + c];
  }
}

// ---------------------------------------------------------------- pass K --
// R rows per block; lines: (row, component) with component 0: Bx -> psi0,
// 1: By -> psi1, 2: k*B0 -> psi2.
__global__ void __launch_bounds__(FFT_NT)
fft_pass_k(const cplx *__restrict__ s0, const cplx *__restrict__ s1,
    const cplx *__restrict__ s2, real *__restrict__ p0, real *__restrict__ p1,
    real *__restrict__ p2, int Ng, int Nkp, int R, size_t nrows,
    FftPlanDev pl, const cplx *__restrict__ twg, EzCicStats *stats) {
  extern __shared__ unsigned char smraw[];
  const int Nh = Ng >> 1;
  const int nl = 3 * R;
  cplx *tw = (cplx *) smraw;            // Nh
  cplx *tg = tw + Nh;                   // Nh: exp(+2 pi i k / Ng)
  cplx *raw = tg + Nh;                  // nl x (Nh+1), line-major
  cplx *ba = raw + (size_t) nl * (Nh + 1);
  cplx *bb = ba + (size_t) Nh * nl;
  for (int e = threadIdx.x; e < Nh; e += blockDim.x) { tw[e] = pl.tw[e]; tg[e] = twg[e]; }
  const size_t row0 = (size_t) blockIdx.x * R;
  // load rows (only k <= Nh is needed)
  for (int e = threadIdx.x; e < nl * (Nh + 1); e += blockDim.x) {
    const int L = e / (Nh + 1), k = e - L * (Nh + 1);
    const int r = L / 3, comp = L - 3 * r;
    const size_t row = row0 + r;
    cplx v; v.x = 0; v.y = 0;
    if (row < nrows) {
      const size_t g = row * Nkp + k;
      if (comp == 0) v = s1[g];
      else if (comp == 1) v = s0[g];
      else { v = s2[g]; v.x *= (rt) k; v.y *= (rt) k; }
    }
    raw[e] = v;
  }
  __syncthreads();
  // even/odd packing: Z[k] = E[k] + i O[k]
  for (int e = threadIdx.x; e < nl * Nh; e += blockDim.x) {
    const int L = e % nl, k = e / nl;
    const cplx *X = raw + (size_t) L * (Nh + 1);
    const rt xr = X[k].x, xi = (k == 0) ? (rt) 0 : X[k].y;
    const rt yr = X[Nh - k].x, yi = (k == 0) ? (rt) 0 : -X[Nh - k].y;
    const rt er = xr + yr, ei = xi + yi;
    const rt dr = xr - yr, di = xi - yi;
    const cplx w = tg[k];
    const rt orr = dr * w.x - di * w.y, oi = dr * w.y + di * w.x;
    cplx z; z.x = er - oi; z.y = ei + orr;
    ba[k * nl + L] = z;
  }
  __syncthreads();
  cplx *res = smem_fft<1>(ba, bb, nl, pl, tw);
  float mx = 0.f;
  for (int e = threadIdx.x; e < nl * Nh; e += blockDim.x) {
    const int L = e / Nh, m = e - L * Nh;
    const int r = L / 3, comp = L - 3 * r;
    const size_t row = row0 + r;
    if (row >= nrows) continue;
    real *dst = (comp == 0) ? p0 : (comp == 1) ? p1 : p2;
    const cplx z = res[m * nl + L];
    cplx *d2 = (cplx *) (dst + row * Ng);
    d2[m] = z;
    mx = fmaxf(mx, fmaxf(fabsf((float) z.x), fabsf((float) z.y)));
  }
  // max |psi|, for the fixed-point scale of the density assignment
#pragma unroll
  for (int o = 16; o; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if ((threadIdx.x & 31) == 0) atomicMax(&stats->psimax_bits, __float_as_uint(mx));
}

// ===================================================== warp-shuffle FFTs ==
//
// Lines of length n = 32 E (E a power of two, E <= 32) are transformed by one
// warp entirely in registers: lane l holds x[32 m + l] (m < E), does an
// E-point DFT in registers, multiplies by exp(S 2 pi i l k / n), and the
// 32-point DFTs across the lanes are done by five radix-2 decimation-in-
// frequency stages with __shfl_xor_sync.  Lane l then holds X[k + E r(l)]
// for k < E, r(l) = 5-bit reversal of l.  Tiles are staged in shared memory
// column-major (one line per column, line stride n + 1) with the element
// index XOR-swizzled by bits 4..7, which keeps both the strided line loads
// and the bit-reversed stores (nearly) free of bank conflicts.

__constant__ cplx c_w32[32];                 // exp(+2 pi i k / 32), rounded to rt

template <int S>
__device__ __forceinline__ cplx w32(int k) {
  cplx r = c_w32[k & 31];
  if (S < 0) r.y = -r.y;
  return r;
}

template <int E, int S> struct RegDft;
template <int S> struct RegDft<1, S> { __device__ static void run(cplx *) {} };
template <int S> struct RegDft<2, S> { __device__ static void run(cplx *v) { dft2<S>(v); } };
template <int S> struct RegDft<4, S> { __device__ static void run(cplx *v) { dft4<S>(v); } };
template <int S> struct RegDft<8, S> { __device__ static void run(cplx *v) { dft8<S>(v); } };
template <int E, int S> struct RegDft {
  // radix-2 decimation in time from two half-size DFTs
  __device__ static void run(cplx *v) {
    cplx ev[E / 2], od[E / 2];
#pragma unroll
    for (int k = 0; k < E / 2; k++) { ev[k] = v[2 * k]; od[k] = v[2 * k + 1]; }
    RegDft<E / 2, S>::run(ev);
    RegDft<E / 2, S>::run(od);
#pragma unroll
    for (int k = 0; k < E / 2; k++) {
      const cplx t = cmul(od[k], w32<S>(k * (32 / E)));
      v[k] = cadd(ev[k], t);
      v[k + E / 2] = csub(ev[k], t);
    }
  }
};

__device__ __forceinline__ int brev5(int l) { return __brev((unsigned) l) >> 27; }

__device__ __forceinline__ cplx shfl_xor_c(cplx v, int m) {
  cplx r;
  r.x = __shfl_xor_sync(0xffffffffu, v.x, m);
  r.y = __shfl_xor_sync(0xffffffffu, v.y, m);
  return r;
}

// tw[e] = exp(+2 pi i e / n) in shared memory
template <int E, int S>
__device__ __forceinline__ void warp_fft(cplx *v, const cplx *tw, int lane) {
  RegDft<E, S>::run(v);
#pragma unroll
  for (int k = 1; k < E; k++) {
    cplx w = tw[lane * k];
    if (S < 0) w.y = -w.y;
    v[k] = cmul(v[k], w);
  }
  // Stage h: the lower lane keeps v + b, the upper lane (b - v) w with
  // w = W_2h^(lane mod h).  Written as (s v + b) w_l with s = -1 and w_l = w
  // on the upper lane, s = 1 and w_l = 1 on the lower one (exact).  The last
  // two stages have w in {1, S i} and {1}: no complex multiply.
#pragma unroll
  for (int h = 16; h >= 4; h >>= 1) {
    const bool hi = (lane & h) != 0;
    const rt sg = hi ? (rt) -1 : (rt) 1;
    cplx w = w32<S>((lane & (h - 1)) * (16 / h));
    if (!hi) { w.x = 1; w.y = 0; }
#pragma unroll
    for (int k = 0; k < E; k++) {
      const cplx b = shfl_xor_c(v[k], h);
      cplx t;
      t.x = fma(sg, v[k].x, b.x);
      t.y = fma(sg, v[k].y, b.y);
      v[k] = cmul(t, w);
    }
  }
  {
    const rt sg = (lane & 2) ? (rt) -1 : (rt) 1;
    const bool rot = (lane & 3) == 3;          // upper lane, w = W_4^1 = S i
#pragma unroll
    for (int k = 0; k < E; k++) {
      const cplx b = shfl_xor_c(v[k], 2);
      cplx t;
      t.x = fma(sg, v[k].x, b.x);
      t.y = fma(sg, v[k].y, b.y);
      if (rot) { const rt x = t.x; t.x = -S * t.y; t.y = S * x; }
      v[k] = t;
    }
  }
  {
    const rt sg = (lane & 1) ? (rt) -1 : (rt) 1;
#pragma unroll
    for (int k = 0; k < E; k++) {
      const cplx b = shfl_xor_c(v[k], 1);
      v[k].x = fma(sg, v[k].x, b.x);
      v[k].y = fma(sg, v[k].y, b.y);
    }
  }
}

// Line transform with one pass through shared memory instead of five
// shuffle stages.  With n = 32 E, x[l + 32 m] (lane l, m < E):
//   Y[l][k]   = sum_m x[l + 32 m] W_E^(m k)          (E-point DFT, registers)
//   Z[l][k]   = Y[l][k] W_n^(l k)
//   X[k + E p] = sum_l Z[l][k] W_32^(l p),   p = q + E r,  l = G j + s (G = 32/E):
//             = sum_s W_G^(s r) [W_32^(s q) sum_j Z[G j + s][k] W_E^(j q)].
// Z goes through the caller's line buffer (n elements, used as scratch:
// lane (k, s) then reads its E values Z[G j + s][k]); the inner sum over j
// is a second register DFT, and the G-point DFT over s runs across the lanes
// that share k, in log2 G shuffle stages (none for E = 32, one for E = 16).
// Lane t then holds X[k(t) + E q + E^2 r(t)] for q < E, r(t) the bit-
// reversed s(t).  The lane mapping and the scratch positions are chosen per
// E so that the scratch writes and reads and the callers' stores to their
// swizzled tiles are free of bank conflicts (E = 4: two-way on the stores).
template <int E> struct W2 {
  static constexpr int G = 32 / E;
  static constexpr bool SHIGH = E >= 16;          // s in the high lane bits
  static __device__ __forceinline__ int k_of(int t) { return SHIGH ? (t & (E - 1)) : (t / G); }
  static __device__ __forceinline__ int s_of(int t) { return SHIGH ? (t / E) : (t & (G - 1)); }
  static __device__ __forceinline__ int pos(int l, int k) {
    return 32 * k + (l ^ (SHIGH ? k : ((G * k) & 31)));
  }
  static __host__ __device__ constexpr int lane_xor(int h) { return SHIGH ? h * E : h; }
  // output index held in register q by lane t
  static __device__ __forceinline__ int out(int t, int q) {
    int r = 0;
    const int s = s_of(t);
#pragma unroll
    for (int b = 1; b < G; b <<= 1) r = (r << 1) | ((s & b) ? 1 : 0);
    return k_of(t) + E * q + E * E * r;
  }
};

template <int E, int S>
__device__ __forceinline__ void warp_fft2(cplx *v, const cplx *tw, int lane, cplx *line) {
  typedef W2<E> M;
  constexpr int G = M::G;
  RegDft<E, S>::run(v);
#pragma unroll
  for (int k = 1; k < E; k++) {
    cplx w = tw[lane * k];
    if (S < 0) w.y = -w.y;
    v[k] = cmul(v[k], w);
  }
  __syncwarp();
#pragma unroll
  for (int k = 0; k < E; k++) line[M::pos(lane, k)] = v[k];
  __syncwarp();
  const int kt = M::k_of(lane), st = M::s_of(lane);
#pragma unroll
  for (int j = 0; j < E; j++) v[j] = line[M::pos(G * j + st, kt)];
  __syncwarp();
  RegDft<E, S>::run(v);
  if (G > 1) {
#pragma unroll
    for (int q = 1; q < E; q++) v[q] = cmul(v[q], w32<S>(st * q));
  }
  // G-point decimation-in-frequency over s across the lanes sharing k: the
  // lower lane keeps v + b, the upper one (b - v) W_2h^(s mod h)
#pragma unroll
  for (int h = G / 2; h >= 1; h >>= 1) {
    const bool hi = (st & h) != 0;
    const rt sg = hi ? (rt) -1 : (rt) 1;
    cplx w = w32<S>((st & (h - 1)) * (16 / h));
    if (!hi) { w.x = 1; w.y = 0; }
#pragma unroll
    for (int q = 0; q < E; q++) {
      const cplx b = shfl_xor_c(v[q], M::lane_xor(h));
      cplx t;
      t.x = fma(sg, v[q].x, b.x);
      t.y = fma(sg, v[q].y, b.y);
      v[q] = cmul(t, w);
    }
  }
}

// The transform a line of a tile goes through, with the output index of
// register q of lane t: the transposed form above (T = true, single
// precision only) or the five shuffle stages (lane t then holds
// X[q + E brev5(t)]).  Measured per pass at 512^3 and 1024^3: the
// transposed form pays where it removes four or five shuffle stages (E = 16
// in passes I and K, E = 32 in pass J), and costs where it adds register
// pressure (pass J at E = 16) or removes only three (E = 8); double
// precision keeps the shuffles (twice the registers per value).
template <int E> __host__ __device__ constexpr bool use_t(int pass) {
  return sizeof(rt) == 4 && (pass == 1 ? E >= 32 : E >= 16);
}
template <int E, int S, bool T>
__device__ __forceinline__ void line_fft(cplx *v, const cplx *tw, int lane, cplx *line) {
  if (T) warp_fft2<E, S>(v, tw, lane, line);
  else { warp_fft<E, S>(v, tw, lane); __syncwarp(); }
}
template <int E, bool T>
__device__ __forceinline__ int line_out(int lane, int q) {
  return T ? W2<E>::out(lane, q) : q + E * brev5(lane);
}

__device__ __forceinline__ int swz(int m) { return m ^ ((m >> 4) & 15); }

constexpr int WNW = 8;                       // warps per block
constexpr int WK = 8;                        // columns per tile (passes I, J)

// pass I: A_x = FFT_i(S k_x), A_0 = FFT_i(S); one column per warp.
// Blocks per SM the launch bounds of pass J plan for: two up to Ng = 512;
// its 1024-point tile (197 KB of shared memory) allows one, so the register
// budget is not halved there (no spills: 10.6 vs 12.1 ms at 1024^3).  Pass I
// keeps two (measured faster at 1024^3 despite small spills).
template <int E> constexpr int wpass_min_blocks() { return E >= 32 ? 1 : 2; }

// pass I: columns per tile = warps per block (512^3: 8 columns 0.71 ms,
// 4 columns with four blocks per SM 0.92 ms, 2 columns 1.31 ms)
constexpr int WKI = 8;
template <int E>
__global__ void __launch_bounds__(32 * WKI, 16 / WKI)
wpass_i(const cplx *__restrict__ S, cplx *__restrict__ Ax, cplx *__restrict__ A0,
    int Ng, int Nkp, const cplx *__restrict__ twn) {
  constexpr int n = 32 * E, LS = n + 1;
  constexpr int WK = WKI, WNW = WKI;
  extern __shared__ unsigned char smraw[];
  cplx *tw = (cplx *) smraw;
  cplx *b0 = tw + n;                         // WK lines: S, then A_0
  cplx *b1 = b0 + WK * LS;                   // WK lines: A_x
  // column tiles of one j run side by side: together they read whole rows
  const int j = blockIdx.y, k0 = blockIdx.x * WK;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int e = threadIdx.x; e < n; e += blockDim.x) tw[e] = twn[e];
  const size_t pst = (size_t) Ng * Nkp;
  // the whole tile is copied asynchronously (no register staging), so all of
  // a thread's loads are in flight at once
#pragma unroll 8
  for (int e = threadIdx.x; e < n * WK; e += 32 * WNW) {
    const int i = e / WK, c = e - i * WK;
    __pipeline_memcpy_async(b0 + c * LS + swz(i), S + i * pst + (size_t) j * Nkp + k0 + c,
        sizeof(cplx));
  }
  __pipeline_commit();
  __pipeline_wait_prior(0);
  __syncthreads();
  for (int c = w; c < WK; c += WNW) {
    cplx v[E];
#pragma unroll
    for (int m = 0; m < E; m++) {
      const int i = 32 * m + lane;
      v[m] = b0[c * LS + swz(i)];
      const rt f = freq_of(i, Ng);
      v[m].x *= f;
      v[m].y *= f;
    }
    line_fft<E, 1, use_t<E>(0)>(v, tw, lane, b1 + c * LS);
#pragma unroll
    for (int q = 0; q < E; q++) b1[c * LS + swz(line_out<E, use_t<E>(0)>(lane, q))] = v[q];
#pragma unroll
    for (int m = 0; m < E; m++) v[m] = b0[c * LS + swz(32 * m + lane)];
    line_fft<E, 1, use_t<E>(0)>(v, tw, lane, b0 + c * LS);
#pragma unroll
    for (int q = 0; q < E; q++) b0[c * LS + swz(line_out<E, use_t<E>(0)>(lane, q))] = v[q];
  }
  __syncthreads();
#pragma unroll 4
  for (int e = threadIdx.x; e < n * WK; e += 32 * WNW) {
    const int i = e / WK, c = e - i * WK;
    const size_t g = i * pst + (size_t) j * Nkp + k0 + c;
    Ax[g] = b1[c * LS + swz(i)];
    A0[g] = b0[c * LS + swz(i)];
  }
}

// pass J: B_x = FFT_j(A_x) -> s1, B_y = FFT_j(A_0 k_y) -> s0,
// B_0 = FFT_j(A_0) -> s2.
template <int E>
__global__ void __launch_bounds__(32 * WNW, wpass_min_blocks<E>())
wpass_j(cplx *__restrict__ s0, cplx *__restrict__ s1, cplx *__restrict__ s2,
    int Ng, int Nkp, const cplx *__restrict__ twn) {
  constexpr int n = 32 * E, LS = n + 1;
  extern __shared__ unsigned char smraw[];
  cplx *tw = (cplx *) smraw;
  cplx *bx = tw + n;                         // A_x -> B_x
  cplx *b0 = bx + WK * LS;                   // A_0 -> B_0
  cplx *by = b0 + WK * LS;                   // B_y
  const int x = blockIdx.y, k0 = blockIdx.x * WK;     // tiles of one plane side by side
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int e = threadIdx.x; e < n; e += blockDim.x) tw[e] = twn[e];
  const size_t base = (size_t) x * Ng * Nkp + k0;
  // asynchronous tile copies: A_x first (group 0), then A_0 (group 1), so B_x
  // is transformed while A_0 is still arriving
#pragma unroll 8
  for (int e = threadIdx.x; e < n * WK; e += 32 * WNW) {
    const int j = e / WK, c = e - j * WK;
    __pipeline_memcpy_async(bx + c * LS + swz(j), s1 + base + (size_t) j * Nkp + c, sizeof(cplx));
  }
  __pipeline_commit();
#pragma unroll 8
  for (int e = threadIdx.x; e < n * WK; e += 32 * WNW) {
    const int j = e / WK, c = e - j * WK;
    __pipeline_memcpy_async(b0 + c * LS + swz(j), s2 + base + (size_t) j * Nkp + c, sizeof(cplx));
  }
  __pipeline_commit();
  __pipeline_wait_prior(1);
  __syncthreads();
  for (int c = w; c < WK; c += WNW) {
    cplx v[E];
#pragma unroll
    for (int m = 0; m < E; m++) v[m] = bx[c * LS + swz(32 * m + lane)];
    line_fft<E, 1, use_t<E>(1)>(v, tw, lane, bx + c * LS);
#pragma unroll
    for (int q = 0; q < E; q++) bx[c * LS + swz(line_out<E, use_t<E>(1)>(lane, q))] = v[q];
  }
  __pipeline_wait_prior(0);
  __syncthreads();
  for (int c = w; c < WK; c += WNW) {
    cplx v[E];
#pragma unroll
    for (int m = 0; m < E; m++) {
      const int jj = 32 * m + lane;
      v[m] = b0[c * LS + swz(jj)];
      const rt f = freq_of(jj, Ng);
      v[m].x *= f;
      v[m].y *= f;
    }
    line_fft<E, 1, use_t<E>(1)>(v, tw, lane, by + c * LS);
#pragma unroll
    for (int q = 0; q < E; q++) by[c * LS + swz(line_out<E, use_t<E>(1)>(lane, q))] = v[q];
#pragma unroll
    for (int m = 0; m < E; m++) v[m] = b0[c * LS + swz(32 * m + lane)];
    line_fft<E, 1, use_t<E>(1)>(v, tw, lane, b0 + c * LS);
#pragma unroll
    for (int q = 0; q < E; q++) b0[c * LS + swz(line_out<E, use_t<E>(1)>(lane, q))] = v[q];
  }
  __syncthreads();
#pragma unroll 4
  for (int e = threadIdx.x; e < n * WK; e += 32 * WNW) {
    const int j = e / WK, c = e - j * WK;
    const size_t g = base + (size_t) j * Nkp + c;
    s1[g] = bx[c * LS + swz(j)];
    s0[g] = by[c * LS + swz(j)];
    s2[g] = b0[c * LS + swz(j)];
  }
}

// ----------------------------------------------------- TMA-staged pass J --
//
// FP32, Ng = 32 E with E = 8 or 16.  The transforms of wpass_j, with tiles of
// WK = 8 columns moved by the Tensor Memory Accelerator: a tile is Ng rows
// (all j of one i) of 64 bytes, copied by 256-row boxes of a tensor map over
// the spectrum (floats, 2 Nkp x Ng x Ng) with the 64-byte swizzle, so that a
// warp reading one column (one line) meets each bank at most twice.  A
// persistent CTA per SM runs a two-stage pipeline: while its eight warps
// transform tile t (one column each, the transposed line form warp_fft2 with
// a per-warp scratch line), the loads of tile t + 1 are in flight; thread 0
// then stores tile t from shared memory and loads tile t + 2 into the
// freed stage.  A_x and A_0 arrive; B_x and B_0 replace them in place and
// B_y goes through a separate tile.  Every wait has an iteration limit; a
// wait that runs out sets stats->tma_err (read by the population) and the
// CTA lets its copies land and returns.  (Pass I through the same pipeline
// measured slower than its cp.async kernel: 1.01 against 0.71 ms at 512^3;
// it does two transforms per loaded tile, and one CTA of eight warps per SM,
// which the 237 registers of the transforms allow, hides less latency than
// the two CTAs of wpass_i.)
constexpr int TP_CW = 8;                           // warps = columns of a tile
constexpr int TP_THREADS = 32 * TP_CW;
constexpr int TP_BOX = 256;                        // rows per box

// element (row, column c) of a swizzled 8-column tile, in complex units
__device__ __forceinline__ int tix(int row, int c) {
  return row * 8 + ((((c >> 1) ^ ((row >> 1) & 3)) << 1) | (c & 1));
}

template <int E>
struct TpLayout {
  static constexpr int n = 32 * E;
  static constexpr size_t tile = (size_t) n * 64;  // bytes of one tile
  // [twiddles n cplx][pad to 1 KB][stage 0: NIN tiles][stage 1][separate tile][scratch][barriers]
  static constexpr size_t tw_bytes = ((size_t) n * 8 + 1023) / 1024 * 1024;
  static size_t bytes(int nin) {
    return tw_bytes + (2 * (size_t) nin + 1) * tile + (size_t) TP_CW * n * 8 + 64 + 1024;
  }
};

template <int E>
__global__ void __launch_bounds__(TP_THREADS, 1)
tpass_j_kernel(const __grid_constant__ CUtensorMap mi0, const __grid_constant__ CUtensorMap mi1,
    const __grid_constant__ CUtensorMap mo0, const __grid_constant__ CUtensorMap mo1,
    const __grid_constant__ CUtensorMap mo2, int Ng, int nkt, int ntiles,
    const cplx *__restrict__ twn, EzCicStats *stats) {
  typedef TpLayout<E> Lay;
  constexpr int n = Lay::n;
  constexpr int NIN = 2;                           // A_x, A_0 per stage
  constexpr int NB = n / TP_BOX > 0 ? n / TP_BOX : 1;   // boxes per tile
  constexpr int BR = n < TP_BOX ? n : TP_BOX;      // rows per box
  extern __shared__ __align__(1024) unsigned char tp_raw[];
  // 1 KB alignment of every tile (the swizzle pattern repeats every 512 B),
  // kept as an offset into the shared array so addresses stay 32-bit
  unsigned char *base = tp_raw + ((1024u - (ez_smem_addr(tp_raw) & 1023u)) & 1023u);
  cplx *tw = (cplx *) base;
  unsigned char *stg = base + Lay::tw_bytes;
  cplx *sep = (cplx *) (stg + 2 * NIN * Lay::tile);
  cplx *scr = (cplx *) ((unsigned char *) sep + Lay::tile);
  uint64_t *bar = (uint64_t *) ((unsigned char *) scr + (size_t) TP_CW * n * 8);
  uint64_t *full = bar, *empty = bar + 2, *sepfree = bar + 4;
  auto in_tile = [&](int s, int a) { return (cplx *) (stg + ((size_t) s * NIN + a) * Lay::tile); };
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int G = gridDim.x;
  const bool producer = threadIdx.x == 0;

  auto coords = [&](int t, int b, int &c0, int &c1, int &c2) {
    const int o = t / nkt, kt = t - o * nkt;
    c0 = 16 * kt;                                  // tile: all j at i = o
    c1 = b * BR;
    c2 = o;
  };
  int nload0 = 0, nload1 = 0;                      // loads issued per stage
  auto issue_load = [&](int it, int s) {
    const int t = blockIdx.x + it * G;
    if (s) nload1++; else nload0++;
    ez_mbar_expect_tx(&full[s], (uint32_t) (NIN * Lay::tile));
#pragma unroll
    for (int a = 0; a < NIN; a++)
#pragma unroll
      for (int b = 0; b < NB; b++) {
        int c0, c1, c2;
        coords(t, b, c0, c1, c2);
        ez_tma_load3((unsigned char *) in_tile(s, a) + (size_t) b * BR * 64, a ? &mi1 : &mi0,
            c0, c1, c2, &full[s]);
      }
  };

  for (int e = threadIdx.x; e < n; e += blockDim.x) tw[e] = twn[e];
  if (producer) {
    ez_mbar_init(&full[0], 1);
    ez_mbar_init(&full[1], 1);
    ez_mbar_init(&empty[0], TP_CW);
    ez_mbar_init(&empty[1], TP_CW);
    ez_mbar_init(sepfree, 1);
    ez_fence_mbar_init();
    ez_prefetch_map(&mi0);
    ez_prefetch_map(&mi1);
    for (int it = 0; it < 2 && blockIdx.x + it * G < ntiles; it++) issue_load(it, it);
  }
  __syncthreads();

  // every warp transforms column c = warp of each tile; thread 0 also issues
  // the copies: after its warp's part of tile t it waits for the other
  // warps, stores tile t, and loads tile t + 2 into the freed stage
  const int c = warp;
  cplx *line = scr + (size_t) warp * n;
  auto col_load = [&](const cplx *tile, bool mulf, cplx *v) {
#pragma unroll
    for (int m = 0; m < E; m++) {
      const int row = 32 * m + lane;
      v[m] = tile[tix(row, c)];
      if (mulf) {
        const rt f = freq_of(row, Ng);
        v[m].x *= f;
        v[m].y *= f;
      }
    }
  };
  auto col_store = [&](cplx *tile, const cplx *v) {
#pragma unroll
    for (int q = 0; q < E; q++) tile[tix(W2<E>::out(lane, q), c)] = v[q];
  };
  bool ok = true;
  for (int it = 0; ok && blockIdx.x + it * G < ntiles; it++) {
    const int s = it & 1, t = blockIdx.x + it * G;
    if (!ez_mbar_wait(&full[s], (it >> 1) & 1)) { atomicExch(&stats->tma_err, 1u); ok = false; }
    cplx v[E];
    if (ok) {
      cplx *Ax = in_tile(s, 0), *A0 = in_tile(s, 1);
      col_load(Ax, false, v);                      // B_x = FFT_j(A_x), in place
      warp_fft2<E, 1>(v, tw, lane, line);
      col_store(Ax, v);
      if (it > 0 && !ez_mbar_wait(sepfree, (it - 1) & 1)) { atomicExch(&stats->tma_err, 1u); ok = false; }
      if (ok) {
        col_load(A0, true, v);                     // B_y = FFT_j(A_0 k_y)
        warp_fft2<E, 1>(v, tw, lane, line);
        col_store(sep, v);
        col_load(A0, false, v);                    // B_0 = FFT_j(A_0), in place
        warp_fft2<E, 1>(v, tw, lane, line);
        col_store(A0, v);
      }
    }
    ez_fence_async_smem();
    ok = __all_sync(0xffffffffu, ok);              // (keeps a warp's lanes together)
    if (ok && lane == 0)
      asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" :: "r"(ez_smem_addr(&empty[s])) : "memory");
    if (producer && ok) {
      if (!ez_mbar_wait(&empty[s], (it >> 1) & 1)) {
        atomicExch(&stats->tma_err, 1u);
        ok = false;
      } else {
        // stores of tile t: B_x, B_0 (in place) -> mo0, mo1, B_y (separate
        // tile) -> mo2
#pragma unroll
        for (int b = 0; b < NB; b++) {
          int c0, c1, c2;
          coords(t, b, c0, c1, c2);
          const size_t off = (size_t) b * BR * 64;
          ez_tma_store3(&mo0, c0, c1, c2, (const unsigned char *) in_tile(s, 0) + off);
          ez_tma_store3(&mo1, c0, c1, c2, (const unsigned char *) in_tile(s, 1) + off);
          ez_tma_store3(&mo2, c0, c1, c2, (const unsigned char *) sep + off);
        }
        ez_tma_commit();
        ez_tma_wait_read<0>();       // the stage and the separate tile are free
        asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" :: "r"(ez_smem_addr(sepfree)) : "memory");
        if (blockIdx.x + (it + 2) * G < ntiles) issue_load(it + 2, s);
      }
    }
    ok = __all_sync(0xffffffffu, ok);
  }
  if (producer) {
    // copies in flight land before the CTA ends (an error path may leave
    // loads unconsumed)
    if (nload0) ez_mbar_wait(&full[0], (nload0 - 1) & 1);
    if (nload1) ez_mbar_wait(&full[1], (nload1 - 1) & 1);
    ez_tma_wait_all();
  }
}

// pass K: per (x, y) row, c2r of B_x (s1), B_y (s0) and k B_0 (s2) through a
// half-length complex FFT (n = Ng/2 = 32 E); one row per warp.
template <int E>
__global__ void __launch_bounds__(32 * WNW, 3)
wpass_k(const cplx *__restrict__ s0, const cplx *__restrict__ s1,
    const cplx *__restrict__ s2, real *__restrict__ p0, real *__restrict__ p1,
    real *__restrict__ p2, int Ng, int Nkp, size_t nrows,
    const cplx *__restrict__ twh, const cplx *__restrict__ twg,
    EzCicStats *stats) {
  constexpr int n = 32 * E, LS = n + 1;      // n = Ng / 2
  extern __shared__ unsigned char smraw[];
  cplx *tw = (cplx *) smraw;                 // n: exp(+2 pi i e / n)
  cplx *tg = tw + n;                         // n: exp(+2 pi i k / Ng)
  cplx *st = tg + n;                         // WNW staging lines
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int e = threadIdx.x; e < n; e += blockDim.x) { tw[e] = twh[e]; tg[e] = twg[e]; }
  __syncthreads();
  cplx *sl = st + w * LS;
  float mx = 0.f;
  for (size_t row = (size_t) blockIdx.x * WNW + w; row < nrows;
       row += (size_t) gridDim.x * WNW) {
#pragma unroll 1
    for (int comp = 0; comp < 3; comp++) {
      const cplx *X = ((comp == 0) ? s1 : (comp == 1) ? s0 : s2) + row * Nkp;
      real *dst = ((comp == 0) ? p0 : (comp == 1) ? p1 : p2) + row * Ng;
      cplx v[E];
#pragma unroll
      for (int m = 0; m < E; m++) {
        const int k = 32 * m + lane;
        cplx a = X[k], b = X[n - k];
        if (comp == 2) {
          a.x *= (rt) k; a.y *= (rt) k;
          b.x *= (rt) (n - k); b.y *= (rt) (n - k);
        }
        const rt xr = a.x, xi = (k == 0) ? (rt) 0 : a.y;
        const rt yr = b.x, yi = (k == 0) ? (rt) 0 : -b.y;
        const rt er = xr + yr, ei = xi + yi;
        const rt dr = xr - yr, di = xi - yi;
        const cplx t = tg[k];
        const rt orr = dr * t.x - di * t.y, oi = dr * t.y + di * t.x;
        v[m].x = er - oi;
        v[m].y = ei + orr;
      }
      line_fft<E, 1, use_t<E>(2)>(v, tw, lane, sl);
#pragma unroll
      for (int q = 0; q < E; q++) sl[swz(line_out<E, use_t<E>(2)>(lane, q))] = v[q];
      __syncwarp();
      cplx *d2 = (cplx *) dst;
#pragma unroll
      for (int m = 0; m < E; m++) {
        const cplx z = sl[swz(32 * m + lane)];
        d2[32 * m + lane] = z;
        mx = fmaxf(mx, fmaxf(fabsf((float) z.x), fabsf((float) z.y)));
      }
      __syncwarp();
    }
  }
#pragma unroll
  for (int o = 16; o; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if (lane == 0) atomicMax(&stats->psimax_bits, __float_as_uint(mx));
}

// ------------------------------------------- forward transforms (r2c) ---
// Row r2c along k (sign -1): even/odd packing into a half-length complex FFT,
// then X[k] = E[k] + exp(-2 pi i k/Ng) O[k] for k = 0..Ng/2.
__global__ void __launch_bounds__(FFT_NT)
fft_r2c_rows(const real *__restrict__ x, cplx *__restrict__ S, int Ng,
    int Nkp, int R, size_t nrows, FftPlanDev pl, const cplx *__restrict__ twg) {
  extern __shared__ unsigned char smraw[];
  const int Nh = Ng >> 1;
  cplx *tw = (cplx *) smraw;
  cplx *tg = tw + Nh;                   // Nh + 1 entries
  cplx *ba = tg + Nh + 1;
  cplx *bb = ba + (size_t) Nh * R;
  for (int e = threadIdx.x; e < Nh; e += blockDim.x) tw[e] = pl.tw[e];
  for (int e = threadIdx.x; e <= Nh; e += blockDim.x) tg[e] = twg[e];
  const size_t row0 = (size_t) blockIdx.x * R;
  for (int e = threadIdx.x; e < R * Nh; e += blockDim.x) {
    const int r = e / Nh, mm = e - r * Nh;
    cplx v; v.x = 0; v.y = 0;
    if (row0 + r < nrows) v = ((const cplx *) (x + (row0 + r) * Ng))[mm];
    ba[mm * R + r] = v;
  }
  __syncthreads();
  cplx *Z = smem_fft<-1>(ba, bb, R, pl, tw);
  for (int e = threadIdx.x; e < R * Nkp; e += blockDim.x) {
    const int r = e / Nkp, k = e - r * Nkp;
    const size_t row = row0 + r;
    if (row >= nrows) continue;
    cplx out; out.x = 0; out.y = 0;
    if (k <= Nh) {
      const int k1 = k % Nh, k2 = (Nh - k) % Nh;
      const cplx a = Z[k1 * R + r], b = Z[k2 * R + r];
      const rt er = (rt) 0.5 * (a.x + b.x), ei = (rt) 0.5 * (a.y - b.y);
      const rt dr = (rt) 0.5 * (a.x - b.x), di = (rt) 0.5 * (a.y + b.y);
      const rt orr = di, oi = -dr;                 // O = (Z - conj)/(2i)
      const cplx w = tg[k];
      const rt c = w.x, s = -w.y;                  // exp(-2 pi i k / Ng)
      out.x = er + orr * c - oi * s;
      out.y = ei + orr * s + oi * c;
    }
    S[row * Nkp + k] = out;
  }
}

// In-place complex transform of one spectrum along axis 0 (i) or 1 (j).
template <int S>
__global__ void __launch_bounds__(FFT_NT)
fft_axis_one(cplx *__restrict__ a, int Ng, int Nkp, int K, int axis,
    FftPlanDev pl) {
  extern __shared__ unsigned char smraw[];
  cplx *tw = (cplx *) smraw;
  cplx *ba = tw + Ng;
  cplx *bb = ba + (size_t) Ng * K;
  const int o = blockIdx.x, k0 = blockIdx.y * K;
  for (int e = threadIdx.x; e < Ng; e += blockDim.x) tw[e] = pl.tw[e];
  const size_t stride = axis == 0 ? (size_t) Ng * Nkp : (size_t) Nkp;
  const size_t base = axis == 0 ? (size_t) o * Nkp + k0 : (size_t) o * Ng * Nkp + k0;
  for (int e = threadIdx.x; e < Ng * K; e += blockDim.x) {
    const int i = e / K, c = e - i * K;
    ba[i * K + c] = a[base + i * stride + c];
  }
  __syncthreads();
  cplx *res = smem_fft<S>(ba, bb, K, pl, tw);
  for (int e = threadIdx.x; e < Ng * K; e += blockDim.x) {
    const int i = e / K, c = e - i * K;
    a[base + i * stride + c] = res[i * K + c];
  }
}

__global__ void scale_kernel(real *a, size_t n, real f) {
  for (size_t i = (size_t) blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (size_t) gridDim.x * blockDim.x)
    a[i] *= f;
}

// --------------------------------------------------------------- host side
struct TwTable {
  cplx *dev = nullptr;
  int n = 0;
};
std::mutex g_tw_mu;
std::map<std::pair<int, int>, cplx *> g_tw;       // (device, n) -> table

cplx *twiddles(int dev, int n) {
  std::lock_guard<std::mutex> lk(g_tw_mu);
  auto key = std::make_pair(dev, n);
  auto it = g_tw.find(key);
  if (it != g_tw.end()) return it->second;
  std::vector<cplx> h(n);
  const long double tpi = 6.283185307179586476925286766559005768L;
  for (int e = 0; e < n; e++) {
    const long double a = tpi * (long double) e / (long double) n;
    h[e].x = (rt) cosl(a);
    h[e].y = (rt) sinl(a);
  }
  cplx *d = nullptr;
  if (!EZ_CUDA_OK(cudaMalloc(&d, sizeof(cplx) * n)) ||
      !EZ_CUDA_OK(cudaMemcpy(d, h.data(), sizeof(cplx) * n, cudaMemcpyHostToDevice)))
    return nullptr;
  g_tw[key] = d;
  return d;
}

bool make_plan(int dev, int n, FftPlanDev *pl) {
  pl->n = n;
  pl->nfac = 0;
  int m = n;
  while (m > 1) {
    int r = 0;
    if (m % 8 == 0) r = 8;
    else if (m % 4 == 0) r = 4;
    else if (m % 2 == 0) r = 2;
    else if (m % 3 == 0) r = 3;
    else if (m % 5 == 0) r = 5;
    else return false;
    if (pl->nfac >= MAXF) return false;
    pl->fac[pl->nfac++] = r;
    m /= r;
  }
  pl->tw = twiddles(dev, n);
  return pl->tw != nullptr;
}

}  // namespace

// Columns per tile for passes I and J: 3 K Ng complex values per buffer stay
// within the shared-memory budget (two ping-pong buffers per block).
int ez_fft_tile_k(int Ng) {
  int K = 16;
  while (K > 1 && (size_t) 3 * K * Ng * sizeof(cplx) > 96 * 1024) K >>= 1;
  return K;
}

// Grid sizes the GPU transforms handle: even, 5-smooth, and small enough that
// one column (pass J, K = 1) and one row (pass K, R = 1) fit shared memory.
bool ez_fft_supported(int Ng) {
  if (Ng < 8 || (Ng & 1)) return false;
  int m = Ng;
  for (int r : {2, 3, 5}) while (m % r == 0) m /= r;
  if (m != 1) return false;
  const size_t Nh = Ng / 2;
  const size_t sm_j = sizeof(cplx) * ((size_t) Ng + 2 * (size_t) Ng * 3);
  const size_t sm_k = sizeof(cplx) * (2 * Nh + 3 * (Nh + 1) + 2 * Nh * 3);
  return sm_j <= 200 * 1024 && sm_k <= 200 * 1024;
}

namespace {
bool w32_ready[64] = {false};

bool set_w32(int dev) {
  if (dev < 0 || dev >= 64) return false;
  if (w32_ready[dev]) return true;
  cplx h[32];
  const long double tpi = 6.283185307179586476925286766559005768L;
  for (int k = 0; k < 32; k++) {
    h[k].x = (rt) cosl(tpi * k / 32);
    h[k].y = (rt) sinl(tpi * k / 32);
  }
  if (!EZ_CUDA_OK(cudaMemcpyToSymbol(c_w32, h, sizeof(h)))) return false;
  w32_ready[dev] = true;
  return true;
}

// E = n / 32 when n is 32 times a power of two up to 32, else 0.
int warp_e(int n) {
  if (n % 32) return 0;
  const int e = n / 32;
  return (e <= 32 && (e & (e - 1)) == 0) ? e : 0;
}

// The warp-shuffle passes serve Ng when Ng and Ng/2 are both 32 E and the
// pass-J tile (three lines of WK columns) fits the 227 KB per-block limit.
bool warp_path(int Ng) {
  if (!warp_e(Ng) || !warp_e(Ng / 2)) return false;
  return sizeof(cplx) * ((size_t) Ng + 3 * WK * (size_t) (Ng + 1)) <= 227 * 1024;
}

}  // namespace

bool ez_tma_encode(CUtensorMap *map, CUtensorMapDataType type, int rank, void *base,
    const uint64_t *dims, const uint64_t *strides_bytes, const uint32_t *box,
    CUtensorMapSwizzle swizzle) {
  typedef CUresult (*EncodeFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
      const cuuint64_t *, const cuuint64_t *, const cuuint32_t *, const cuuint32_t *,
      CUtensorMapInterleave, CUtensorMapSwizzle, CUtensorMapL2promotion,
      CUtensorMapFloatOOBfill);
  static std::mutex mu;
  static EncodeFn fn = nullptr;
  static bool tried = false;
  {
    std::lock_guard<std::mutex> lk(mu);
    if (!tried) {
      tried = true;
      void *p = nullptr;
      cudaDriverEntryPointQueryResult q;
      if (EZ_CUDA_OK(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q)) &&
          q == cudaDriverEntryPointSuccess)
        fn = (EncodeFn) p;
      else
        cudaGetLastError();
    }
  }
  if (!fn) return false;
  cuuint64_t d[5], st[4];
  cuuint32_t bx[5], es[5];
  for (int i = 0; i < rank; i++) { d[i] = dims[i]; bx[i] = box[i]; es[i] = 1; }
  for (int i = 0; i + 1 < rank; i++) st[i] = strides_bytes[i];
  return fn(map, type, (cuuint32_t) rank, base, d, st, bx, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
            swizzle, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
         CUDA_SUCCESS;
}

namespace {

// Pass J through tpass_j_kernel (FP32, E = 8 or 16).  False if nothing was
// launched (no tensor maps or a failed launch): the cp.async pass runs then.
template <int E>
bool run_tpass_j(EzMesh *m, const FftPlanDev &pn) {
  const int Ng = m->Ng;
  if (sizeof(rt) != 4 || 32 * E != Ng) return false;
  const uint64_t dims[3] = {2 * (uint64_t) m->Nkp, (uint64_t) Ng, (uint64_t) Ng};
  const uint64_t str[2] = {2 * (uint64_t) m->Nkp * sizeof(rt),
                           2 * (uint64_t) m->Nkp * Ng * sizeof(rt)};
  const uint32_t box[3] = {16, (uint32_t) std::min(Ng, TP_BOX), 1};
  CUtensorMap mj[3];
  for (int a = 0; a < 3; a++)
    if (!ez_tma_encode(&mj[a], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, m->spec[a], dims, str, box,
                       CU_TENSOR_MAP_SWIZZLE_64B))
      return false;
  const size_t smj = TpLayout<E>::bytes(2);
  if (!EZ_CUDA_OK(cudaFuncSetAttribute(tpass_j_kernel<E>,
          cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smj))) {
    cudaGetLastError();
    return false;
  }
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, m->device);
  const int nkt = (m->Nk + WK - 1) / WK;
  const int ntiles = Ng * nkt;
  const unsigned grid = (unsigned) std::min(nsm, ntiles);
  ez_stage_begin(m, ST_FFT_J);
  // A_x (spec1), A_0 (spec2) -> B_x (spec1), B_0 (spec2), B_y (spec0)
  tpass_j_kernel<E><<<grid, TP_THREADS, smj, m->stream>>>(mj[1], mj[2], mj[1], mj[2], mj[0],
      Ng, nkt, ntiles, pn.tw, (EzCicStats *) m->stats); ez_count_launch();
  ez_stage_end(m, ST_FFT_J);
  return EZ_CUDA_OK(cudaGetLastError());
}

// pass I with row-major tiles of 8 columns (the 64-byte-swizzled layout of
// the TMA pass J, so a warp reading one column meets each bank at most
// twice), copied in 16-byte chunks (two columns of a row) and stored as
// 16-byte chunks, half the copy instructions of wpass_i; a per-warp scratch
// line for the transforms.  The same transforms, so the same results.
template <int E>
__global__ void __launch_bounds__(32 * WKI, 2)
wpass_i_rm(const cplx *__restrict__ S, cplx *__restrict__ Ax, cplx *__restrict__ A0,
    int Ng, int Nkp, const cplx *__restrict__ twn) {
  static_assert(WKI == 8, "one warp per column of an 8-column tile");
  constexpr int n = 32 * E;
  extern __shared__ __align__(16) unsigned char smraw[];
  cplx *tw = (cplx *) smraw;                 // n
  cplx *b0 = tw + n;                         // n x 8: S, then A_0
  cplx *b1 = b0 + 8 * n;                     // n x 8: A_x
  cplx *scr = b1 + 8 * n;                    // a scratch line per warp
  const int j = blockIdx.y, k0 = blockIdx.x * 8;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int e = threadIdx.x; e < n; e += blockDim.x) tw[e] = twn[e];
  const size_t pst = (size_t) Ng * Nkp;
  const cplx *src = S + (size_t) j * Nkp + k0;
#pragma unroll 4
  for (int q = threadIdx.x; q < n * 4; q += 32 * WKI) {
    const int row = q >> 2, c = (q & 3) << 1;
    __pipeline_memcpy_async(b0 + tix(row, c), src + row * pst + c, 16);
  }
  __pipeline_commit();
  __pipeline_wait_prior(0);
  __syncthreads();
  const int c = w;
  cplx *line = scr + (size_t) w * n;
  cplx v[E];
#pragma unroll
  for (int m = 0; m < E; m++) {
    const int i = 32 * m + lane;
    v[m] = b0[tix(i, c)];
    const rt f = freq_of(i, Ng);
    v[m].x *= f;
    v[m].y *= f;
  }
  line_fft<E, 1, use_t<E>(0)>(v, tw, lane, line);
#pragma unroll
  for (int q = 0; q < E; q++) b1[tix(line_out<E, use_t<E>(0)>(lane, q), c)] = v[q];
#pragma unroll
  for (int m = 0; m < E; m++) v[m] = b0[tix(32 * m + lane, c)];
  __syncwarp();
  line_fft<E, 1, use_t<E>(0)>(v, tw, lane, line);
#pragma unroll
  for (int q = 0; q < E; q++) b0[tix(line_out<E, use_t<E>(0)>(lane, q), c)] = v[q];
  __syncthreads();
  cplx *dx = Ax + (size_t) j * Nkp + k0, *d0 = A0 + (size_t) j * Nkp + k0;
#pragma unroll 4
  for (int q = threadIdx.x; q < n * 4; q += 32 * WKI) {
    const int row = q >> 2, c2 = (q & 3) << 1;
    const size_t g = row * pst + c2;
    *reinterpret_cast<float4 *>(dx + g) = *reinterpret_cast<const float4 *>(b1 + tix(row, c2));
    *reinterpret_cast<float4 *>(d0 + g) = *reinterpret_cast<const float4 *>(b0 + tix(row, c2));
  }
}

// Pass I with its tiles moved by the Tensor Memory Accelerator (FP32): one
// CTA per tile, the transforms of wpass_i_rm (so the results are the same
// bit for bit), but the S tile arrives by tensor copies of 256-row boxes
// (2 KC floats x 1 j x 256 i of the spectrum, swizzled) and A_x and A_0
// leave the same way, so the load/store unit only carries the transforms'
// own shared-memory traffic, not the cp.async fills and the 16-byte
// shared-to-global copies of wpass_i_rm.  Thread 0 issues the copies;
// the mbarrier wait is bounded, and a wait that runs out sets
// stats->tma_err (read by the population), skips the tile and lets the
// copies land before the CTA returns.
// KC columns per tile (one warp each): 8 (64-byte rows, 64-byte swizzle, the
// layout of tix) or 4 (32-byte rows, 32-byte swizzle: the 16-byte half of a
// row is flipped by bit 2 of the row).
template <int KC>
__device__ __forceinline__ int tixk(int row, int c) {
  if constexpr (KC == 8) return tix(row, c);
  else return row * 4 + ((((c >> 1) ^ ((row >> 2) & 1)) << 1) | (c & 1));
}
template <int E, int KC> constexpr int tpi_min_blocks() {
  return KC == 4 ? (E == 16 ? 4 : 2) : (E == 16 ? 2 : 1);
}
template <int E, int KC> struct TpiLayout {
  static constexpr int n = 32 * E;
  static constexpr size_t tile = (size_t) n * KC * 8;
  static constexpr size_t tw_bytes = ((size_t) n * 8 + 1023) / 1024 * 1024;
  static constexpr bool T = use_t<E>(0);
  static constexpr size_t scr_bytes = T ? (size_t) KC * n * 8 : 0;
  // [twiddles][tile S -> A_0][tile A_x][scratch lines][barrier] + alignment
  static constexpr size_t bytes = tw_bytes + 2 * tile + scr_bytes + 64 + 1024;
};

template <int E, int KC>
__global__ void __launch_bounds__(32 * KC, (tpi_min_blocks<E, KC>()))
tpass_i_tile(const __grid_constant__ CUtensorMap ms, const __grid_constant__ CUtensorMap mx,
    const __grid_constant__ CUtensorMap m0, int Ng, int nkt, const cplx *__restrict__ twn,
    EzCicStats *stats) {
  typedef TpiLayout<E, KC> Lay;
  constexpr int n = Lay::n;
  constexpr int NB = n / TP_BOX > 0 ? n / TP_BOX : 1;   // boxes per tile
  constexpr int BR = n < TP_BOX ? n : TP_BOX;           // rows per box
  constexpr int RB = KC * 8;                            // bytes per row
  extern __shared__ __align__(1024) unsigned char tpi_raw[];
  // 1 KB alignment of the tiles (the swizzle patterns repeat every 256 or
  // 512 B), kept as an offset into the shared array so addresses stay 32-bit
  unsigned char *base = tpi_raw + ((1024u - (ez_smem_addr(tpi_raw) & 1023u)) & 1023u);
  cplx *tw = (cplx *) base;
  cplx *b0 = (cplx *) (base + Lay::tw_bytes);              // S, then A_0
  cplx *b1 = (cplx *) ((unsigned char *) b0 + Lay::tile);  // A_x
  cplx *scr = (cplx *) ((unsigned char *) b1 + Lay::tile);
  uint64_t *full = (uint64_t *) ((unsigned char *) scr + Lay::scr_bytes);
  const int lane = threadIdx.x & 31, c = threadIdx.x >> 5;
  const bool producer = threadIdx.x == 0;
  if (producer) {
    const int j = blockIdx.x / nkt, kt = blockIdx.x - j * nkt;
    ez_mbar_init(full, 1);
    ez_fence_mbar_init();
    ez_mbar_expect_tx(full, (uint32_t) Lay::tile);
#pragma unroll
    for (int b = 0; b < NB; b++)
      ez_tma_load3((unsigned char *) b0 + (size_t) b * BR * RB, &ms, 2 * KC * kt, j, b * BR,
                   full);
  }
  for (int e = threadIdx.x; e < n; e += blockDim.x) tw[e] = twn[e];
  __syncthreads();
  // a wait that runs out leaves the tile unwritten and skips the stores
  const bool ok = ez_mbar_wait(full, 0);
  {
    cplx *line = scr + (size_t) c * n;
    cplx v[E];
#pragma unroll
    for (int m = 0; m < E; m++) {
      const int i = 32 * m + lane;
      v[m] = b0[tixk<KC>(i, c)];
      const rt f = freq_of(i, Ng);
      v[m].x *= f;
      v[m].y *= f;
    }
    line_fft<E, 1, Lay::T>(v, tw, lane, line);
#pragma unroll
    for (int q = 0; q < E; q++) b1[tixk<KC>(line_out<E, Lay::T>(lane, q), c)] = v[q];
#pragma unroll
    for (int m = 0; m < E; m++) v[m] = b0[tixk<KC>(32 * m + lane, c)];
    __syncwarp();
    line_fft<E, 1, Lay::T>(v, tw, lane, line);
#pragma unroll
    for (int q = 0; q < E; q++) b0[tixk<KC>(line_out<E, Lay::T>(lane, q), c)] = v[q];
  }
  ez_fence_async_smem();
  const bool all = __syncthreads_and(ok);
  if (producer) {
    if (all) {
      const int j = blockIdx.x / nkt, kt = blockIdx.x - j * nkt;
#pragma unroll
      for (int b = 0; b < NB; b++) {
        const size_t off = (size_t) b * BR * RB;
        ez_tma_store3(&mx, 2 * KC * kt, j, b * BR, (const unsigned char *) b1 + off);
        ez_tma_store3(&m0, 2 * KC * kt, j, b * BR, (const unsigned char *) b0 + off);
      }
      ez_tma_commit();
      ez_tma_wait_read<0>();                 // the tiles are read before the CTA ends
    } else {
      atomicExch(&stats->tma_err, 1u);
      ez_mbar_wait(full, 0);                 // the load lands before the CTA ends
    }
  }
}

// Pass I through tpass_i_tile (FP32, Ng = 32 E with E = 16 or 32).  False if
// nothing was launched (no tensor maps or shared memory): the cp.async
// kernels run then.
template <int E, int KC>
bool run_tpass_i(EzMesh *m, const FftPlanDev &pn) {
  const int Ng = m->Ng;
  if (sizeof(rt) != 4 || 32 * E != Ng || E < 16 || E > 32) return false;
  const uint64_t dims[3] = {2 * (uint64_t) m->Nkp, (uint64_t) Ng, (uint64_t) Ng};
  const uint64_t str[2] = {2 * (uint64_t) m->Nkp * sizeof(rt),
                           2 * (uint64_t) m->Nkp * Ng * sizeof(rt)};
  const uint32_t box[3] = {2 * KC, 1, (uint32_t) std::min(Ng, TP_BOX)};
  CUtensorMap mp[3];
  for (int a = 0; a < 3; a++)
    if (!ez_tma_encode(&mp[a], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, m->spec[a], dims, str, box,
                       KC == 8 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_32B))
      return false;
  const size_t sm = TpiLayout<E, KC>::bytes;
  if (!EZ_CUDA_OK(cudaFuncSetAttribute(tpass_i_tile<E, KC>,
          cudaFuncAttributeMaxDynamicSharedMemorySize, (int) sm))) {
    cudaGetLastError();
    return false;
  }
  const int nkt = (m->Nk + KC - 1) / KC;
  ez_stage_begin(m, ST_FFT_I);
  tpass_i_tile<E, KC><<<(unsigned) (Ng * nkt), 32 * KC, sm, m->stream>>>(mp[0], mp[1], mp[2],
      Ng, nkt, pn.tw, (EzCicStats *) m->stats); ez_count_launch();
  ez_stage_end(m, ST_FFT_I);
  return EZ_CUDA_OK(cudaGetLastError());
}

template <int E>
int run_wpass_i(EzMesh *m, const FftPlanDev &pn) {
  // With the tensor copies: 512^3 0.720 -> 0.643 ms on 8-column tiles, 0.613
  // on 4-column tiles (four CTAs of four warps per SM); 1024^3 5.73 -> 5.02
  // ms on 8-column tiles (8.64 on 4-column ones).  At 256^3 the column-major
  // tiles of wpass_i stay faster (0.095 against 0.132 ms).
  if constexpr (E >= 16) {
    if (m->fft_tma && m->fft_tma_i && run_tpass_i<E, E == 16 ? 4 : 8>(m, pn)) return 0;
  }
  const int Ng = m->Ng;
  const size_t n = 32 * E, LS = n + 1;
  const int nkt = (m->Nk + WKI - 1) / WKI;
  ez_stage_begin(m, ST_FFT_I);
#ifdef SINGLE_PREC
  // 512^3 (E = 16): 0.739 -> 0.713 ms with the row-major tiles; at 256^3 they
  // measured slower (0.094 -> 0.145 ms: fewer blocks per SM) and at 1024^3
  // the same
  if constexpr (E == 16) {
    const size_t sm_r = sizeof(cplx) * (n + 16 * n + WKI * n);
    cudaFuncSetAttribute(wpass_i_rm<E>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) sm_r);
    wpass_i_rm<E><<<dim3(nkt, Ng), 32 * WKI, sm_r, m->stream>>>(m->spec[0], m->spec[1],
        m->spec[2], Ng, m->Nkp, pn.tw); ez_count_launch();
    ez_stage_end(m, ST_FFT_I);
    return 0;
  }
#endif
  const size_t sm_i = sizeof(cplx) * (n + 2 * WKI * LS);
  cudaFuncSetAttribute(wpass_i<E>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) sm_i);
  wpass_i<E><<<dim3(nkt, Ng), 32 * WKI, sm_i, m->stream>>>(m->spec[0], m->spec[1],
      m->spec[2], Ng, m->Nkp, pn.tw); ez_count_launch();
  ez_stage_end(m, ST_FFT_I);
  return 0;
}

template <int E>
int run_wpass_j(EzMesh *m, const FftPlanDev &pn) {
  const int Ng = m->Ng;
  const size_t n = 32 * E, LS = n + 1;
  const size_t sm_j = sizeof(cplx) * (n + 3 * WK * LS);
  cudaFuncSetAttribute(wpass_j<E>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) sm_j);
  const int nkt = (m->Nk + WK - 1) / WK;
  ez_stage_begin(m, ST_FFT_J);
  wpass_j<E><<<dim3(nkt, Ng), 32 * WNW, sm_j, m->stream>>>(m->spec[0], m->spec[1],
      m->spec[2], Ng, m->Nkp, pn.tw); ez_count_launch();
  ez_stage_end(m, ST_FFT_J);
  return 0;
}

template <int E>
int run_wpass_ij(EzMesh *m, const FftPlanDev &pn) {
  run_wpass_i<E>(m, pn);
  if constexpr (E == 8 || E == 16) {
    if (m->fft_tma && run_tpass_j<E>(m, pn)) return 0;
  }
  return run_wpass_j<E>(m, pn);
}

template <int E>
int run_wpass_k(EzMesh *m, const FftPlanDev &ph, const cplx *twg) {
  const int Ng = m->Ng;
  const size_t n = 32 * E;
  const size_t sm = sizeof(cplx) * (2 * n + WNW * (n + 1));
  cudaFuncSetAttribute(wpass_k<E>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) sm);
  const size_t nrows = (size_t) Ng * Ng;
  const unsigned nb = (unsigned) std::min<size_t>((nrows + WNW - 1) / WNW, 148 * 16);
  ez_stage_begin(m, ST_FFT_K);
  wpass_k<E><<<nb, 32 * WNW, sm, m->stream>>>(m->spec[0], m->spec[1], m->spec[2],
      m->psi[0], m->psi[1], m->psi[2], Ng, m->Nkp, nrows, ph.tw, twg,
      (EzCicStats *) m->stats); ez_count_launch();
  ez_stage_end(m, ST_FFT_K);
  return 0;
}
}  // namespace

int ez_fft_c2r_psi(EzMesh *m) {
  const int Ng = m->Ng, Nkp = m->Nkp, Nh = Ng / 2;
  const int Ei = warp_e(Ng), Ek = warp_e(Nh);
  if (warp_path(Ng) && m->Nkp % WK == 0 && set_w32(m->device)) {
    FftPlanDev pn, ph;
    if (!make_plan(m->device, Ng, &pn) || !make_plan(m->device, Nh, &ph))
      return EZMOCK_ERR_UNKNOWN;
    const cplx *twg = twiddles(m->device, Ng);
    if (!twg) return EZMOCK_ERR_UNKNOWN;
    cudaMemsetAsync(&((EzCicStats *) m->stats)->tma_err, 0, sizeof(unsigned int), m->stream);
    switch (Ei) {
      case 2: run_wpass_ij<2>(m, pn); break;
      case 4: run_wpass_ij<4>(m, pn); break;
      case 8: run_wpass_ij<8>(m, pn); break;
      case 16: run_wpass_ij<16>(m, pn); break;
      default: run_wpass_ij<32>(m, pn); break;
    }
    cudaMemsetAsync(&((EzCicStats *) m->stats)->psimax_bits, 0, sizeof(unsigned int), m->stream);
    switch (Ek) {
      case 1: run_wpass_k<1>(m, ph, twg); break;
      case 2: run_wpass_k<2>(m, ph, twg); break;
      case 4: run_wpass_k<4>(m, ph, twg); break;
      case 8: run_wpass_k<8>(m, ph, twg); break;
      default: run_wpass_k<16>(m, ph, twg); break;
    }
    m->psimax_valid = true;
    return EZ_CUDA_OK(cudaGetLastError()) ? 0 : EZMOCK_ERR_UNKNOWN;
  }
  const int K = ez_fft_tile_k(Ng);
  FftPlanDev pn, ph;
  if (!make_plan(m->device, Ng, &pn) || !make_plan(m->device, Nh, &ph))
    return EZMOCK_ERR_UNKNOWN;
  const cplx *twg = twiddles(m->device, Ng);
  if (!twg) return EZMOCK_ERR_UNKNOWN;

  const size_t sm_i = sizeof(cplx) * ((size_t) Ng + 2 * (size_t) Ng * 2 * K);
  const size_t sm_j = sizeof(cplx) * ((size_t) Ng + 2 * (size_t) Ng * 3 * K);
  int R = 4;
  while (R > 1 && sizeof(cplx) * (2 * (size_t) Nh + 3 * R * (Nh + 1) + 2 * (size_t) Nh * 3 * R) > 160 * 1024) R >>= 1;
  const size_t sm_k = sizeof(cplx) * (2 * (size_t) Nh + 3 * R * (size_t) (Nh + 1) + 2 * (size_t) Nh * 3 * R);
  // per-device function attributes: set on every call (current device)
  if (!EZ_CUDA_OK(cudaFuncSetAttribute(fft_pass_i, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024)) ||
      !EZ_CUDA_OK(cudaFuncSetAttribute(fft_pass_j, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024)) ||
      !EZ_CUDA_OK(cudaFuncSetAttribute(fft_pass_k, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024)))
    return EZMOCK_ERR_UNKNOWN;
  const int nkt = (m->Nk + K - 1) / K;
  ez_stage_begin(m, ST_FFT_I);
  fft_pass_i<<<dim3(Ng, nkt), FFT_NT, sm_i, m->stream>>>(m->spec[0], m->spec[1],
      m->spec[2], Ng, Nkp, K, pn); ez_count_launch();
  ez_stage_end(m, ST_FFT_I);
  ez_stage_begin(m, ST_FFT_J);
  fft_pass_j<<<dim3(Ng, nkt), FFT_NT, sm_j, m->stream>>>(m->spec[0], m->spec[1],
      m->spec[2], Ng, Nkp, K, pn); ez_count_launch();
  ez_stage_end(m, ST_FFT_J);
  const size_t nrows = (size_t) Ng * Ng;
  cudaMemsetAsync(&((EzCicStats *) m->stats)->psimax_bits, 0, sizeof(unsigned int), m->stream);
  ez_stage_begin(m, ST_FFT_K);
  fft_pass_k<<<(unsigned) ((nrows + R - 1) / R), FFT_NT, sm_k, m->stream>>>(
      m->spec[0], m->spec[1], m->spec[2], m->psi[0], m->psi[1], m->psi[2], Ng,
      Nkp, R, nrows, ph, twg, (EzCicStats *) m->stats); ez_count_launch();
  ez_stage_end(m, ST_FFT_K);
  m->psimax_valid = true;
  return EZ_CUDA_OK(cudaGetLastError()) ? 0 : EZMOCK_ERR_UNKNOWN;
}

// r2c(delta) (sign -1, unnormalised) into spec[0]
// (libEZmock/EZmock/dens_field.c:195-201).
int ez_fft_r2c_delta(EzMesh *m, const real *d_delta) {
  return ez_fft_r2c(m->device, m->stream, d_delta, m->spec[0], m->Ng, m->Nkp);
}

// Forward (sign -1, unnormalised) r2c of an Ng^3 real grid into half-complex
// rows of Nkp >= Ng/2 + 1 values (FFTW's r2c layout, padded).
int ez_fft_r2c(int dev, cudaStream_t st, const real *in, cplx *out, int Ng, int Nkp) {
  const int Nh = Ng / 2;
  const int Nk = Nh + 1;
  FftPlanDev pn, ph;
  if (!make_plan(dev, Ng, &pn) || !make_plan(dev, Nh, &ph))
    return EZMOCK_ERR_UNKNOWN;
  const cplx *twg = twiddles(dev, Ng);
  if (!twg) return EZMOCK_ERR_UNKNOWN;
  int R = 8;
  while (R > 1 && sizeof(cplx) * (2 * (size_t) Nh + 1 + 2 * (size_t) Nh * R) > 160 * 1024) R >>= 1;
  const size_t sm_r = sizeof(cplx) * (2 * (size_t) Nh + 1 + 2 * (size_t) Nh * R);
  const int K = ez_fft_tile_k(Ng);
  const size_t sm_a = sizeof(cplx) * ((size_t) Ng + 2 * (size_t) Ng * K);
  if (!EZ_CUDA_OK(cudaFuncSetAttribute(fft_r2c_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024)) ||
      !EZ_CUDA_OK(cudaFuncSetAttribute(fft_axis_one<-1>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024)))
    return EZMOCK_ERR_UNKNOWN;
  const size_t nrows = (size_t) Ng * Ng;
  fft_r2c_rows<<<(unsigned) ((nrows + R - 1) / R), FFT_NT, sm_r, st>>>(
      in, out, Ng, Nkp, R, nrows, ph, twg); ez_count_launch();
  const int nkt = (Nk + K - 1) / K;
  fft_axis_one<-1><<<dim3(Ng, nkt), FFT_NT, sm_a, st>>>(out, Ng, Nkp, K, 1, pn); ez_count_launch();
  fft_axis_one<-1><<<dim3(Ng, nkt), FFT_NT, sm_a, st>>>(out, Ng, Nkp, K, 0, pn); ez_count_launch();
  return EZ_CUDA_OK(cudaGetLastError()) ? 0 : EZMOCK_ERR_UNKNOWN;
}

int ez_scale_psi(EzMesh *m, real f) {
  scale_kernel<<<148 * 16, 256, 0, m->stream>>>(m->psi[0], 3 * m->N, f); ez_count_launch();
  return EZ_CUDA_OK(cudaGetLastError()) ? 0 : EZMOCK_ERR_UNKNOWN;
}
