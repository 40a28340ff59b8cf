// ez_ic.cu -- Fourier-space initial field S(k) (the reference's `rhok`
// before its multiplication by k_i; libEZmock/EZmock/perturb.c:78-359).
//
// Cell c of the half-complex grid (row-major, Ng x Ng x (Ng/2+1), origin
// skipped) uses draws 2(c-1) (amplitude, get_double_pos) and 2(c-1)+1
// (phase, get_double); with fixed amplitudes only draw c-1 (phase).  On the
// k=0 and Nyquist planes the reference samples the lower half plane and
// writes the partner (-i,-j) with its real part negated; here every thread
// computes its own cell, upper-half cells from their partner's draws, so the
// kernel needs no scattered writes.  The real parts at the seven non-origin
// self-conjugate corners are zeroed (perturb.c:344-359).  All arithmetic is
// FP64 (log, sqrt, sin, cos and the cubic-spline P(k)), rounded to `real` on
// store, in the reference's expression order.  The interpolated P(k) is
// tabulated per integer k^2 (pkq_kernel), which changes no result.
#include "ez_internal.cuh"

namespace {

constexpr int IC_NT = 128;

// bin search + natural cubic spline (linear_pk.c:36-51, 194-202;
// cspline.c:91-105)
__device__ __forceinline__ double pk_eval(const double *__restrict__ kt,
    const double *__restrict__ Pt, const double *__restrict__ P2, int n,
    double kv) {
  int l = 0, u = n - 1, idx = -1;
  while (l <= u) {
    const int i = (l + u) >> 1;
    if (i >= n - 1) { idx = (kt[n - 1] == kv) ? n - 1 : -1; break; }
    if (kt[i + 1] <= kv) l = i + 1;
    else if (kt[i] > kv) u = i - 1;
    else { idx = i; break; }
  }
  if (idx == n - 1) return Pt[idx];
  if (idx < 0) {
    if (kv >= kt[n - 1]) return Pt[n - 1];
    return Pt[0];
  }
  const int j = idx + 1;
  const double ba = kt[j] - kt[idx];
  const double xa = kv - kt[idx];
  const double bx = kt[j] - kv;
  const double ba2 = ba * ba;
  const double lower = xa * Pt[j] + bx * Pt[idx];
  const double c = (xa * xa - ba2) * xa * P2[j];
  const double d = (bx * bx - ba2) * bx * P2[idx];
  return (lower + 0x1.5555555555555p-3 * (c + d)) / ba;
}

// The interpolated power depends on the cell only through the integer
// ksq = ki^2 + kj^2 + k^2 (exact in double), so it is tabulated once per
// field: q[ksq] = exp(P/2) for a log table, P otherwise (the per-cell
// expressions below then apply exactly the reference's operations).
// The FP32 build also tabulates the amplitude factor of a mode in single
// precision, qa[ksq] = (Q or sqrt Q) Pfac / (ksq kfac), so that a cell needs
// one multiplication by the square root of its -log u.
__global__ void pkq_kernel(double *__restrict__ q, int nq,
    const double *__restrict__ tab, int npk, int logpk, double kfac,
    double logkfac, float *__restrict__ qa, double Pfac) {
  const double *kt = tab, *Pt = tab + npk, *P2 = tab + 2 * npk;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < nq; s += gridDim.x * blockDim.x) {
    if (s == 0) { q[0] = 0; if (qa) qa[0] = 0; continue; }   // the origin is never sampled
    const double ksq = (double) s;
    const double kmod = logpk ? log(ksq) * 0.5 + logkfac : kfac * sqrt(ksq);
    const double P = pk_eval(kt, Pt, P2, npk, kmod);
    q[s] = logpk ? exp(P * 0.5) : P;
    if (qa) qa[s] = (float) ((logpk ? q[s] : sqrt(q[s])) * Pfac / (ksq * kfac));
  }
}

#ifdef SINGLE_PREC
// -log(u) for u = ez_upos(ran, x) in single precision, without branches
// (a warp's draws take both halves).  The logarithm is the classical atanh
// series, log((1 + s)/(1 - s)) = 2 (s + s^3/3 + s^5/5 + ...): for u < 1/2,
// u = m 2^e with m in [1, 2) and s = (m - 1)/(m + 1); for u >= 1/2 the exact
// 1 - u = w is formed in integers and -log(1 - w) = 2 atanh(w / (2 - w)), so
// the result keeps its relative accuracy where -log(u) is small.  s <= 1/3:
// nine terms leave a truncation below 2^-30.  Measured against long double
// over 4e7 random and 2e4 edge draws: at most 5.2 ulp (3.1e-7 relative).
__device__ __forceinline__ float neglog_upos_f(int ran, uint32_t x) {
  const bool hi = x >= 0x80000000u;
  float v;                                     // u (lower half) or w = 1 - u
  if (ran)                                     // u = (x + 1/2) 2^-32
    v = ((float) (hi ? 0xFFFFFFFFu - x : x) + 0.5f) * 2.3283064365386963e-10f;
  else                                         // u = x / 4294967088
    v = (float) (hi ? 4294967088u - x : x) * 2.3283065e-10f;
  const int bits = __float_as_int(v);
  const int e = ((bits >> 23) & 0xff) - 127;
  const float m = __int_as_float((bits & 0x007fffff) | 0x3f800000);
  const float s = __fdividef(hi ? v : m - 1.f, hi ? 2.f - v : m + 1.f);
  const float s2 = s * s;
  float p = 1.f / 17.f;
  p = fmaf(p, s2, 1.f / 15.f);
  p = fmaf(p, s2, 1.f / 13.f);
  p = fmaf(p, s2, 1.f / 11.f);
  p = fmaf(p, s2, 1.f / 9.f);
  p = fmaf(p, s2, 1.f / 7.f);
  p = fmaf(p, s2, 1.f / 5.f);
  p = fmaf(p, s2, 1.f / 3.f);
  p = fmaf(p, s2, 1.f);
  const float at = s * p;                      // atanh(s)
  return hi ? 2.f * at : fmaf((float) -e, 0.693147180559945309f, -2.f * at);
}

// sin(pi x) and cos(pi x) for x in [0, 2]: x = q/2 + r with q = rint(2x) and
// |r| <= 1/4 (r exact by Sterbenz's lemma), then sin(pi r) = r S(r^2) and
// cos(pi r) = C(r^2), degree-4 polynomials fitted to sin(pi r)/r and
// cos(pi r) by relative least squares on 4000 Chebyshev nodes of [-1/4, 1/4]
// (at most 1.7 ulp in single precision), and the quadrant's signs and swap.
#ifndef EZ_IC_OWN_SINCOS
#define EZ_IC_OWN_SINCOS 1
#endif
__device__ __forceinline__ void sincospi_unit(float x, float *s, float *c) {
#if EZ_IC_OWN_SINCOS
  const float qf = rintf(2.f * x);
  const float r = fmaf(qf, -0.5f, x);
  const int q = (int) qf;
  const float t = r * r;
  const float ps = r * fmaf(fmaf(fmaf(fmaf(0.08099576830863953f, t, -0.5992013216018677f), t,
      2.5501625537872314f), t, -5.167712688446045f), t, 3.1415927410125732f);
  const float pc = fmaf(fmaf(fmaf(fmaf(0.23126046359539032f, t, -1.335035800933838f), t,
      4.058706760406494f), t, -4.934802055358887f), t, 1.f);
  const bool sw = q & 1;
  const float sv = sw ? pc : ps, cv = sw ? ps : pc;
  *s = (q & 2) ? -sv : sv;
  *c = ((q + 1) & 2) ? -cv : cv;
#else
  sincospif(x, s, c);
#endif
}

// 2 u for u = ez_u(ran, x), the argument of sincospi for the phase 2 pi u.
__device__ __forceinline__ float twice_u_f(int ran, uint32_t x) {
  return ran ? (float) x * 4.656612873077393e-10f      // 2^-31
             : (float) x * 4.656613e-10f;              // 2 / 4294967088
}
#endif

// One warp per (i, j) row of the half-complex grid.  The generator (RAN),
// the draws per cell (PER: 2, or 1 with fixed amplitudes) and the inverted
// phase (IPH) are template parameters; a row's draws and output are
// addressed from per-row pointers, and the two draws of a cell come as one
// 8-byte load (512^3: 0.52 -> 0.47 ms with the polynomial sincospi).  A
// separate path for the interior columns (no partner draws or sign changes)
// measured no faster.
template <int RAN, int PER, bool IPH>
__device__ __forceinline__ cplx ic_mode(const uint32_t *__restrict__ draws, size_t src,
    const double *__restrict__ pkq, const float *__restrict__ pka, int logpk, int isq,
    double kfac, double Pfac) {
  uint32_t da, dp;                                // amplitude and phase draws
  if (PER == 2) {
    const uint2 d = reinterpret_cast<const uint2 *>(draws)[src];
    da = d.x;
    dp = d.y;
  } else {
    da = 0;
    dp = draws[src];
  }
  cplx out;
#ifdef SINGLE_PREC
  // FP32 production mode: amplitude and phase in single precision from the
  // same bit-exact draws (about 2e-7 relative per mode)
  float P = pka[isq];
  if (PER == 2) P *= sqrtf(neglog_upos_f(RAN, da));
  float sn, cs;
  sincospi_unit(twice_u_f(RAN, dp), &sn, &cs);
  if (IPH) { sn = -sn; cs = -cs; }
  out.x = -P * sn;
  out.y = P * cs;
#else
  const double ksq = (double) isq;
  const double Q = pkq[isq];
  double P;
  if (PER == 1) P = logpk ? Q : sqrt(Q);
  else {
    const double amp = -log(ez_upos(RAN, da));
    P = logpk ? Q * sqrt(amp) : sqrt(Q * amp);
  }
  P *= Pfac;
  double phase = ez_u(RAN, dp) * 2 * EZ_PI;
  if (IPH) phase += EZ_PI;
  P /= (ksq * kfac);
  out.x = -P * sin(phase);
  out.y = P * cos(phase);
#endif
  return out;
}

template <int RAN, int PER, bool IPH>
__global__ void __launch_bounds__(IC_NT)
ic_kernel(cplx *__restrict__ S, const uint32_t *__restrict__ draws,
    const double *__restrict__ pkq, const float *__restrict__ pka, int logpk, int Ng,
    int Nk, int Nkp, double kfac, double Pfac) {
  const int Ngh = Ng >> 1;
  // one warp per row: the row's set-up is shared by the 8 cells (512^3) a
  // lane computes (with a block per row it was about half of the kernel's
  // instructions)
  const int i = blockIdx.y, j = blockIdx.x * (IC_NT / 32) + (threadIdx.x >> 5);
  if (j >= Ng) return;
  const int row = i * Ng + j;
  const int ki = (i <= Ngh) ? i : i - Ng;
  const int kj = (j <= Ngh) ? j : j - Ng;
  const int ni = (i == 0) ? 0 : Ng - i, nj = (j == 0) ? 0 : Ng - j;
  const int kij = ki * ki + kj * kj;
  const bool lower = (i == ni && j <= Ngh) || (i != ni && i <= Ngh);
  const bool selfp = (i == ni && j == nj);
  const bool even = (Ng & 1) == 0;
  // self-conjugate corners (0|Ngh, 0|Ngh, 0|Ngh), the origin excepted
  const bool crow = even && (i == 0 || i == Ngh) && (j == 0 || j == Ngh);
  // draws of cell c = row * Nk + k (c >= 1) start at (c - 1) PER
  const size_t rowc = (size_t) row * Nk, prowc = ((size_t) ni * Ng + nj) * Nk;
  cplx *Srow = S + (size_t) row * Nkp;
  for (int k = threadIdx.x & 31; k < Nkp; k += 32) {
    cplx out;
    out.x = 0; out.y = 0;
    if (k < Nk && (row | k) != 0) {
      // k = 0 or Ng/2: the reference samples the lower half plane and writes
      // the partner (-i, -j) with its real part negated
      const bool plane = (k == 0) || (even && k == Ngh);
      out = ic_mode<RAN, PER, IPH>(draws, ((!plane || lower) ? rowc : prowc) + k - 1, pkq, pka,
          logpk, kij + k * k, kfac, Pfac);
      if (plane && (!lower || selfp)) out.x = -out.x;
      if (crow && plane) out.x = 0;
    }
    Srow[k] = out;
  }
}

// White-noise input: S = i sqrt(P)/(k^2 kf) L^-1.5 r2c(delta)
// (perturb.c:476-554), applied to the forward transform already in S.
__global__ void __launch_bounds__(IC_NT)
wn_scale_kernel(cplx *__restrict__ S, const double *__restrict__ pkq,
    int logpk, int Ng, int Nk, int Nkp, double kfac, double Pfac) {
  const int Ngh = Ng >> 1;
  const int row = blockIdx.x;
  const int i = row / Ng, j = row - i * Ng;
  const int ki = (i <= Ngh) ? i : i - Ng;
  const int kj = (j <= Ngh) ? j : j - Ng;
  const int kij = ki * ki + kj * kj;
  for (int k = threadIdx.x; k < Nkp; k += blockDim.x) {
    const size_t g = (size_t) row * Nkp + k;
    cplx w = S[g], out;
    out.x = 0; out.y = 0;
    if (k < Nk && !(row == 0 && k == 0)) {
      const int isq = kij + k * k;
      const double ksq = (double) isq;
      double P = pkq[isq];
      P = logpk ? P : sqrt(P);
      P *= Pfac / (ksq * kfac);
      out.x = -P * w.y;
      out.y = P * w.x;
    }
    S[g] = out;
  }
}

}  // namespace

namespace {
// q[ksq] for ksq = 0 .. 3 (Ng/2)^2 on the mesh's device, followed (FP32
// build) by the single-precision amplitude factors.
int pkq_build(EzMesh *m, const EzPk *pk, double kfac, double logkfac, double Pfac) {
  const int Ngh = m->Ng >> 1;
  const int nq = 3 * Ngh * Ngh + 1;
  if (!m->pkq && !EZ_CUDA_OK(cudaMalloc(&m->pkq, (size_t) nq * (sizeof(double) + sizeof(float))))) {
    m->pkq = nullptr;
    cudaGetLastError();
    return EZMOCK_ERR_MEMORY;
  }
#ifdef SINGLE_PREC
  float *qa = (float *) (m->pkq + nq);
#else
  float *qa = nullptr;
#endif
  pkq_kernel<<<(nq + 255) / 256, 256, 0, m->stream>>>(m->pkq, nq, pk->d_tab, pk->n,
      pk->log ? 1 : 0, kfac, logkfac, qa, Pfac); ez_count_launch();
  return 0;
}
}  // namespace

int ez_ic_spectrum(EzMesh *m, const EzPk *pk, double Lbox, int ran,
    int fixamp, int iphase, const uint32_t *draws) {
  const int Ng = m->Ng;
  const double kfac = EZ_PI * 2 / Lbox;
  const double logkfac = log(kfac);
  const double Pfac = pow(Lbox, -1.5);
  // (the draws of a cell as one 8-byte load: the buffer is 8-byte aligned)
  if (((uintptr_t) draws & 7) != 0) return EZMOCK_ERR_UNKNOWN;
  ez_stage_begin(m, ST_IC);
  int e = pkq_build(m, pk, kfac, logkfac, Pfac);
  if (e) return e;
  const int nq = 3 * (Ng >> 1) * (Ng >> 1) + 1;
  auto kern = iphase
      ? (ran ? (fixamp ? ic_kernel<1, 1, true> : ic_kernel<1, 2, true>)
             : (fixamp ? ic_kernel<0, 1, true> : ic_kernel<0, 2, true>))
      : (ran ? (fixamp ? ic_kernel<1, 1, false> : ic_kernel<1, 2, false>)
             : (fixamp ? ic_kernel<0, 1, false> : ic_kernel<0, 2, false>));
  kern<<<dim3((unsigned) ((Ng + IC_NT / 32 - 1) / (IC_NT / 32)), (unsigned) Ng), IC_NT, 0,
      m->stream>>>(
      m->spec[0], draws, m->pkq, (const float *) (m->pkq + nq), pk->log ? 1 : 0, Ng, m->Nk,
      m->Nkp, kfac, Pfac); ez_count_launch();
  ez_stage_end(m, ST_IC);
  return EZ_CUDA_OK(cudaGetLastError()) ? 0 : EZMOCK_ERR_UNKNOWN;
}

int ez_wn_scale(EzMesh *m, const EzPk *pk, double Lbox) {
  const int Ng = m->Ng;
  const double kfac = EZ_PI * 2 / Lbox;
  int e = pkq_build(m, pk, kfac, log(kfac), pow(Lbox, -1.5));
  if (e) return e;
  wn_scale_kernel<<<(unsigned) ((size_t) Ng * Ng), IC_NT, 0, m->stream>>>(
      m->spec[0], m->pkq, pk->log ? 1 : 0, Ng, m->Nk, m->Nkp, kfac,
      pow(Lbox, -1.5)); ez_count_launch();
  return EZ_CUDA_OK(cudaGetLastError()) ? 0 : EZMOCK_ERR_UNKNOWN;
}
