// ez_pk.cu -- power-spectrum multipoles and count-in-cell PDF of a tracer
// catalogue in the periodic box of an instance.
//
// The reference measures clustering with external programs
// (example/fit/pyclustering.py:173-186, POWSPEC configured by
// example/fit/conf/powspec.conf: cubic box, CIC assignment on 256^3 with grid
// interlacing, multipoles 0 and 2, linear k bins).  This is the same standard
// periodic-box estimator on the GPU:
//   * tracers (optionally moved to redshift space along z, z + rsd_fac v_z,
//     wrapped into [0, L) as save_res.c:147-158 writes them) are assigned
//     with CIC to grid points x_i = i h, and with interlacing also to the
//     grid x_i + h/2;
//   * both grids are transformed (forward r2c), combined as
//     F = (F_0 + exp(-i k.h/2) F_1) / 2, and divided by the CIC window
//     prod_d sinc^2(pi k_d / Ng);
//   * P(k) = L^3 |F|^2 / N^2; the multipoles P_l = (2l+1) <P L_l(mu)> over
//     the modes of each bin (mu = k_z / |k|, both halves of the half-complex
//     grid counted), with the shot noise L^3 / N subtracted from P_0.
//     Bin sums are accumulated in FP64.
// Count-in-cell PDF: tracers counted per cell of an Ng^3 grid (nearest grid
// cell, cell i covering [i h, (i+1) h)); pdf[c] is the fraction of cells
// holding c tracers, the last bin collecting c >= nbin - 1.
#include "ez_internal.cuh"
#include "ezmock_b200.h"

#include <cmath>
#include <vector>

namespace {

constexpr int PK_NT = 256;
constexpr int PK_MAXBIN = 1024;

// Grid coordinate in [0, Ng) of position p (box length L).
__device__ __forceinline__ double gcoord(double p, double ig, int Ng) {
  double u = p * ig;
  u -= floor(u / Ng) * Ng;
  if (u >= Ng) u -= Ng;
  if (u < 0) u = 0;
  return u;
}

__device__ __forceinline__ double zpos(const real *z, const real *vz, size_t t,
    double rsd, double L) {
  double v = z[t];
  if (vz && rsd != 0) {
    v += rsd * vz[t];
    if (v < 0) v += L;
    else if (v >= L) v -= L;
  }
  return v;
}

// CIC assignment; shift = 0.5 places the grid points at (i + 1/2) h.
__global__ void __launch_bounds__(PK_NT)
assign_kernel(const real *__restrict__ x, const real *__restrict__ y,
    const real *__restrict__ z, const real *__restrict__ vz, size_t n,
    double rsd, double L, int Ng, double shift, real *__restrict__ g) {
  const double ig = Ng / L;
  for (size_t t = (size_t) blockIdx.x * PK_NT + threadIdx.x; t < n;
       t += (size_t) gridDim.x * PK_NT) {
    double u[3] = {gcoord(x[t], ig, Ng) - shift, gcoord(y[t], ig, Ng) - shift,
                   gcoord(zpos(z, vz, t, rsd, L), ig, Ng) - shift};
    int i0[3], i1[3];
    double w1[3];
#pragma unroll
    for (int d = 0; d < 3; d++) {
      double f = floor(u[d]);
      w1[d] = u[d] - f;
      int c = (int) f;
      if (c < 0) c += Ng;
      if (c >= Ng) c -= Ng;
      i0[d] = c;
      i1[d] = (c + 1 == Ng) ? 0 : c + 1;
    }
#pragma unroll
    for (int a = 0; a < 2; a++)
#pragma unroll
      for (int b = 0; b < 2; b++)
#pragma unroll
        for (int c = 0; c < 2; c++) {
          const double w = (a ? w1[0] : 1 - w1[0]) * (b ? w1[1] : 1 - w1[1]) *
                           (c ? w1[2] : 1 - w1[2]);
          const size_t id = ((size_t) (a ? i1[0] : i0[0]) * Ng + (b ? i1[1] : i0[1])) * Ng +
                            (c ? i1[2] : i0[2]);
          atomicAdd(g + id, (real) w);
        }
  }
}

__device__ __forceinline__ double sinc(double x) { return x == 0 ? 1.0 : sin(x) / x; }

// Mode sums per bin: [0] modes, [1] sum |k|, [2] sum P, [3] sum P L2(mu).
__global__ void __launch_bounds__(PK_NT)
modes_kernel(const cplx *__restrict__ F0, const cplx *__restrict__ F1, int Ng,
    int Nkp, double kf, double kmin, double dk, int nbin, double pnorm,
    double *__restrict__ acc) {
  __shared__ double s[4 * PK_MAXBIN];
  for (int e = threadIdx.x; e < 4 * nbin; e += PK_NT) s[e] = 0;
  __syncthreads();
  const int Nh = Ng / 2, Nk = Nh + 1;
  const size_t ncell = (size_t) Ng * Ng * Nk;
  for (size_t c = (size_t) blockIdx.x * PK_NT + threadIdx.x; c < ncell;
       c += (size_t) gridDim.x * PK_NT) {
    const int k = (int) (c % Nk);
    const size_t ij = c / Nk;
    const int j = (int) (ij % Ng), i = (int) (ij / Ng);
    const int ki = (i <= Nh) ? i : i - Ng, kj = (j <= Nh) ? j : j - Ng;
    const long long q2 = (long long) ki * ki + (long long) kj * kj + (long long) k * k;
    if (!q2) continue;
    const double kmag = kf * sqrt((double) q2);
    const double fb = floor((kmag - kmin) / dk);
    if (fb < 0 || fb >= nbin) continue;
    const int b = (int) fb;
    const size_t g = ij * Nkp + k;
    double re = F0[g].x, im = F0[g].y;
    if (F1) {
      // exp(-i pi (ki + kj + k) / Ng) F_1
      double sn, cs;
      sincospi(-(double) (ki + kj + k) / Ng, &sn, &cs);
      const double r1 = F1[g].x, i1 = F1[g].y;
      re = 0.5 * (re + cs * r1 - sn * i1);
      im = 0.5 * (im + cs * i1 + sn * r1);
    }
    const double w = sinc(EZ_PI * ki / Ng) * sinc(EZ_PI * kj / Ng) * sinc(EZ_PI * k / Ng);
    const double w2 = w * w;
    re /= w2;
    im /= w2;
    const double P = (re * re + im * im) * pnorm;
    const double mu2 = (double) k * k / (double) q2;
    const double L2 = 1.5 * mu2 - 0.5;
    const double m = (k == 0 || k == Nh) ? 1.0 : 2.0;
    atomicAdd(&s[4 * b], m);
    atomicAdd(&s[4 * b + 1], m * kmag);
    atomicAdd(&s[4 * b + 2], m * P);
    atomicAdd(&s[4 * b + 3], m * P * L2);
  }
  __syncthreads();
  for (int e = threadIdx.x; e < 4 * nbin; e += PK_NT)
    if (s[e] != 0) atomicAdd(acc + e, s[e]);
}

// Nearest-cell counts.
__global__ void __launch_bounds__(PK_NT)
count_kernel(const real *__restrict__ x, const real *__restrict__ y,
    const real *__restrict__ z, const real *__restrict__ vz, size_t n,
    double rsd, double L, int Ng, unsigned int *__restrict__ cnt) {
  const double ig = Ng / L;
  for (size_t t = (size_t) blockIdx.x * PK_NT + threadIdx.x; t < n;
       t += (size_t) gridDim.x * PK_NT) {
    int c[3] = {(int) gcoord(x[t], ig, Ng), (int) gcoord(y[t], ig, Ng),
                (int) gcoord(zpos(z, vz, t, rsd, L), ig, Ng)};
#pragma unroll
    for (int d = 0; d < 3; d++) if (c[d] >= Ng) c[d] = Ng - 1;
    atomicAdd(cnt + ((size_t) c[0] * Ng + c[1]) * Ng + c[2], 1u);
  }
}

__global__ void __launch_bounds__(PK_NT)
hist_kernel(const unsigned int *__restrict__ cnt, size_t ncell, int nbin,
    unsigned long long *__restrict__ hist) {
  __shared__ unsigned int s[PK_MAXBIN];
  for (int e = threadIdx.x; e < nbin; e += PK_NT) s[e] = 0;
  __syncthreads();
  for (size_t c = (size_t) blockIdx.x * PK_NT + threadIdx.x; c < ncell;
       c += (size_t) gridDim.x * PK_NT) {
    const unsigned int v = cnt[c];
    atomicAdd(&s[v < (unsigned) nbin ? v : nbin - 1], 1u);
  }
  __syncthreads();
  for (int e = threadIdx.x; e < nbin; e += PK_NT)
    if (s[e]) atomicAdd(hist + e, (unsigned long long) s[e]);
}

unsigned grid_of(size_t n) {
  const size_t b = (n + PK_NT - 1) / PK_NT;
  return (unsigned) (b < 148 * 16 ? (b ? b : 1) : 148 * 16);
}

// The catalogue on the device: the instance's last catalogue (x == NULL) or
// host arrays copied into the estimator buffer.
struct Cat {
  const real *x, *y, *z, *vz;
  size_t n;
};

int get_cat(EzMesh *m, const real *x, const real *y, const real *z,
    const real *vz, size_t n, char *stage, Cat *c) {
  if (!x) {
    if (!m->cat || !m->cat_n) return EZMOCK_ERR_ARG_NULL;
    const size_t nc = m->cat_n;
    c->x = m->cat;
    c->y = m->cat + nc;
    c->z = m->cat + 2 * nc;
    c->vz = m->cat + 5 * nc;
    c->n = nc;
    return 0;
  }
  if (!y || !z) return EZMOCK_ERR_ARG_NULL;
  real *d = (real *) stage;
  const size_t b = n * sizeof(real);
  if (!EZ_CUDA_OK(cudaMemcpyAsync(d, x, b, cudaMemcpyHostToDevice, m->stream)) ||
      !EZ_CUDA_OK(cudaMemcpyAsync(d + n, y, b, cudaMemcpyHostToDevice, m->stream)) ||
      !EZ_CUDA_OK(cudaMemcpyAsync(d + 2 * n, z, b, cudaMemcpyHostToDevice, m->stream)) ||
      (vz && !EZ_CUDA_OK(cudaMemcpyAsync(d + 3 * n, vz, b, cudaMemcpyHostToDevice, m->stream))))
    return EZMOCK_ERR_UNKNOWN;
  c->x = d;
  c->y = d + n;
  c->z = d + 2 * n;
  c->vz = vz ? d + 3 * n : nullptr;
  c->n = n;
  return 0;
}

// Estimator buffer of the mesh, grown on demand.
int est_buffer(EzMesh *m, size_t bytes) {
  if (bytes <= m->est_cap) return 0;
  if (m->est) {
    cudaStreamSynchronize(m->stream);
    cudaFree(m->est);
  }
  m->est = nullptr;
  m->est_cap = 0;
  if (!EZ_CUDA_OK(cudaMalloc(&m->est, bytes))) { cudaGetLastError(); return EZMOCK_ERR_MEMORY; }
  m->est_cap = bytes;
  return 0;
}

size_t align256(size_t b) { return (b + 255) / 256 * 256; }

}  // namespace

int ez_powspec(EzMesh *m, double L, const real *x, const real *y, const real *z,
    const real *vz, size_t n, double rsd, int Ng, int interlace, double kmin,
    double kmax, int nbin, double *kavg, double *nmodes, double *p0, double *p2) {
  if (Ng < 8 || !ez_fft_supported(Ng)) return EZMOCK_ERR_ARG_NGRID;
  if (nbin < 1 || nbin > PK_MAXBIN || !(kmax > kmin) || kmin < 0) return EZMOCK_ERR_ARG_NBIN;
  const size_t N3 = (size_t) Ng * Ng * Ng;
  const int Nkp = (Ng / 2 + 1 + EZ_KPAD - 1) / EZ_KPAD * EZ_KPAD;
  const size_t nspec = (size_t) Ng * Ng * Nkp;
  const size_t g_b = align256(N3 * sizeof(real)), s_b = align256(nspec * sizeof(cplx));
  const size_t a_b = align256(4 * (size_t) nbin * sizeof(double));
  const size_t c_b = x ? align256(4 * n * sizeof(real)) : 0;
  const int ng = interlace ? 2 : 1;
  int e = est_buffer(m, ng * (g_b + s_b) + a_b + c_b);
  if (e) return e;
  char *base = (char *) m->est;
  real *g[2] = {(real *) base, (real *) (base + g_b)};
  cplx *F[2] = {(cplx *) (base + ng * g_b), (cplx *) (base + ng * g_b + s_b)};
  double *acc = (double *) (base + ng * (g_b + s_b));
  Cat c;
  if ((e = get_cat(m, x, y, z, vz, n, base + ng * (g_b + s_b) + a_b, &c))) return e;
  if (!c.n) return EZMOCK_ERR_ARG_NDATA;
  cudaStream_t st = m->stream;
  for (int s = 0; s < ng; s++) {
    if (!EZ_CUDA_OK(cudaMemsetAsync(g[s], 0, N3 * sizeof(real), st))) return EZMOCK_ERR_UNKNOWN;
    assign_kernel<<<grid_of(c.n), PK_NT, 0, st>>>(c.x, c.y, c.z, c.vz, c.n, rsd, L, Ng,
        s ? 0.5 : 0.0, g[s]); ez_count_launch();
    if ((e = ez_fft_r2c(m->device, st, g[s], F[s], Ng, Nkp))) return e;
  }
  if (!EZ_CUDA_OK(cudaMemsetAsync(acc, 0, 4 * (size_t) nbin * sizeof(double), st)))
    return EZMOCK_ERR_UNKNOWN;
  const double kf = 2 * EZ_PI / L, dk = (kmax - kmin) / nbin;
  const double V = L * L * L, nd = (double) c.n;
  const size_t ncell = (size_t) Ng * Ng * (Ng / 2 + 1);
  modes_kernel<<<grid_of(ncell), PK_NT, 0, st>>>(F[0], interlace ? F[1] : nullptr, Ng, Nkp,
      kf, kmin, dk, nbin, V / (nd * nd), acc); ez_count_launch();
  std::vector<double> h(4 * (size_t) nbin);
  if (!EZ_CUDA_OK(cudaMemcpyAsync(h.data(), acc, h.size() * sizeof(double),
          cudaMemcpyDeviceToHost, st)) || !EZ_CUDA_OK(cudaStreamSynchronize(st)))
    return EZMOCK_ERR_UNKNOWN;
  const double shot = V / nd;
  for (int b = 0; b < nbin; b++) {
    const double nm = h[4 * b];
    nmodes[b] = nm;
    kavg[b] = nm ? h[4 * b + 1] / nm : kmin + (b + 0.5) * dk;
    p0[b] = nm ? h[4 * b + 2] / nm - shot : 0;
    p2[b] = nm ? 5 * h[4 * b + 3] / nm : 0;
  }
  return 0;
}

int ez_cic_pdf(EzMesh *m, double L, const real *x, const real *y, const real *z,
    const real *vz, size_t n, double rsd, int Ng, int nbin, double *pdf) {
  if (Ng < 1 || Ng > 4096) return EZMOCK_ERR_ARG_NGRID;
  if (nbin < 1 || nbin > PK_MAXBIN) return EZMOCK_ERR_ARG_NBIN;
  const size_t N3 = (size_t) Ng * Ng * Ng;
  const size_t c_b = align256(N3 * sizeof(unsigned int));
  const size_t h_b = align256((size_t) nbin * sizeof(unsigned long long));
  const size_t s_b = x ? align256(4 * n * sizeof(real)) : 0;
  int e = est_buffer(m, c_b + h_b + s_b);
  if (e) return e;
  char *base = (char *) m->est;
  unsigned int *cnt = (unsigned int *) base;
  unsigned long long *hist = (unsigned long long *) (base + c_b);
  Cat c;
  if ((e = get_cat(m, x, y, z, vz, n, base + c_b + h_b, &c))) return e;
  cudaStream_t st = m->stream;
  if (!EZ_CUDA_OK(cudaMemsetAsync(cnt, 0, N3 * sizeof(unsigned int), st)) ||
      !EZ_CUDA_OK(cudaMemsetAsync(hist, 0, (size_t) nbin * sizeof(unsigned long long), st)))
    return EZMOCK_ERR_UNKNOWN;
  if (c.n) {
    count_kernel<<<grid_of(c.n), PK_NT, 0, st>>>(c.x, c.y, c.z, c.vz, c.n, rsd, L, Ng, cnt);
    ez_count_launch();
  }
  hist_kernel<<<grid_of(N3), PK_NT, 0, st>>>(cnt, N3, nbin, hist); ez_count_launch();
  std::vector<unsigned long long> h(nbin);
  if (!EZ_CUDA_OK(cudaMemcpyAsync(h.data(), hist, h.size() * sizeof(unsigned long long),
          cudaMemcpyDeviceToHost, st)) || !EZ_CUDA_OK(cudaStreamSynchronize(st)))
    return EZMOCK_ERR_UNKNOWN;
  for (int b = 0; b < nbin; b++) pdf[b] = (double) h[b] / (double) N3;
  return 0;
}
