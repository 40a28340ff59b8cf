// ez_cic.cu -- particle displacement fused with cloud-in-cell assignment.
//
// Particle (i,j,k) moves to x = psi * Ng/L + (i,j,k) and deposits the eight
// CIC weights (libEZmock/EZmock/dens_field.c:233-310).  The same pass also
// deposits the three displacement-weighted grids that the reference builds
// later, one dimension at a time, for tracer velocities
// (libEZmock/EZmock/pop_tracer.c:593-683, before its division by rho), so
// the displacement fields are read once.  Expression order and `real`
// rounding of positions and weights follow the reference.
//
// Two accumulation modes:
//   0  float/double atomics in L2 (order-dependent rounding, as the
//      reference's `omp atomic`);
//   1  deterministic: contributions converted to 64-bit fixed point
//      (2^-50 resolution for rho, 2^-40 for the momenta) and added with
//      integer atomics, which are associative, then converted back.  Results
//      are independent of scheduling.
#include "ez_internal.cuh"

namespace {

constexpr int CIC_NT = 256;

__device__ __forceinline__ void cic_axis(real p, real igs, int i, int Ng,
    int *c0, int *c1, real *w0, real *w1) {
  const real x = p * igs + i;
  int x0 = (int) floor((double) x);
  *w1 = x - x0;
  *w0 = 1 - *w1;
  if (x0 < 0) x0 += Ng;
  else if (x0 >= Ng) x0 -= Ng;
  // Displacements beyond one box length are never produced by the Zel'dovich
  // fields; keep the index in range regardless.
  if (x0 < 0 || x0 >= Ng) { x0 %= Ng; if (x0 < 0) x0 += Ng; }
  *c0 = x0;
  *c1 = (x0 == Ng - 1) ? 0 : x0 + 1;
}

__device__ __forceinline__ size_t idx3(int Ng, int a, int b, int c) {
  return ((size_t) a * Ng + b) * Ng + c;
}

template <bool PAINT>
__global__ void __launch_bounds__(CIC_NT)
cic_atomic_kernel(const real *__restrict__ p0, const real *__restrict__ p1,
    const real *__restrict__ p2, real *rho, real *q0, real *q1, real *q2,
    int Ng, real igs, size_t N) {
  for (size_t id = (size_t) blockIdx.x * blockDim.x + threadIdx.x; id < N;
       id += (size_t) gridDim.x * blockDim.x) {
    const int k = (int) (id % Ng);
    const size_t ij = id / Ng;
    const int j = (int) (ij % Ng), i = (int) (ij / Ng);
    const real a = p0[id], b = p1[id], c = p2[id];
    int x0, x1, y0, y1, z0, z1;
    real wx0, wx1, wy0, wy1, wz0, wz1;
    cic_axis(a, igs, i, Ng, &x0, &x1, &wx0, &wx1);
    cic_axis(b, igs, j, Ng, &y0, &y1, &wy0, &wy1);
    cic_axis(c, igs, k, Ng, &z0, &z1, &wz0, &wz1);
    const size_t c000 = idx3(Ng, x0, y0, z0), c001 = idx3(Ng, x0, y0, z1);
    const size_t c010 = idx3(Ng, x0, y1, z0), c011 = idx3(Ng, x0, y1, z1);
    const size_t c100 = idx3(Ng, x1, y0, z0), c101 = idx3(Ng, x1, y0, z1);
    const size_t c110 = idx3(Ng, x1, y1, z0), c111 = idx3(Ng, x1, y1, z1);
    atomicAdd(rho + c000, wx0 * wy0 * wz0);
    atomicAdd(rho + c001, wx0 * wy0 * wz1);
    atomicAdd(rho + c010, wx0 * wy1 * wz0);
    atomicAdd(rho + c011, wx0 * wy1 * wz1);
    atomicAdd(rho + c100, wx1 * wy0 * wz0);
    atomicAdd(rho + c101, wx1 * wy0 * wz1);
    atomicAdd(rho + c110, wx1 * wy1 * wz0);
    atomicAdd(rho + c111, wx1 * wy1 * wz1);
    if (PAINT) {
      const real pv[3] = {a, b, c};
      real *q[3] = {q0, q1, q2};
#pragma unroll
      for (int d = 0; d < 3; d++) {
        const real u0 = wx0 * pv[d], u1 = wx1 * pv[d];
        atomicAdd(q[d] + c000, u0 * wy0 * wz0);
        atomicAdd(q[d] + c001, u0 * wy0 * wz1);
        atomicAdd(q[d] + c010, u0 * wy1 * wz0);
        atomicAdd(q[d] + c011, u0 * wy1 * wz1);
        atomicAdd(q[d] + c100, u1 * wy0 * wz0);
        atomicAdd(q[d] + c101, u1 * wy0 * wz1);
        atomicAdd(q[d] + c110, u1 * wy1 * wz0);
        atomicAdd(q[d] + c111, u1 * wy1 * wz1);
      }
    }
  }
}

// ---- deterministic mode: 64-bit fixed point ----
constexpr double FIX_RHO = 1125899906842624.0;    // 2^50: rho < 8192 per cell
constexpr double FIX_MOM = 1099511627776.0;       // 2^40: |sum psi w| < 2^23

__device__ __forceinline__ void fadd(unsigned long long *a, double v, double s) {
  atomicAdd(a, (unsigned long long) (long long) llrint(v * s));
}

__global__ void __launch_bounds__(CIC_NT)
cic_fixed_kernel(const real *__restrict__ p0, const real *__restrict__ p1,
    const real *__restrict__ p2, unsigned long long *acc, int Ng, real igs,
    size_t N) {
  // acc layout: 4 grids of N words (rho, q0, q1, q2)
  for (size_t id = (size_t) blockIdx.x * blockDim.x + threadIdx.x; id < N;
       id += (size_t) gridDim.x * blockDim.x) {
    const int k = (int) (id % Ng);
    const size_t ij = id / Ng;
    const int j = (int) (ij % Ng), i = (int) (ij / Ng);
    const real pv[3] = {p0[id], p1[id], p2[id]};
    int x0, x1, y0, y1, z0, z1;
    real wx0, wx1, wy0, wy1, wz0, wz1;
    cic_axis(pv[0], igs, i, Ng, &x0, &x1, &wx0, &wx1);
    cic_axis(pv[1], igs, j, Ng, &y0, &y1, &wy0, &wy1);
    cic_axis(pv[2], igs, k, Ng, &z0, &z1, &wz0, &wz1);
    const size_t cs[8] = {idx3(Ng, x0, y0, z0), idx3(Ng, x0, y0, z1),
                          idx3(Ng, x0, y1, z0), idx3(Ng, x0, y1, z1),
                          idx3(Ng, x1, y0, z0), idx3(Ng, x1, y0, z1),
                          idx3(Ng, x1, y1, z0), idx3(Ng, x1, y1, z1)};
    const real ws[8] = {wx0 * wy0 * wz0, wx0 * wy0 * wz1, wx0 * wy1 * wz0,
                        wx0 * wy1 * wz1, wx1 * wy0 * wz0, wx1 * wy0 * wz1,
                        wx1 * wy1 * wz0, wx1 * wy1 * wz1};
#pragma unroll
    for (int c = 0; c < 8; c++) {
      fadd(acc + cs[c], (double) ws[c], FIX_RHO);
#pragma unroll
      for (int d = 0; d < 3; d++)
        fadd(acc + (size_t) (d + 1) * N + cs[c], (double) ws[c] * (double) pv[d], FIX_MOM);
    }
  }
}

__global__ void fixed_to_real(const unsigned long long *__restrict__ acc,
    real *rho, real *q0, real *q1, real *q2, size_t N) {
  for (size_t id = (size_t) blockIdx.x * blockDim.x + threadIdx.x; id < N;
       id += (size_t) gridDim.x * blockDim.x) {
    rho[id] = (real) ((double) (long long) acc[id] / FIX_RHO);
    q0[id] = (real) ((double) (long long) acc[N + id] / FIX_MOM);
    q1[id] = (real) ((double) (long long) acc[2 * N + id] / FIX_MOM);
    q2[id] = (real) ((double) (long long) acc[3 * N + id] / FIX_MOM);
  }
}

}  // namespace

int ez_cic(EzMesh *m, double Lbox) {
  const int Ng = m->Ng;
  const size_t N = m->N;
  const real igs = Ng / Lbox;
  const unsigned grid = (unsigned) ((N + CIC_NT - 1) / CIC_NT < 148u * 64u
      ? (N + CIC_NT - 1) / CIC_NT : 148u * 64u);
  ez_stage_begin(m, ST_CIC);
  if (m->cic_mode == 1) {
    // 4 x N 64-bit accumulators, allocated on first use
    const size_t need = 4 * N * sizeof(unsigned long long);
    if (!m->fixacc && !EZ_CUDA_OK(cudaMalloc(&m->fixacc, need))) {
      m->fixacc = nullptr;
      return EZMOCK_ERR_MEMORY;
    }
    unsigned long long *acc = m->fixacc;
    if (!EZ_CUDA_OK(cudaMemsetAsync(acc, 0, need, m->stream))) return EZMOCK_ERR_UNKNOWN;
    cic_fixed_kernel<<<grid, CIC_NT, 0, m->stream>>>(m->psi[0], m->psi[1],
        m->psi[2], acc, Ng, igs, N); ez_count_launch();
    fixed_to_real<<<grid, CIC_NT, 0, m->stream>>>(acc, m->rho, m->paint[0],
        m->paint[1], m->paint[2], N); ez_count_launch();
  }
  else {
    if (!EZ_CUDA_OK(cudaMemsetAsync(m->rho, 0, N * sizeof(real), m->stream))) return EZMOCK_ERR_UNKNOWN;
    for (int d = 0; d < 3; d++)
      if (!EZ_CUDA_OK(cudaMemsetAsync(m->paint[d], 0, N * sizeof(real), m->stream)))
        return EZMOCK_ERR_UNKNOWN;
    cic_atomic_kernel<true><<<grid, CIC_NT, 0, m->stream>>>(m->psi[0], m->psi[1],
        m->psi[2], m->rho, m->paint[0], m->paint[1], m->paint[2], Ng, igs, N); ez_count_launch();
  }
  ez_stage_end(m, ST_CIC);
  return EZ_CUDA_OK(cudaGetLastError()) ? 0 : EZMOCK_ERR_UNKNOWN;
}
