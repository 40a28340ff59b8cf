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

#ifdef SINGLE_PREC
// ---- slab kernel: shared-memory accumulation with a sliding z window ----
//
// A CTA owns the particles of a 16 x 16 column of Lagrangian cells and walks
// it along z in chunks of 8 slices.  Contributions land in a shared-memory
// ring of 16 z slices covering the column widened by H = 2 cells on each
// side (plus the CIC neighbour), for rho and the three momenta.  After each
// chunk the slices no later particle can reach are added to global memory
// with 16-byte vector atomics (4 consecutive z cells) and cleared.  Particles
// displaced by more than H cells fall back to direct global atomics.  Needs
// Ng a multiple of 16.
constexpr int ST = 16;                       // column tile (x and y)
constexpr int SH = 2;                        // halo
constexpr int SB = ST + 2 * SH + 1;          // box side = 21
constexpr int SKZ = 8;                       // z slices per chunk
constexpr int SRING = 16;                    // ring length (z slices)
constexpr int SLAB_NT = 512;
constexpr int SQ = SB * SB * SRING;          // floats per quantity

__device__ __forceinline__ void gadd(real *g, real v) { atomicAdd(g, v); }

__global__ void __launch_bounds__(SLAB_NT)
cic_slab_kernel(const real *__restrict__ p0, const real *__restrict__ p1,
    const real *__restrict__ p2, real *rho, real *q0, real *q1, real *q2,
    int Ng, real igs) {
  extern __shared__ float ring[];            // [4][SB][SB][SRING]
  const int ntile = Ng / ST;
  const int i0 = (blockIdx.x / ntile) * ST, j0 = (blockIdx.x % ntile) * ST;
  for (int e = threadIdx.x; e < 4 * SQ; e += SLAB_NT) ring[e] = 0;
  __syncthreads();
  int U = -4;                                // oldest unflushed z (multiple of 4)
  const int nchunk = Ng / SKZ;
  for (int c = 0; c <= nchunk; c++) {
    if (c < nchunk) {
      const int zc = c * SKZ;
      for (int p = threadIdx.x; p < ST * ST * SKZ; p += SLAB_NT) {
        const int kz = p & (SKZ - 1), tj = (p >> 3) & (ST - 1), ti = p >> 7;
        const int i = i0 + ti, j = j0 + tj, k = zc + kz;
        const size_t id = ((size_t) i * Ng + j) * Ng + k;
        const real pv[3] = {p0[id], p1[id], p2[id]};
        // positions and weights as in dens_field.c:262-289 (unwrapped cells)
        const real x = pv[0] * igs + i, y = pv[1] * igs + j, z = pv[2] * igs + k;
        const int x0 = (int) floor((double) x), y0 = (int) floor((double) y),
                  z0 = (int) floor((double) z);
        const real wx1 = x - x0, wx0 = 1 - wx1;
        const real wy1 = y - y0, wy0 = 1 - wy1;
        const real wz1 = z - z0, wz0 = 1 - wz1;
        const int rx = x0 - (i0 - SH), ry = y0 - (j0 - SH);
        const bool inbox = rx >= 0 && rx <= SB - 2 && ry >= 0 && ry <= SB - 2 &&
            z0 >= zc - SH && z0 <= zc + SKZ - 1 + SH;
        const real wxs[2] = {wx0, wx1}, wys[2] = {wy0, wy1}, wzs[2] = {wz0, wz1};
        if (inbox) {
#pragma unroll
          for (int a = 0; a < 2; a++)
#pragma unroll
            for (int b = 0; b < 2; b++)
#pragma unroll
              for (int cz = 0; cz < 2; cz++) {
                const int base = ((rx + a) * SB + (ry + b)) * SRING + ((z0 + cz) & (SRING - 1));
                const real w = wxs[a] * wys[b] * wzs[cz];
                atomicAdd(ring + base, (float) w);
#pragma unroll
                for (int d = 0; d < 3; d++)
                  atomicAdd(ring + (d + 1) * SQ + base, (float) ((wxs[a] * pv[d]) * wys[b] * wzs[cz]));
              }
        }
        else {
          int xs[2], ys[2], zs[2];
          xs[0] = ((x0 % Ng) + Ng) % Ng; xs[1] = (xs[0] == Ng - 1) ? 0 : xs[0] + 1;
          ys[0] = ((y0 % Ng) + Ng) % Ng; ys[1] = (ys[0] == Ng - 1) ? 0 : ys[0] + 1;
          zs[0] = ((z0 % Ng) + Ng) % Ng; zs[1] = (zs[0] == Ng - 1) ? 0 : zs[0] + 1;
#pragma unroll
          for (int a = 0; a < 2; a++)
#pragma unroll
            for (int b = 0; b < 2; b++)
#pragma unroll
              for (int cz = 0; cz < 2; cz++) {
                const size_t g = ((size_t) xs[a] * Ng + ys[b]) * Ng + zs[cz];
                gadd(rho + g, wxs[a] * wys[b] * wzs[cz]);
                gadd(q0 + g, (wxs[a] * pv[0]) * wys[b] * wzs[cz]);
                gadd(q1 + g, (wxs[a] * pv[1]) * wys[b] * wzs[cz]);
                gadd(q2 + g, (wxs[a] * pv[2]) * wys[b] * wzs[cz]);
              }
        }
      }
    }
    __syncthreads();
    // flush the quads of z slices no later particle can reach
    const int zfinal = (c < nchunk) ? (c + 1) * SKZ - SH : Ng + SH + 2;
    int nq = 0;
    while (U + 4 * (nq + 1) <= zfinal) nq++;
    const int ntask = nq * 4 * SB * SB;
    for (int t = threadIdx.x; t < ntask; t += SLAB_NT) {
      const int qd = t / (4 * SB * SB);
      const int r = t - qd * 4 * SB * SB;
      const int q = r / (SB * SB), col = r - q * SB * SB;
      const int rx = col / SB, ry = col - rx * SB;
      const int zq = U + 4 * qd;
      float4 *src = (float4 *) (ring + q * SQ + col * SRING + (zq & (SRING - 1)));
      const float4 v = *src;
      *src = make_float4(0.f, 0.f, 0.f, 0.f);
      if (v.x == 0.f && v.y == 0.f && v.z == 0.f && v.w == 0.f) continue;
      const int gx = (((i0 - SH + rx) % Ng) + Ng) % Ng;
      const int gy = (((j0 - SH + ry) % Ng) + Ng) % Ng;
      const int gz = ((zq % Ng) + Ng) % Ng;
      real *gq = (q == 0) ? rho : (q == 1) ? q0 : (q == 2) ? q1 : q2;
      atomicAdd((float4 *) (gq + ((size_t) gx * Ng + gy) * Ng + gz), v);
    }
    U += 4 * nq;
    __syncthreads();
  }
}
#endif

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
#ifdef SINGLE_PREC
    if (Ng % ST == 0 && Ng >= 2 * ST) {
      static bool attr = false;
      const size_t smem = 4 * SQ * sizeof(float);
      if (!attr) {
        cudaFuncSetAttribute(cic_slab_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem);
        attr = true;
      }
      cic_slab_kernel<<<(unsigned) ((Ng / ST) * (Ng / ST)), SLAB_NT, smem, m->stream>>>(
          m->psi[0], m->psi[1], m->psi[2], m->rho, m->paint[0], m->paint[1],
          m->paint[2], Ng, igs); ez_count_launch();
    }
    else
#endif
    {
      cic_atomic_kernel<true><<<grid, CIC_NT, 0, m->stream>>>(m->psi[0], m->psi[1],
          m->psi[2], m->rho, m->paint[0], m->paint[1], m->paint[2], Ng, igs, N); ez_count_launch();
    }
  }
  ez_stage_end(m, ST_CIC);
  return EZ_CUDA_OK(cudaGetLastError()) ? 0 : EZMOCK_ERR_UNKNOWN;
}
