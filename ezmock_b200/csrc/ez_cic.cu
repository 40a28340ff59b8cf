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
// ---- owner-computes kernel (FP32) ----
//
// A CTA owns a 16 x 16 column of output cells (all z) and walks it along z in
// chunks of 8 slices.  For each chunk it reads every particle whose cloud can
// reach the column -- Lagrangian cells i0 - OH - 1 .. i0 + 15 + OH in x (the
// lower corner moves by at most OH cells, the upper corner lies one cell
// above it) and likewise in y, (17 + 2 OH)^2 x 8 particles -- and keeps the
// CIC contributions that land in its own cells, in a shared-memory ring of
// three z chunks.  OH is 2 or 3: an instance starts with 3 and uses 2 while
// fewer than 1/4096 of the particles lie farther than 2 cells from their
// Lagrangian cell (every launch counts them).  Accumulation is in 32-bit
// fixed point (integer shared-memory atomics are exact and fast): rho in
// units of 2^-21 per cell, the momenta in units of 2^-s with s chosen from
// the largest |psi| so that no sum can overflow while rho < 1024.  A chunk is
// final once the particles of the next chunk are in; it is then written with
// plain coalesced stores, so every output cell is written exactly once and
// no global atomics are needed.  Particles displaced by more than OH cells in
// any direction are listed by their own CTA and deposited afterwards with
// global atomics (fixup_kernel).  No in-kernel sum can overflow: a cell is
// reached only by particles within OH + 1 Lagrangian cells on each axis,
// (2 OH + 2)^3 <= 512 of them, each with weight <= 1, so rho < 2^9 and the
// momenta stay below 512 max|psi| scale <= 2^30.
constexpr int OT = 16;                       // owned column tile (x and y)
constexpr int OKZ = 8;                       // z slices per chunk
constexpr int ORS = 3 * OKZ;                 // ring: three chunks
constexpr int OWN_NT = 512;
constexpr int OQS = OT * OT * ORS;           // ints per quantity
constexpr float RHO_SCALE = 2097152.f;       // 2^21

typedef EzCicStats CicStats;

// max |psi| over the three displacement fields (for the fixed-point scale)
__global__ void psi_absmax_kernel(const real *__restrict__ p, size_t n,
    CicStats *stats) {
  float mx = 0.f;
  for (size_t i = (size_t) blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (size_t) gridDim.x * blockDim.x)
    mx = fmaxf(mx, fabsf((float) p[i]));
#pragma unroll
  for (int o = 16; o; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if ((threadIdx.x & 31) == 0) atomicMax(&stats->psimax_bits, __float_as_uint(mx));
}

// Wraps an index that lies within one box length of [0, Ng).
__device__ __forceinline__ int wrap1(int v, int Ng) {
  return v < 0 ? v + Ng : (v >= Ng ? v - Ng : v);
}

// Float to integer on the FMA/ALU pipes instead of the conversion unit:
// adding 1.5 * 2^23 places the integer part of |v| < 2^22 in the low
// mantissa bits, rounded to nearest even (the default rounding of the add),
// so the result equals __float2int_rn(v).
constexpr float RMAGIC = 12582912.f;         // 1.5 * 2^23
// round(a * b) of the exact product, |a * b| < 2^22: the magic addition is
// fused into the multiply (one rounding).
__device__ __forceinline__ int fmround(float a, float b) {
  return __float_as_int(__fmaf_rn(a, b, RMAGIC)) - 0x4B400000;
}
// floor(v) for |v| < 2^22, exact: round, then step down where rounding went up.
__device__ __forceinline__ int ffloor(float v) {
  const float t = v + RMAGIC;
  const float r = t - RMAGIC;                // v rounded to an integer, exact
  return __float_as_int(t) - 0x4B400000 - (r > v ? 1 : 0);
}

template <int OH>
__global__ void __launch_bounds__(OWN_NT, 2)
cic_owner_kernel(const real *__restrict__ p0, const real *__restrict__ p1,
    const real *__restrict__ p2, real *rho, real *q0, real *q1, real *q2,
    int Ng, real igs, CicStats *stats, unsigned int *list) {
  constexpr int OW = OT + 2 * OH + 1;        // particle read width
  constexpr int OB = OH + 1;                 // read origin: i0 - OB, j0 - OB
  extern __shared__ __align__(16) int iring[];       // [4][OT*OT][ORS]
  const int nt = Ng / OT;
  const int i0 = (blockIdx.x / nt) * OT, j0 = (blockIdx.x % nt) * OT;
  // momentum scale: 1023 * max|psi| * scale < 2^31
  const float pmax = fmaxf(__uint_as_float(stats->psimax_bits), 1e-30f);
  const float mscale = exp2f(floorf(log2f(2147483647.f / (1024.f * pmax))));
  const float minv = 1.f / mscale;
  for (int e = threadIdx.x; e < OQS; e += OWN_NT)
    reinterpret_cast<int4 *>(iring)[e] = make_int4(0, 0, 0, 0);
  __syncthreads();
  const int nch = Ng / OKZ;
  const int lane = threadIdx.x & 31;
  for (int c = -1; c <= nch; c++) {
    // ring offsets of the chunks c-1, c, c+1 (slices 8(c-1) .. 8c+15)
    const int rb0 = ((c + 2) % 3) * OKZ, rb1 = ((c + 3) % 3) * OKZ, rb2 = ((c + 4) % 3) * OKZ;
    const bool cown = c >= 0 && c < nch;
    // particle p's displacements are loaded one iteration ahead
    auto locate = [&](int p, int &li, int &lj, int &zu, int &iw, int &jw, int &zw) {
      const int kz = p & (OKZ - 1), lc = p >> 3;
      li = lc / OW;
      lj = lc - li * OW;
      iw = wrap1(i0 - OB + li, Ng);
      jw = wrap1(j0 - OB + lj, Ng);
      zu = c * OKZ + kz;
      zw = wrap1(zu, Ng);
      return ((size_t) iw * Ng + jw) * Ng + zw;
    };
    int nli, nlj, nzu, niw, njw, nzw;
    size_t nid = 0;
    real na = 0, nb = 0, nc = 0;
    if (threadIdx.x < OW * OW * OKZ) {
      nid = locate(threadIdx.x, nli, nlj, nzu, niw, njw, nzw);
      na = p0[nid]; nb = p1[nid]; nc = p2[nid];
    }
    for (int p = threadIdx.x; p < OW * OW * OKZ; p += OWN_NT) {
      const int li = nli, lj = nlj, zu = nzu, iw = niw, jw = njw, zw = nzw;
      const size_t id = nid;
      const real pa = na, pb = nb, pc = nc;
      if (p + OWN_NT < OW * OW * OKZ) {
        nid = locate(p + OWN_NT, nli, nlj, nzu, niw, njw, nzw);
        na = p0[nid]; nb = p1[nid]; nc = p2[nid];
      }
      // positions and weights as dens_field.c:262-275 (floor of a float is
      // exact, so the single-precision floor equals the reference's)
      const real x = pa * igs + iw, y = pb * igs + jw, z = pc * igs + zw;
      const int x0 = ffloor(x), y0 = ffloor(y), z0 = ffloor(z);
      const int dx = x0 - iw, dy = y0 - jw, dz = z0 - zw;
      const bool far = dx < -OH || dx > OH || dy < -OH || dy > OH || dz < -OH || dz > OH;
      const bool own = cown && li >= OB && li < OB + OT && lj >= OB && lj < OB + OT;
      const unsigned am = __activemask();
      if (OH > 2) {
        // particles that a launch with OH = 2 would list
        const bool far2 = dx < -2 || dx > 2 || dy < -2 || dy > 2 || dz < -2 || dz > 2;
        const unsigned f2 = __ballot_sync(am, far2 && own);
        if (f2 && lane == __ffs(f2) - 1) atomicAdd(&stats->nfar2, (unsigned) __popc(f2));
      }
      const unsigned fm = __ballot_sync(am, far && own);
      if (fm) {
        const int leader = __ffs(fm) - 1;
        unsigned int base = 0;
        if (lane == leader) {
          base = atomicAdd(&stats->nlist, (unsigned) __popc(fm));
          if (OH == 2) atomicAdd(&stats->nfar2, (unsigned) __popc(fm));
        }
        base = __shfl_sync(am, base, leader);
        if (far && own) list[base + __popc(fm & ((1u << lane) - 1))] = (unsigned int) id;
      }
      if (far) continue;
      // tile coordinates of the lower corner; skip particles whose cloud
      // misses the tile
      const int cx = li - OB + dx, cy = lj - OB + dy, zz = zu + dz;
      const bool ax0 = (unsigned) cx < (unsigned) OT, ax1 = (unsigned) (cx + 1) < (unsigned) OT;
      const bool by0 = (unsigned) cy < (unsigned) OT, by1 = (unsigned) (cy + 1) < (unsigned) OT;
      const bool cz0 = (unsigned) zz < (unsigned) Ng, cz1 = (unsigned) (zz + 1) < (unsigned) Ng;
      if (!((ax0 || ax1) && (by0 || by1) && (cz0 || cz1))) continue;
      const real wx1 = x - x0, wx0 = 1 - wx1;
      const real wy1 = y - y0, wy0 = 1 - wy1;
      const real wz1 = z - z0, wz0 = 1 - wz1;
      // slot of zz and zz + 1 in the ring (zz >> 3 is one of c-1, c, c+1)
      const int k0 = (zz >> 3) - c, k1 = ((zz + 1) >> 3) - c;
      const int s0 = (k0 < 0 ? rb0 : (k0 == 0 ? rb1 : rb2)) + (zz & (OKZ - 1));
      const int s1 = (k1 < 0 ? rb0 : (k1 == 0 ? rb1 : rb2)) + ((zz + 1) & (OKZ - 1));
      const int ox0 = cx * (OT * ORS), ox1 = ox0 + OT * ORS;
      const int oy0 = cy * ORS, oy1 = oy0 + ORS;
      // z weights scaled per quantity: rho, then the three momenta
      const float sm1 = pa * mscale, sm2 = pb * mscale, sm3 = pc * mscale;
      const float zr[2] = {wz0 * RHO_SCALE, wz1 * RHO_SCALE};
      const float za[2] = {wz0 * sm1, wz1 * sm1};
      const float zb[2] = {wz0 * sm2, wz1 * sm2};
      const float zc[2] = {wz0 * sm3, wz1 * sm3};
      const float wxy[4] = {wx0 * wy0, wx0 * wy1, wx1 * wy0, wx1 * wy1};
      const bool okx[2] = {ax0, ax1}, oky[2] = {by0, by1}, okz[2] = {cz0, cz1};
      const int oxs[2] = {ox0, ox1}, oys[2] = {oy0, oy1}, ss[2] = {s0, s1};
#pragma unroll
      for (int ab = 0; ab < 4; ab++) {
        const int ia = ab >> 1, ib = ab & 1;
        if (!(okx[ia] && oky[ib])) continue;
        const int oxy = oxs[ia] + oys[ib];
        const float w = wxy[ab];
#pragma unroll
        for (int ic = 0; ic < 2; ic++) {
          if (!okz[ic]) continue;
          int *r = iring + oxy + ss[ic];
          atomicAdd(r, fmround(w, zr[ic]));
          atomicAdd(r + OQS, fmround(w, za[ic]));
          atomicAdd(r + 2 * OQS, fmround(w, zb[ic]));
          atomicAdd(r + 3 * OQS, fmround(w, zc[ic]));
        }
      }
    }
    __syncthreads();
    const int o = c - 1;                     // output chunk now complete
    if (o >= 0 && o < nch) {
      // one (quantity, column) per thread and pass: 8 slices = two int4
      const int ro = (o % 3) * OKZ;
      for (int t = threadIdx.x; t < 4 * OT * OT; t += OWN_NT) {
        const int q = t / (OT * OT), col = t - q * (OT * OT);
        int4 *src = reinterpret_cast<int4 *>(iring + q * OQS + col * ORS + ro);
        const int4 va = src[0], vb = src[1];
        src[0] = make_int4(0, 0, 0, 0);
        src[1] = make_int4(0, 0, 0, 0);
        const float f = (q == 0) ? (1.f / RHO_SCALE) : minv;
        real *g = (q == 0) ? rho : (q == 1) ? q0 : (q == 2) ? q1 : q2;
        const int cx = col / OT, cy = col - cx * OT;
        float4 *dst = reinterpret_cast<float4 *>(
            g + ((size_t) (i0 + cx) * Ng + (j0 + cy)) * Ng + o * OKZ);
        dst[0] = make_float4(va.x * f, va.y * f, va.z * f, va.w * f);
        dst[1] = make_float4(vb.x * f, vb.y * f, vb.z * f, vb.w * f);
      }
    }
    __syncthreads();
  }
}

// ---- owner-computes kernel on 16 x 32 column tiles (FP32, Ng % 32 == 0) ----
//
// A CTA owns 16 (x) by 32 (y) columns of cells over a z range [zs, ze) (the
// grid is also cut along z so that the CTAs, one per SM, fill whole waves)
// and walks it eight slices at a time.  Each thread owns two of the
// (16 + 2 OH + 1) x (32 + 2 OH + 1) Lagrangian columns whose particles can
// reach the tile, for the whole walk.  A column's next eight particles (one
// 32-byte sector per displacement field, a 256-bit load) are loaded into
// registers while its current eight are deposited, so every sector is read
// from memory once.  Accumulation is 32-bit fixed point (rho in units of
// 2^-21, the momenta in units of 2^-s from max |psi|, as in the kernel above)
// in a shared ring of 24 slices laid out [quantity][slice][x][y] with y
// fastest: the lanes of a warp hold consecutive Lagrangian columns along y,
// so a deposit's bank is its y cell.  Particles z = 8p .. 8p+7 reach slices
// 8p-3 .. 8p+11; after them the eight slices 8p-8 .. 8p-1 are final and are
// written with plain 32-byte stores (one sector per cell and quantity), and
// cleared; at most 20 slices are live at once.  Deposits use `red.shared` on
// 32-bit shared addresses.  Particles displaced by more than OH cells are
// listed by the CTA that owns their Lagrangian cell and deposited by
// fixup_kernel; the overflow bound is the same as above.
constexpr int TX = 16;                        // tile rows (x)
constexpr int TY = 32;                        // tile columns (y): one per bank
constexpr int TZ = 8;                         // particles per column and step
constexpr int TRS = 24;                       // ring slices
constexpr int TSLOT = TX * TY;                // ints per slice and quantity
constexpr int TQS = TRS * TSLOT;              // ints per quantity
constexpr int TNT = 480;                      // threads: two columns each
constexpr size_t TSMEM = 4 * (size_t) TQS * sizeof(int);

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t) __cvta_generic_to_shared(p);
}

__device__ __forceinline__ void red_add(uint32_t addr, int v) {
  asm volatile("red.shared.add.s32 [%0], %1;" :: "r"(addr), "r"(v) : "memory");
}

// 32-byte global accesses (one sector, 32-byte aligned) as single 256-bit
// instructions: the lanes of a warp touch 32 different sectors here (one per
// Lagrangian column or output cell), so each access instruction costs a
// load/store-unit pass per sector, and one 256-bit access instead of two
// 128-bit ones halves those passes.
__device__ __forceinline__ void ld8(const float *p, float4 &a, float4 &b) {
  asm volatile("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=f"(a.x), "=f"(a.y), "=f"(a.z), "=f"(a.w), "=f"(b.x), "=f"(b.y), "=f"(b.z),
                 "=f"(b.w)
               : "l"(p));
}
__device__ __forceinline__ void st8(float *p, float4 a, float4 b) {
  asm volatile("st.global.v8.f32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};"
               :: "l"(p), "f"(a.x), "f"(a.y), "f"(a.z), "f"(a.w), "f"(b.x), "f"(b.y), "f"(b.z),
                  "f"(b.w)
               : "memory");
}

template <int OH>
__global__ void __launch_bounds__(TNT, 1)
cic_tile_kernel(const real *__restrict__ p0, const real *__restrict__ p1,
    const real *__restrict__ p2, real *rho, float4 *pq,
    int Ng, real igs, CicStats *stats, unsigned int *list, int nzs) {
  constexpr int OWX = TX + 2 * OH + 1;        // Lagrangian columns along x
  constexpr int OWY = TY + 2 * OH + 1;        // and along y
  constexpr int OB = OH + 1;                  // read origin: i0 - OB, j0 - OB
  constexpr int NCOL = OWX * OWY;
  static_assert(NCOL <= 2 * TNT, "two columns per thread");
  extern __shared__ __align__(128) int tring[];   // [4][TRS][TX][TY]
  const uint32_t ringb = smem_u32(tring);
  const int nty = Ng / TY;
  const int tile = blockIdx.x / nzs, zsp = blockIdx.x - tile * nzs;
  const int i0 = (tile / nty) * TX, j0 = (tile % nty) * TY;
  const int zlen = Ng / nzs;
  const int zs = zsp * zlen, ze = zs + zlen;
  // steps p cover particles z = 8p .. 8p + 7; those that reach [zs, ze) lie
  // in z = zs - 4 .. ze + 2
  const int pfirst = zs / TZ - 1, plast = ze / TZ;
  const float pmax = fmaxf(__uint_as_float(stats->psimax_bits), 1e-30f);
  const float mscale = exp2f(floorf(log2f(2147483647.f / (1024.f * pmax))));
  const float minv = 1.f / mscale;
  for (int e = threadIdx.x; e < TQS; e += TNT)      // 4 * TQS ints as int4
    reinterpret_cast<int4 *>(tring)[e] = make_int4(0, 0, 0, 0);

  // the thread's two columns (the second may be past the last one)
  struct Col {
    int cxo, cyo;          // tile coordinates of the Lagrangian column
    int iw, jw;            // wrapped lattice indices
    bool own, valid;
  };
  auto setup = [&](int col, Col &C) {
    C.valid = col < NCOL;
    const int cc = C.valid ? col : 0;
    const int li = cc / OWY, lj = cc - (cc / OWY) * OWY;
    C.cxo = li - OB;
    C.cyo = lj - OB;
    C.iw = wrap1(i0 + C.cxo, Ng);
    C.jw = wrap1(j0 + C.cyo, Ng);
    C.own = C.valid && (unsigned) C.cxo < (unsigned) TX && (unsigned) C.cyo < (unsigned) TY;
  };
  Col colA, colB;
  setup(threadIdx.x, colA);
  setup(threadIdx.x + TNT, colB);
  auto zwrap = [&](int p) { const int z = p * TZ; return z < 0 ? z + Ng : (z >= Ng ? z - Ng : z); };
  // [column][field][half]: a step's particles of both columns; a column's
  // next step is loaded as soon as its particles of this step are taken
  float4 cur[2][3][2];
  auto load = [&](int k, int p) {
    const Col &C = k ? colB : colA;
    if (!C.valid) return;
    const size_t o = ((size_t) C.iw * Ng + C.jw) * Ng + zwrap(p);
    const real *src[3] = {p0 + o, p1 + o, p2 + o};
#pragma unroll
    for (int a = 0; a < 3; a++) ld8(src[a], cur[k][a][0], cur[k][a][1]);
  };
#pragma unroll
  for (int k = 0; k < 2; k++)
#pragma unroll
    for (int a = 0; a < 3; a++) cur[k][a][0] = cur[k][a][1] = make_float4(0, 0, 0, 0);
  load(0, pfirst);
  load(1, pfirst);
  unsigned int nfar2 = 0;
  __syncthreads();

  for (int p = pfirst; p <= plast; p++) {
    const int zc = zwrap(p);
    // ring slice of the unwrapped slice 8p - 8 (slices 8p-8 .. 8p+15 map to
    // rbase + 0 .. 23, wrapping past 24)
    const int rbase = (((p - 1) % 3) + 3) % 3 * TZ;
#pragma unroll
    for (int k = 0; k < 2; k++) {
      const Col &C = k ? colB : colA;
#pragma unroll
      for (int kz = 0; kz < TZ; kz++) {
        const int h = kz >> 2, e = kz & 3;
        const float pa = (&cur[k][0][h].x)[e], pb = (&cur[k][1][h].x)[e];
        const float pc = (&cur[k][2][h].x)[e];
        if (kz == TZ - 1 && p < plast) load(k, p + 1);
        const int zu = p * TZ + kz;
        const bool ownp = C.own && zu >= zs && zu < ze;
        // positions and weights as dens_field.c:262-275: separate single-
        // precision multiply and add; floor by rounding to an integer with
        // a magic addition (exact for |v| < 2^22); w1 = v - floor(v), one
        // rounding, as the reference's `x - x0`
        const float x = __fadd_rn(__fmul_rn(pa, igs), (float) C.iw);
        const float y = __fadd_rn(__fmul_rn(pb, igs), (float) C.jw);
        const float z = __fadd_rn(__fmul_rn(pc, igs), (float) (zc + kz));
        const float tx = __fadd_rn(x, RMAGIC), ty = __fadd_rn(y, RMAGIC), tz = __fadd_rn(z, RMAGIC);
        const float ex = __fsub_rn(x, __fsub_rn(tx, RMAGIC));
        const float ey = __fsub_rn(y, __fsub_rn(ty, RMAGIC));
        const float ez = __fsub_rn(z, __fsub_rn(tz, RMAGIC));
        const int nx = ex < 0, ny = ey < 0, nz = ez < 0;
        const int dx = __float_as_int(tx) - 0x4B400000 - nx - C.iw;
        const int dy = __float_as_int(ty) - 0x4B400000 - ny - C.jw;
        const int dz = __float_as_int(tz) - 0x4B400000 - nz - (zc + kz);
        const int mad = max(max(abs(dx), abs(dy)), abs(dz));
        nfar2 += (ownp && mad > 2) ? 1u : 0u;
        if (mad > OH) {
          if (ownp) {
            const unsigned int slot = atomicAdd(&stats->nlist, 1u);
            list[slot] = (unsigned int) (((size_t) C.iw * Ng + C.jw) * Ng + (zc + kz));
          }
          continue;
        }
        const int cx = C.cxo + dx, cy = C.cyo + dy;
        const bool ax0 = (unsigned) cx < (unsigned) TX, ax1 = (unsigned) (cx + 1) < (unsigned) TX;
        const bool by0 = (unsigned) cy < (unsigned) TY, by1 = (unsigned) (cy + 1) < (unsigned) TY;
        if (!C.valid || !((ax0 || ax1) && (by0 || by1))) continue;
        const float wx1 = nx ? ex + 1.f : ex, wx0 = 1.f - wx1;
        const float wy1 = ny ? ey + 1.f : ey, wy0 = 1.f - wy1;
        const float wz1 = nz ? ez + 1.f : ez, wz0 = 1.f - wz1;
        // ring slices of s and s + 1: s - (8p - 8) is in 5 .. 19
        int r0 = rbase + (kz + dz + TZ);
        r0 -= (r0 >= TRS) ? TRS : 0;
        int r1 = r0 + 1;
        r1 -= (r1 >= TRS) ? TRS : 0;
        const uint32_t cell = ringb + 4u * (uint32_t) (cx * TY + cy);
        const uint32_t b0 = cell + 4u * (uint32_t) (r0 * TSLOT);
        const uint32_t b1 = cell + 4u * (uint32_t) (r1 * TSLOT);
        const float sm1 = pa * mscale, sm2 = pb * mscale, sm3 = pc * mscale;
        const float zq[2][4] = {{wz0 * RHO_SCALE, wz0 * sm1, wz0 * sm2, wz0 * sm3},
                                {wz1 * RHO_SCALE, wz1 * sm1, wz1 * sm2, wz1 * sm3}};
        const float wxy[4] = {wx0 * wy0, wx0 * wy1, wx1 * wy0, wx1 * wy1};
        const bool ok[4] = {ax0 && by0, ax0 && by1, ax1 && by0, ax1 && by1};
        constexpr uint32_t QB = 4u * TQS;
#pragma unroll
        for (int ab = 0; ab < 4; ab++) {
          if (!ok[ab]) continue;
          const uint32_t off = 4u * (uint32_t) ((ab >> 1) * TY + (ab & 1));
#pragma unroll
          for (int ic = 0; ic < 2; ic++) {
            const uint32_t r = (ic ? b1 : b0) + off;
#pragma unroll
            for (int q = 0; q < 4; q++) red_add(r + q * QB, fmround(wxy[ab], zq[ic][q]));
          }
        }
      }
    }
    // slices 8p-8 .. 8p-1 are final: written if the CTA owns them and
    // cleared.  First the density of each cell's eight slices (one 32-byte
    // sector of rho per thread), then one (slice pair, cell) per thread,
    // cells fastest: the four quantities of two slices go out as two float4
    // of the interleaved grid (q0, q1, q2, rho per cell: one sector) and the
    // ring slots are cleared.
    __syncthreads();
    const int zo = (p - 1) * TZ;
    const bool wr = zo >= zs && zo < ze;
    const float fr = 1.f / RHO_SCALE;
    if (wr) {
      for (int cc = threadIdx.x; cc < TSLOT; cc += TNT) {
        const int *src = tring + rbase * TSLOT + cc;
        int v[TZ];
#pragma unroll
        for (int kk = 0; kk < TZ; kk++) v[kk] = src[kk * TSLOT];
        const int cx = cc / TY, cy = cc - (cc / TY) * TY;
        st8(rho + ((size_t) (i0 + cx) * Ng + (j0 + cy)) * Ng + zo,
            make_float4(v[0] * fr, v[1] * fr, v[2] * fr, v[3] * fr),
            make_float4(v[4] * fr, v[5] * fr, v[6] * fr, v[7] * fr));
      }
      __syncthreads();
    }
    for (int t = threadIdx.x; t < (TZ / 2) * TSLOT; t += TNT) {
      const int sp = t / TSLOT, cc = t - sp * TSLOT;
      int v[4][2];
#pragma unroll
      for (int q = 0; q < 4; q++)
#pragma unroll
        for (int h = 0; h < 2; h++) {
          int *src = tring + q * TQS + (rbase + 2 * sp + h) * TSLOT + cc;
          v[q][h] = *src;
          *src = 0;
        }
      if (wr) {
        const int cx = cc / TY, cy = cc - (cc / TY) * TY;
        const size_t g = ((size_t) (i0 + cx) * Ng + (j0 + cy)) * Ng + zo + 2 * sp;
        st8(reinterpret_cast<float *>(pq + g),
            make_float4(v[1][0] * minv, v[2][0] * minv, v[3][0] * minv, v[0][0] * fr),
            make_float4(v[1][1] * minv, v[2][1] * minv, v[3][1] * minv, v[0][1] * fr));
      }
    }
    __syncthreads();
  }
  // particles displaced beyond two cells, for the next field's halo
#pragma unroll
  for (int o = 16; o; o >>= 1) nfar2 += __shfl_xor_sync(0xffffffffu, nfar2, o);
  if ((threadIdx.x & 31) == 0 && nfar2) atomicAdd(&stats->nfar2, nfar2);
}

// Deposits the listed far-displaced particles with global atomics, into rho
// and the separate painted grids q0..q2, or (IL) into rho and the
// interleaved grid pq = (q0, q1, q2, rho) per cell.
template <bool IL>
__global__ void __launch_bounds__(CIC_NT)
fixup_kernel(const real *__restrict__ p0, const real *__restrict__ p1,
    const real *__restrict__ p2, real *rho, real *q0, real *q1, real *q2, real *pq,
    int Ng, real igs, const CicStats *stats, const unsigned int *list) {
  const unsigned int n = stats->nlist;
  for (unsigned int t = blockIdx.x * blockDim.x + threadIdx.x; t < n;
       t += gridDim.x * blockDim.x) {
    const size_t id = list[t];
    const int k = (int) (id % Ng);
    const size_t ij = id / Ng;
    const int j = (int) (ij % Ng), i = (int) (ij / Ng);
    const real pv[3] = {p0[id], p1[id], p2[id]};
    int x0, x1, y0, y1, z0, z1;
    real wx0, wx1, wy0, wy1, wz0, wz1;
    cic_axis(pv[0], igs, i, Ng, &x0, &x1, &wx0, &wx1);
    cic_axis(pv[1], igs, j, Ng, &y0, &y1, &wy0, &wy1);
    cic_axis(pv[2], igs, k, Ng, &z0, &z1, &wz0, &wz1);
    const int xs[2] = {x0, x1}, ys[2] = {y0, y1}, zs[2] = {z0, z1};
    const real wxs[2] = {wx0, wx1}, wys[2] = {wy0, wy1}, wzs[2] = {wz0, wz1};
#pragma unroll
    for (int a = 0; a < 2; a++)
#pragma unroll
      for (int b = 0; b < 2; b++)
#pragma unroll
        for (int cz = 0; cz < 2; cz++) {
          const size_t g = idx3(Ng, xs[a], ys[b], zs[cz]);
          const real w = wxs[a] * wys[b] * wzs[cz];
          atomicAdd(rho + g, w);
          if (IL) {
            atomicAdd(pq + 4 * g, (wxs[a] * pv[0]) * wys[b] * wzs[cz]);
            atomicAdd(pq + 4 * g + 1, (wxs[a] * pv[1]) * wys[b] * wzs[cz]);
            atomicAdd(pq + 4 * g + 2, (wxs[a] * pv[2]) * wys[b] * wzs[cz]);
            atomicAdd(pq + 4 * g + 3, w);
          } else {
            atomicAdd(q0 + g, (wxs[a] * pv[0]) * wys[b] * wzs[cz]);
            atomicAdd(q1 + g, (wxs[a] * pv[1]) * wys[b] * wzs[cz]);
            atomicAdd(q2 + g, (wxs[a] * pv[2]) * wys[b] * wzs[cz]);
          }
        }
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
  m->paint_il = false;                       // set by the 16 x 32 tile assignment
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
#ifdef SINGLE_PREC
    if (Ng % OT == 0 && Ng >= 2 * OT) {
      const size_t smem = 4 * OQS * sizeof(int);
      // the shared-memory limit is a property of the function in each
      // device's context: set it on every call (the instance's device is
      // current)
      if (!EZ_CUDA_OK(cudaFuncSetAttribute(cic_owner_kernel<2>,
              cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem)) ||
          !EZ_CUDA_OK(cudaFuncSetAttribute(cic_owner_kernel<3>,
              cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem)))
        return EZMOCK_ERR_UNKNOWN;
      CicStats *stats = (CicStats *) m->stats;
      unsigned int *list = m->draws;                  // free after the spectrum
      if (!m->psimax_valid) {
        cudaMemsetAsync(&stats->psimax_bits, 0, sizeof(unsigned int), m->stream);
        psi_absmax_kernel<<<148 * 8, 256, 0, m->stream>>>(m->psi[0], 3 * N, stats); ez_count_launch();
      }
      // the halo: set by the caller, else from the previous field's count if
      // it has arrived
      if (m->cic_oh_set) m->cic_oh_set = false;
      else if (m->h_cic && cudaEventQuery(m->ev_cic) == cudaSuccess)
        m->cic_oh = ((size_t) m->h_cic[0] * 4096 < N) ? 2 : 3;
      cudaMemsetAsync(&stats->nlist, 0, 2 * sizeof(int), m->stream);
      if (Ng % TY == 0 && Ng >= 2 * TY && !m->cic_legacy) {
        // 16 x 32 tiles; the z range is cut so that the CTAs (one per SM)
        // fill whole waves: pick the cut count with the least time per
        // wave-slot, counting each range's two extra steps
        if (!EZ_CUDA_OK(cudaFuncSetAttribute(cic_tile_kernel<2>,
                cudaFuncAttributeMaxDynamicSharedMemorySize, (int) TSMEM)) ||
            !EZ_CUDA_OK(cudaFuncSetAttribute(cic_tile_kernel<3>,
                cudaFuncAttributeMaxDynamicSharedMemorySize, (int) TSMEM)))
          return EZMOCK_ERR_UNKNOWN;
        int nsm = 148;
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, m->device);
        const long tiles = (long) (Ng / TX) * (Ng / TY);
        int nzs = 1;
        double best = 1e300;
        for (int s = 1; s <= 64 && Ng % s == 0 && (Ng / s) % TZ == 0 && Ng / s >= 2 * TZ;
             s *= 2) {
          const long waves = (tiles * s + nsm - 1) / nsm;
          const double cost = (double) waves * (Ng / s / TZ + 2);
          if (cost < best * 0.999) { best = cost; nzs = s; }
        }
        const unsigned nblk = (unsigned) (tiles * nzs);
        float4 *pq = reinterpret_cast<float4 *>(m->pq);
        if (m->cic_oh != 2)
          cic_tile_kernel<3><<<nblk, TNT, TSMEM, m->stream>>>(m->psi[0], m->psi[1],
              m->psi[2], m->rho, pq, Ng, igs, stats, list, nzs);
        else
          cic_tile_kernel<2><<<nblk, TNT, TSMEM, m->stream>>>(m->psi[0], m->psi[1],
              m->psi[2], m->rho, pq, Ng, igs, stats, list, nzs);
        m->paint_il = true;
      }
      else {
        const unsigned nblk = (unsigned) ((Ng / OT) * (Ng / OT));
        m->paint_il = false;
        if (m->cic_oh != 2)
          cic_owner_kernel<3><<<nblk, OWN_NT, smem, m->stream>>>(m->psi[0], m->psi[1],
              m->psi[2], m->rho, m->paint[0], m->paint[1], m->paint[2], Ng, igs, stats, list);
        else
          cic_owner_kernel<2><<<nblk, OWN_NT, smem, m->stream>>>(m->psi[0], m->psi[1],
              m->psi[2], m->rho, m->paint[0], m->paint[1], m->paint[2], Ng, igs, stats, list);
      }
      ez_count_launch();
      if (m->paint_il)
        fixup_kernel<true><<<148 * 4, CIC_NT, 0, m->stream>>>(m->psi[0], m->psi[1],
            m->psi[2], m->rho, m->paint[0], m->paint[1], m->paint[2], m->pq, Ng, igs,
            stats, list);
      else
        fixup_kernel<false><<<148 * 4, CIC_NT, 0, m->stream>>>(m->psi[0], m->psi[1],
            m->psi[2], m->rho, m->paint[0], m->paint[1], m->paint[2], m->pq, Ng, igs,
            stats, list);
      ez_count_launch();
      // this field's count of particles beyond 2 cells, for the next field's
      // halo (2 only while almost none move farther; those take the
      // global-atomic fixup); read into pinned memory without waiting
      if (!m->h_cic) {
        if (!EZ_CUDA_OK(cudaMallocHost(&m->h_cic, sizeof(unsigned int))) ||
            !EZ_CUDA_OK(cudaEventCreateWithFlags(&m->ev_cic, cudaEventDisableTiming))) {
          m->h_cic = nullptr;
          return EZMOCK_ERR_MEMORY;
        }
      }
      if (!EZ_CUDA_OK(cudaMemcpyAsync(m->h_cic, &stats->nfar2, sizeof(unsigned int),
              cudaMemcpyDeviceToHost, m->stream)) ||
          !EZ_CUDA_OK(cudaEventRecord(m->ev_cic, m->stream)))
        return EZMOCK_ERR_UNKNOWN;
    }
    else
#endif
    {
      if (!EZ_CUDA_OK(cudaMemsetAsync(m->rho, 0, N * sizeof(real), m->stream))) return EZMOCK_ERR_UNKNOWN;
      for (int d = 0; d < 3; d++)
        if (!EZ_CUDA_OK(cudaMemsetAsync(m->paint[d], 0, N * sizeof(real), m->stream)))
          return EZMOCK_ERR_UNKNOWN;
      cic_atomic_kernel<true><<<grid, CIC_NT, 0, m->stream>>>(m->psi[0], m->psi[1],
          m->psi[2], m->rho, m->paint[0], m->paint[1], m->paint[2], Ng, igs, N); ez_count_launch();
    }
  }
  ez_stage_end(m, ST_CIC);
  return EZ_CUDA_OK(cudaGetLastError()) ? 0 : EZMOCK_ERR_UNKNOWN;
}
