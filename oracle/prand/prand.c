/*
 * prand.c -- CPU restatement of the random-number generators behind the
 * EZmock `prand` API (oracle only; see prand.h for the definitions chosen).
 *
 * MT19937 (Matsumoto & Nishimura 1998) is kept as a 624-word window
 * w[(pos+k) % 624] = x_{m+k}; one step computes x_{m+624} in place.  This is
 * the same sequence as the block-twist formulation of the published
 * reference generator.  Skip-ahead follows Haramoto et al. (2008): the
 * characteristic polynomial phi of the output recurrence is recovered with
 * Berlekamp-Massey, the table X[k] = x^(2^k) mod phi is built by repeated
 * squaring over GF(2), and a jump by J applies p(T) = sum c_i T^i with
 * Horner's rule for each set bit of J.
 *
 * MRG32k3a (L'Ecuyer 1999) uses the standard component recurrences and
 * skip-ahead by powers of the 3x3 transition matrices modulo m1 and m2.
 */
#include "prand.h"
#include <stdlib.h>
#include <string.h>
#include <pthread.h>

/*============================================================================*\
                                   MT19937
\*============================================================================*/

#define MT_N 624
#define MT_M 397
#define MT_MATRIX_A 0x9908b0dfU
#define MT_UPPER 0x80000000U
#define MT_LOWER 0x7fffffffU
#define MT_DEG 19937
#define MT_PW 312            /* 64-bit words holding a poly of degree <= 19937 */
#define MT_SEQ_SKIP_BITS 22  /* jumps below 2^22 are done by plain stepping */

typedef struct {
  uint32_t w[MT_N];
  int pos;
} mt_state;

static void mt_init_genrand(uint32_t *mt, uint32_t s) {
  mt[0] = s;
  for (int i = 1; i < MT_N; i++)
    mt[i] = 1812433253U * (mt[i - 1] ^ (mt[i - 1] >> 30)) + (uint32_t) i;
}

static void mt_init_by_array(uint32_t *mt, const uint32_t *key, int len) {
  mt_init_genrand(mt, 19650218U);
  int i = 1, j = 0;
  for (int k = (MT_N > len ? MT_N : len); k; k--) {
    mt[i] = (mt[i] ^ ((mt[i - 1] ^ (mt[i - 1] >> 30)) * 1664525U)) + key[j]
        + (uint32_t) j;
    i++; j++;
    if (i >= MT_N) { mt[0] = mt[MT_N - 1]; i = 1; }
    if (j >= len) j = 0;
  }
  for (int k = MT_N - 1; k; k--) {
    mt[i] = (mt[i] ^ ((mt[i - 1] ^ (mt[i - 1] >> 30)) * 1566083941U))
        - (uint32_t) i;
    i++;
    if (i >= MT_N) { mt[0] = mt[MT_N - 1]; i = 1; }
  }
  mt[0] = 0x80000000U;
}

static void mt_seed(mt_state *s, uint64_t seed) {
  if (seed <= 0xffffffffULL) mt_init_genrand(s->w, (uint32_t) seed);
  else {
    uint32_t key[2] = {(uint32_t) seed, (uint32_t) (seed >> 32)};
    mt_init_by_array(s->w, key, 2);
  }
  s->pos = 0;
}

/* One step of the linear recurrence: x_{m+624} replaces x_m. */
static inline uint32_t mt_step(mt_state *s) {
  const int p = s->pos;
  const int p1 = (p + 1 == MT_N) ? 0 : p + 1;
  const int pm = (p + MT_M >= MT_N) ? p + MT_M - MT_N : p + MT_M;
  const uint32_t y = (s->w[p] & MT_UPPER) | (s->w[p1] & MT_LOWER);
  const uint32_t x = s->w[pm] ^ (y >> 1) ^ ((y & 1U) ? MT_MATRIX_A : 0U);
  s->w[p] = x;
  s->pos = p1;
  return x;
}

static inline uint32_t mt_temper(uint32_t y) {
  y ^= y >> 11;
  y ^= (y << 7) & 0x9d2c5680U;
  y ^= (y << 15) & 0xefc60000U;
  y ^= y >> 18;
  return y;
}

/* ---- GF(2) polynomial helpers for the skip-ahead ---- */

static uint64_t mt_phi[MT_PW + 1];            /* characteristic polynomial */
static uint64_t mt_phi_sh[64][MT_PW + 2];     /* phi << s, s = 0..63       */
static uint64_t mt_xpow[64][MT_PW];           /* x^(2^k) mod phi           */
static int mt_tables_ok = 0;
static pthread_once_t mt_once = PTHREAD_ONCE_INIT;

static inline int bit_get(const uint64_t *a, long b) {
  return (int) ((a[b >> 6] >> (b & 63)) & 1ULL);
}

/* Berlekamp-Massey on one bit stream of the raw words; returns the degree. */
static int mt_find_phi(void) {
  const long len = 2L * MT_DEG + 128;
  const long nw = (len + 63) / 64 + 2;
  uint64_t *rev = calloc(nw, sizeof(uint64_t));
  uint64_t *C = calloc(nw, sizeof(uint64_t));
  uint64_t *B = calloc(nw, sizeof(uint64_t));
  uint64_t *T = calloc(nw, sizeof(uint64_t));
  if (!rev || !C || !B || !T) { free(rev); free(C); free(B); free(T); return -1; }

  mt_state s;
  mt_seed(&s, 5489U);
  for (long n = 0; n < len; n++) {
    const uint32_t x = mt_step(&s);
    const long t = len - 1 - n;           /* reversed position */
    if (x >> 31) rev[t >> 6] |= 1ULL << (t & 63);
  }

  C[0] = B[0] = 1;
  long L = 0, m = 1;
  for (long n = 0; n < len; n++) {
    /* d = sum_{i=0}^{L} C_i s[n-i], with s[n-i] = rev[len-1-n+i] */
    const long o = len - 1 - n;
    const long lw = L / 64 + 1;
    uint64_t acc = 0;
    for (long w = 0; w < lw; w++) {
      const long b = o + 64 * w;
      const long bw = b >> 6, bs = b & 63;
      uint64_t v = rev[bw] >> bs;
      if (bs && bw + 1 < nw) v |= rev[bw + 1] << (64 - bs);
      acc ^= C[w] & v;          /* deg C <= L, so higher bits of C are 0 */
    }
    const int d = __builtin_parityll(acc);
    if (!d) { m++; continue; }
    if (2 * L <= n) {
      memcpy(T, C, nw * sizeof(uint64_t));
      /* C += x^m B */
      const long ws = m >> 6, bs = m & 63;
      for (long w = nw - 1; w >= 0; w--) {
        uint64_t v = 0;
        if (w - ws >= 0) v = B[w - ws] << bs;
        if (bs && w - ws - 1 >= 0) v |= B[w - ws - 1] >> (64 - bs);
        C[w] ^= v;
      }
      L = n + 1 - L;
      memcpy(B, T, nw * sizeof(uint64_t));
      m = 1;
    }
    else {
      const long ws = m >> 6, bs = m & 63;
      for (long w = nw - 1; w >= 0; w--) {
        uint64_t v = 0;
        if (w - ws >= 0) v = B[w - ws] << bs;
        if (bs && w - ws - 1 >= 0) v |= B[w - ws - 1] >> (64 - bs);
        C[w] ^= v;
      }
      m++;
    }
  }

  /* phi(x) = x^L C(1/x): coefficient of x^j is C_{L-j}. */
  memset(mt_phi, 0, sizeof(mt_phi));
  if (L == MT_DEG) {
    for (long j = 0; j <= L; j++)
      if (bit_get(C, L - j)) mt_phi[j >> 6] |= 1ULL << (j & 63);
  }
  free(rev); free(C); free(B); free(T);
  return (int) L;
}

/* r (2*MT_PW words, degree < 2*MT_DEG) reduced modulo phi, in place. */
static void mt_poly_reduce(uint64_t *r) {
  for (long b = 2L * MT_DEG; b >= MT_DEG; b--) {
    if (!bit_get(r, b)) continue;
    const long t = b - MT_DEG;
    const long ws = t >> 6;
    const uint64_t *ph = mt_phi_sh[t & 63];
    for (long w = 0; w < MT_PW + 2 && ws + w < 2 * MT_PW + 2; w++)
      r[ws + w] ^= ph[w];
  }
}

static inline uint64_t spread32(uint32_t v) {
  uint64_t x = v;
  x = (x | (x << 16)) & 0x0000ffff0000ffffULL;
  x = (x | (x << 8)) & 0x00ff00ff00ff00ffULL;
  x = (x | (x << 4)) & 0x0f0f0f0f0f0f0f0fULL;
  x = (x | (x << 2)) & 0x3333333333333333ULL;
  x = (x | (x << 1)) & 0x5555555555555555ULL;
  return x;
}

static void mt_build_tables(void) {
  if (mt_find_phi() != MT_DEG) return;
  for (int s = 0; s < 64; s++) {
    memset(mt_phi_sh[s], 0, sizeof(mt_phi_sh[s]));
    for (int w = 0; w <= MT_PW; w++) {
      mt_phi_sh[s][w] ^= mt_phi[w] << s;
      if (s) mt_phi_sh[s][w + 1] ^= mt_phi[w] >> (64 - s);
    }
  }
  uint64_t r[2 * MT_PW + 4];
  memset(mt_xpow[0], 0, sizeof(mt_xpow[0]));
  mt_xpow[0][0] = 2;                              /* x */
  for (int k = 1; k < 64; k++) {
    memset(r, 0, sizeof(r));
    for (int w = 0; w < MT_PW; w++) {
      r[2 * w] = spread32((uint32_t) mt_xpow[k - 1][w]);
      r[2 * w + 1] = spread32((uint32_t) (mt_xpow[k - 1][w] >> 32));
    }
    mt_poly_reduce(r);
    memcpy(mt_xpow[k], r, sizeof(mt_xpow[k]));
  }
  mt_tables_ok = 1;
}

/* s <- p(T) s by Horner's rule (p of degree < MT_DEG). */
static void mt_horner(mt_state *s, const uint64_t *p) {
  uint32_t wl[MT_N];
  for (int k = 0; k < MT_N; k++) wl[k] = s->w[(s->pos + k) % MT_N];
  mt_state r;
  memset(&r, 0, sizeof(r));
  long deg = MT_DEG - 1;
  while (deg >= 0 && !bit_get(p, deg)) deg--;
  for (long i = deg; i >= 0; i--) {
    mt_step(&r);
    if (bit_get(p, i)) {
      const int head = MT_N - r.pos;
      for (int k = 0; k < head; k++) r.w[r.pos + k] ^= wl[k];
      for (int k = head; k < MT_N; k++) r.w[k - head] ^= wl[k];
    }
  }
  *s = r;
}

static void mt_jump(mt_state *s, uint64_t J, int *err) {
  const uint64_t small = J & ((1ULL << MT_SEQ_SKIP_BITS) - 1);
  for (uint64_t i = 0; i < small; i++) mt_step(s);
  J >>= MT_SEQ_SKIP_BITS;
  if (!J) return;
  pthread_once(&mt_once, mt_build_tables);
  if (!mt_tables_ok) { if (err) *err = PRAND_ERR_RNG; return; }
  for (int k = MT_SEQ_SKIP_BITS; J; k++, J >>= 1)
    if (J & 1ULL) mt_horner(s, mt_xpow[k]);
}

static void mt_reset(void *state, const uint64_t seed, const uint64_t skip,
    int *err) {
  mt_state *s = (mt_state *) state;
  mt_seed(s, seed);
  mt_jump(s, skip, err);
}

static double mt_get_double(void *state) {
  return (double) mt_temper(mt_step((mt_state *) state)) *
      (1.0 / 4294967296.0);
}

static double mt_get_double_pos(void *state) {
  return ((double) mt_temper(mt_step((mt_state *) state)) + 0.5) *
      (1.0 / 4294967296.0);
}

/*============================================================================*\
                                  MRG32k3a
\*============================================================================*/

#define MRG_M1 4294967087ULL
#define MRG_M2 4294944443ULL
#define MRG_A12 1403580ULL
#define MRG_A13N 810728ULL
#define MRG_A21 527612ULL
#define MRG_A23N 1370589ULL
#define MRG_NORM 2.328306549295727688e-10

typedef struct {
  uint64_t s1[3], s2[3];   /* (x_{n-3}, x_{n-2}, x_{n-1}) of each component */
} mrg_state;

static uint64_t mrg_pow1[64][9], mrg_pow2[64][9];   /* A^(2^k) mod m */
static pthread_once_t mrg_once = PTHREAD_ONCE_INIT;

static void mat_mul_mod(const uint64_t *a, const uint64_t *b, uint64_t *c,
    uint64_t m) {
  uint64_t t[9];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      unsigned __int128 acc = 0;
      for (int k = 0; k < 3; k++)
        acc += (unsigned __int128) a[3 * i + k] * b[3 * k + j];
      t[3 * i + j] = (uint64_t) (acc % m);
    }
  memcpy(c, t, sizeof(t));
}

static void mrg_build_tables(void) {
  const uint64_t a1[9] = {0, 1, 0, 0, 0, 1, MRG_M1 - MRG_A13N, MRG_A12, 0};
  const uint64_t a2[9] = {0, 1, 0, 0, 0, 1, MRG_M2 - MRG_A23N, 0, MRG_A21};
  memcpy(mrg_pow1[0], a1, sizeof(a1));
  memcpy(mrg_pow2[0], a2, sizeof(a2));
  for (int k = 1; k < 64; k++) {
    mat_mul_mod(mrg_pow1[k - 1], mrg_pow1[k - 1], mrg_pow1[k], MRG_M1);
    mat_mul_mod(mrg_pow2[k - 1], mrg_pow2[k - 1], mrg_pow2[k], MRG_M2);
  }
}

static void mat_vec_mod(const uint64_t *a, uint64_t *v, uint64_t m) {
  uint64_t t[3];
  for (int i = 0; i < 3; i++) {
    unsigned __int128 acc = 0;
    for (int k = 0; k < 3; k++) acc += (unsigned __int128) a[3 * i + k] * v[k];
    t[i] = (uint64_t) (acc % m);
  }
  memcpy(v, t, sizeof(t));
}

static uint64_t splitmix64(uint64_t *z) {
  uint64_t r = (*z += 0x9e3779b97f4a7c15ULL);
  r = (r ^ (r >> 30)) * 0xbf58476d1ce4e5b9ULL;
  r = (r ^ (r >> 27)) * 0x94d049bb133111ebULL;
  return r ^ (r >> 31);
}

static void mrg_seed(mrg_state *s, uint64_t seed) {
  uint64_t z = seed;
  for (int j = 0; j < 3; j++) s->s1[j] = splitmix64(&z) % MRG_M1;
  for (int j = 0; j < 3; j++) s->s2[j] = splitmix64(&z) % MRG_M2;
  if (!s->s1[0] && !s->s1[1] && !s->s1[2]) s->s1[0] = 1;
  if (!s->s2[0] && !s->s2[1] && !s->s2[2]) s->s2[0] = 1;
}

static inline uint32_t mrg_step(mrg_state *s) {
  const uint64_t p1 = (MRG_A12 * s->s1[1] % MRG_M1 +
      (MRG_M1 - MRG_A13N) * s->s1[0] % MRG_M1) % MRG_M1;
  const uint64_t p2 = (MRG_A21 * s->s2[2] % MRG_M2 +
      (MRG_M2 - MRG_A23N) * s->s2[0] % MRG_M2) % MRG_M2;
  s->s1[0] = s->s1[1]; s->s1[1] = s->s1[2]; s->s1[2] = p1;
  s->s2[0] = s->s2[1]; s->s2[1] = s->s2[2]; s->s2[2] = p2;
  return (uint32_t) ((p1 > p2) ? p1 - p2 : p1 + MRG_M1 - p2);
}

static void mrg_reset(void *state, const uint64_t seed, const uint64_t skip,
    int *err) {
  (void) err;
  mrg_state *s = (mrg_state *) state;
  mrg_seed(s, seed);
  pthread_once(&mrg_once, mrg_build_tables);
  uint64_t J = skip;
  for (int k = 0; J; k++, J >>= 1) {
    if (J & 1ULL) {
      mat_vec_mod(mrg_pow1[k], s->s1, MRG_M1);
      mat_vec_mod(mrg_pow2[k], s->s2, MRG_M2);
    }
  }
}

static double mrg_get_double(void *state) {
  return (double) mrg_step((mrg_state *) state) * MRG_NORM;
}

/*============================================================================*\
                                 Public API
\*============================================================================*/

prand_t *prand_init(const prand_rng_enum type, const uint64_t seed,
    const int nstream, const uint64_t step, int *err) {
  if (!err) return NULL;
  if (type != PRAND_RNG_MRG32K3A && type != PRAND_RNG_MT19937) {
    *err = PRAND_ERR_RNG; return NULL;
  }
  if (nstream <= 0) { *err = PRAND_ERR_NSTREAM; return NULL; }
  prand_t *r = calloc(1, sizeof(prand_t));
  if (!r) { *err = PRAND_ERR_MEMORY; return NULL; }
  r->type = type;
  r->nstream = nstream;
  const size_t ssize = (type == PRAND_RNG_MT19937) ? sizeof(mt_state)
      : sizeof(mrg_state);
  r->state = calloc(1, ssize);
  r->state_stream = calloc(nstream, sizeof(void *));
  if (!r->state || !r->state_stream) {
    prand_destroy(r); *err = PRAND_ERR_MEMORY; return NULL;
  }
  if (type == PRAND_RNG_MT19937) {
    r->reset = mt_reset;
    r->get_double = mt_get_double;
    r->get_double_pos = mt_get_double_pos;
  }
  else {
    r->reset = mrg_reset;
    r->get_double = mrg_get_double;
    r->get_double_pos = mrg_get_double;
  }
  r->reset(r->state, seed, 0, err);
  for (int i = 0; i < nstream; i++) {
    if (!(r->state_stream[i] = calloc(1, ssize))) {
      prand_destroy(r); *err = PRAND_ERR_MEMORY; return NULL;
    }
    r->reset(r->state_stream[i], seed, step * (uint64_t) i, err);
  }
  return r;
}

void prand_destroy(prand_t *rng) {
  if (!rng) return;
  if (rng->state_stream) {
    for (int i = 0; i < rng->nstream; i++) free(rng->state_stream[i]);
    free(rng->state_stream);
  }
  free(rng->state);
  free(rng);
}

uint32_t prand_raw_next(prand_t *rng, void *state) {
  if (rng->type == PRAND_RNG_MT19937)
    return mt_temper(mt_step((mt_state *) state));
  return mrg_step((mrg_state *) state);
}

void prand_fill_raw(const int type, const uint64_t seed, const uint64_t start,
    const uint64_t count, uint32_t *out) {
  int err = 0;
  if (type == PRAND_RNG_MT19937) {
    mt_state s;
    mt_reset(&s, seed, start, &err);
    for (uint64_t i = 0; i < count; i++) out[i] = mt_temper(mt_step(&s));
  }
  else {
    mrg_state s;
    mrg_reset(&s, seed, start, &err);
    for (uint64_t i = 0; i < count; i++) out[i] = mrg_step(&s);
  }
}
