// ez_gf2.cpp -- host arithmetic in GF(2)[x] modulo the MT19937 characteristic
// polynomial phi (degree 19937), for the jump polynomials x^J mod phi.
//
// Products use carry-less multiplication (PCLMULQDQ when the CPU has it, a
// portable shift-and-xor loop otherwise) and are reduced with Barrett's
// method, which is exact over GF(2): with mu = floor(x^(2n) / phi) and
// deg(a) < 2n, floor(a / phi) = floor(floor(a / x^n) * mu / x^n).
#include "ez_gf2.h"

#include <cstring>
#include <vector>

#include <emmintrin.h>
#include <wmmintrin.h>

namespace {

int g_n = 0;                    // degree of phi
int g_w = 0;                    // words of a reduced polynomial
std::vector<uint64_t> g_phi;    // g_w words
std::vector<uint64_t> g_mu;     // g_w words (degree n)
bool g_hw = false;

__attribute__((target("pclmul,sse2")))
void mul_hw(const uint64_t *a, const uint64_t *b, int n, uint64_t *c) {
  std::memset(c, 0, sizeof(uint64_t) * 2 * n);
  for (int i = 0; i < n; i++) {
    if (!a[i]) continue;
    const __m128i ai = _mm_cvtsi64_si128((long long) a[i]);
    uint64_t carry = 0;
    for (int j = 0; j < n; j++) {
      const __m128i p = _mm_clmulepi64_si128(ai, _mm_cvtsi64_si128((long long) b[j]), 0x00);
      c[i + j] ^= (uint64_t) _mm_cvtsi128_si64(p) ^ carry;
      carry = (uint64_t) _mm_cvtsi128_si64(_mm_unpackhi_epi64(p, p));
    }
    c[i + n] ^= carry;
  }
}

void clmul_sw(uint64_t a, uint64_t b, uint64_t *lo, uint64_t *hi) {
  uint64_t l = 0, h = 0;
  for (int k = 0; k < 64; k++)
    if ((b >> k) & 1) {
      l ^= a << k;
      if (k) h ^= a >> (64 - k);
    }
  *lo = l;
  *hi = h;
}

void mul_sw(const uint64_t *a, const uint64_t *b, int n, uint64_t *c) {
  std::memset(c, 0, sizeof(uint64_t) * 2 * n);
  for (int i = 0; i < n; i++) {
    if (!a[i]) continue;
    uint64_t carry = 0;
    for (int j = 0; j < n; j++) {
      uint64_t lo, hi;
      clmul_sw(a[i], b[j], &lo, &hi);
      c[i + j] ^= lo ^ carry;
      carry = hi;
    }
    c[i + n] ^= carry;
  }
}

void mul(const uint64_t *a, const uint64_t *b, int n, uint64_t *c) {
  if (g_hw) mul_hw(a, b, n, c);
  else mul_sw(a, b, n, c);
}

// dst (w words) = src >> sh (bits), src having `sw` words
void shr(const uint64_t *src, int sw, int sh, uint64_t *dst, int w) {
  const int ws = sh >> 6, bs = sh & 63;
  for (int i = 0; i < w; i++) {
    const int s = i + ws;
    uint64_t v = (s < sw) ? src[s] >> bs : 0;
    if (bs && s + 1 < sw) v |= src[s + 1] << (64 - bs);
    dst[i] = v;
  }
}

inline int bit(const uint64_t *a, long b) { return (int) ((a[b >> 6] >> (b & 63)) & 1ULL); }

}  // namespace

bool ez_gf2_init(const uint64_t *phi, int n, int w) {
  g_hw = __builtin_cpu_supports("pclmul") && __builtin_cpu_supports("sse2");
  g_n = n;
  g_w = w;
  if (n <= 0 || (n + 1 + 63) / 64 > w) return false;
  g_phi.assign(phi, phi + w);
  // mu = floor(x^(2n) / phi) by long division: r runs over 2n + 1 bits
  const int rw = (2 * n + 1 + 63) / 64 + 1;
  std::vector<uint64_t> r(rw, 0), mu(w, 0);
  r[(2 * n) >> 6] |= 1ULL << ((2 * n) & 63);
  for (long b = 2L * n; b >= n; b--) {
    if (!bit(r.data(), b)) continue;
    const long t = b - n;                   // quotient bit
    mu[t >> 6] |= 1ULL << (t & 63);
    const long ws = t >> 6, bs = t & 63;
    for (int i = 0; i < w; i++) {
      const uint64_t v = g_phi[i];
      if (!v) continue;
      r[ws + i] ^= v << bs;
      if (bs && ws + i + 1 < rw) r[ws + i + 1] ^= v >> (64 - bs);
    }
  }
  g_mu = mu;
  return true;
}

void ez_gf2_mulmod(const uint64_t *a, const uint64_t *b, uint64_t *out) {
  const int w = g_w, n = g_n;
  std::vector<uint64_t> c(2 * w), q(w), q2(2 * w), t(2 * w);
  mul(a, b, w, c.data());                   // deg < 2n
  shr(c.data(), 2 * w, n, q.data(), w);     // floor(c / x^n), deg < n
  mul(q.data(), g_mu.data(), w, q2.data()); // deg < 2n
  shr(q2.data(), 2 * w, n, q.data(), w);    // quotient, deg < n
  mul(q.data(), g_phi.data(), w, t.data());
  for (int i = 0; i < w; i++) out[i] = c[i] ^ t[i];
  // the remainder has degree < n: clear the bits above (they cancel)
  const int top = n >> 6;
  if (top < w) {
    out[top] &= (n & 63) ? ((1ULL << (n & 63)) - 1) : 0;
    for (int i = top + 1; i < w; i++) out[i] = 0;
  }
}
