// ez_gf2.h -- host arithmetic in GF(2)[x] modulo a fixed polynomial phi.
#pragma once

#include <cstdint>

// Sets phi (w words, bit i = coefficient of x^i, degree n) and precomputes
// the Barrett constant.  Not thread-safe; call once under the caller's lock.
bool ez_gf2_init(const uint64_t *phi, int n, int w);

// out = a * b mod phi; a, b reduced (degree < n), all w words.
void ez_gf2_mulmod(const uint64_t *a, const uint64_t *b, uint64_t *out);
