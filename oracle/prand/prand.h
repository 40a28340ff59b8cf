/*
 * prand.h -- CPU restatement of the random-number API that the EZmock
 * library calls (test infrastructure: oracle only, never shipped).
 *
 * The reference declares `libEZmock/prand` as a git submodule
 * (`.gitmodules:1-3`) but the directory is empty, so the generator sources
 * are not available.  This header restates the interface exactly as the
 * reference's call sites use it:
 *   - prand_init(type, seed, nstream, step, &err)   libEZmock/EZmock/EZmock.c:85
 *   - PRAND_IS_ERROR / PRAND_IS_WARN                 libEZmock/EZmock/EZmock.c:86
 *   - prand_t::{state, state_stream[], reset,
 *              get_double, get_double_pos}          libEZmock/EZmock/perturb.c:112-164
 *   - prand_destroy                                  libEZmock/EZmock/structs.c:30
 *   - PRAND_RNG_MRG32K3A = 0, PRAND_RNG_MT19937 = 1  libEZmock/EZmock/save_res.c:138
 *
 * Generator definitions (published algorithms, restated here):
 *   MT19937  : Matsumoto & Nishimura (1998).  Seeded with init_genrand(seed)
 *              when seed < 2^32, otherwise init_by_array({lo32, hi32}).
 *              One 32-bit output per draw:
 *                get_double     = x * 2^-32          in [0,1)
 *                get_double_pos = (x + 0.5) * 2^-32  in (0,1)
 *              Skip-ahead by the characteristic polynomial (Haramoto et al.
 *              2008): x^J mod phi(x), applied with Horner's rule.
 *   MRG32k3a : L'Ecuyer (1999).  One step per draw, output d in [1, m1],
 *              get_double = get_double_pos = d * 2.328306549295727688e-10.
 *              Seeded from splitmix64(seed); skip-ahead by 3x3 matrix powers.
 *
 * Bit-exactness against the upstream `cheng-zhao/prand` cannot be checked
 * (its source is absent): parity of the random streams with the reference's
 * generator is unpinned.  What the reference does pin -- and what this
 * restatement honours -- is the stream-offset contract: `reset(state, seed,
 * s)` positions a stream at absolute draw index s of the stream seeded by
 * `seed`.
 */
#ifndef EZ_ORACLE_PRAND_H
#define EZ_ORACLE_PRAND_H

#include <stdint.h>
/* The reference's save_res.c uses FILE/fopen without including <stdio.h>
   itself; it receives it through this header (libEZmock/EZmock/structs.h:34). */
#include <stdio.h>

typedef enum {
  PRAND_RNG_MRG32K3A = 0,
  PRAND_RNG_MT19937 = 1
} prand_rng_enum;

#define PRAND_ERR_NONE   0
#define PRAND_ERR_MEMORY 1
#define PRAND_ERR_RNG    2
#define PRAND_ERR_SEED   3
#define PRAND_ERR_NSTREAM 4

#define PRAND_IS_ERROR(e)  ((e) > 0)
#define PRAND_IS_WARN(e)   ((e) < 0)

typedef struct prand_struct {
  prand_rng_enum type;
  int nstream;
  void *state;            /* the serial stream                                */
  void **state_stream;    /* one stream per thread                            */
  void (*reset)(void *state, const uint64_t seed, const uint64_t skip,
      int *err);
  double (*get_double)(void *state);      /* [0,1)                            */
  double (*get_double_pos)(void *state);  /* (0,1)                            */
} prand_t;

prand_t *prand_init(const prand_rng_enum type, const uint64_t seed,
    const int nstream, const uint64_t step, int *err);
void prand_destroy(prand_t *rng);

/* Extra entry points used by the tests (not part of the reference API). */
uint32_t prand_raw_next(prand_t *rng, void *state);   /* raw 32-bit draw */
void prand_fill_raw(const int type, const uint64_t seed, const uint64_t start,
    const uint64_t count, uint32_t *out);

#endif
