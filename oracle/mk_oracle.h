/*
 * mk_oracle.h -- storage shared by the oracle's translation units.
 *
 * TEST INFRASTRUCTURE ONLY (see mk_oracle.c): the checker, the host
 * generators it uses to draw the benchmark's inputs without the product
 * library (mk_gen.c), and the multithreaded CPU baseline (mk_cpu.c).
 */
#ifndef MK_ORACLE_H_
#define MK_ORACLE_H_

#include <stdint.h>

#define OK_EMPTY (~0ull)
#define OK_INF 0xFFFFFFFFu

static inline uint64_t mixk(uint64_t x) {
  x ^= x >> 33;
  x *= 0xff51afd7ed558ccdull;
  x ^= x >> 33;
  x *= 0xc4ceb9fe1a85ec53ull;
  x ^= x >> 33;
  return x;
}

typedef struct {
  uint64_t *keys;
  uint32_t *wt;
  uint32_t *pos;
  uint64_t cap, size;
} omap;

/* Out-neighbours of one vertex with their weights (same order). */
typedef struct {
  uint32_t *a; /* neighbours */
  uint32_t *w; /* weights    */
  uint32_t n, cap;
} ivec;

typedef struct og {
  uint32_t V;
  int T;
  omap *shard;
  ivec *adj;
} og;

int og_has_edge(const og *g, uint32_t u, uint32_t v, uint32_t *w);

#endif /* MK_ORACLE_H_ */
