/*
 * mk_gen.c -- the benchmark's synthetic inputs, drawn on the host without the
 * product library.
 *
 * TEST INFRASTRUCTURE ONLY.  bench.py's reference arm (the CPU baseline)
 * draws its R-MAT graph and update batches here so that arm loads nothing
 * but the oracle.  The streams restate the product generators' definitions
 * (meerkat_b200/csrc/gen.cpp), and tests/test_oracle_gen.py checks that both
 * give the same edges and batches:
 *
 *   R-MAT   candidate i draws `scale` quadrant choices from the counter-based
 *           stream splitmix(key ^ splitmix(32 i + l/2)) (two 32-bit draws per
 *           64-bit word), key = splitmix(seed ^ "RMAT"); self loops are
 *           dropped and the graph keeps the first `num_edges` distinct
 *           candidates in candidate order.  Weight i = w_lo + draw(i) % range
 *           from the key splitmix(seed ^ "WGHT").
 *   absent  inserts draw (u, v) = (x mod V, (x >> 32) mod V) from stream
 *           splitmix(seed ^ "ABST"), skipping self loops and edges present in
 *           the set, and add each drawn edge to the set.
 *   present deletes take index draw(i) mod |set| of the set's dense edge
 *           list (stream splitmix(seed ^ "PRST")), removing it by moving the
 *           last edge into its place.
 *
 * The reference itself reads text edge lists and batch files
 * (src/BFS.cu:27-36, :76-91); none ship with it.
 */
#include <omp.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

static inline uint64_t sm64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

static inline uint64_t draw(uint64_t key, uint64_t i) { return sm64(key ^ sm64(i)); }

#define GE_EMPTY (~0ull)

static uint64_t pow2_ge(uint64_t n) {
  uint64_t c = 1024;
  while (c < n) c <<= 1;
  return c;
}

/* ------------------------------------------------------------------ R-MAT */

/* Returns 0, or -1 on a bad argument or a graph too dense to generate. */
int og_gen_rmat(uint32_t scale, uint64_t num_edges, double a, double b, double c, uint64_t seed,
                uint32_t w_lo, uint32_t w_hi, uint32_t *src, uint32_t *dst, uint32_t *w) {
  if (scale == 0 || scale > 31 || !src || !dst || w_hi < w_lo) return -1;
  if (a < 0 || b < 0 || c < 0 || a + b + c > 1.0) return -1;
  const double V = (double)(1ull << scale);
  if ((double)num_edges > 0.5 * V * (V - 1)) return -1;
  const double S = 4294967296.0;
  const uint32_t ta = (uint32_t)(a * S < S - 1 ? a * S : S - 1);
  const uint32_t tab = (uint32_t)((a + b) * S < S - 1 ? (a + b) * S : S - 1);
  const uint32_t tabc = (uint32_t)((a + b + c) * S < S - 1 ? (a + b + c) * S : S - 1);
  const uint64_t key = sm64(seed ^ 0x524D4154ull);
  int T = omp_get_max_threads();
  if (T < 1) T = 1;
  /* candidates are processed in chunks of at most 4 Mi; the kept edges are
     the first distinct ones in candidate order whatever the chunking */
  const uint64_t chunk_max = (1u << 22) < num_edges + num_edges / 4 + 1024
                                 ? (1u << 22) : num_edges + num_edges / 4 + 1024;
  /* one open-addressing table per hash shard, shard t owned by thread t,
     sized for every distinct key the chunks can show (num_edges + one chunk)
     at load <= 1/2 on average; a shard past 3/4 full stops the generator */
  const uint64_t shard_cap = pow2_ge(2 * (num_edges + chunk_max) / (uint64_t)T + 4096);
  uint64_t *tables = (uint64_t *)malloc((size_t)T * shard_cap * 8);
  uint64_t *fill = (uint64_t *)calloc((size_t)T, 8);
  memset(tables, 0xFF, (size_t)T * shard_cap * 8);
  uint64_t *cand = (uint64_t *)malloc(chunk_max * 8);
  uint8_t *first = (uint8_t *)malloc(chunk_max);
  uint64_t have = 0, next = 0;
  int overflow = 0;
  while (have < num_edges && !overflow) {
    const uint64_t want = num_edges - have;
    const uint64_t chunk = want + want / 4 + 1024 < chunk_max ? want + want / 4 + 1024 : chunk_max;
#pragma omp parallel for schedule(static)
    for (int64_t j = 0; j < (int64_t)chunk; ++j) {
      const uint64_t i = next + (uint64_t)j;
      uint32_t u = 0, v = 0;
      uint64_t word = 0;
      for (uint32_t l = 0; l < scale; ++l) {
        if ((l & 1) == 0) word = draw(key, i * 32 + (l >> 1));
        const uint32_t r = (l & 1) ? (uint32_t)(word >> 32) : (uint32_t)word;
        const uint32_t bu = r >= tab, bv = (r >= ta && r < tab) || r >= tabc;
        u = (u << 1) | bu;
        v = (v << 1) | bv;
      }
      cand[j] = u == v ? GE_EMPTY : (((uint64_t)u << 32) | v);
      first[j] = 0;
    }
#pragma omp parallel num_threads(T)
    {
      const int t = omp_get_thread_num();
      uint64_t *tab_t = tables + (size_t)t * shard_cap;
      const uint64_t mask = shard_cap - 1;
      for (uint64_t j = 0; j < chunk; ++j) {
        const uint64_t k = cand[j];
        if (k == GE_EMPTY) continue;
        const uint64_t h = sm64(k);
        if ((int)(h % (uint64_t)T) != t) continue;
        if (4 * fill[t] > 3 * shard_cap) break;
        uint64_t p = (h >> 8) & mask;
        while (tab_t[p] != GE_EMPTY && tab_t[p] != k) p = (p + 1) & mask;
        if (tab_t[p] == GE_EMPTY) {
          tab_t[p] = k;
          first[j] = 1;
          fill[t]++;
        }
      }
    }
    for (int t = 0; t < T; ++t)
      if (4 * fill[t] > 3 * shard_cap) overflow = 1;
    for (uint64_t j = 0; j < chunk && have < num_edges; ++j)
      if (first[j]) {
        src[have] = (uint32_t)(cand[j] >> 32);
        dst[have] = (uint32_t)cand[j];
        ++have;
      }
    next += chunk;
    /* a graph too dense for R-MAT to reach num_edges distinct edges */
    if (next > 64 * (num_edges + chunk_max)) overflow = 1;
  }
  free(cand);
  free(first);
  free(tables);
  free(fill);
  if (overflow) return -1;
  if (w) {
    const uint64_t wkey = sm64(seed ^ 0x57474854ull);
    const uint64_t range = (uint64_t)w_hi - w_lo + 1;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)num_edges; ++i) w[i] = w_lo + (uint32_t)(draw(wkey, i) % range);
  }
  return 0;
}

/* --------------------------------------------------------------- edge set */

typedef struct oes {
  uint32_t V;
  uint64_t *edges; /* dense list of keys u << 32 | v */
  uint64_t n, ecap;
  uint64_t *keys;  /* open addressing set of the same keys */
  uint64_t mask;
} oes;

static uint64_t oes_slot(const oes *s, uint64_t k) {
  uint64_t p = sm64(k) & s->mask;
  while (s->keys[p] != GE_EMPTY && s->keys[p] != k) p = (p + 1) & s->mask;
  return p;
}

static void oes_rehash(oes *s, uint64_t cap) {
  free(s->keys);
  s->keys = (uint64_t *)malloc(cap * 8);
  memset(s->keys, 0xFF, cap * 8);
  s->mask = cap - 1;
  for (uint64_t i = 0; i < s->n; ++i) s->keys[oes_slot(s, s->edges[i])] = s->edges[i];
}

static int oes_contains(const oes *s, uint64_t k) { return s->keys[oes_slot(s, k)] == k; }

static void oes_add(oes *s, uint64_t k) {
  if ((s->n + 1) * 2 > s->mask + 1) oes_rehash(s, (s->mask + 1) * 2);
  if (s->n == s->ecap) {
    s->ecap = s->ecap ? s->ecap * 2 : 1024;
    s->edges = (uint64_t *)realloc(s->edges, s->ecap * 8);
  }
  s->edges[s->n++] = k;
  s->keys[oes_slot(s, k)] = k;
}

/* backward-shift deletion */
static void oes_erase(oes *s, uint64_t k) {
  uint64_t p = oes_slot(s, k);
  if (s->keys[p] != k) return;
  s->keys[p] = GE_EMPTY;
  uint64_t q = (p + 1) & s->mask;
  while (s->keys[q] != GE_EMPTY) {
    const uint64_t home = sm64(s->keys[q]) & s->mask;
    const int in_range = (p <= q) ? (home > p && home <= q) : (home > p || home <= q);
    if (!in_range) {
      s->keys[p] = s->keys[q];
      s->keys[q] = GE_EMPTY;
      p = q;
    }
    q = (q + 1) & s->mask;
  }
}

oes *oes_create(uint32_t V, const uint32_t *src, const uint32_t *dst, uint64_t n) {
  oes *s = (oes *)calloc(1, sizeof(oes));
  s->V = V;
  s->ecap = n > 1024 ? n : 1024;
  s->edges = (uint64_t *)malloc(s->ecap * 8);
  s->keys = NULL;
  oes_rehash(s, pow2_ge(2 * n + 16));
  for (uint64_t i = 0; i < n; ++i) {
    if (src[i] == dst[i] || src[i] >= V || dst[i] >= V) continue;
    const uint64_t k = ((uint64_t)src[i] << 32) | dst[i];
    if (!oes_contains(s, k)) oes_add(s, k);
  }
  return s;
}

void oes_destroy(oes *s) {
  if (!s) return;
  free(s->edges);
  free(s->keys);
  free(s);
}

uint64_t oes_size(const oes *s) { return s->n; }

/* n distinct absent edges (u != v), added to the set.  0, or -1 if the
 * graph is too dense to find them. */
int oes_sample_absent(oes *s, uint64_t n, uint64_t seed, uint32_t *src, uint32_t *dst) {
  const uint64_t key = sm64(seed ^ 0x41425354ull);
  uint64_t got = 0, i = 0;
  while (got < n) {
    const uint64_t x = draw(key, i++);
    const uint32_t u = (uint32_t)((x & 0xFFFFFFFFull) % s->V), v = (uint32_t)((x >> 32) % s->V);
    if (u == v) continue;
    const uint64_t k = ((uint64_t)u << 32) | v;
    if (oes_contains(s, k)) continue;
    oes_add(s, k);
    src[got] = u;
    dst[got] = v;
    ++got;
    if (i > 64 * (n + 1024)) return -1;
  }
  return 0;
}

/* n present edges drawn uniformly, removed from the set.  0, or -1 if the set
 * holds fewer than n edges. */
int oes_sample_present(oes *s, uint64_t n, uint64_t seed, uint32_t *src, uint32_t *dst) {
  if (n > s->n) return -1;
  const uint64_t key = sm64(seed ^ 0x50525354ull);
  for (uint64_t i = 0; i < n; ++i) {
    const uint64_t idx = draw(key, i) % s->n;
    const uint64_t k = s->edges[idx];
    src[i] = (uint32_t)(k >> 32);
    dst[i] = (uint32_t)k;
    oes_erase(s, k);
    s->edges[idx] = s->edges[s->n - 1];
    s->n--;
  }
  return 0;
}
