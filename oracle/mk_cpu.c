/*
 * mk_cpu.c -- multithreaded CPU implementation of the dynamic queries: the
 * CPU baseline that bench.py times beside the GPU.
 *
 * TEST INFRASTRUCTURE ONLY (the product never links it).  It runs on the
 * oracle's hash-set adjacency (mk_oracle.h) with OpenMP, one parallel loop
 * per frontier level, and is checked against the oracle's sequential
 * definitions (og_bfs, og_sssp, og_pagerank, og_triangles, og_wcc) by
 * tests/test_oracle_cpu.py.  The algorithms are those of the reference's
 * GPU path restated for a multicore host:
 *
 *   BFS / SSSP    packed dist << 32 | parent words relaxed by a 64-bit
 *                 atomic minimum (include/Algorithms/definitions.cuh:14-17,
 *                 BFSImpl.cuh:296-382, SSSPImpl.cuh:280-364), level by level
 *                 over a vertex frontier (Bellman-Ford for SSSP).
 *     incremental seeds from the batch edges, then relaxes to a fixed point
 *                 (BFSImpl.cuh:270-382).
 *     decremental invalidates the subtrees below deleted tree edges level by
 *                 level over out-edges, re-seeds every invalidated vertex
 *                 from its valid in-neighbours with one sweep over all
 *                 vertices (the reference's strategy, BFSImpl.cuh:419-440),
 *                 then relaxes; when more than a tenth of the vertices were
 *                 invalidated it recomputes from the source instead (the GPU
 *                 path's default rule).
 *   PageRank      FP64 pull over a transposed CSR built per solve
 *                 (PageRankImpl.cuh:3-62, :89-216), same teleport and
 *                 dangling terms as og_pagerank.
 *   TC            symmetrised simple graph, degree-ordered orientation,
 *                 merge intersections (TCImpl.cuh:149-214).
 *   WCC           union-find with CAS hooking of the larger root under the
 *                 smaller (include/Util/UnionFind.cuh:194-215), min-id labels.
 */
#include <omp.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "mk_oracle.h"

#define OC_INFINF (~0ull)
#define OC_DIST(x) ((uint32_t)((x) >> 32))
#define OC_PARENT(x) ((uint32_t)(x))
#define OC_PACK(d, p) (((uint64_t)(d) << 32) | (uint32_t)(p))

/* 64-bit atomic minimum; returns the value seen before a successful store,
 * or a value <= x when nothing was stored. */
static inline uint64_t oc_atomic_min(uint64_t *p, uint64_t x) {
  uint64_t cur = __atomic_load_n(p, __ATOMIC_RELAXED);
  while (x < cur) {
    if (__atomic_compare_exchange_n(p, &cur, x, 1, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) return cur;
  }
  return cur <= x ? cur : x;
}

typedef struct otrav {
  const og *g;
  uint32_t V, src;
  int weighted; /* 1 = SSSP */
  uint64_t *packed;
  uint32_t *front, *next;
  uint64_t nfront;
  uint32_t *stamp; /* frontier dedupe: stamp[v] == epoch when queued */
  uint32_t epoch;
  uint8_t *invalid;
  uint32_t levels;
  uint64_t invalidated;
  int recomputed;
} otrav;

otrav *otrav_create(const og *g, uint32_t src, int weighted) {
  otrav *t = (otrav *)calloc(1, sizeof(otrav));
  t->g = g;
  t->V = g->V;
  t->src = src;
  t->weighted = weighted;
  t->packed = (uint64_t *)malloc((size_t)t->V * 8);
  t->front = (uint32_t *)malloc((size_t)t->V * 4 + 4);
  t->next = (uint32_t *)malloc((size_t)t->V * 4 + 4);
  t->stamp = (uint32_t *)calloc(t->V, 4);
  t->invalid = (uint8_t *)calloc(t->V, 1);
  return t;
}

void otrav_destroy(otrav *t) {
  if (!t) return;
  free(t->packed);
  free(t->front);
  free(t->next);
  free(t->stamp);
  free(t->invalid);
  free(t);
}

/* Appends the vertices a thread found to `out` in blocks of 1,024. */
typedef struct {
  uint32_t buf[1024];
  uint32_t n;
} oc_local;

static inline void oc_flush(oc_local *l, uint32_t *out, uint64_t *count) {
  if (!l->n) return;
  const uint64_t at = __atomic_fetch_add(count, l->n, __ATOMIC_RELAXED);
  memcpy(out + at, l->buf, (size_t)l->n * 4);
  l->n = 0;
}

static inline void oc_push(otrav *t, oc_local *l, uint32_t *out, uint64_t *count, uint32_t v) {
  if (__atomic_exchange_n(&t->stamp[v], t->epoch, __ATOMIC_RELAXED) == t->epoch) return;
  l->buf[l->n++] = v;
  if (l->n == 1024) oc_flush(l, out, count);
}

static void oc_new_epoch(otrav *t) {
  if (++t->epoch == 0) {
    memset(t->stamp, 0, (size_t)t->V * 4);
    t->epoch = 1;
  }
}

/* Relaxes from the current frontier until it is empty. */
static void oc_relax(otrav *t) {
  const og *g = t->g;
  while (t->nfront) {
    oc_new_epoch(t);
    uint64_t nnext = 0;
#pragma omp parallel
    {
      oc_local l;
      l.n = 0;
#pragma omp for schedule(dynamic, 64)
      for (int64_t i = 0; i < (int64_t)t->nfront; ++i) {
        const uint32_t u = t->front[i];
        const uint32_t du = OC_DIST(__atomic_load_n(&t->packed[u], __ATOMIC_RELAXED));
        const ivec *a = &g->adj[u];
        for (uint32_t j = 0; j < a->n; ++j) {
          const uint32_t v = a->a[j];
          const uint64_t nd = (uint64_t)du + (t->weighted ? a->w[j] : 1u);
          if (nd >= OK_INF) continue;
          const uint64_t cand = OC_PACK(nd, u);
          const uint64_t old = oc_atomic_min(&t->packed[v], cand);
          if (old > cand && OC_DIST(old) > nd) oc_push(t, &l, t->next, &nnext, v);
        }
      }
      oc_flush(&l, t->next, &nnext);
    }
    uint32_t *x = t->front;
    t->front = t->next;
    t->next = x;
    t->nfront = nnext;
    t->levels++;
  }
}

void otrav_static(otrav *t) {
  const uint32_t V = t->V;
#pragma omp parallel for schedule(static)
  for (int64_t v = 0; v < (int64_t)V; ++v) t->packed[v] = OC_INFINF;
  t->packed[t->src] = OC_PACK(0, t->src);
  t->front[0] = t->src;
  t->nfront = 1;
  t->levels = 0;
  t->invalidated = 0;
  t->recomputed = 0;
  oc_relax(t);
}

/* After the batch was inserted: seeds from its edges, then relaxes. */
void otrav_incremental(otrav *t, const uint32_t *src, const uint32_t *dst, uint64_t n) {
  const og *g = t->g;
  oc_new_epoch(t);
  uint64_t nf = 0;
  t->levels = 0;
  t->invalidated = 0;
  t->recomputed = 0;
#pragma omp parallel
  {
    oc_local l;
    l.n = 0;
#pragma omp for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
      const uint32_t u = src[i], v = dst[i];
      if (u >= t->V || v >= t->V || u == v) continue;
      const uint64_t pu = __atomic_load_n(&t->packed[u], __ATOMIC_RELAXED);
      if (pu == OC_INFINF) continue;
      uint32_t w = 0;
      if (!og_has_edge(g, u, v, &w)) continue;
      const uint64_t nd = (uint64_t)OC_DIST(pu) + (t->weighted ? w : 1u);
      if (nd >= OK_INF) continue;
      const uint64_t cand = OC_PACK(nd, u);
      const uint64_t old = oc_atomic_min(&t->packed[v], cand);
      if (old > cand && OC_DIST(old) > nd) oc_push(t, &l, t->front, &nf, v);
    }
    oc_flush(&l, t->front, &nf);
  }
  t->nfront = nf;
  oc_relax(t);
}

/* After the batch was deleted: invalidates, re-seeds, relaxes. */
void otrav_decremental(otrav *t, const uint32_t *src, const uint32_t *dst, uint64_t n) {
  const og *g = t->g;
  const uint32_t V = t->V;
  t->levels = 0;
  t->recomputed = 0;
  /* 1. the heads of deleted tree edges */
  oc_new_epoch(t);
  uint64_t nf = 0;
#pragma omp parallel
  {
    oc_local l;
    l.n = 0;
#pragma omp for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
      const uint32_t u = src[i], v = dst[i];
      if (u >= V || v >= V || u == v || v == t->src) continue;
      const uint64_t pv = t->packed[v];
      if (pv == OC_INFINF || OC_PARENT(pv) != u) continue;
      if (og_has_edge(g, u, v, NULL)) continue;
      if (__atomic_exchange_n(&t->invalid[v], 1, __ATOMIC_RELAXED)) continue;
      oc_push(t, &l, t->front, &nf, v);
    }
    oc_flush(&l, t->front, &nf);
  }
  /* 2. their subtrees, level by level over out-edges; every invalidated
        vertex is appended to `next` beyond the frontier region */
  uint64_t total = 0;
  uint32_t *all = (uint32_t *)malloc((size_t)V * 4 + 4);
  while (nf) {
    memcpy(all + total, t->front, nf * 4);
    total += nf;
    oc_new_epoch(t);
    uint64_t nn = 0;
#pragma omp parallel
    {
      oc_local l;
      l.n = 0;
#pragma omp for schedule(dynamic, 64)
      for (int64_t i = 0; i < (int64_t)nf; ++i) {
        const uint32_t x = t->front[i];
        const ivec *a = &g->adj[x];
        for (uint32_t j = 0; j < a->n; ++j) {
          const uint32_t y = a->a[j];
          const uint64_t py = t->packed[y];
          if (py == OC_INFINF || OC_PARENT(py) != x || y == t->src) continue;
          if (__atomic_exchange_n(&t->invalid[y], 1, __ATOMIC_RELAXED)) continue;
          oc_push(t, &l, t->next, &nn, y);
        }
      }
      oc_flush(&l, t->next, &nn);
    }
    uint32_t *x = t->front;
    t->front = t->next;
    t->next = x;
    nf = nn;
  }
  t->invalidated = total;
  if (total * 10 > V) { /* most of the tree is gone: recompute */
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)total; ++i) t->invalid[all[i]] = 0;
    free(all);
    otrav_static(t);
    t->invalidated = total;
    t->recomputed = 1;
    return;
  }
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)total; ++i) t->packed[all[i]] = OC_INFINF;
  /* 3. re-seed: every valid vertex offers itself to its invalid out-neighbours */
  if (total) {
#pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t uu = 0; uu < (int64_t)V; ++uu) {
      const uint32_t u = (uint32_t)uu;
      if (t->invalid[u]) continue;
      const uint64_t pu = t->packed[u];
      if (pu == OC_INFINF) continue;
      const ivec *a = &g->adj[u];
      for (uint32_t j = 0; j < a->n; ++j) {
        const uint32_t y = a->a[j];
        if (!t->invalid[y]) continue;
        const uint64_t nd = (uint64_t)OC_DIST(pu) + (t->weighted ? a->w[j] : 1u);
        if (nd >= OK_INF) continue;
        oc_atomic_min(&t->packed[y], OC_PACK(nd, u));
      }
    }
  }
  /* 4. relax from the re-seeded vertices */
  uint64_t k = 0;
  for (uint64_t i = 0; i < total; ++i) {
    const uint32_t y = all[i];
    t->invalid[y] = 0;
    if (t->packed[y] != OC_INFINF) t->front[k++] = y;
  }
  free(all);
  t->nfront = k;
  oc_relax(t);
}

void otrav_distances(const otrav *t, uint32_t *out) {
#pragma omp parallel for schedule(static)
  for (int64_t v = 0; v < (int64_t)t->V; ++v)
    out[v] = t->packed[v] == OC_INFINF ? OK_INF : OC_DIST(t->packed[v]);
}

void otrav_packed(const otrav *t, uint64_t *out) { memcpy(out, t->packed, (size_t)t->V * 8); }

/* levels of the last call, vertices invalidated, whether it recomputed */
void otrav_stats(const otrav *t, uint32_t *levels, uint64_t *invalidated, int *recomputed) {
  if (levels) *levels = t->levels;
  if (invalidated) *invalidated = t->invalidated;
  if (recomputed) *recomputed = t->recomputed;
}

/* ------------------------------------------------------------- PageRank */

/* FP64 pull PageRank; pr holds a warm start when warm != 0.  Returns the
 * iterations run. */
uint32_t oc_pagerank(const og *g, double d, double tol, uint32_t max_iter, int warm, double *pr) {
  const uint32_t V = g->V;
  uint64_t *rp = (uint64_t *)calloc((size_t)V + 1, 8);
  for (uint32_t u = 0; u < V; ++u)
    for (uint32_t j = 0; j < g->adj[u].n; ++j) rp[g->adj[u].a[j] + 1]++;
  for (uint32_t v = 0; v < V; ++v) rp[v + 1] += rp[v];
  uint32_t *in = (uint32_t *)malloc(rp[V] ? rp[V] * 4 : 4);
  uint64_t *fill = (uint64_t *)malloc((size_t)V * 8);
  memcpy(fill, rp, (size_t)V * 8);
  for (uint32_t u = 0; u < V; ++u)
    for (uint32_t j = 0; j < g->adj[u].n; ++j) in[fill[g->adj[u].a[j]]++] = u;
  free(fill);
  double *contrib = (double *)malloc((size_t)V * 8);
  double *nx = (double *)malloc((size_t)V * 8);
  if (!warm)
    for (uint32_t i = 0; i < V; ++i) pr[i] = 1.0 / V;
  uint32_t it = 0;
  for (; it < max_iter; ++it) {
    double dang = 0;
#pragma omp parallel for schedule(static) reduction(+ : dang)
    for (int64_t u = 0; u < (int64_t)V; ++u) {
      const uint32_t n = g->adj[u].n;
      contrib[u] = n ? pr[u] / n : 0.0;
      if (!n) dang += pr[u];
    }
    const double base = (1.0 - d) / V + d * dang / V;
    double delta = 0;
#pragma omp parallel for schedule(dynamic, 1024) reduction(+ : delta)
    for (int64_t v = 0; v < (int64_t)V; ++v) {
      double s = 0;
      for (uint64_t k = rp[v]; k < rp[v + 1]; ++k) s += contrib[in[k]];
      nx[v] = base + d * s;
      const double x = nx[v] - pr[v];
      delta += x < 0 ? -x : x;
    }
    memcpy(pr, nx, (size_t)V * 8);
    if (delta <= tol) {
      ++it;
      break;
    }
  }
  free(rp);
  free(in);
  free(contrib);
  free(nx);
  return it;
}

/* ------------------------------------------------------------------- TC */

static int oc_cmp_u32(const void *a, const void *b) {
  const uint32_t x = *(const uint32_t *)a, y = *(const uint32_t *)b;
  return (x > y) - (x < y);
}

/* Triangles of the symmetrised simple graph. */
uint64_t oc_triangles(const og *g) {
  const uint32_t V = g->V;
  uint64_t *cnt = (uint64_t *)calloc((size_t)V + 1, 8);
#pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t u = 0; u < (int64_t)V; ++u) {
    __atomic_fetch_add(&cnt[u + 1], g->adj[u].n, __ATOMIC_RELAXED);
    for (uint32_t j = 0; j < g->adj[u].n; ++j)
      __atomic_fetch_add(&cnt[g->adj[u].a[j] + 1], 1, __ATOMIC_RELAXED);
  }
  for (uint32_t v = 0; v < V; ++v) cnt[v + 1] += cnt[v];
  uint32_t *col = (uint32_t *)malloc(cnt[V] ? cnt[V] * 4 : 4);
  uint64_t *fill = (uint64_t *)malloc((size_t)V * 8);
  memcpy(fill, cnt, (size_t)V * 8);
#pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t u = 0; u < (int64_t)V; ++u)
    for (uint32_t j = 0; j < g->adj[u].n; ++j) {
      const uint32_t v = g->adj[u].a[j];
      col[__atomic_fetch_add(&fill[u], 1, __ATOMIC_RELAXED)] = v;
      col[__atomic_fetch_add(&fill[v], 1, __ATOMIC_RELAXED)] = (uint32_t)u;
    }
  /* sort + unique each row in place; fill[u] = its distinct count */
#pragma omp parallel for schedule(dynamic, 256)
  for (int64_t u = 0; u < (int64_t)V; ++u) {
    uint32_t *r = col + cnt[u];
    const uint64_t n = cnt[u + 1] - cnt[u];
    qsort(r, n, 4, oc_cmp_u32);
    uint64_t k = 0;
    for (uint64_t i = 0; i < n; ++i)
      if (i == 0 || r[i] != r[i - 1]) r[k++] = r[i];
    fill[u] = k;
  }
  /* oriented rows (higher (degree, id) neighbours), kept in place */
  uint64_t *olen = (uint64_t *)malloc((size_t)V * 8);
#pragma omp parallel for schedule(dynamic, 256)
  for (int64_t u = 0; u < (int64_t)V; ++u) {
    uint32_t *r = col + cnt[u];
    const uint64_t du = fill[u];
    uint64_t k = 0;
    for (uint64_t i = 0; i < du; ++i) {
      const uint32_t v = r[i];
      const uint64_t dv = fill[v];
      if (du < dv || (du == dv && (uint32_t)u < v)) r[k++] = v;
    }
    olen[u] = k;
  }
  uint64_t total = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : total)
  for (int64_t u = 0; u < (int64_t)V; ++u) {
    const uint32_t *ru = col + cnt[u];
    for (uint64_t i = 0; i < olen[u]; ++i) {
      const uint32_t v = ru[i];
      const uint32_t *rv = col + cnt[v];
      uint64_t a = 0, b = 0;
      const uint64_t ae = olen[u], be = olen[v];
      while (a < ae && b < be) {
        if (ru[a] < rv[b])
          ++a;
        else if (ru[a] > rv[b])
          ++b;
        else {
          ++total;
          ++a;
          ++b;
        }
      }
    }
  }
  free(cnt);
  free(col);
  free(fill);
  free(olen);
  return total;
}

/* ------------------------------------------------------------------ WCC */

static inline uint32_t oc_find(uint32_t *p, uint32_t x) {
  for (;;) {
    uint32_t y = __atomic_load_n(&p[x], __ATOMIC_RELAXED);
    if (y == x) return x;
    const uint32_t z = __atomic_load_n(&p[y], __ATOMIC_RELAXED);
    if (z != y) /* path halving: x skips to its grandparent if unchanged */
      __atomic_compare_exchange_n(&p[x], &y, z, 0, __ATOMIC_RELAXED, __ATOMIC_RELAXED);
    x = z;
  }
}

static inline void oc_union(uint32_t *p, uint32_t a, uint32_t b) {
  for (;;) {
    a = oc_find(p, a);
    b = oc_find(p, b);
    if (a == b) return;
    if (a > b) {
      const uint32_t t = a;
      a = b;
      b = t;
    }
    uint32_t expect = b;
    if (__atomic_compare_exchange_n(&p[b], &expect, a, 0, __ATOMIC_RELAXED, __ATOMIC_RELAXED))
      return;
  }
}

/* Static WCC: labels = min vertex id of each component. */
void oc_wcc(const og *g, uint32_t *labels) {
  const uint32_t V = g->V;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)V; ++i) labels[i] = (uint32_t)i;
#pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t u = 0; u < (int64_t)V; ++u)
    for (uint32_t j = 0; j < g->adj[u].n; ++j) oc_union(labels, (uint32_t)u, g->adj[u].a[j]);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)V; ++i) {
    uint32_t x = (uint32_t)i;
    while (labels[x] != x) x = labels[x];
    labels[i] = x;
  }
}

/* Incremental WCC: labels hold min-id labels of the graph before the batch
 * (every label is its component's root); unions the batch edges. */
void oc_wcc_incremental(uint32_t V, uint32_t *labels, const uint32_t *src, const uint32_t *dst,
                        uint64_t n) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)n; ++i)
    if (src[i] < V && dst[i] < V) oc_union(labels, src[i], dst[i]);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)V; ++i) {
    uint32_t x = (uint32_t)i;
    while (labels[x] != x) x = labels[x];
    labels[i] = x;
  }
}
