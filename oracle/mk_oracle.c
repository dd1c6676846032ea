/*
 * mk_oracle.c -- CPU restatement of the reference's dynamic-graph semantics.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA path: the
 * tests, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it;
 * the product library never links or calls it.
 *
 * Parity status: the reference (meerkat-pkd/Meerkat) cannot be compiled here
 * -- its slab allocator / slab hash submodule is absent
 * (include/Graph/SlabGraph.cuh:4 includes the missing slab_hash.cuh) -- and it
 * ships no golden vectors and no algorithm tests.  The structural checks of
 * test/GraphTest.cu (degrees, adjacency sets, weights, tombstones after a
 * full delete) are mirrored by the tests; for the algorithms parity is
 * unpinned against the reference itself and the oracle is cross-checked
 * against independent implementations (scipy.sparse.csgraph, networkx) in
 * tests/test_oracle.py.
 *
 * Semantics restated (reference file:line):
 *   insert  skip self loops (include/Graph/device/InsertEdgeKernel.cuh:21-26);
 *           an edge already present is not duplicated (set semantics of the
 *           slab-hash insertKey, include/Graph/warp/InsertEdge.cuh:86-98); on
 *           weighted graphs the stored weight becomes the minimum of the live
 *           weight and every inserted copy (upsert-min; the reference's
 *           weighted insertPair duplicates keys, which is unpinned).
 *   delete  a present edge is removed, absent ones ignored
 *           (include/Graph/warp/DeleteEdge.cuh:7-39).
 *   BFS     hop levels from the source (BFSImpl.cuh:498-588), MK_INF for
 *           unreachable vertices.
 *   SSSP    uint32 shortest distances with integer weights
 *           (SSSPImpl.cuh:490-605).
 *   PR      PR'[u] = (1-d)/N + d*sum_{v->u} PR[v]/outdeg[v]
 *                    + d*sum_{outdeg v = 0} PR[v]/N, PR0 = 1/N
 *           (PageRankImpl.cuh:3-62, :89-144, PageRank.cuh:42-43), in FP64.
 *   TC      triangles of the symmetrised simple graph (TCImpl.cuh:149-214,
 *           total / 6 at :368).
 *   WCC     union-find hooking larger roots under smaller ones
 *           (include/Util/UnionFind.cuh:194-215): label = min vertex id of
 *           the weakly connected component.
 *
 * Storage: T shards (vertex u belongs to shard u % T); each shard holds an
 * open-addressing map (u,v) -> (weight, position) and the per-vertex
 * adjacency arrays of its vertices, so batch application runs one thread
 * per shard in batch order with no locks and gives the same result for any
 * thread count.
 */
#include <omp.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "mk_oracle.h"

static void omap_init(omap *m, uint64_t cap) {
  m->cap = cap;
  m->size = 0;
  m->keys = (uint64_t *)malloc(cap * 8);
  m->wt = (uint32_t *)malloc(cap * 4);
  m->pos = (uint32_t *)malloc(cap * 4);
  memset(m->keys, 0xFF, cap * 8);
}

static void omap_free(omap *m) {
  free(m->keys);
  free(m->wt);
  free(m->pos);
}

static uint64_t omap_slot(const omap *m, uint64_t k) {
  uint64_t p = mixk(k) & (m->cap - 1);
  while (m->keys[p] != OK_EMPTY && m->keys[p] != k) p = (p + 1) & (m->cap - 1);
  return p;
}

static void omap_grow(omap *m) {
  omap n;
  omap_init(&n, m->cap * 2);
  for (uint64_t i = 0; i < m->cap; ++i)
    if (m->keys[i] != OK_EMPTY) {
      uint64_t p = omap_slot(&n, m->keys[i]);
      n.keys[p] = m->keys[i];
      n.wt[p] = m->wt[i];
      n.pos[p] = m->pos[i];
    }
  n.size = m->size;
  omap_free(m);
  *m = n;
}

static void omap_erase_slot(omap *m, uint64_t p) {
  uint64_t mask = m->cap - 1;
  m->keys[p] = OK_EMPTY;
  m->size--;
  uint64_t q = (p + 1) & mask;
  while (m->keys[q] != OK_EMPTY) {
    uint64_t home = mixk(m->keys[q]) & mask;
    int in_range = (p <= q) ? (home > p && home <= q) : (home > p || home <= q);
    if (!in_range) {
      m->keys[p] = m->keys[q];
      m->wt[p] = m->wt[q];
      m->pos[p] = m->pos[q];
      m->keys[q] = OK_EMPTY;
      p = q;
    }
    q = (q + 1) & mask;
  }
}

static void ivec_push(ivec *v, uint32_t x, uint32_t w) {
  if (v->n == v->cap) {
    v->cap = v->cap ? v->cap * 2 : 4;
    v->a = (uint32_t *)realloc(v->a, (size_t)v->cap * 4);
    v->w = (uint32_t *)realloc(v->w, (size_t)v->cap * 4);
  }
  v->w[v->n] = w;
  v->a[v->n++] = x;
}

og *og_create(uint32_t V, int threads) {
  og *g = (og *)calloc(1, sizeof(og));
  g->V = V;
  g->T = threads > 0 ? threads : 1;
  g->shard = (omap *)calloc((size_t)g->T, sizeof(omap));
  for (int t = 0; t < g->T; ++t) omap_init(&g->shard[t], 1024);
  g->adj = (ivec *)calloc(V, sizeof(ivec));
  return g;
}

void og_destroy(og *g) {
  if (!g) return;
  for (int t = 0; t < g->T; ++t) omap_free(&g->shard[t]);
  free(g->shard);
  for (uint32_t i = 0; i < g->V; ++i) {
    free(g->adj[i].a);
    free(g->adj[i].w);
  }
  free(g->adj);
  free(g);
}

static int og_insert_one(og *g, omap *m, uint32_t u, uint32_t v, uint32_t w) {
  uint64_t k = ((uint64_t)u << 32) | v;
  if ((m->size + 1) * 2 > m->cap) omap_grow(m);
  uint64_t p = omap_slot(m, k);
  if (m->keys[p] == k) { /* live edge: keep the smaller weight (upsert-min) */
    if (w < m->wt[p]) {
      m->wt[p] = w;
      g->adj[u].w[m->pos[p]] = w;
    }
    return 0;
  }
  m->keys[p] = k;
  m->wt[p] = w;
  m->pos[p] = g->adj[u].n;
  m->size++;
  ivec_push(&g->adj[u], v, w);
  return 1;
}

static int og_delete_one(og *g, omap *m, uint32_t u, uint32_t v) {
  uint64_t k = ((uint64_t)u << 32) | v;
  uint64_t p = omap_slot(m, k);
  if (m->keys[p] != k) return 0;
  uint32_t pos = m->pos[p];
  omap_erase_slot(m, p);
  ivec *a = &g->adj[u];
  uint32_t last = a->a[a->n - 1];
  uint32_t lastw = a->w[a->n - 1];
  a->n--;
  if (pos < a->n) {
    a->a[pos] = last;
    a->w[pos] = lastw;
    uint64_t q = omap_slot(m, ((uint64_t)u << 32) | last);
    m->pos[q] = pos;
  }
  return 1;
}

/* Applies an insert batch; applied[i] = 1 when edge i was added. */
uint64_t og_insert(og *g, const uint32_t *src, const uint32_t *dst, const uint32_t *w,
                   uint64_t n, uint8_t *applied) {
  uint64_t total = 0;
#pragma omp parallel num_threads(g->T) reduction(+ : total)
  {
    int t = omp_get_thread_num();
    omap *m = &g->shard[t];
    for (uint64_t i = 0; i < n; ++i) {
      uint32_t u = src[i], v = dst[i];
      if (u >= g->V || v >= g->V || u == v) {
        if (t == 0 && applied) applied[i] = 0;
        continue;
      }
      if ((int)(u % (uint32_t)g->T) != t) continue;
      int a = og_insert_one(g, m, u, v, w ? w[i] : 0u);
      if (applied) applied[i] = (uint8_t)a;
      total += (uint64_t)a;
    }
  }
  return total;
}

uint64_t og_delete(og *g, const uint32_t *src, const uint32_t *dst, uint64_t n, uint8_t *applied) {
  uint64_t total = 0;
#pragma omp parallel num_threads(g->T) reduction(+ : total)
  {
    int t = omp_get_thread_num();
    omap *m = &g->shard[t];
    for (uint64_t i = 0; i < n; ++i) {
      uint32_t u = src[i], v = dst[i];
      if (u >= g->V || v >= g->V || u == v) {
        if (t == 0 && applied) applied[i] = 0;
        continue;
      }
      if ((int)(u % (uint32_t)g->T) != t) continue;
      int a = og_delete_one(g, m, u, v);
      if (applied) applied[i] = (uint8_t)a;
      total += (uint64_t)a;
    }
  }
  return total;
}

int og_has_edge(const og *g, uint32_t u, uint32_t v, uint32_t *w) {
  if (u >= g->V || v >= g->V) return 0;
  const omap *m = &g->shard[u % (uint32_t)g->T];
  uint64_t k = ((uint64_t)u << 32) | v;
  uint64_t p = omap_slot(m, k);
  if (m->keys[p] != k) return 0;
  if (w) *w = m->wt[p];
  return 1;
}

uint64_t og_num_edges(const og *g) {
  uint64_t e = 0;
  for (int t = 0; t < g->T; ++t) e += g->shard[t].size;
  return e;
}

void og_degrees(const og *g, uint32_t *out) {
  for (uint32_t u = 0; u < g->V; ++u) out[u] = g->adj[u].n;
}

static int cmp_u32(const void *a, const void *b) {
  uint32_t x = *(const uint32_t *)a, y = *(const uint32_t *)b;
  return (x > y) - (x < y);
}

/* CSR with rows sorted by neighbour id; w may be NULL. */
void og_export_csr(const og *g, uint64_t *row_ptr, uint32_t *col, uint32_t *w) {
  uint64_t p = 0;
  for (uint32_t u = 0; u < g->V; ++u) {
    row_ptr[u] = p;
    memcpy(col + p, g->adj[u].a, (size_t)g->adj[u].n * 4);
    qsort(col + p, g->adj[u].n, 4, cmp_u32);
    if (w)
      for (uint32_t i = 0; i < g->adj[u].n; ++i) og_has_edge(g, u, col[p + i], &w[p + i]);
    p += g->adj[u].n;
  }
  row_ptr[g->V] = p;
}

/* BFS hop levels (sequential queue). */
void og_bfs(const og *g, uint32_t src, uint32_t *dist) {
  for (uint32_t i = 0; i < g->V; ++i) dist[i] = OK_INF;
  uint32_t *q = (uint32_t *)malloc((size_t)g->V * 4);
  uint64_t h = 0, t = 0;
  dist[src] = 0;
  q[t++] = src;
  while (h < t) {
    uint32_t u = q[h++];
    const ivec *a = &g->adj[u];
    for (uint32_t i = 0; i < a->n; ++i) {
      uint32_t v = a->a[i];
      if (dist[v] == OK_INF) {
        dist[v] = dist[u] + 1;
        q[t++] = v;
      }
    }
  }
  free(q);
}

/* Dijkstra with a binary heap of (dist << 32 | vertex). Returns -1 when a
 * distance does not fit in uint32. */
int og_sssp(const og *g, uint32_t src, uint32_t *dist) {
  uint64_t *d64 = (uint64_t *)malloc((size_t)g->V * 8);
  for (uint32_t i = 0; i < g->V; ++i) d64[i] = UINT64_MAX;
  uint64_t cap = 1024, n = 0;
  uint64_t *heap = (uint64_t *)malloc(cap * 16);
  /* heap of (key = dist, vertex) stored as two u64 */
#define HK(i) heap[2 * (i)]
#define HV(i) heap[2 * (i) + 1]
  d64[src] = 0;
  HK(0) = 0;
  HV(0) = src;
  n = 1;
  while (n) {
    uint64_t dk = HK(0), u = HV(0);
    --n;
    if (n) {
      HK(0) = HK(n);
      HV(0) = HV(n);
      uint64_t i = 0;
      for (;;) {
        uint64_t l = 2 * i + 1, r = l + 1, s = i;
        if (l < n && HK(l) < HK(s)) s = l;
        if (r < n && HK(r) < HK(s)) s = r;
        if (s == i) break;
        uint64_t tk = HK(i), tv = HV(i);
        HK(i) = HK(s);
        HV(i) = HV(s);
        HK(s) = tk;
        HV(s) = tv;
        i = s;
      }
    }
    if (dk != d64[u]) continue;
    const ivec *a = &g->adj[u];
    for (uint32_t j = 0; j < a->n; ++j) {
      uint32_t v = a->a[j], w = a->w[j];
      uint64_t nd = dk + w;
      if (nd < d64[v]) {
        d64[v] = nd;
        if (n == cap) {
          cap *= 2;
          heap = (uint64_t *)realloc(heap, cap * 16);
        }
        uint64_t i = n++;
        HK(i) = nd;
        HV(i) = v;
        while (i) {
          uint64_t p = (i - 1) / 2;
          if (HK(p) <= HK(i)) break;
          uint64_t tk = HK(i), tv = HV(i);
          HK(i) = HK(p);
          HV(i) = HV(p);
          HK(p) = tk;
          HV(p) = tv;
          i = p;
        }
      }
    }
  }
#undef HK
#undef HV
  int ok = 0;
  for (uint32_t i = 0; i < g->V; ++i) {
    if (d64[i] == UINT64_MAX)
      dist[i] = OK_INF;
    else if (d64[i] >= OK_INF) {
      dist[i] = OK_INF;
      ok = -1;
    } else
      dist[i] = (uint32_t)d64[i];
  }
  free(d64);
  free(heap);
  return ok;
}

/* Checks a packed dist<<32|parent array: every reachable v != src has a live
 * edge (p, v) with dist[p] + w(p, v) == dist[v] (w = 1 if !weighted).
 * Returns the number of violations. */
uint64_t og_check_parents(const og *g, uint32_t src, const uint64_t *packed, int weighted) {
  uint64_t bad = 0;
  for (uint32_t v = 0; v < g->V; ++v) {
    uint64_t x = packed[v];
    if (x == ~0ull) continue;
    uint32_t dv = (uint32_t)(x >> 32), p = (uint32_t)x;
    if (v == src) {
      bad += (dv != 0);
      continue;
    }
    uint32_t w = 0;
    if (p >= g->V || !og_has_edge(g, p, v, &w) || packed[p] == ~0ull) {
      ++bad;
      continue;
    }
    uint32_t dp = (uint32_t)(packed[p] >> 32);
    if ((uint64_t)dp + (weighted ? w : 1u) != dv) ++bad;
  }
  return bad;
}

/* FP64 PageRank over the edges as stored (u -> v), iterated until the L1
 * change is <= tol or max_iter.  pr may hold a warm start when warm != 0. */
uint32_t og_pagerank(const og *g, double d, double tol, uint32_t max_iter, int warm, double *pr) {
  const uint32_t V = g->V;
  double *nx = (double *)malloc((size_t)V * 8);
  if (!warm)
    for (uint32_t i = 0; i < V; ++i) pr[i] = 1.0 / V;
  uint32_t it = 0;
  for (; it < max_iter; ++it) {
    double dang = 0;
    for (uint32_t u = 0; u < V; ++u)
      if (g->adj[u].n == 0) dang += pr[u];
    double base = (1.0 - d) / V + d * dang / V;
    for (uint32_t u = 0; u < V; ++u) nx[u] = base;
    for (uint32_t u = 0; u < V; ++u) {
      const ivec *a = &g->adj[u];
      if (!a->n) continue;
      double c = d * pr[u] / a->n;
      for (uint32_t i = 0; i < a->n; ++i) nx[a->a[i]] += c;
    }
    double delta = 0;
    for (uint32_t u = 0; u < V; ++u) {
      double x = nx[u] - pr[u];
      delta += x < 0 ? -x : x;
      pr[u] = nx[u];
    }
    if (delta <= tol) {
      ++it;
      break;
    }
  }
  free(nx);
  return it;
}

/* Symmetrised simple undirected adjacency (sorted rows). */
static void sym_csr(const og *g, uint64_t **rp_out, uint32_t **col_out) {
  const uint32_t V = g->V;
  uint64_t *cnt = (uint64_t *)calloc((size_t)V + 1, 8);
  for (uint32_t u = 0; u < V; ++u)
    for (uint32_t i = 0; i < g->adj[u].n; ++i) {
      cnt[u]++;
      cnt[g->adj[u].a[i]]++;
    }
  uint64_t *rp = (uint64_t *)malloc(((size_t)V + 1) * 8);
  uint64_t s = 0;
  for (uint32_t u = 0; u < V; ++u) {
    rp[u] = s;
    s += cnt[u];
  }
  rp[V] = s;
  uint32_t *col = (uint32_t *)malloc(s ? s * 4 : 4);
  uint64_t *fill = cnt;
  for (uint32_t u = 0; u < V; ++u) fill[u] = rp[u];
  for (uint32_t u = 0; u < V; ++u)
    for (uint32_t i = 0; i < g->adj[u].n; ++i) {
      uint32_t v = g->adj[u].a[i];
      col[fill[u]++] = v;
      col[fill[v]++] = u;
    }
  /* sort + unique each row in place (rows in parallel), then compact */
  uint64_t *len = cnt;
#pragma omp parallel for schedule(dynamic, 256)
  for (int64_t uu = 0; uu < (int64_t)V; ++uu) {
    uint64_t b = rp[uu], e = rp[uu + 1], k = b;
    qsort(col + b, e - b, 4, cmp_u32);
    for (uint64_t i = b; i < e; ++i)
      if (i == b || col[i] != col[i - 1]) col[k++] = col[i];
    len[uu] = k - b;
  }
  uint64_t w = 0;
  for (uint32_t u = 0; u < V; ++u) {
    uint64_t b = rp[u];
    rp[u] = w;
    memmove(col + w, col + b, (size_t)len[u] * 4);
    w += len[u];
  }
  rp[V] = w;
  free(cnt);
  *rp_out = rp;
  *col_out = col;
}

/* Triangles of the symmetrised graph: forward algorithm, merge intersection. */
uint64_t og_triangles(const og *g) {
  uint64_t *rp;
  uint32_t *col;
  sym_csr(g, &rp, &col);
  const uint32_t V = g->V;
  /* oriented rows: neighbours of higher rank (degree, id) */
  uint64_t *orp = (uint64_t *)malloc(((size_t)V + 1) * 8);
  uint32_t *ocol = (uint32_t *)malloc(rp[V] ? rp[V] * 4 : 4);
  uint64_t p = 0;
  for (uint32_t u = 0; u < V; ++u) {
    orp[u] = p;
    uint64_t du = rp[u + 1] - rp[u];
    for (uint64_t i = rp[u]; i < rp[u + 1]; ++i) {
      uint32_t v = col[i];
      uint64_t dv = rp[v + 1] - rp[v];
      if (du < dv || (du == dv && u < v)) ocol[p++] = v;
    }
  }
  orp[V] = p;
  uint64_t total = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : total)
  for (int64_t uu = 0; uu < (int64_t)V; ++uu) {
    uint32_t u = (uint32_t)uu;
    for (uint64_t i = orp[u]; i < orp[u + 1]; ++i) {
      uint32_t v = ocol[i];
      uint64_t a = orp[u], ae = orp[u + 1], b = orp[v], be = orp[v + 1];
      while (a < ae && b < be) {
        if (ocol[a] < ocol[b])
          ++a;
        else if (ocol[a] > ocol[b])
          ++b;
        else {
          ++total;
          ++a;
          ++b;
        }
      }
    }
  }
  free(rp);
  free(col);
  free(orp);
  free(ocol);
  return total;
}

static uint32_t uf_find(uint32_t *p, uint32_t x) {
  while (p[x] != x) {
    p[x] = p[p[x]];
    x = p[x];
  }
  return x;
}

/* Weakly connected components, label = min vertex id. */
void og_wcc(const og *g, uint32_t *labels) {
  const uint32_t V = g->V;
  for (uint32_t i = 0; i < V; ++i) labels[i] = i;
  for (uint32_t u = 0; u < V; ++u)
    for (uint32_t i = 0; i < g->adj[u].n; ++i) {
      uint32_t a = uf_find(labels, u), b = uf_find(labels, g->adj[u].a[i]);
      if (a == b) continue;
      if (a < b)
        labels[b] = a;
      else
        labels[a] = b;
    }
  for (uint32_t i = 0; i < V; ++i) labels[i] = uf_find(labels, i);
}
