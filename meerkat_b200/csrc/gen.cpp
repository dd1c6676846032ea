// Seeded synthetic inputs: R-MAT graphs, 2D grids with shortcuts, and an
// edge-set tracker that draws valid update batches (absent-edge inserts,
// present-edge deletes).  Host only; results do not depend on the thread
// count.
//
// The reference reads text edge lists and "<prefix>.batch.<i>" files
// (src/BFS.cu:27-36, :76-91); none ship with it, so these generators produce
// inputs of the benchmark shapes instead.
#include <omp.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../../include/meerkat_b200.h"

namespace {

inline uint64_t splitmix(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

// Counter-based stream: value i of stream `key`.
inline uint64_t rnd(uint64_t key, uint64_t i) { return splitmix(key ^ splitmix(i)); }

inline uint64_t hkey(uint64_t k) { return splitmix(k); }

constexpr uint64_t kEmpty = ~0ull;

uint64_t pow2_at_least(uint64_t n) {
  uint64_t c = 1024;
  while (c < n) c <<= 1;
  return c;
}

// One R-MAT edge from the random words of candidate i.
inline void rmat_edge(uint64_t seed, uint64_t i, uint32_t scale, uint32_t ta, uint32_t tab,
                      uint32_t tabc, uint32_t &u, uint32_t &v) {
  u = 0;
  v = 0;
  uint64_t word = 0;
  for (uint32_t l = 0; l < scale; ++l) {
    if ((l & 1) == 0) word = rnd(seed, i * 32 + (l >> 1));
    uint32_t r = (l & 1) ? (uint32_t)(word >> 32) : (uint32_t)word;
    uint32_t bu, bv;
    if (r < ta) {
      bu = 0;
      bv = 0;
    } else if (r < tab) {
      bu = 0;
      bv = 1;
    } else if (r < tabc) {
      bu = 1;
      bv = 0;
    } else {
      bu = 1;
      bv = 1;
    }
    u = (u << 1) | bu;
    v = (v << 1) | bv;
  }
}

// Marks keep[i] = 1 for the first occurrence of every key in cand[0..n),
// skipping keys flagged invalid (kEmpty).  Parallel over hash shards.
void first_occurrences(const std::vector<uint64_t> &cand, std::vector<uint8_t> &keep) {
  const size_t n = cand.size();
  keep.assign(n, 0);
  int T = omp_get_max_threads();
  if (T < 1) T = 1;
  const uint64_t cap_total = pow2_at_least(2 * n + 16);
  const int shards = T;
  const uint64_t cap = pow2_at_least(cap_total / shards + 16);
#pragma omp parallel num_threads(T)
  {
    int t = omp_get_thread_num();
    for (int sh = t; sh < shards; sh += T) {
      std::vector<uint64_t> table(cap, kEmpty);
      for (size_t i = 0; i < n; ++i) {
        uint64_t k = cand[i];
        if (k == kEmpty) continue;
        uint64_t h = hkey(k);
        if ((int)(h % (uint64_t)shards) != sh) continue;
        uint64_t p = (h >> 8) & (cap - 1);
        while (true) {
          if (table[p] == kEmpty) {
            table[p] = k;
            keep[i] = 1;
            break;
          }
          if (table[p] == k) break;
          p = (p + 1) & (cap - 1);
        }
      }
    }
  }
}

}  // namespace

struct mk_edgeset {
  uint32_t V = 0;
  std::vector<uint64_t> edges;  // dense list (u << 32 | v)
  std::vector<uint64_t> keys;   // open addressing table of edge keys
  std::vector<uint64_t> pos;    // index of the key in `edges`
  uint64_t mask = 0;
  uint64_t draws = 0;           // stream position for sampling

  void rebuild(uint64_t cap) {
    keys.assign(cap, kEmpty);
    pos.assign(cap, 0);
    mask = cap - 1;
    for (uint64_t i = 0; i < edges.size(); ++i) put(edges[i], i);
  }
  uint64_t slot_of(uint64_t k) const {
    uint64_t p = hkey(k) & mask;
    while (keys[p] != kEmpty && keys[p] != k) p = (p + 1) & mask;
    return p;
  }
  bool contains(uint64_t k) const { return keys[slot_of(k)] == k; }
  void put(uint64_t k, uint64_t i) {
    uint64_t p = slot_of(k);
    keys[p] = k;
    pos[p] = i;
  }
  void maybe_grow() {
    if ((edges.size() + 1) * 2 > keys.size()) rebuild(keys.size() * 2);
  }
  void add(uint64_t k) {
    maybe_grow();
    edges.push_back(k);
    put(k, edges.size() - 1);
  }
  // backward-shift deletion of key k
  void erase_key(uint64_t k) {
    uint64_t p = slot_of(k);
    if (keys[p] != k) return;
    keys[p] = kEmpty;
    uint64_t q = (p + 1) & mask;
    while (keys[q] != kEmpty) {
      uint64_t home = hkey(keys[q]) & mask;
      // move q back to p if home is not in the cyclic range (p, q]
      bool in_range = (p <= q) ? (home > p && home <= q) : (home > p || home <= q);
      if (!in_range) {
        keys[p] = keys[q];
        pos[p] = pos[q];
        keys[q] = kEmpty;
        p = q;
      }
      q = (q + 1) & mask;
    }
  }
  void remove_at(uint64_t i) {
    uint64_t k = edges[i];
    erase_key(k);
    uint64_t last = edges.back();
    edges.pop_back();
    if (i < edges.size()) {
      edges[i] = last;
      pos[slot_of(last)] = i;
    }
  }
};

extern "C" {

mk_status mk_gen_rmat(uint32_t scale, uint64_t num_edges, double a, double b, double c,
                      uint64_t seed, uint32_t w_lo, uint32_t w_hi, uint32_t *h_src,
                      uint32_t *h_dst, uint32_t *h_w) {
  if (scale == 0 || scale > 31 || !h_src || !h_dst) return MK_ERR_INVALID;
  if (a < 0 || b < 0 || c < 0 || a + b + c > 1.0) return MK_ERR_INVALID;
  const double V = (double)(1ull << scale);
  if ((double)num_edges > 0.5 * V * (V - 1)) return MK_ERR_INVALID;
  if (w_hi < w_lo) return MK_ERR_INVALID;
  const double s = 4294967296.0;
  const uint32_t ta = (uint32_t)std::min(a * s, s - 1);
  const uint32_t tab = (uint32_t)std::min((a + b) * s, s - 1);
  const uint32_t tabc = (uint32_t)std::min((a + b + c) * s, s - 1);
  const uint64_t eseed = splitmix(seed ^ 0x524D4154ull);
  uint64_t have = 0;
  uint64_t next_cand = 0;
  std::vector<uint64_t> kept;  // keys of accepted edges, in candidate order
  kept.reserve(num_edges);
  std::vector<uint64_t> all;   // every candidate so far (for first-occurrence)
  while (have < num_edges) {
    uint64_t want = num_edges - have;
    uint64_t batch = want + want / 4 + 1024;
    uint64_t base = next_cand;
    all.resize(base + batch);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)batch; ++i) {
      uint32_t u, v;
      rmat_edge(eseed, base + i, scale, ta, tab, tabc, u, v);
      all[base + i] = (u == v) ? kEmpty : (((uint64_t)u << 32) | v);
    }
    next_cand = base + batch;
    std::vector<uint8_t> keep;
    first_occurrences(all, keep);
    kept.clear();
    for (uint64_t i = 0; i < all.size() && kept.size() < num_edges; ++i)
      if (keep[i]) kept.push_back(all[i]);
    have = kept.size();
  }
  const uint64_t wseed = splitmix(seed ^ 0x57474854ull);
  const uint64_t range = (uint64_t)w_hi - w_lo + 1;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)num_edges; ++i) {
    h_src[i] = (uint32_t)(kept[i] >> 32);
    h_dst[i] = (uint32_t)kept[i];
    if (h_w) h_w[i] = w_lo + (uint32_t)(rnd(wseed, i) % range);
  }
  return MK_OK;
}

mk_status mk_gen_grid(uint32_t side, uint64_t shortcuts, uint64_t seed, uint32_t w_lo,
                      uint32_t w_hi, uint32_t *h_src, uint32_t *h_dst, uint32_t *h_w,
                      uint64_t *h_num_edges) {
  if (side < 2 || (uint64_t)side * side >= 0xFFFFFFF0ull || !h_num_edges) return MK_ERR_INVALID;
  if (w_hi < w_lo) return MK_ERR_INVALID;
  const uint64_t grid_edges = 4ull * side * (side - 1);
  const uint64_t total = grid_edges + shortcuts;
  *h_num_edges = total;
  if (!h_src || !h_dst) return MK_OK;
  const uint64_t V = (uint64_t)side * side;
  // grid edges: for each vertex, right and down neighbours in both directions
#pragma omp parallel for schedule(static)
  for (int64_t r = 0; r < (int64_t)side; ++r) {
    for (uint32_t cc = 0; cc < side; ++cc) {
      const uint64_t id = (uint64_t)r * side + cc;
      // edges before row r: r * (side-1) horizontal pairs + r * side vertical pairs
      uint64_t k = 2ull * ((uint64_t)r * (side - 1) + (uint64_t)r * side);
      // within row r before column cc: cc horizontal pairs + cc vertical pairs (if r < side-1)
      k += 2ull * cc + (r + 1 < (int64_t)side ? 2ull * cc : 0ull);
      if (cc + 1 < side) {
        h_src[k] = (uint32_t)id;
        h_dst[k] = (uint32_t)(id + 1);
        h_src[k + 1] = (uint32_t)(id + 1);
        h_dst[k + 1] = (uint32_t)id;
        k += 2;
      }
      if (r + 1 < (int64_t)side) {
        h_src[k] = (uint32_t)id;
        h_dst[k] = (uint32_t)(id + side);
        h_src[k + 1] = (uint32_t)(id + side);
        h_dst[k + 1] = (uint32_t)id;
      }
    }
  }
  // shortcuts: distinct random directed pairs that are not grid neighbours
  const uint64_t sseed = splitmix(seed ^ 0x53485254ull);
  std::vector<uint64_t> cand;
  uint64_t got = 0, next = 0;
  std::vector<uint64_t> chosen;
  while (got < shortcuts) {
    uint64_t batch = (shortcuts - got) * 2 + 1024;
    uint64_t base = next;
    cand.resize(base + batch);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)batch; ++i) {
      uint64_t x = rnd(sseed, base + i);
      uint32_t u = (uint32_t)((x & 0xFFFFFFFFull) % V), v = (uint32_t)((x >> 32) % V);
      uint32_t ur = u / side, uc = u % side, vr = v / side, vc = v % side;
      bool nb = (ur == vr && (uc + 1 == vc || vc + 1 == uc)) || (uc == vc && (ur + 1 == vr || vr + 1 == ur));
      cand[base + i] = (u == v || nb) ? kEmpty : (((uint64_t)u << 32) | v);
    }
    next = base + batch;
    std::vector<uint8_t> keep;
    first_occurrences(cand, keep);
    chosen.clear();
    for (uint64_t i = 0; i < cand.size() && chosen.size() < shortcuts; ++i)
      if (keep[i]) chosen.push_back(cand[i]);
    got = chosen.size();
  }
  for (uint64_t i = 0; i < shortcuts; ++i) {
    h_src[grid_edges + i] = (uint32_t)(chosen[i] >> 32);
    h_dst[grid_edges + i] = (uint32_t)chosen[i];
  }
  if (h_w) {
    const uint64_t wseed = splitmix(seed ^ 0x57474854ull);
    const uint64_t range = (uint64_t)w_hi - w_lo + 1;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)total; ++i) h_w[i] = w_lo + (uint32_t)(rnd(wseed, i) % range);
  }
  return MK_OK;
}

mk_status mk_edgeset_create(uint32_t num_vertices, const uint32_t *h_src, const uint32_t *h_dst,
                            uint64_t n, mk_edgeset **out) {
  if (!out || num_vertices < 2 || (n && (!h_src || !h_dst))) return MK_ERR_INVALID;
  mk_edgeset *s = new mk_edgeset();
  s->V = num_vertices;
  s->edges.reserve(n);
  s->rebuild(pow2_at_least(2 * n + 16));
  for (uint64_t i = 0; i < n; ++i) {
    if (h_src[i] == h_dst[i] || h_src[i] >= num_vertices || h_dst[i] >= num_vertices) continue;
    uint64_t k = ((uint64_t)h_src[i] << 32) | h_dst[i];
    if (!s->contains(k)) s->add(k);
  }
  *out = s;
  return MK_OK;
}

mk_status mk_edgeset_destroy(mk_edgeset *s) {
  delete s;
  return MK_OK;
}

uint64_t mk_edgeset_size(const mk_edgeset *s) { return s ? s->edges.size() : 0; }

mk_status mk_edgeset_sample_absent(mk_edgeset *s, uint64_t n, uint64_t seed, uint32_t *h_src,
                                   uint32_t *h_dst) {
  if (!s || (n && (!h_src || !h_dst))) return MK_ERR_INVALID;
  const uint64_t key = splitmix(seed ^ 0x41425354ull);
  uint64_t got = 0, i = 0;
  while (got < n) {
    uint64_t x = rnd(key, i++);
    uint32_t u = (uint32_t)((x & 0xFFFFFFFFull) % s->V), v = (uint32_t)((x >> 32) % s->V);
    if (u == v) continue;
    uint64_t k = ((uint64_t)u << 32) | v;
    if (s->contains(k)) continue;
    s->add(k);
    h_src[got] = u;
    h_dst[got] = v;
    ++got;
    if (i > 64 * (n + 1024)) return MK_ERR_INVALID;  // graph too dense
  }
  return MK_OK;
}

mk_status mk_edgeset_sample_present(mk_edgeset *s, uint64_t n, uint64_t seed, uint32_t *h_src,
                                    uint32_t *h_dst) {
  if (!s || (n && (!h_src || !h_dst))) return MK_ERR_INVALID;
  if (n > s->edges.size()) return MK_ERR_INVALID;
  const uint64_t key = splitmix(seed ^ 0x50525354ull);
  for (uint64_t i = 0; i < n; ++i) {
    uint64_t idx = rnd(key, i) % s->edges.size();
    uint64_t k = s->edges[idx];
    h_src[i] = (uint32_t)(k >> 32);
    h_dst[i] = (uint32_t)k;
    s->remove_at(idx);
  }
  return MK_OK;
}

}  // extern "C"
