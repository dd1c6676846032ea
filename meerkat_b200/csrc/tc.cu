// Triangle counting on a symmetric slab graph.
//
// Reference (include/Algorithms/impl/TCImpl.cuh): Static collects all edges,
// orients each from its lower-degree endpoint and counts, per edge (u, v),
// the w in N(u) with (w, v) present, dividing the total by 6 (:149-214,
// :288-380).  Incremental/Decremental combine three batch-local counts
// (:431-565); that combination is broken as written (the batch graph is
// built with zero vertices before the mapping is known, and the decremental
// path divides by a zero load factor), so this build keeps the contract --
// the count of triangles of the current graph after each call -- and
// re-derives the update rule:
//
//   every changed undirected edge e = {a, b} (an edge the last update applied)
//   counts the triangles {a, b, w} of the new graph (insert) or of the old
//   graph (delete) whose other changed edges all order after e; each changed
//   triangle is therefore counted exactly once, at its smallest changed edge.
//
// B200 design.  Static: degree-ordered orientation (rank = (deg, id)),
// oriented CSR built from the slabs (count, scan, fill), then the forward
// algorithm: a warp stages N+(u) in a shared-memory hash set and streams
// N+(v) for every v in N+(u) with coalesced 128-byte reads; vertices with a
// large N+(u) use a block and a global-memory set.  Dynamic: one 8-lane group
// per changed edge walks the slabs of the lower-degree endpoint and probes the
// other endpoint's slab hash per candidate (one lane per candidate).
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "mk_internal.h"
#include "mk_slab.cuh"

namespace mk {

__device__ __forceinline__ bool rank_less(uint32_t du, uint32_t u, uint32_t dv, uint32_t v) {
  return du < dv || (du == dv && u < v);
}

// Oriented CSR from the slabs, one 8-lane group per bucket (balanced under
// degree skew): per-bucket counts, a scan over buckets, then the fill.
template <bool kW>
__global__ void k_orient_count(GraphView g, uint32_t *__restrict__ bcnt) {
  const Lanes L = lanes();
  const uint32_t group = (blockIdx.x * blockDim.x + threadIdx.x) >> 3;
  const uint32_t ngroups = (gridDim.x * blockDim.x) >> 3;
  for (uint32_t b = group; b < g.nbuckets; b += ngroups) {
    const uint32_t u = g.bowner[b];
    const uint32_t du = g.deg[u];
    uint32_t c = 0;
    if (du) {
      walk_bucket(g, L, b, [&](const uint4 &q) {
        uint32_t k[4], w[4];
        lane_keys<kW>(q, L.gl, k, w);
#pragma unroll
        for (int i = 0; i < keys_per_lane<kW>(); ++i)
          if (k[i] < kTombKey && k[i] != u && rank_less(du, u, g.deg[k[i]], k[i])) ++c;
      });
    }
    c = __reduce_add_sync(L.gmask, c);
    if (L.gl == 0) bcnt[b] = c;
  }
}

__global__ void k_tc_rows(const uint32_t *__restrict__ boff, uint32_t V, uint32_t nb,
                          const unsigned long long *__restrict__ bpos,
                          unsigned long long *__restrict__ row_ptr) {
  for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u <= V; u += gridDim.x * blockDim.x)
    row_ptr[u] = bpos[u < V ? boff[u] : nb];
}

template <bool kW>
__global__ void k_orient_fill(GraphView g, const unsigned long long *__restrict__ bpos,
                              uint32_t *__restrict__ ocol) {
  const Lanes L = lanes();
  const uint32_t group = (blockIdx.x * blockDim.x + threadIdx.x) >> 3;
  const uint32_t ngroups = (gridDim.x * blockDim.x) >> 3;
  for (uint32_t b = group; b < g.nbuckets; b += ngroups) {
    unsigned long long pos = bpos[b];
    const unsigned long long end = bpos[b + 1];
    if (pos == end) continue;
    const uint32_t u = g.bowner[b];
    const uint32_t du = g.deg[u];
    walk_bucket(g, L, b, [&](const uint4 &q) {
      uint32_t k[4], w[4];
      lane_keys<kW>(q, L.gl, k, w);
      uint32_t keep[4];
      uint32_t cnt = 0;
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        keep[i] = (i < keys_per_lane<kW>()) && k[i] < kTombKey && k[i] != u &&
                  rank_less(du, u, g.deg[k[i]], k[i]);
        cnt += keep[i];
      }
      uint32_t incl = cnt;
#pragma unroll
      for (int o = 1; o < 8; o <<= 1) {
        uint32_t y = __shfl_up_sync(L.gmask, incl, o, 8);
        if (L.gl >= (uint32_t)o) incl += y;
      }
      uint32_t total = __shfl_sync(L.gmask, incl, L.gbase + 7);
      unsigned long long p = pos + (incl - cnt);
#pragma unroll
      for (int i = 0; i < 4; ++i)
        if (keep[i]) {
          if (p < end) ocol[p] = k[i];
          ++p;
        }
      pos += total;
    });
  }
}

constexpr int kTcWarps = 4;           // warps per block in the small kernel (32 KB of sets)
constexpr int kTcSetCap = 2048;       // per-warp shared hash capacity (entries)
constexpr uint32_t kTcSmallMax = 1024;  // N+(u) handled by one warp

// Open-addressing sets of capacity 2^k (k >= 6), at most half full (a
// quarter where the warp's share of shared memory allows), with
// Fibonacci hashing: the slot is the top k bits of key * 2654435769 (one
// multiply and one shift per probe; the sets are probed far more often than
// built).  shift = 32 - k.  Probes are bounded by the capacity.
__device__ __forceinline__ uint32_t set_slot(uint32_t key, uint32_t shift) {
  return (key * 2654435769u) >> shift;
}

__device__ __forceinline__ void set_insert(uint32_t *set, uint32_t cap_mask, uint32_t shift,
                                           uint32_t key) {
  uint32_t h = set_slot(key, shift);
  for (uint32_t it = 0; it <= cap_mask; ++it) {
    uint32_t old = atomicCAS(set + h, kEmptyKey, key);
    if (old == kEmptyKey || old == key) return;
    h = (h + 1) & cap_mask;
  }
}

__device__ __forceinline__ bool set_contains(const uint32_t *set, uint32_t cap_mask, uint32_t shift,
                                             uint32_t key) {
  uint32_t h = set_slot(key, shift);
  for (uint32_t it = 0; it <= cap_mask; ++it) {
    uint32_t k = set[h];
    if (k == key) return true;
    if (k == kEmptyKey) return false;
    h = (h + 1) & cap_mask;
  }
  return false;
}

// Same probe for a set in global memory, read through L2 (the set is
// rebuilt for every vertex, so L1 may hold stale lines).
__device__ __forceinline__ bool set_contains_cg(const uint32_t *set, uint32_t cap_mask,
                                                uint32_t shift, uint32_t key) {
  uint32_t h = set_slot(key, shift);
  for (uint32_t it = 0; it <= cap_mask; ++it) {
    uint32_t k = __ldcg(set + h);
    if (k == key) return true;
    if (k == kEmptyKey) return false;
    h = (h + 1) & cap_mask;
  }
  return false;
}

constexpr uint32_t kTcChunk = 32;  // N+(u) entries per work item (one per lane)
constexpr int kTcSteps = 4;        // 32-entry probe steps with their loads in flight together

// Work items of the forward algorithm: (u, chunk c) covers N+(u)[32c, 32c+32).
// Per-vertex work is heavy-tailed (a hub's neighbours have long N+ lists),
// so vertices are split into chunks and handed out dynamically.  Vertices
// with N+(u) larger than kTcSmallMax go to the big list instead.
__global__ void k_tc_item_count(uint32_t V, const unsigned long long *__restrict__ orow,
                                uint32_t *__restrict__ icnt, uint32_t *big_list, uint32_t *big_n,
                                uint32_t *big_max) {
  for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < V; u += gridDim.x * blockDim.x) {
    const uint32_t du = (uint32_t)(orow[u + 1] - orow[u]);
    uint32_t c = 0;
    if (du >= 2) {  // a triangle needs two oriented edges out of u
      if (du > kTcSmallMax) {
        big_list[atomicAdd(big_n, 1u)] = u;
        atomicMax(big_max, du);
      } else
        c = (du + kTcChunk - 1) / kTcChunk;
    }
    icnt[u] = c;
  }
}

__global__ void k_tc_item_fill(uint32_t V, const uint32_t *__restrict__ icnt,
                               const unsigned long long *__restrict__ ioff,
                               unsigned long long *__restrict__ items) {
  for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < V; u += gridDim.x * blockDim.x) {
    const uint32_t c = icnt[u];
    const unsigned long long b = ioff[u];
    for (uint32_t j = 0; j < c; ++j) items[b + j] = ((unsigned long long)j << 32) | u;
  }
}

// Persistent warps take work items from a global counter.  For item (u, c)
// the warp stages N+(u) in a shared-memory hash set and streams the N+(v)
// lists of the item's 32 neighbours v as one concatenated range with
// coalesced reads, probing the set.
__global__ void __launch_bounds__(kTcWarps * 32)
    k_tc_small(const unsigned long long *__restrict__ orow, const uint32_t *__restrict__ ocol,
               const unsigned long long *__restrict__ items, const unsigned long long *nitems_p,
               uint32_t *next, unsigned long long *count) {
  __shared__ uint32_t sets[kTcWarps][kTcSetCap];
  const uint32_t lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  uint32_t *set = sets[wib];
  const unsigned long long nitems = *nitems_p;
  unsigned long long c = 0;
  uint32_t have_u = 0xFFFFFFFFu;  // vertex whose set is staged
  uint32_t cap = 64;
  for (;;) {
    uint32_t it = 0;
    if (lane == 0) it = atomicAdd(next, 1u);
    it = __shfl_sync(0xFFFFFFFFu, it, 0);
    if (it >= nitems) break;
    const unsigned long long item = items[it];
    const uint32_t u = (uint32_t)item, chunk = (uint32_t)(item >> 32);
    const unsigned long long r0 = orow[u], r1 = orow[u + 1];
    const uint32_t du = (uint32_t)(r1 - r0);
    if (u != have_u) {
      __syncwarp();
      // load at most 1/4 (1/2 for the largest sets): most probes miss, and a
      // miss walks the probe run to an EMPTY slot
      cap = 64;
      while (cap < 4 * du && cap < (uint32_t)kTcSetCap) cap <<= 1;
      for (uint32_t i = lane; i < cap; i += 32) set[i] = kEmptyKey;
      __syncwarp();
      for (uint32_t i = lane; i < du; i += 32) set_insert(set, cap - 1, __clz(cap) + 1, ocol[r0 + i]);
      __syncwarp();
      have_u = u;
    }
    // the item's (up to 32) neighbours v, one per lane; their N+(v) lists
    // are walked as one concatenated range, 32 entries per step and
    // kTcSteps steps of loads in flight, so short lists do not idle lanes
    const uint32_t shift = __clz(cap) + 1;
    const uint32_t i0 = chunk * kTcChunk, m = min(du, i0 + kTcChunk) - i0;
    unsigned long long s0 = 0;
    uint32_t len = 0;
    if (lane < m) {
      const uint32_t v = ocol[r0 + i0 + lane];
      s0 = orow[v];
      len = (uint32_t)(orow[v + 1] - s0);
    }
    uint32_t incl = len;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
      if (lane >= (uint32_t)o) incl += y;
    }
    const uint32_t off = incl - len;
    const uint32_t T = __shfl_sync(0xFFFFFFFFu, incl, 31);
    const unsigned long long basej = s0 - off;  // entry x of lane l's list is ocol[basej(l) + x]
    for (uint32_t x0 = 0; x0 < T; x0 += 32u * kTcSteps) {
      uint32_t key[kTcSteps];
#pragma unroll
      for (int q = 0; q < kTcSteps; ++q) {
        const uint32_t x = x0 + 32u * q + lane;
        uint32_t lo = 0;  // last lane whose list starts at or before x
#pragma unroll
        for (int st = 16; st > 0; st >>= 1) {
          const uint32_t cand = lo + (uint32_t)st;
          if (__shfl_sync(0xFFFFFFFFu, off, cand) <= x) lo = cand;
        }
        const unsigned long long bj = __shfl_sync(0xFFFFFFFFu, basej, lo);
        key[q] = x < T ? ocol[bj + x] : kEmptyKey;
      }
#pragma unroll
      for (int q = 0; q < kTcSteps; ++q)
        if (key[q] != kEmptyKey) c += set_contains(set, cap - 1, shift, key[q]);
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xFFFFFFFFu, c, o);
  if (lane == 0 && c) atomicAdd(count, c);
}

__global__ void k_tc_big(const unsigned long long *__restrict__ orow,
                         const uint32_t *__restrict__ ocol, const uint32_t *__restrict__ big_list,
                         const uint32_t *__restrict__ big_n, uint32_t *scratch, uint32_t cap,
                         unsigned long long *count) {
  __shared__ unsigned long long red[32];
  uint32_t *set = scratch + (size_t)blockIdx.x * cap;
  unsigned long long c = 0;
  const uint32_t nbig = *big_n;
  for (uint32_t bi = blockIdx.x; bi < nbig; bi += gridDim.x) {
    const uint32_t u = big_list[bi];
    const unsigned long long r0 = orow[u], r1 = orow[u + 1];
    const uint32_t du = (uint32_t)(r1 - r0);
    uint32_t cp = 64;
    while (cp < 2 * du && cp < cap) cp <<= 1;
    for (uint32_t i = threadIdx.x; i < cp; i += blockDim.x) set[i] = kEmptyKey;
    __syncthreads();
    const uint32_t shift = __clz(cp) + 1;
    for (uint32_t i = threadIdx.x; i < du; i += blockDim.x) set_insert(set, cp - 1, shift, ocol[r0 + i]);
    __syncthreads();
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (uint32_t i = warp; i < du; i += nw) {
      const uint32_t v = ocol[r0 + i];
      const unsigned long long s0 = orow[v], s1 = orow[v + 1];
      for (unsigned long long j = s0 + lane; j < s1; j += 32) c += set_contains_cg(set, cp - 1, shift, ocol[j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xFFFFFFFFu, c, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long t = 0;
    for (uint32_t i = 0; i < (blockDim.x >> 5); ++i) t += red[i];
    if (t) atomicAdd(count, t);
  }
}

// ---- dynamic counting ------------------------------------------------------

__device__ __forceinline__ unsigned long long pair_key(uint32_t a, uint32_t b) {
  return a < b ? ((unsigned long long)a << 32) | b : ((unsigned long long)b << 32) | a;
}

__device__ __forceinline__ unsigned long long hmix64(unsigned long long x) {
  x ^= x >> 33;
  x *= 0xff51afd7ed558ccdull;
  x ^= x >> 33;
  x *= 0xc4ceb9fe1a85ec53ull;
  x ^= x >> 33;
  return x;
}

// Elects one batch entry per changed undirected pair (lowest index).
__global__ void k_pairs_elect(const uint32_t *__restrict__ src, const uint32_t *__restrict__ dst,
                              const uint8_t *__restrict__ applied, uint32_t n,
                              unsigned long long *keys, uint32_t *idx, uint32_t mask) {
  uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n || !applied[e]) return;
  uint32_t a = src[e], b = dst[e];
  if (a == b) return;
  unsigned long long key = pair_key(a, b);
  uint32_t h = (uint32_t)hmix64(key) & mask;
  for (uint32_t it = 0; it <= mask; ++it) {
    unsigned long long k = __ldcg(keys + h);
    if (k == key) {
      atomicMin(idx + h, e);
      return;
    }
    if (k == ~0ull) {
      unsigned long long old = atomicCAS(keys + h, ~0ull, key);
      if (old == ~0ull || old == key) {
        atomicMin(idx + h, e);
        return;
      }
    }
    h = (h + 1) & mask;
  }
}

__device__ __forceinline__ uint32_t pairs_find(const unsigned long long *keys, const uint32_t *idx,
                                               uint32_t mask, unsigned long long key) {
  uint32_t h = (uint32_t)hmix64(key) & mask;
  for (uint32_t it = 0; it <= mask; ++it) {
    unsigned long long k = keys[h];
    if (k == key) return idx[h];
    if (k == ~0ull) return kEmptyKey;
    h = (h + 1) & mask;
  }
  return kEmptyKey;
}

// Batch adjacency (both directions) of the elected pairs, for deletions.
__global__ void k_pairs_degree(const uint32_t *__restrict__ src, const uint32_t *__restrict__ dst,
                               const uint8_t *__restrict__ applied, uint32_t n,
                               const unsigned long long *keys, const uint32_t *idx, uint32_t mask,
                               uint32_t *bcnt) {
  uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n || !applied[e]) return;
  uint32_t a = src[e], b = dst[e];
  if (a == b || pairs_find(keys, idx, mask, pair_key(a, b)) != e) return;
  atomicAdd(bcnt + a, 1u);
  atomicAdd(bcnt + b, 1u);
}

__global__ void k_pairs_fill(const uint32_t *__restrict__ src, const uint32_t *__restrict__ dst,
                             const uint8_t *__restrict__ applied, uint32_t n,
                             const unsigned long long *keys, const uint32_t *idx, uint32_t mask,
                             const unsigned long long *brow, uint32_t *bfill, uint32_t *bcol) {
  uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n || !applied[e]) return;
  uint32_t a = src[e], b = dst[e];
  if (a == b || pairs_find(keys, idx, mask, pair_key(a, b)) != e) return;
  bcol[brow[a] + atomicAdd(bfill + a, 1u)] = b;
  bcol[brow[b] + atomicAdd(bfill + b, 1u)] = a;
}

// Lane-level membership test of (u, v) in the slab graph.  The eight 16-byte
// loads of a slab are all issued before any is examined, so a probe costs one
// memory round trip per slab of the chain, not one per load.
template <bool kW>
__device__ __forceinline__ bool lane_find(const GraphView &g, uint32_t u, uint32_t v) {
  const uint32_t b0 = g.boff[u];
  const uint32_t nb = g.boff[u + 1] - b0;
  uint32_t s = b0 + bucket_of(v, nb);
  for (uint32_t it = 0; it < (1u << 24) && s != kNoSlab; ++it) {
    const uint4 *p = g.slabs + 8ull * s;
    uint4 q[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) q[j] = __ldg(p + j);
    bool hit = false;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      if (!kW)
        hit |= q[j].x == v || q[j].y == v || q[j].z == v || (j != 7 && q[j].w == v);
      else
        hit |= q[j].x == v || (j != 7 && q[j].z == v);
    }
    if (hit) return true;
    s = q[7].w;
  }
  return false;
}

template <bool kW>
__global__ void k_tc_delta(GraphView g, const uint32_t *__restrict__ src,
                           const uint32_t *__restrict__ dst, const uint8_t *__restrict__ applied,
                           uint32_t n, const unsigned long long *keys, const uint32_t *idx,
                           uint32_t mask, const unsigned long long *__restrict__ brow,
                           const uint32_t *__restrict__ bcol, bool deletion,
                           unsigned long long *acc) {
  const Lanes L = lanes();
  const uint32_t group = (blockIdx.x * blockDim.x + threadIdx.x) >> 3;
  const uint32_t ngroups = (gridDim.x * blockDim.x) >> 3;
  unsigned long long c = 0;
  for (uint32_t e = group; e < n; e += ngroups) {
    if (!applied[e]) continue;
    uint32_t a = src[e], b = dst[e];
    if (a == b) continue;
    const unsigned long long ke = pair_key(a, b);
    if (pairs_find(keys, idx, mask, ke) != e) continue;
    // iterate the lower-degree endpoint
    uint32_t x = a, y = b;
    uint32_t dx = g.deg[a] + (deletion ? (uint32_t)(brow[a + 1] - brow[a]) : 0u);
    uint32_t dy = g.deg[b] + (deletion ? (uint32_t)(brow[b + 1] - brow[b]) : 0u);
    if (dy < dx) {
      x = b;
      y = a;
    }
    auto consider = [&](uint32_t w) {
      if (w == x || w == y || w >= kTombKey) return;
      unsigned long long k1 = pair_key(x, w);
      if (pairs_find(keys, idx, mask, k1) != kEmptyKey && k1 < ke) return;
      unsigned long long k2 = pair_key(y, w);
      bool in_b2 = pairs_find(keys, idx, mask, k2) != kEmptyKey;
      if (in_b2 && k2 < ke) return;
      bool present = lane_find<kW>(g, y, w) || (deletion && in_b2);
      if (present) ++c;
    };
    walk_vertex(g, L, x, [&](const uint4 &q) {
      uint32_t k[4], w[4];
      lane_keys<kW>(q, L.gl, k, w);
#pragma unroll
      for (int i = 0; i < keys_per_lane<kW>(); ++i) consider(k[i]);
    });
    if (deletion) {
      for (unsigned long long j = brow[x] + L.gl; j < brow[x + 1]; j += 8) consider(bcol[j]);
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xFFFFFFFFu, c, o);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(acc, c);
}

__global__ void k_tc_apply(unsigned long long *count, const unsigned long long *acc, int sign) {
  if (sign > 0)
    *count += *acc;
  else
    *count -= *acc;
}

// ---- triangles of one vertex range of a directed graph -----------------
// The symmetrised member is never built: its edges come from a CSR export
// of the member's out-edges, each edge (u, v) probes the slab table of v for
// the reverse edge (v, u), and the symmetric degree is out + in - reciprocal.
// An undirected edge present in both directions is kept once (from its
// smaller endpoint), then oriented by (symmetric degree, id) like the static
// path, and the same forward algorithm counts.

// rowid[e] = local row of CSR edge e: one warp per row, so hubs are written
// with coalesced stores.
__global__ void k_trc_rows(const unsigned long long *__restrict__ rp, uint32_t n,
                           uint32_t *__restrict__ rowid) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = (gridDim.x * (uint64_t)blockDim.x) >> 5;
  for (uint64_t u = warp; u < n; u += nwarps)
    for (unsigned long long e = rp[u] + lane; e < rp[u + 1]; e += 32) rowid[e] = (uint32_t)u;
}

// Per edge (u, v): range check, reverse-edge probe, in-degree and
// reciprocal counts.  rflag[e] = 1 when (v, u) is present, 0 when not, 2 for
// an edge leaving the range (skipped; sets kErrInvalidId on the graph).
template <bool kW>
__global__ void k_trc_probe(GraphView g, uint32_t lo, uint32_t n, const uint32_t *__restrict__ rowid,
                            const uint32_t *__restrict__ col, unsigned long long E,
                            uint8_t *__restrict__ rflag, uint32_t *__restrict__ indeg,
                            uint32_t *__restrict__ recip) {
  for (unsigned long long e = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; e < E;
       e += (unsigned long long)gridDim.x * blockDim.x) {
    const uint32_t u = rowid[e], v = col[e];
    if (v < lo || v - lo >= n) {
      atomicOr(g.err, kErrInvalidId);
      rflag[e] = 2;
      continue;
    }
    const bool r = lane_find<kW>(g, v, lo + u);
    rflag[e] = r ? 1 : 0;
    atomicAdd(indeg + (v - lo), 1u);
    if (r) atomicAdd(recip + u, 1u);
  }
}

__global__ void k_trc_dsym(const uint32_t *__restrict__ deg, uint32_t lo, uint32_t n,
                           const uint32_t *__restrict__ indeg, const uint32_t *__restrict__ recip,
                           uint32_t *__restrict__ dsym) {
  for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < n; u += gridDim.x * blockDim.x)
    dsym[u] = deg[lo + u] + indeg[u] - recip[u];
}

// Orientation of the undirected edges: kFill = false counts the oriented
// degree of each lower-ranked endpoint, kFill = true writes the higher one
// into its row (positions taken with an atomic per row; the forward
// algorithm does not need sorted rows).
template <bool kFill>
__global__ void k_trc_orient(const uint32_t *__restrict__ rowid, const uint32_t *__restrict__ col,
                             uint32_t lo, unsigned long long E, const uint8_t *__restrict__ rflag,
                             const uint32_t *__restrict__ dsym, uint32_t *__restrict__ ocnt,
                             const unsigned long long *__restrict__ orow, uint32_t *__restrict__ ocol) {
  for (unsigned long long e = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; e < E;
       e += (unsigned long long)gridDim.x * blockDim.x) {
    const uint8_t f = rflag[e];
    if (f == 2) continue;
    const uint32_t u = rowid[e], v = col[e] - lo;
    if (f == 1 && u > v) continue;  // both directions present: keep (min, max) once
    const bool ux = rank_less(dsym[u], u, dsym[v], v);
    const uint32_t x = ux ? u : v, y = ux ? v : u;
    if (!kFill)
      atomicAdd(ocnt + x, 1u);
    else
      ocol[orow[x] + atomicAdd(ocnt + x, 1u)] = y;
  }
}

}  // namespace mk

using namespace mk;

struct mk_tc {
  mk_graph *g = nullptr;
  unsigned long long *dcount = nullptr;  // [0] count, [1] scratch accumulator
  uint32_t *small = nullptr;             // [0] big_n
  DevBuf<uint32_t> ocnt, ocol, big_list, big_scratch, bcnt, bfill, bcol, pidx;
  DevBuf<unsigned long long> orow, tmp, brow, pkeys, bpos, items;
  Timer timer;
};

struct mk_tc_range {
  mk_tc core;  // orow / ocol and the counting scratch; core.g is the directed graph
  DevBuf<unsigned long long> rp;
  DevBuf<uint32_t> col, rowid, indeg, recip, dsym;
  DevBuf<uint8_t> rflag;
};

static int groups_grid(uint64_t items, int device) {
  uint64_t b = items * 8 / 256 + 1;
  uint64_t cap = (uint64_t)device_sm_count(device) * 8;
  return (int)std::min(b, cap);
}

static mk_status tc_count_oriented(mk_tc *t, uint32_t V, int device, cudaStream_t s);

static mk_status tc_static(mk_tc *t, cudaStream_t s) {
  mk_graph *g = t->g;
  const uint32_t V = g->V;
  const uint32_t nb = (uint32_t)g->num_buckets;
  size_t acc = 0;
  MK_CHECK(t->ocnt.reserve(nb, &acc));
  MK_CHECK(t->bpos.reserve((size_t)nb + 1, &acc));
  MK_CHECK(t->orow.reserve((size_t)V + 1, &acc));
  GraphView gv = g->view();
  int blocks = groups_grid(nb, g->device);
  if (g->weighted)
    k_orient_count<true><<<blocks, 256, 0, s>>>(gv, t->ocnt.ptr);
  else
    k_orient_count<false><<<blocks, 256, 0, s>>>(gv, t->ocnt.ptr);
  MK_CHECK(scan_u32_to_u64(t->ocnt.ptr, t->bpos.ptr, nb, t->tmp, s));
  k_tc_rows<<<(V + 256) / 256, 256, 0, s>>>(g->boff, V, nb, t->bpos.ptr, t->orow.ptr);
  unsigned long long total = 0;
  MK_CUDA(cudaMemcpyAsync(&total, t->bpos.ptr + nb, 8, cudaMemcpyDeviceToHost, s));
  MK_CUDA(cudaStreamSynchronize(s));
  MK_CHECK(t->ocol.reserve(std::max<unsigned long long>(total, 1), &acc));
  if (g->weighted)
    k_orient_fill<true><<<blocks, 256, 0, s>>>(gv, t->bpos.ptr, t->ocol.ptr);
  else
    k_orient_fill<false><<<blocks, 256, 0, s>>>(gv, t->bpos.ptr, t->ocol.ptr);
  MK_CUDA(cudaGetLastError());
  return tc_count_oriented(t, V, g->device, s);
}

// The forward algorithm on the oriented CSR in t->orow / t->ocol over V
// vertices; the count lands in t->dcount[0].  t->ocnt (>= V words) and
// t->bpos (>= V + 1) serve as scratch.
static mk_status tc_count_oriented(mk_tc *t, uint32_t V, int device, cudaStream_t s) {
  size_t acc = 0;
  MK_CHECK(t->big_list.reserve(V, &acc));
  MK_CUDA(cudaMemsetAsync(t->dcount, 0, 8, s));
  // [0] big count, [1] work-item counter, [2] largest big oriented degree
  MK_CUDA(cudaMemsetAsync(t->small, 0, 16, s));
  // work items (the orientation scratch is free again: ocnt >= V words,
  // bpos >= V + 1)
  const int vb = (int)std::min<uint64_t>((uint64_t)V / 256 + 1, (uint64_t)device_sm_count(device) * 8);
  k_tc_item_count<<<vb, 256, 0, s>>>(V, t->orow.ptr, t->ocnt.ptr, t->big_list.ptr, t->small,
                                     t->small + 2);
  MK_CHECK(scan_u32_to_u64(t->ocnt.ptr, t->bpos.ptr, V, t->tmp, s));
  unsigned long long nitems = 0;
  uint32_t hs[4] = {0, 0, 0, 0};  // [0] big vertices, [2] their largest oriented degree
  MK_CUDA(cudaMemcpyAsync(&nitems, t->bpos.ptr + V, 8, cudaMemcpyDeviceToHost, s));
  MK_CUDA(cudaMemcpyAsync(hs, t->small, 16, cudaMemcpyDeviceToHost, s));
  MK_CUDA(cudaStreamSynchronize(s));
  MK_CHECK(t->items.reserve(std::max<unsigned long long>(nitems, 1), &acc));
  k_tc_item_fill<<<vb, 256, 0, s>>>(V, t->ocnt.ptr, t->bpos.ptr, t->items.ptr);
  int per_sm = 0;
  MK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_tc_small, kTcWarps * 32, 0));
  const int sblocks = device_sm_count(device) * std::max(per_sm, 1);
  k_tc_small<<<sblocks, kTcWarps * 32, 0, s>>>(t->orow.ptr, t->ocol.ptr, t->items.ptr,
                                              t->bpos.ptr + V, t->small + 1, t->dcount);
  // big vertices: one block each, global-memory set
  const uint32_t nbig = hs[0];
  if (nbig) {
    // capacity: next power of two >= 2 * largest oriented degree of a big vertex
    const uint32_t mx = hs[2];
    uint32_t cap = 64;
    while (cap < 2ull * mx) cap <<= 1;
    int bb = std::min<uint32_t>(nbig, (uint32_t)device_sm_count(device) * 2);
    MK_CHECK(t->big_scratch.reserve((size_t)bb * cap, &acc));
    k_tc_big<<<bb, 512, 0, s>>>(t->orow.ptr, t->ocol.ptr, t->big_list.ptr, t->small,
                                t->big_scratch.ptr, cap, t->dcount);
  }
  MK_CUDA(cudaGetLastError());
  return MK_OK;
}

static mk_status tc_dynamic(mk_tc *t, const uint32_t *d_src, const uint32_t *d_dst,
                            uint32_t n, bool deletion, void *stream, float *ms_out) {
  mk_graph *g = t->g;
  DeviceGuard dg(g->device);
  cudaStream_t s = as_stream(stream);
  MK_CHECK(t->timer.start(s, ms_out != nullptr));
  const bool matches = n == g->last_n && d_src == g->last_src && d_dst == g->last_dst &&
                       g->last_op == (deletion ? 2 : 1);
  if (!matches) {
    // the batch is not the one the graph just applied: recount from scratch
    MK_CHECK(tc_static(t, s));
    return t->timer.stop(ms_out);
  }
  if (n == 0) return t->timer.stop(ms_out);
  size_t acc = 0;
  uint32_t cap = 1024;
  while (cap < 2ull * n) cap <<= 1;
  MK_CHECK(t->pkeys.reserve(cap, &acc));
  MK_CHECK(t->pidx.reserve(cap, &acc));
  MK_CUDA(cudaMemsetAsync(t->pkeys.ptr, 0xFF, (size_t)cap * 8, s));
  MK_CUDA(cudaMemsetAsync(t->pidx.ptr, 0xFF, (size_t)cap * 4, s));
  const uint8_t *applied = g->applied.ptr;
  k_pairs_elect<<<(n + 255) / 256, 256, 0, s>>>(d_src, d_dst, applied, n, t->pkeys.ptr,
                                                t->pidx.ptr, cap - 1);
  const uint32_t V = g->V;
  if (deletion) {
    MK_CHECK(t->bcnt.reserve(V, &acc));
    MK_CHECK(t->bfill.reserve(V, &acc));
    MK_CHECK(t->brow.reserve((size_t)V + 1, &acc));
    MK_CHECK(t->bcol.reserve(2ull * n + 1, &acc));
    MK_CUDA(cudaMemsetAsync(t->bcnt.ptr, 0, (size_t)V * 4, s));
    MK_CUDA(cudaMemsetAsync(t->bfill.ptr, 0, (size_t)V * 4, s));
    k_pairs_degree<<<(n + 255) / 256, 256, 0, s>>>(d_src, d_dst, applied, n, t->pkeys.ptr,
                                                   t->pidx.ptr, cap - 1, t->bcnt.ptr);
    MK_CHECK(scan_u32_to_u64(t->bcnt.ptr, t->brow.ptr, V, t->tmp, s));
    k_pairs_fill<<<(n + 255) / 256, 256, 0, s>>>(d_src, d_dst, applied, n, t->pkeys.ptr,
                                                 t->pidx.ptr, cap - 1, t->brow.ptr,
                                                 t->bfill.ptr, t->bcol.ptr);
  }
  MK_CUDA(cudaMemsetAsync(t->dcount + 1, 0, 8, s));
  int blocks = groups_grid(n, g->device);
  if (g->weighted)
    k_tc_delta<true><<<blocks, 256, 0, s>>>(g->view(), d_src, d_dst, applied, n, t->pkeys.ptr,
                                            t->pidx.ptr, cap - 1, t->brow.ptr, t->bcol.ptr,
                                            deletion, t->dcount + 1);
  else
    k_tc_delta<false><<<blocks, 256, 0, s>>>(g->view(), d_src, d_dst, applied, n, t->pkeys.ptr,
                                             t->pidx.ptr, cap - 1, t->brow.ptr, t->bcol.ptr,
                                             deletion, t->dcount + 1);
  k_tc_apply<<<1, 1, 0, s>>>(t->dcount, t->dcount + 1, deletion ? -1 : 1);
  MK_CUDA(cudaGetLastError());
  return t->timer.stop(ms_out);
}

extern "C" {

mk_status mk_tc_create(mk_graph *g, mk_tc **out) {
  if (!g || !out) return fail(MK_ERR_INVALID, "mk_tc_create: null argument");
  DeviceGuard dg(g->device);
  mk_tc *t = new mk_tc();
  t->g = g;
  cudaError_t e = cudaMalloc(&t->dcount, 16);
  if (e == cudaSuccess) e = cudaMalloc(&t->small, 16);
  if (e == cudaSuccess) e = cudaMemset(t->dcount, 0, 16);
  if (e != cudaSuccess) {
    mk_tc_destroy(t);
    return cuda_fail(e, "mk_tc_create");
  }
  *out = t;
  return MK_OK;
}

mk_status mk_tc_static(mk_tc *t, void *stream, float *ms_out) {
  if (!t) return fail(MK_ERR_INVALID, "mk_tc_static: null handle");
  DeviceGuard dg(t->g->device);
  cudaStream_t s = as_stream(stream);
  MK_CHECK(t->timer.start(s, ms_out != nullptr));
  MK_CHECK(tc_static(t, s));
  return t->timer.stop(ms_out);
}

mk_status mk_tc_incremental(mk_tc *t, const uint32_t *d_src, const uint32_t *d_dst,
                            uint32_t n, void *stream, float *ms_out) {
  if (!t) return fail(MK_ERR_INVALID, "mk_tc_incremental: null handle");
  return tc_dynamic(t, d_src, d_dst, n, false, stream, ms_out);
}

mk_status mk_tc_decremental(mk_tc *t, const uint32_t *d_src, const uint32_t *d_dst,
                            uint32_t n, void *stream, float *ms_out) {
  if (!t) return fail(MK_ERR_INVALID, "mk_tc_decremental: null handle");
  return tc_dynamic(t, d_src, d_dst, n, true, stream, ms_out);
}

mk_status mk_tc_count(mk_tc *t, uint64_t *h_count) {
  if (!t || !h_count) return fail(MK_ERR_INVALID, "mk_tc_count: null argument");
  DeviceGuard dg(t->g->device);
  MK_CUDA(cudaDeviceSynchronize());
  unsigned long long c = 0;
  MK_CUDA(cudaMemcpy(&c, t->dcount, 8, cudaMemcpyDeviceToHost));
  *h_count = c;
  return MK_OK;
}

mk_status mk_tc_range_create(mk_graph *g, mk_tc_range **out) {
  if (!g || !out) return fail(MK_ERR_INVALID, "mk_tc_range_create: null argument");
  if (g->reverse) return fail(MK_ERR_INVALID, "mk_tc_range_create: needs an out-edge graph");
  *out = nullptr;
  DeviceGuard dg(g->device);
  mk_tc_range *t = new mk_tc_range();
  t->core.g = g;
  cudaError_t e = cudaMalloc(&t->core.dcount, 16);
  if (e == cudaSuccess) e = cudaMalloc(&t->core.small, 16);
  if (e == cudaSuccess) e = cudaMemset(t->core.dcount, 0, 16);
  if (e != cudaSuccess) {
    mk_tc_range_destroy(t);
    return cuda_fail(e, "mk_tc_range_create");
  }
  *out = t;
  return MK_OK;
}

mk_status mk_tc_range_run(mk_tc_range *t, uint32_t v_begin, uint32_t v_end, void *stream,
                          float *ms_out) {
  if (!t) return fail(MK_ERR_INVALID, "mk_tc_range_run: null handle");
  mk_graph *g = t->core.g;
  if (v_begin >= v_end || v_end > g->V) return fail(MK_ERR_INVALID, "mk_tc_range_run: bad vertex range");
  DeviceGuard dg(g->device);
  cudaStream_t s = as_stream(stream);
  MK_CHECK(t->core.timer.start(s, ms_out != nullptr));
  const uint32_t lo = v_begin, n = v_end - v_begin;
  uint64_t E = 0;
  MK_CHECK(mk_graph_count_edges_range(g, v_begin, v_end, stream, &E));
  const size_t e1 = std::max<uint64_t>(E, 1);
  size_t acc = 0;
  MK_CHECK(t->rp.reserve((size_t)n + 1, &acc));
  MK_CHECK(t->col.reserve(e1, &acc));
  MK_CHECK(t->rowid.reserve(e1, &acc));
  MK_CHECK(t->rflag.reserve(e1, &acc));
  MK_CHECK(t->indeg.reserve(n, &acc));
  MK_CHECK(t->recip.reserve(n, &acc));
  MK_CHECK(t->dsym.reserve(n, &acc));
  mk_tc *c = &t->core;
  MK_CHECK(c->ocnt.reserve(n, &acc));
  MK_CHECK(c->bpos.reserve((size_t)n + 1, &acc));
  MK_CHECK(c->orow.reserve((size_t)n + 1, &acc));
  MK_CHECK(c->ocol.reserve(e1, &acc));
  MK_CHECK(mk_graph_export_csr_range(g, v_begin, v_end, reinterpret_cast<uint64_t *>(t->rp.ptr),
                                     t->col.ptr, nullptr, stream));
  MK_CUDA(cudaMemsetAsync(t->indeg.ptr, 0, (size_t)n * 4, s));
  MK_CUDA(cudaMemsetAsync(t->recip.ptr, 0, (size_t)n * 4, s));
  MK_CUDA(cudaMemsetAsync(c->ocnt.ptr, 0, (size_t)n * 4, s));
  const int sms = device_sm_count(g->device);
  const int rb = (int)std::min<uint64_t>((uint64_t)n / 8 + 1, (uint64_t)sms * 8);
  k_trc_rows<<<rb, 256, 0, s>>>(t->rp.ptr, n, t->rowid.ptr);
  const int eb = (int)std::min<uint64_t>(E / 256 + 1, (uint64_t)sms * 16);
  if (g->weighted)
    k_trc_probe<true><<<eb, 256, 0, s>>>(g->view(), lo, n, t->rowid.ptr, t->col.ptr, E,
                                         t->rflag.ptr, t->indeg.ptr, t->recip.ptr);
  else
    k_trc_probe<false><<<eb, 256, 0, s>>>(g->view(), lo, n, t->rowid.ptr, t->col.ptr, E,
                                          t->rflag.ptr, t->indeg.ptr, t->recip.ptr);
  const int vb = (int)std::min<uint64_t>((uint64_t)n / 256 + 1, (uint64_t)sms * 8);
  k_trc_dsym<<<vb, 256, 0, s>>>(g->deg, lo, n, t->indeg.ptr, t->recip.ptr, t->dsym.ptr);
  k_trc_orient<false><<<eb, 256, 0, s>>>(t->rowid.ptr, t->col.ptr, lo, E, t->rflag.ptr,
                                         t->dsym.ptr, c->ocnt.ptr, nullptr, nullptr);
  MK_CHECK(scan_u32_to_u64(c->ocnt.ptr, c->orow.ptr, n, c->tmp, s));
  MK_CUDA(cudaMemsetAsync(c->ocnt.ptr, 0, (size_t)n * 4, s));
  k_trc_orient<true><<<eb, 256, 0, s>>>(t->rowid.ptr, t->col.ptr, lo, E, t->rflag.ptr,
                                        t->dsym.ptr, c->ocnt.ptr, c->orow.ptr, c->ocol.ptr);
  MK_CUDA(cudaGetLastError());
  MK_CHECK(tc_count_oriented(c, n, g->device, s));
  return c->timer.stop(ms_out);
}

mk_status mk_tc_range_count(mk_tc_range *t, uint64_t *h_count) {
  if (!t) return fail(MK_ERR_INVALID, "mk_tc_range_count: null handle");
  return mk_tc_count(&t->core, h_count);
}

mk_status mk_tc_range_count_async(mk_tc_range *t, uint64_t *h_count, void *stream) {
  if (!t || !h_count) return fail(MK_ERR_INVALID, "mk_tc_range_count_async: null argument");
  DeviceGuard dg(t->core.g->device);
  MK_CUDA(cudaMemcpyAsync(h_count, t->core.dcount, 8, cudaMemcpyDeviceToHost, as_stream(stream)));
  return MK_OK;
}

mk_status mk_tc_range_destroy(mk_tc_range *t) {
  if (!t) return MK_OK;
  DeviceGuard dg(t->core.g->device);
  t->rp.release();
  t->col.release();
  t->rowid.release();
  t->indeg.release();
  t->recip.release();
  t->dsym.release();
  t->rflag.release();
  // the core's buffers are released by its own destructor path
  mk_tc *c = &t->core;
  cudaFree(c->dcount);
  cudaFree(c->small);
  c->ocnt.release();
  c->ocol.release();
  c->big_list.release();
  c->big_scratch.release();
  c->orow.release();
  c->tmp.release();
  c->bpos.release();
  c->items.release();
  delete t;
  return MK_OK;
}

mk_status mk_tc_destroy(mk_tc *t) {
  if (!t) return MK_OK;
  DeviceGuard dg(t->g->device);
  cudaFree(t->dcount);
  cudaFree(t->small);
  t->ocnt.release();
  t->ocol.release();
  t->big_list.release();
  t->big_scratch.release();
  t->bcnt.release();
  t->bfill.release();
  t->bcol.release();
  t->pidx.release();
  t->orow.release();
  t->tmp.release();
  t->brow.release();
  t->pkeys.release();
  t->bpos.release();
  t->items.release();
  delete t;
  return MK_OK;
}

}  // extern "C"
