// BFS and SSSP: static, incremental and decremental, one persistent
// cooperative launch per call.
//
// Reference semantics followed (include/Algorithms/impl/BFSImpl.cuh,
// include/Algorithms/impl/SSSPImpl.cuh):
//   * distances are packed dist<<32 | parent in a u64 and relaxed with
//     atomicMin (definitions.cuh:14-17, BFSImpl.cuh:307-314); the source holds
//     PACK(0, src) (BFS.cuh:47-52); unreachable = INFINF;
//   * incremental: after the inserts are in the graph, every batch edge (s, d)
//     with finite dist[s] seeds d, then frontier relaxation runs to a fixed
//     point (BFSImpl.cuh:296-381, SSSPImpl.cuh:280-364);
//   * decremental: a deleted edge (s, d) with PARENT(dist[d]) == s
//     invalidates d and its whole shortest-path subtree; invalidated vertices
//     are re-seeded from valid in-neighbours and relaxed again
//     (BFSImpl.cuh:3-42, :384-496).
//
// B200 design differences:
//   * vertex frontiers (not edge frontiers), deduplicated per level with a
//     stamp word per vertex, staged in a shared-memory queue per block;
//   * the subtree is invalidated level by level along tree edges
//     (O(sum of subtree out-degrees)) instead of walking every vertex's parent
//     chain (O(V * depth), BFSImpl.cuh:17-42);
//   * re-seeding streams every valid vertex's slabs once (the reference's own
//     strategy, BFSImpl.cuh:419-440), skipping vertices of degree 0;
//   * the stored edge weight is probed for every seeding batch edge, so a
//     batch entry that did not change the graph cannot seed a wrong distance;
//   * frontier entries are work items (vertex, chunk of `chunk` buckets), so a
//     hub's buckets spread over many 8-lane groups instead of one; a group
//     reads 128-byte slabs with 16-byte loads, up to 4 head slabs at once;
//   * the re-seed sweep runs over buckets (bucket -> owner map), not vertices,
//     so it is balanced whatever the degree skew;
//   * grid-wide barriers are bounded (MK_ERR_TIMEOUT, never a hang).
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "mk_internal.h"
#include "mk_slab.cuh"
#include "mk_members.cuh"

namespace mk {

enum TravMode : uint32_t { kStatic = 0, kIncremental = 1, kDecremental = 2 };

// ctl words (u32)
enum Ctl : int {
  kBar0 = 0,      // barrier arrival
  kBar1 = 1,      // barrier generation
  kErr = 2,       // sticky error bits
  kThr = 3,       // near-far SSSP: distance threshold of the near frontier
  kSz0 = 4,       // frontier sizes kSz0 + (level % 3): words 4, 5, 6
  kRestart = 7,   // decremental: 1 when the call recomputed from the sources
  kInvCount = 8,  // invalidated vertices so far (append cursor of inv_list)
  kLevels = 9,    // relaxation levels run by the last call
  kDSz0 = 10,     // invalidation frontier sizes kDSz0 + (level % 3)
  kFarN0 = 13,    // near-far SSSP: far list sizes kFarN0 + (list 0 / 1): words 13, 14
  kRound = 15,    // stamp base, persists across calls
  kFarMin0 = 16,  // near-far SSSP: smallest distance on far list 0 / 1 (set in-kernel)
  kTrimN = 20,    // BFS repair: seeds (heads of deleted tree edges)
  kTrimLo = 21,   // BFS repair: lowest / highest seed level
  kTrimHi = 22,
  kTCand0 = 23,   // BFS repair: candidate list sizes, words 23, 24 (round parity)
  kTItem0 = 25,   // BFS repair: support-search item counts, words 25, 26
  kTChild = 27,   // BFS repair: child-scan items of the level
  kTReseed = 28,  // decremental with a reverse graph: re-seed items
  kEarly = 29,    // decremental: deleted tree edges counted before an immediate recompute
  kCtlWords = 32
};
constexpr uint32_t kRepairChunk = 8;  // buckets per repair / re-seed work item
constexpr uint32_t kTrimMaxRounds = 256;  // BFS repair levels before a recompute

struct TravArgs {
  GraphView g;
  unsigned long long *dist;
  uint32_t *stamp;
  uint32_t *inval;  // bitmap, one bit per vertex
  unsigned long long *fr0;  // work items (chunk << 32 | vertex)
  unsigned long long *fr1;
  uint32_t *inv_list;
  uint32_t *ctl;
  unsigned long long *pushed;
  const uint32_t *bsrc;
  const uint32_t *bdst;
  uint32_t bn;
  const uint32_t *sources;  // distinct source vertices (one per query)
  uint32_t nsources;
  uint32_t chunk;           // buckets per frontier work item
  uint32_t mode;
  uint32_t delta;           // near-far SSSP step (0: plain level-synchronous)
  uint32_t recompute_inv;   // decremental: invalidated vertices from which to recompute (0: never)
  GraphView rg;             // in-edges of the same graph (static BFS pull levels), rg.V == 0: none
  uint32_t pull_items;      // static BFS: frontier size from which a level is pulled (0: never)
  uint32_t *far0, *far1;    // far lists (vertex ids), one is appended at a time
  uint32_t *fbits;          // bit per vertex: on a far list
  unsigned long long limit_ns;
  // decremental with the reverse graph: BFS repair (trim != 0) -- seeds
  // (level << 32 | vertex), candidate lists and support-search items per
  // round parity, child-scan items, each candidate's best support (tpar,
  // kEmptyKey when none) -- and the chunked re-seed items (BFS and SSSP)
  uint32_t trim;
  unsigned long long *tseeds;
  uint32_t *tcand0, *tcand1, *tpar;
  unsigned long long *titems0, *titems1, *tchild, *treseed;
};

constexpr int kTravBlock = 256;
constexpr int kQueueCap = 2048;
constexpr uint32_t kDefaultChunk = 4;  // buckets per frontier work item

__host__ __device__ __forceinline__ unsigned long long item(uint32_t v, uint32_t chunk) {
  return ((unsigned long long)chunk << 32) | v;
}

struct BlockQueue {
  unsigned long long *q;
  uint32_t *qn;
};

// Pushes vertex v as ceil(buckets / chunk) work items.
__device__ __forceinline__ void push_vertex(const TravArgs &a, const BlockQueue &Q, uint32_t v,
                                            unsigned long long *gfr, uint32_t *gsz) {
  const uint32_t nb = a.g.boff[v + 1] - a.g.boff[v];
  const uint32_t k = (nb + a.chunk - 1) / a.chunk;
  if (k <= 1) {
    uint32_t pos = atomicAdd(Q.qn, 1u);
    if (pos < kQueueCap) {
      Q.q[pos] = item(v, 0);
    } else {
      gfr[atomicAdd(gsz, 1u)] = item(v, 0);
    }
  } else {
    uint32_t base = atomicAdd(gsz, k);
    for (uint32_t j = 0; j < k; ++j) gfr[base + j] = item(v, j);
  }
}

// Work items (chunk << 32 | v) over v's buckets in `gv`, kRepairChunk
// buckets each (one item for a vertex with no bucket beyond the first).
__device__ __forceinline__ void push_items(const GraphView &gv, uint32_t v, unsigned long long *list,
                                           uint32_t *cnt) {
  const uint32_t nb = gv.boff[v + 1] - gv.boff[v];
  const uint32_t k = max(1u, (nb + kRepairChunk - 1) / kRepairChunk);
  const uint32_t base = atomicAdd(cnt, k);
  for (uint32_t j = 0; j < k; ++j) list[base + j] = item(v, j);
}

// The vertex and bucket range [b0, b1) of a work item of push_items.
__device__ __forceinline__ void item_buckets(const GraphView &gv, unsigned long long it, uint32_t &v,
                                             uint32_t &b0, uint32_t &b1) {
  v = (uint32_t)it;
  const uint32_t c = (uint32_t)(it >> 32);
  const uint32_t s = gv.boff[v], e = gv.boff[v + 1];
  b0 = min(s + c * kRepairChunk, e);
  b1 = min(b0 + kRepairChunk, e);
}

// Frontier buffers, sizes and dist words are rewritten by other SMs inside
// this launch, so every read of them goes through L2 (__ldcg / acquire).

// Flushes the block queue into the global frontier; all threads call it.
__device__ __forceinline__ void queue_flush(const BlockQueue &Q, unsigned long long *gfr,
                                            uint32_t *gsz, unsigned long long *pushed,
                                            uint32_t *base_s) {
  __syncthreads();
  uint32_t cnt = min(*Q.qn, (uint32_t)kQueueCap);
  if (threadIdx.x == 0) {
    *base_s = cnt ? atomicAdd(gsz, cnt) : 0u;
    uint32_t total = *Q.qn;
    if (total) atomicAdd(pushed, (unsigned long long)total);
  }
  __syncthreads();
  uint32_t base = *base_s;
  for (uint32_t i = threadIdx.x; i < cnt; i += blockDim.x) gfr[base + i] = Q.q[i];
  __syncthreads();
  if (threadIdx.x == 0) *Q.qn = 0;
  __syncthreads();
}

__device__ __forceinline__ bool inval_test(const uint32_t *bits, uint32_t v) {
  return (__ldcg(bits + (v >> 5)) >> (v & 31)) & 1u;
}
// Sets v's bit; true if this call set it.
__device__ __forceinline__ bool inval_set(uint32_t *bits, uint32_t v) {
  uint32_t m = 1u << (v & 31);
  return (atomicOr(bits + (v >> 5), m) & m) == 0;
}

__device__ __forceinline__ unsigned long long ld_dist(const unsigned long long *p) {
  return __ldcg(p);
}

// Near-far split of static SSSP: an improved vertex whose new distance is
// below `thr` joins the next level; otherwise it goes (once) onto the far
// list, which is drained when the near frontier runs dry.  thr = kNoFar
// sends everything to the next level.
constexpr uint32_t kNoFar = 0xFFFFFFFFu;
struct NearFar {
  uint32_t thr;
  uint32_t *far;   // list being appended
  uint32_t *farn;  // its size
};

__device__ __forceinline__ void far_push(const TravArgs &a, const NearFar &nf, uint32_t v) {
  const uint32_t m = 1u << (v & 31);
  if ((atomicOr(a.fbits + (v >> 5), m) & m) == 0) nf.far[atomicAdd(nf.farn, 1u)] = v;
}

// Pushes v, whose distance just improved to nd, to the next level or the far list.
__device__ __forceinline__ void push_improved(const TravArgs &a, const BlockQueue &Q,
                                              const NearFar &nf, uint32_t v,
                                              unsigned long long nd, uint32_t stamp_next,
                                              unsigned long long *gfr, uint32_t *gsz) {
  if (nd < nf.thr) {
    if (atomicExch(a.stamp + v, stamp_next) != stamp_next) push_vertex(a, Q, v, gfr, gsz);
  } else {
    far_push(a, nf, v);
  }
}

// Relaxes v with candidate distance nd via parent u; pushes v on improvement.
__device__ __forceinline__ void relax(const TravArgs &a, const BlockQueue &Q, const NearFar &nf,
                                      uint32_t v, unsigned long long nd, uint32_t u,
                                      uint32_t stamp_next, unsigned long long *gfr,
                                      uint32_t *gsz) {
  if (nd >= kInf) return;
  unsigned long long cur = ld_dist(a.dist + v);
  if (nd >= pack_hi(cur)) return;
  unsigned long long cand = pack((uint32_t)nd, u);
  unsigned long long old = atomicMin(a.dist + v, cand);
  if (pack_hi(old) > nd) push_improved(a, Q, nf, v, nd, stamp_next, gfr, gsz);
}

// Relaxes the live out-neighbours held by one slab quarter.
template <bool kW, bool kUseW>
__device__ __forceinline__ void relax_slab(const TravArgs &a, const Lanes &L,
                                           const BlockQueue &Q, const NearFar &nf,
                                           const uint4 &q, uint32_t u,
                                           uint32_t du, uint32_t stamp_next,
                                           unsigned long long *gfr, uint32_t *gsz,
                                           bool only_invalid) {
  uint32_t k[4], w[4];
  lane_keys<kW>(q, L.gl, k, w);
#pragma unroll
  for (int i = 0; i < keys_per_lane<kW>(); ++i) {
    uint32_t v = k[i];
    if (v < kTombKey && v != u) {
      if (only_invalid && !inval_test(a.inval, v)) continue;
      unsigned long long nd = (unsigned long long)du + (kUseW ? w[i] : 1u);
      relax(a, Q, nf, v, nd, u, stamp_next, gfr, gsz);
    }
  }
}

// Relaxes the keys of up to 4 slab quarters at once: every dist word is
// loaded before any is used, so a lane keeps up to 16 loads in flight.
template <bool kW, bool kUseW>
__device__ __forceinline__ void relax_slabs4(const TravArgs &a, const Lanes &L,
                                             const BlockQueue &Q, const NearFar &nf,
                                             const uint4 (&q)[4], uint32_t nq,
                                             uint32_t u, uint32_t du, uint32_t stamp_next,
                                             unsigned long long *gfr, uint32_t *gsz) {
  constexpr int KP = keys_per_lane<kW>();
  uint32_t k[4][4], w[4][4];
  unsigned long long cur[4][KP];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    lane_keys<kW>(q[j], L.gl, k[j], w[j]);
#pragma unroll
    for (int i = 0; i < KP; ++i) {
      const uint32_t v = k[j][i];
      const bool live = (uint32_t)j < nq && v < kTombKey && v != u;
      if (!live) k[j][i] = kEmptyKey;
      cur[j][i] = live ? ld_dist(a.dist + v) : 0ull;
    }
  }
#pragma unroll
  for (int j = 0; j < 4; ++j) {
#pragma unroll
    for (int i = 0; i < KP; ++i) {
      const uint32_t v = k[j][i];
      if (v == kEmptyKey) continue;
      const unsigned long long nd = (unsigned long long)du + (kUseW ? w[j][i] : 1u);
      if (nd >= kInf || nd >= pack_hi(cur[j][i])) continue;
      const unsigned long long old = atomicMin(a.dist + v, pack((uint32_t)nd, u));
      if (pack_hi(old) > nd) push_improved(a, Q, nf, v, nd, stamp_next, gfr, gsz);
    }
  }
}

// Expands buckets [b0, b1) of vertex u: head slabs 4 at a time (batched
// relaxation), overflow chains slab by slab.
template <bool kW, bool kUseW>
__device__ __forceinline__ void expand_range(const TravArgs &a, const Lanes &L,
                                             const BlockQueue &Q, const NearFar &nf, uint32_t u,
                                             uint32_t du,
                                             uint32_t b0, uint32_t b1, uint32_t stamp_next,
                                             unsigned long long *gfr, uint32_t *gsz) {
  for (uint32_t b = b0; b < b1; b += 4) {
    const uint32_t nq = min(4u, b1 - b);
    uint4 q[4];
#pragma unroll
    for (int j = 0; j < 4; ++j)
      q[j] = ((uint32_t)j < nq) ? ld_slab_ro(a.g.slabs + 8ull * (b + j) + L.gl)
                                : make_uint4(kEmptyKey, kEmptyKey, kEmptyKey, kNoSlab);
    relax_slabs4<kW, kUseW>(a, L, Q, nf, q, nq, u, du, stamp_next, gfr, gsz);
    // overflow chains level by level: the next slabs of all running chains
    // are loaded together (a finished chain contributes an empty slab)
    uint32_t nx[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) nx[j] = __shfl_sync(L.gmask, q[j].w, L.gbase + 7);
    while ((nx[0] & nx[1] & nx[2] & nx[3]) != kNoSlab) {
#pragma unroll
      for (int j = 0; j < 4; ++j)
        q[j] = nx[j] != kNoSlab ? ld_slab_ro(a.g.slabs + 8ull * nx[j] + L.gl)
                                : make_uint4(kEmptyKey, kEmptyKey, kEmptyKey, kNoSlab);
      relax_slabs4<kW, kUseW>(a, L, Q, nf, q, 4u, u, du, stamp_next, gfr, gsz);
#pragma unroll
      for (int j = 0; j < 4; ++j) nx[j] = __shfl_sync(L.gmask, q[j].w, L.gbase + 7);
    }
  }
}

// Bucket range of a work item.
__device__ __forceinline__ void item_range(const GraphView &g, unsigned long long it, uint32_t chunk,
                                           uint32_t &v, uint32_t &b0, uint32_t &b1) {
  v = (uint32_t)it;
  const uint32_t c = (uint32_t)(it >> 32);
  const uint32_t lo = g.boff[v], hi = g.boff[v + 1];
  b0 = lo + c * chunk;
  b1 = min(hi, b0 + chunk);
}

// A source holds PACK(0, itself) (BFS.cuh:47-52) and is the only vertex whose
// parent is itself, so sources are never invalidated.
__device__ __forceinline__ bool is_source(unsigned long long p, uint32_t v) {
  return p == pack(0, v);
}

// Bottom-up BFS level: every unvisited vertex walks its in-edges (in the
// reverse graph) until it meets a vertex on level lvl; it then takes level
// lvl + 1 with that parent and joins the next frontier.  One 8-lane group per
// vertex, stopping at the first slab that holds a parent.
template <bool kRW>
__device__ __forceinline__ void pull_level(const TravArgs &a, const Lanes &L, const BlockQueue &Q,
                                           uint32_t group, uint32_t ngroups, uint32_t lvl,
                                           uint32_t stamp_next, unsigned long long *nxt,
                                           uint32_t *nsz) {
  const GraphView &rg = a.rg;
  for (uint32_t v = group; v < rg.V; v += ngroups) {
    unsigned long long pv = 0;
    if (L.gl == 0) pv = ld_dist(a.dist + v);
    pv = __shfl_sync(L.gmask, pv, L.gbase);
    if (pv != kInfInf) continue;
    uint32_t parent = kNoSlab;
    for (uint32_t b = rg.boff[v]; b < rg.boff[v + 1] && parent == kNoSlab; ++b) {
      uint32_t s = b;
      for (uint32_t hop = 0; s != kNoSlab && hop < (1u << 24); ++hop) {
        const uint4 q = ld_slab_ro(rg.slabs + 8ull * s + L.gl);
        uint32_t k[4], w[4];
        lane_keys<kRW>(q, L.gl, k, w);
        uint32_t mine = kNoSlab;
#pragma unroll
        for (int j = 0; j < keys_per_lane<kRW>(); ++j)
          if (mine == kNoSlab && k[j] < kTombKey && k[j] != v &&
              pack_hi(ld_dist(a.dist + k[j])) == lvl)
            mine = k[j];
        const uint32_t hit = __ballot_sync(L.gmask, mine != kNoSlab) >> L.gbase;
        if (hit) {
          parent = __shfl_sync(L.gmask, mine, L.gbase + __ffs(hit) - 1);
          break;
        }
        s = __shfl_sync(L.gmask, q.w, L.gbase + 7);
      }
    }
    if (parent != kNoSlab && L.gl == 0) {
      a.dist[v] = pack(lvl + 1, parent);
      if (atomicExch(a.stamp + v, stamp_next) != stamp_next) push_vertex(a, Q, v, nxt, nsz);
    }
  }
}

// Decremental re-seed by pull: every invalidated vertex takes the best
// distance offered by its in-neighbours that are still valid (reverse graph;
// its weights when SSSP), instead of a sweep over every bucket of the graph.
template <bool kRW, bool kUseW>
__device__ __forceinline__ void pull_reseed(const TravArgs &a, const Lanes &L, const BlockQueue &Q,
                                            uint32_t group, uint32_t ngroups, uint32_t nitems,
                                            uint32_t stamp_next, unsigned long long *gfr,
                                            uint32_t *gsz) {
  // one work item per chunk of an invalidated vertex's in-edge buckets
  // (a hub's in-edges spread over many groups); each item offers the best
  // of its chunk with an atomic minimum
  const GraphView &rg = a.rg;
  for (uint32_t i = group; i < nitems; i += ngroups) {
    uint32_t v, b0, b1;
    item_buckets(rg, __ldcg(a.treseed + i), v, b0, b1);
    unsigned long long best = kInfInf;  // pack(candidate distance, parent)
    for (uint32_t b = b0; b < b1; ++b) {
      uint32_t s = b;
      for (uint32_t hop = 0; s != kNoSlab && hop < (1u << 24); ++hop) {
        const uint4 q = ld_slab_ro(rg.slabs + 8ull * s + L.gl);
        uint32_t k[4], w[4];
        lane_keys<kRW>(q, L.gl, k, w);
#pragma unroll
        for (int j = 0; j < keys_per_lane<kRW>(); ++j) {
          const uint32_t u = k[j];
          if (u >= kTombKey || u == v || inval_test(a.inval, u)) continue;
          const unsigned long long pu = ld_dist(a.dist + u);
          if (pu == kInfInf) continue;
          const unsigned long long nd = (unsigned long long)pack_hi(pu) + (kUseW ? w[j] : 1u);
          if (nd < kInf) best = min(best, pack((uint32_t)nd, u));
        }
        s = __shfl_sync(L.gmask, q.w, L.gbase + 7);
      }
    }
#pragma unroll
    for (int o = 4; o > 0; o >>= 1) best = min(best, __shfl_xor_sync(L.gmask, best, o, 8));
    if (L.gl == 0 && best != kInfInf) {
      const unsigned long long old = atomicMin(a.dist + v, best);
      if (old > best && atomicExch(a.stamp + v, stamp_next) != stamp_next)
        push_vertex(a, Q, v, gfr, gsz);
    }
  }
}

template <bool kW, bool kUseW>
__global__ void __launch_bounds__(kTravBlock) k_traverse(TravArgs a) {
  __shared__ unsigned long long q_s[kQueueCap];
  __shared__ uint32_t qn_s;
  __shared__ uint32_t base_s;
  if (threadIdx.x == 0) qn_s = 0;
  __syncthreads();
  BlockQueue Q{q_s, &qn_s};
  const Lanes L = lanes();
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t nthreads = gridDim.x * blockDim.x;
  const uint32_t group = tid >> 3;
  const uint32_t ngroups = nthreads >> 3;
  const unsigned long long t_start = global_ns();
  uint32_t *ctl = a.ctl;
  uint32_t *err = ctl + kErr;
  unsigned long long *fr[2] = {a.fr0, a.fr1};
  const uint32_t round = ld_acquire_u32(ctl + kRound);
  bool nearfar = kUseW && a.mode == kStatic && a.delta != 0 && a.far0 != nullptr;
  const NearFar all_near{kNoFar, nullptr, nullptr};
  uint32_t fb = 0;  // far list being appended
  if (nearfar && tid == 0) {
    ctl[kThr] = a.delta;
    ctl[kFarMin0] = kNoFar;
    ctl[kFarMin0 + 1] = kNoFar;
  }

  // ---- seeding (level -1 pushes into fr[0] / sz[0]) ----
  if (a.mode == kStatic) {
    // every source seeds its own work items (a hub source has many)
    for (uint32_t i = tid; i < a.nsources; i += nthreads) {
      const uint32_t src = a.sources[i];
      a.dist[src] = pack(0, src);
      a.stamp[src] = round + 1;
      const uint32_t nb = a.g.boff[src + 1] - a.g.boff[src];
      const uint32_t k = max(1u, (nb + a.chunk - 1) / a.chunk);
      const uint32_t base = atomicAdd(ctl + kSz0, k);
      for (uint32_t j = 0; j < k; ++j) a.fr0[base + j] = item(src, j);
      atomicAdd(a.pushed, 1ull);
    }
  } else if (a.mode == kIncremental) {
    for (uint32_t e = group; e < a.bn; e += ngroups) {
      uint32_t s = a.bsrc[e], d = a.bdst[e];
      if (s == d || s >= a.g.V || d >= a.g.V) continue;
      // one lane loads, the group decides together
      unsigned long long ps = 0, pd = 0;
      if (L.gl == 0) {
        ps = ld_dist(a.dist + s);
        pd = ld_dist(a.dist + d);
      }
      ps = __shfl_sync(L.gmask, ps, L.gbase);
      pd = __shfl_sync(L.gmask, pd, L.gbase);
      if (ps == kInfInf) continue;
      uint32_t ds = pack_hi(ps);
      if (ds >= pack_hi(pd)) continue;
      uint32_t wv = 1;
      bool present = find_edge<kW>(a.g, L, s, d, &wv);
      if (!present) continue;
      if (L.gl == 0) {
        unsigned long long nd = (unsigned long long)ds + (kUseW ? wv : 1u);
        relax(a, Q, all_near, d, nd, s, round + 1, a.fr0, ctl + kSz0);
      }
    }
  } else {  // kDecremental
    uint64_t walked = 0;
    bool restart = false;
    if (!kUseW && a.trim) {
      // BFS repair, level by level in the old levels.  A candidate at level
      // L (a head of a deleted tree edge, or a tree child of a vertex that
      // lost its level) keeps level L when some in-neighbour still at level
      // L - 1 is not affected: that neighbour becomes its parent.  Otherwise
      // its level rises: it is marked affected (invalidated) and its tree
      // children become candidates of level L + 1.  Every vertex of level
      // L - 1 is decided before level L is examined (a barrier per level), so
      // the affected set is exact: only vertices whose level really rises
      // are invalidated and re-seeded, not whole subtrees.
      for (uint32_t e = tid; e < a.bn; e += nthreads) {
        const uint32_t s = a.bsrc[e], d = a.bdst[e];
        if (s == d || s >= a.g.V || d >= a.g.V) continue;
        const unsigned long long pd = ld_dist(a.dist + d);
        if (pd == kInfInf || is_source(pd, d) || pack_lo(pd) != s) continue;
        if (atomicExch(a.stamp + d, round) == round) continue;  // already a candidate
        const uint32_t lvl = pack_hi(pd);
        a.tseeds[atomicAdd(ctl + kTrimN, 1u)] = ((unsigned long long)lvl << 32) | d;
        atomicMin(ctl + kTrimLo, lvl);
        atomicMax(ctl + kTrimHi, lvl);
      }
      if (!grid_barrier(ctl + kBar0, err, a.limit_ns)) return;
      const uint32_t nseeds = ld_acquire_u32(ctl + kTrimN);
      const uint32_t lo = ld_acquire_u32(ctl + kTrimLo), hi_l = ld_acquire_u32(ctl + kTrimHi);
      // the seeds of one level become candidates, with their support-search
      // work items (chunks of their in-edge buckets)
      auto seed_level = [&](uint32_t lev, uint32_t *cand, uint32_t *ncand,
                            unsigned long long *items, uint32_t *nitems) {
        for (uint32_t i = tid; i < nseeds; i += nthreads) {
          const unsigned long long sd = __ldcg(a.tseeds + i);
          if ((uint32_t)(sd >> 32) != lev) continue;
          const uint32_t v = (uint32_t)sd;
          cand[atomicAdd(ncand, 1u)] = v;
          push_items(a.rg, v, items, nitems);
        }
      };
      if (nseeds) {
        seed_level(lo, a.tcand0, ctl + kTCand0, a.titems0, ctl + kTItem0);
        if (!grid_barrier(ctl + kBar0, err, a.limit_ns)) return;
      }
      // Each level in three steps, a barrier after each:
      //   A  every support-search item scans its chunk of a candidate's
      //      in-edges for a neighbour one level up that is not affected
      //      (the smallest such id wins, by atomicMin on tpar);
      //   B  a candidate with a support keeps its level under that parent;
      //      one without is affected: invalidated, queued for the re-seed,
      //      and its out-edges queued (in chunks) for the child scan;
      //   C  the child-scan items find the tree children of the affected
      //      vertices (the next level's candidates) and the next level's
      //      seeds join them.
      // Hubs are split into many items, so no vertex serialises a level.
      for (uint32_t r = 0; nseeds; ++r) {
        const uint32_t lev = lo + r, cb = r & 1u, nb = cb ^ 1u;
        const uint32_t ncand = ld_acquire_u32(ctl + kTCand0 + cb);
        const uint32_t nit = ld_acquire_u32(ctl + kTItem0 + cb);
        if (ncand == 0 && lev >= hi_l) break;
        if (r >= kTrimMaxRounds || (a.recompute_inv && ld_acquire_u32(ctl + kInvCount) >= a.recompute_inv)) {
          restart = true;
          break;
        }
        const uint32_t *cand = cb ? a.tcand1 : a.tcand0;
        const unsigned long long *items = cb ? a.titems1 : a.titems0;
        uint32_t *cand_n = nb ? a.tcand1 : a.tcand0;
        unsigned long long *items_n = nb ? a.titems1 : a.titems0;
        if (tid == 0) {
          ctl[kTCand0 + nb] = 0;
          ctl[kTItem0 + nb] = 0;
          ctl[kTChild] = 0;
        }
        // A
        const GraphView &rg = a.rg;
        for (uint32_t i = group; i < nit; i += ngroups) {
          uint32_t v, b0, b1;
          item_buckets(rg, __ldcg(items + i), v, b0, b1);
          if (__ldcg(a.tpar + v) != kEmptyKey) continue;  // another chunk found one
          uint32_t found = kEmptyKey;
          for (uint32_t b = b0; b < b1 && found == kEmptyKey; ++b) {
            uint32_t sl = b;
            for (uint32_t hop = 0; sl != kNoSlab && hop < (1u << 24) && found == kEmptyKey; ++hop) {
              const uint4 q = ld_slab_ro(rg.slabs + 8ull * sl + L.gl);
              uint32_t k[4], w[4];
              if (rg.weighted)
                lane_keys<true>(q, L.gl, k, w);
              else
                lane_keys<false>(q, L.gl, k, w);
              uint32_t mine = kEmptyKey;
#pragma unroll
              for (int j = 0; j < 4; ++j) {
                const uint32_t u = k[j];
                if (u >= kTombKey || u == v || u >= mine || inval_test(a.inval, u)) continue;
                const unsigned long long pu = ld_dist(a.dist + u);
                if (pu != kInfInf && pack_hi(pu) + 1u == lev) mine = u;
              }
              found = __reduce_min_sync(L.gmask, mine);
              sl = __shfl_sync(L.gmask, q.w, L.gbase + 7);
            }
          }
          if (found != kEmptyKey && L.gl == 0) atomicMin(a.tpar + v, found);
        }
        if (!grid_barrier(ctl + kBar0, err, a.limit_ns)) return;
        // B
        for (uint32_t i = tid; i < ncand; i += nthreads) {
          const uint32_t v = __ldcg(cand + i);
          const uint32_t w = __ldcg(a.tpar + v);
          if (w != kEmptyKey) {
            a.tpar[v] = kEmptyKey;
            a.dist[v] = pack(lev, w);  // same level, new parent
          } else {
            inval_set(a.inval, v);
            a.dist[v] = kInfInf;
            a.inv_list[atomicAdd(ctl + kInvCount, 1u)] = v;
            push_items(a.g, v, a.tchild, ctl + kTChild);
            push_items(rg, v, a.treseed, ctl + kTReseed);
          }
        }
        if (!grid_barrier(ctl + kBar0, err, a.limit_ns)) return;
        // C
        const uint32_t nch = ld_acquire_u32(ctl + kTChild);
        for (uint32_t i = group; i < nch; i += ngroups) {
          uint32_t v, b0, b1;
          item_buckets(a.g, __ldcg(a.tchild + i), v, b0, b1);
          walk_buckets(a.g, L, b0, b1, [&](const uint4 &q) {
            uint32_t k[4], w[4];
            lane_keys<kW>(q, L.gl, k, w);
#pragma unroll
            for (int j = 0; j < keys_per_lane<kW>(); ++j) {
              const uint32_t x = k[j];
              if (x >= kTombKey || x == v) continue;
              const unsigned long long px = ld_dist(a.dist + x);
              if (px == kInfInf || pack_lo(px) != v || pack_hi(px) != lev + 1u) continue;
              if (atomicExch(a.stamp + x, round) == round) continue;
              cand_n[atomicAdd(ctl + kTCand0 + nb, 1u)] = x;
              push_items(rg, x, items_n, ctl + kTItem0 + nb);
            }
          });
        }
        if (lev + 1u <= hi_l) seed_level(lev + 1u, cand_n, ctl + kTCand0 + nb, items_n, ctl + kTItem0 + nb);
        if (!grid_barrier(ctl + kBar0, err, a.limit_ns)) return;
      }
      walked = ld_acquire_u32(ctl + kInvCount);
    } else {
    // D1: children of deleted tree edges.  Every invalidated vertex goes to
    // inv_list (for the final flag reset) and to the invalidation frontier.
    auto invalidate = [&](uint32_t v, unsigned long long *gfr, uint32_t *gsz) {
      a.dist[v] = kInfInf;
      a.inv_list[atomicAdd(ctl + kInvCount, 1u)] = v;
      if (a.rg.V && a.treseed) push_items(a.rg, v, a.treseed, ctl + kTReseed);
      const uint32_t nb = a.g.boff[v + 1] - a.g.boff[v];
      const uint32_t k = max(1u, (nb + a.chunk - 1) / a.chunk);
      const uint32_t base = atomicAdd(gsz, k);
      for (uint32_t j = 0; j < k; ++j) gfr[base + j] = item(v, j);
    };
    auto tree_edge = [&](uint32_t e, uint32_t &d) {
      const uint32_t s = a.bsrc[e];
      d = a.bdst[e];
      if (s == d || s >= a.g.V || d >= a.g.V) return false;
      const unsigned long long pd = ld_dist(a.dist + d);
      return pd != kInfInf && !is_source(pd, d) && pack_lo(pd) == s;
    };
    if (a.recompute_inv) {
      // count the deleted tree edges first: when they alone reach the
      // recompute threshold, recompute without invalidating anything
      uint32_t c = 0;
      for (uint32_t e = tid; e < a.bn; e += nthreads) {
        uint32_t d;
        c += tree_edge(e, d) ? 1u : 0u;
      }
      c = __reduce_add_sync(0xFFFFFFFFu, c);
      if ((threadIdx.x & 31u) == 0 && c) atomicAdd(ctl + kEarly, c);
      if (!grid_barrier(ctl + kBar0, err, a.limit_ns)) return;
      if (ld_acquire_u32(ctl + kEarly) >= a.recompute_inv) restart = true;
    }
    if (!restart) {
      if (tid == 0) ctl[kEarly] = 0u;
      for (uint32_t e = tid; e < a.bn; e += nthreads) {
        uint32_t d;
        if (tree_edge(e, d) && inval_set(a.inval, d)) invalidate(d, a.fr0, ctl + kDSz0);
      }
      if (!grid_barrier(ctl + kBar0, err, a.limit_ns)) return;
    }
    // D2: invalidate whole subtrees along tree edges, level by level.  Sizes
    // rotate over three counters so no block reads a counter that another
    // block is already filling for the next level.
    // The running total of the level sizes (each read after a barrier, the
    // same in every thread) stops the walk early once a recompute is due.
    for (uint32_t dl = 0; !restart; ++dl) {
      const uint32_t n = ld_acquire_u32(ctl + kDSz0 + (dl % 3));
      if (n == 0) break;
      walked += n;
      if (a.recompute_inv && walked >= a.recompute_inv) {
        restart = true;
        break;
      }
      if (tid == 0) ctl[kDSz0 + ((dl + 2) % 3)] = 0;
      const unsigned long long *cur = fr[dl & 1];
      unsigned long long *nxt = fr[(dl + 1) & 1];
      uint32_t *nsz = ctl + kDSz0 + ((dl + 1) % 3);
      for (uint32_t i = group; i < n; i += ngroups) {
        uint32_t x, b0, b1;
        item_range(a.g, __ldcg(cur + i), a.chunk, x, b0, b1);
        walk_buckets(a.g, L, b0, b1, [&](const uint4 &q) {
          uint32_t k[4], w[4];
          lane_keys<kW>(q, L.gl, k, w);
#pragma unroll
          for (int j = 0; j < keys_per_lane<kW>(); ++j) {
            uint32_t y = k[j];
            if (y < kTombKey && y != x && !inval_test(a.inval, y)) {
              unsigned long long py = ld_dist(a.dist + y);
              if (py != kInfInf && !is_source(py, y) && pack_lo(py) == x && inval_set(a.inval, y))
                invalidate(y, nxt, nsz);
            }
          }
        });
      }
      if (!grid_barrier(ctl + kBar0, err, a.limit_ns)) return;
    }
    }  // whole-subtree invalidation
    (void)walked;
    const uint32_t hi = ld_acquire_u32(ctl + kInvCount);
    if (restart) {
      // Most of the tree is gone: a recompute from the sources costs less
      // than re-seeding and repairing this many vertices.  The invalidation
      // bits are cleared in the epilogue as usual.
      for (uint32_t v = tid; v < a.g.V; v += nthreads) a.dist[v] = kInfInf;
      if (tid == 0) {
        ctl[kRestart] = 1u;
        ctl[kThr] = a.delta;
        ctl[kFarMin0] = kNoFar;
        ctl[kFarMin0 + 1] = kNoFar;
      }
      if (!grid_barrier(ctl + kBar0, err, a.limit_ns)) return;
      for (uint32_t i = tid; i < a.nsources; i += nthreads) {
        const uint32_t src = a.sources[i];
        a.dist[src] = pack(0, src);
        a.stamp[src] = round + 1;
        const uint32_t nb = a.g.boff[src + 1] - a.g.boff[src];
        const uint32_t k = max(1u, (nb + a.chunk - 1) / a.chunk);
        const uint32_t base = atomicAdd(ctl + kSz0, k);
        for (uint32_t j = 0; j < k; ++j) a.fr0[base + j] = item(src, j);
        atomicAdd(a.pushed, 1ull);
      }
      nearfar = kUseW && a.delta != 0 && a.far0 != nullptr;
    } else if (hi > 0 && a.rg.V && a.treseed) {
      // D3 with the reverse graph: pull from each invalidated vertex's in-edges
      const uint32_t nri = ld_acquire_u32(ctl + kTReseed);
      if (a.rg.weighted)
        pull_reseed<true, kUseW>(a, L, Q, group, ngroups, nri, round + 1, a.fr0, ctl + kSz0);
      else
        pull_reseed<false, kUseW>(a, L, Q, group, ngroups, nri, round + 1, a.fr0, ctl + kSz0);
    } else if (hi > 0) {
      // D3: re-seed invalidated vertices from valid in-neighbours: one sweep
      // over all buckets (balanced by construction)
      for (uint32_t b = group; b < a.g.nbuckets; b += ngroups) {
        const uint32_t u = a.g.bowner[b];
        if (a.g.deg[u] == 0 || inval_test(a.inval, u)) continue;
        unsigned long long pu = 0;
        if (L.gl == 0) pu = ld_dist(a.dist + u);
        pu = __shfl_sync(L.gmask, pu, L.gbase);
        if (pu == kInfInf) continue;
        walk_bucket(a.g, L, b, [&](const uint4 &q) {
          relax_slab<kW, kUseW>(a, L, Q, all_near, q, u, pack_hi(pu), round + 1, a.fr0, ctl + kSz0,
                                true);
        });
      }
    }
  }
  queue_flush(Q, a.fr0, ctl + kSz0, a.pushed, &base_s);
  if (!grid_barrier(ctl + kBar0, err, a.limit_ns)) return;

  // ---- relaxation levels ----
  // A level expands the frontier; with near-far SSSP, a level whose frontier
  // is empty instead drains the far list: the threshold moves to the far
  // list's smallest distance plus delta, vertices below it join the next
  // level and the rest move to the other far list.
  // The level loop ends when the frontier (and the far lists) run dry; as a
  // guard against a logic error that would keep it going with every barrier
  // met, a launch that has run longer than 64 wait limits (at least 60 s)
  // reports a timeout and stops.
  const unsigned long long guard_ns = max(64ull * a.limit_ns, 60000000000ull);
  uint32_t lv = 0;
  for (;; ++lv) {
    if (global_ns() - t_start > guard_ns) {
      if (tid == 0) atomicOr(err, kErrTimeout);
      break;
    }
    const uint32_t n = ld_acquire_u32(ctl + kSz0 + (lv % 3));
    uint32_t nfar = 0;
    if (n == 0) {
      if (!nearfar) break;
      nfar = ld_acquire_u32(ctl + kFarN0 + fb);
      if (nfar == 0) break;
    }
    if (tid == 0) ctl[kSz0 + ((lv + 2) % 3)] = 0;
    const unsigned long long *cur = fr[lv & 1];
    unsigned long long *nxt = fr[(lv + 1) & 1];
    uint32_t *nsz = ctl + kSz0 + ((lv + 1) % 3);
    const uint32_t stamp_next = round + 2 + lv;
    const uint32_t thr = nearfar ? ld_acquire_u32(ctl + kThr) : kNoFar;
    if (n && !kUseW && a.mode == kStatic && a.pull_items && n >= a.pull_items) {
      // large BFS frontier: pull this level from the unvisited side
      if (a.rg.weighted)
        pull_level<true>(a, L, Q, group, ngroups, lv, stamp_next, nxt, nsz);
      else
        pull_level<false>(a, L, Q, group, ngroups, lv, stamp_next, nxt, nsz);
    } else if (n) {
      const NearFar nf = nearfar ? NearFar{thr, fb ? a.far1 : a.far0, ctl + kFarN0 + fb} : all_near;
      for (uint32_t i = group; i < n; i += ngroups) {
        uint32_t u, b0, b1;
        item_range(a.g, __ldcg(cur + i), a.chunk, u, b0, b1);
        unsigned long long pu = 0;
        if (L.gl == 0) pu = ld_dist(a.dist + u);
        pu = __shfl_sync(L.gmask, pu, L.gbase);
        if (pu == kInfInf) continue;
        expand_range<kW, kUseW>(a, L, Q, nf, u, pack_hi(pu), b0, b1, stamp_next, nxt, nsz);
      }
    } else {
      const uint32_t *fc = fb ? a.far1 : a.far0;
      uint32_t *fo = fb ? a.far0 : a.far1;
      for (uint32_t i = tid; i < nfar; i += nthreads)
        atomicMin(ctl + kFarMin0 + fb, pack_hi(ld_dist(a.dist + __ldcg(fc + i))));
      if (!grid_barrier(ctl + kBar0, err, a.limit_ns)) return;
      const uint32_t lo = max(thr, ld_acquire_u32(ctl + kFarMin0 + fb));
      const uint32_t nthr = lo > kNoFar - a.delta ? kNoFar : lo + a.delta;
      for (uint32_t i = tid; i < nfar; i += nthreads) {
        const uint32_t v = __ldcg(fc + i);
        const uint32_t d = pack_hi(ld_dist(a.dist + v));
        if (d < nthr) {
          atomicAnd(a.fbits + (v >> 5), ~(1u << (v & 31)));
          if (atomicExch(a.stamp + v, stamp_next) != stamp_next) push_vertex(a, Q, v, nxt, nsz);
        } else {
          fo[atomicAdd(ctl + kFarN0 + (fb ^ 1u), 1u)] = v;
        }
      }
      if (tid == 0) {
        ctl[kThr] = nthr;
        ctl[kFarN0 + fb] = 0;
        // the other list's minimum is read by the next drain, not this one
        ctl[kFarMin0 + (fb ^ 1u)] = kNoFar;
      }
      fb ^= 1u;
    }
    queue_flush(Q, nxt, nsz, a.pushed, &base_s);
    if (!grid_barrier(ctl + kBar0, err, a.limit_ns)) return;
  }

  // ---- epilogue: clear invalidation flags, publish counters ----
  if (a.mode == kDecremental) {
    uint32_t ninv = ld_acquire_u32(ctl + kInvCount);
    for (uint32_t i = tid; i < ninv; i += nthreads) a.inval[__ldcg(a.inv_list + i) >> 5] = 0u;
  }
  if (tid == 0) {
    ctl[kLevels] = lv;
    ctl[kRound] = round + 3 + lv;
  }
}


// ---- static BFS of ranges held in shared memory ----
// One CTA per range (a member of a graph set that holds one source), the
// member's state in shared memory (bfs_member).  CTAs take ranges from a
// counter, largest first.  rng[r] = (first vertex, end vertex, first bucket,
// end bucket) of a range of at most kMemLocalMax vertices, src[r] its source
// (global id).  items holds one word per bucket of the graph, found one per
// vertex.  dist must already hold INFINF.
template <bool kW>
__global__ void __launch_bounds__(kMemThreads, 1)
    k_bfs_members(GraphView g, const uint4 *__restrict__ rng, const uint32_t *__restrict__ src,
                  uint32_t nr, uint32_t *counter, unsigned long long *__restrict__ dist,
                  uint32_t *__restrict__ items, uint32_t *__restrict__ found, uint32_t *err) {
  extern __shared__ uint32_t smem[];
  __shared__ uint32_t s_range, s_nfound, s_nitems;
  const Lanes L = lanes();
  for (;;) {
    if (threadIdx.x == 0) s_range = atomicAdd(counter, 1u);
    __syncthreads();
    const uint32_t r = s_range;
    if (r >= nr) break;
    bfs_member<kW, false>(g, L, rng[r], src[r], dist, items, found, err, smem, s_nfound, s_nitems);
  }
}

}  // namespace mk

using namespace mk;

struct mk_traversal {
  mk_graph *g = nullptr;
  uint32_t nsources = 0;
  uint32_t src_cap = 0;
  uint32_t *sources = nullptr;  // device copy
  bool sssp = false;
  bool has_static = false;
  int nblocks = 0;
  unsigned long long *dist = nullptr;
  uint32_t *stamp = nullptr;
  uint32_t *inval = nullptr;
  unsigned long long *fr0 = nullptr, *fr1 = nullptr;
  uint32_t *inv_list = nullptr;
  uint32_t *ctl = nullptr;
  unsigned long long *pushed = nullptr;
  uint32_t *far0 = nullptr, *far1 = nullptr, *fbits = nullptr;  // near-far SSSP
  mk_graph *rev = nullptr;  // in-edges of the same graph, for pull levels (BFS)
  // decremental with a reverse graph (allocated when one is attached): the
  // BFS repair's lists and the re-seed items (TravArgs has the layout)
  unsigned long long *tseeds = nullptr, *titems0 = nullptr, *titems1 = nullptr;
  unsigned long long *tchild = nullptr, *treseed = nullptr;
  uint32_t *tcand0 = nullptr, *tcand1 = nullptr, *tpar = nullptr;
  size_t rcap = 0;  // re-seed / support item capacity
  std::vector<uint32_t> h_sources;
  // prepared member table (BFS): counter word, uint4 (lo, hi, b0, b1) per
  // small range (largest first), their sources, then the sources whose
  // range is too large for shared memory
  DevBuf<uint32_t> members;
  uint32_t n_small = 0, n_large = 0, small_max = 0;
  int small_grid = 0;
  bool members_prepared = false;
  PinnedRing staging;  // stream-ordered source uploads
  Timer timer;
};

// A launch that gave up on a wait leaves its error word set, its stamps
// and invalidation bits behind and the round counter not advanced, so the
// next call's stamps could collide with them.  Run before the next launch
// clears the control words: when the error word holds a timeout, clear the
// stamps and the bits and restart the round count.
__global__ void k_trav_recover(uint32_t *ctl, uint32_t *stamp, uint32_t *inval, uint32_t *tpar,
                               uint32_t V) {
  if (!(ld_relaxed_u32(ctl + kErr) & kErrTimeout)) return;
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, n = gridDim.x * blockDim.x;
  for (uint32_t v = tid; v < V; v += n) {
    stamp[v] = 0u;
    if (tpar) tpar[v] = kEmptyKey;
  }
  for (uint32_t w = tid; w < (V + 31) / 32; w += n) inval[w] = 0u;
  if (tid == 0) ctl[kRound] = 1u;
}

__global__ void k_set_sources(unsigned long long *dist, const uint32_t *sources, uint32_t n) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    dist[sources[i]] = pack(0, sources[i]);
}

static mk_status check_sources(const mk_graph *g, const uint32_t *h_sources, uint32_t n,
                               const char *what) {
  std::vector<uint32_t> sorted(h_sources, h_sources + n);
  std::sort(sorted.begin(), sorted.end());
  if (sorted.back() >= g->V) return fail(MK_ERR_INVALID, std::string(what) + ": source out of range");
  if (std::adjacent_find(sorted.begin(), sorted.end()) != sorted.end())
    return fail(MK_ERR_INVALID, std::string(what) + ": repeated source");
  return MK_OK;
}

static mk_status trav_create(mk_graph *g, const uint32_t *h_sources, uint32_t nsrc, bool sssp,
                             mk_traversal **out) {
  if (!g || !out || !h_sources) return fail(MK_ERR_INVALID, "traversal create: null argument");
  *out = nullptr;
  if (nsrc == 0) return fail(MK_ERR_INVALID, "traversal create: no source");
  if (g->reverse) return fail(MK_ERR_INVALID, "traversal create: graph must store out-edges");
  if (sssp && !g->weighted) return fail(MK_ERR_INVALID, "SSSP needs a weighted graph");
  MK_CHECK(check_sources(g, h_sources, nsrc, "traversal create"));
  DeviceGuard dg(g->device);
  mk_traversal *t = new mk_traversal();
  t->g = g;
  t->nsources = nsrc;
  t->src_cap = nsrc;
  t->sssp = sssp;
  t->h_sources.assign(h_sources, h_sources + nsrc);
  const size_t V = g->V;
  cudaError_t e = cudaSuccess;
  auto A = [&](void **p, size_t bytes) {
    if (e == cudaSuccess) e = cudaMalloc(p, bytes);
  };
  A((void **)&t->dist, V * 8);
  A((void **)&t->stamp, V * 4);
  A((void **)&t->inval, (V + 31) / 32 * 4);
  // a level holds every vertex at most once, as at most one item per bucket
  // (any chunk size >= 1)
  const size_t items = g->num_buckets + 64;
  A((void **)&t->fr0, items * 8);
  A((void **)&t->fr1, items * 8);
  A((void **)&t->inv_list, V * 4 + 16);
  A((void **)&t->ctl, kCtlWords * 4);
  A((void **)&t->pushed, 8);
  A((void **)&t->sources, (size_t)nsrc * 4);
  if (sssp) {  // far lists: a vertex is on at most one of them at a time
    A((void **)&t->far0, V * 4 + 16);
    A((void **)&t->far1, V * 4 + 16);
    A((void **)&t->fbits, (V + 31) / 32 * 4);
  }
  if (e == cudaSuccess)
    e = cudaMemcpy(t->sources, h_sources, (size_t)nsrc * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(t->dist, 0xFF, V * 8);
  if (e == cudaSuccess) e = cudaMemset(t->stamp, 0, V * 4);
  if (e == cudaSuccess) e = cudaMemset(t->inval, 0, (V + 31) / 32 * 4);
  if (e == cudaSuccess) e = cudaMemset(t->ctl, 0, kCtlWords * 4);
  if (e == cudaSuccess) {
    // dist[src] = PACK(0, src) as the reference constructor does (BFS.cuh:49-52)
    k_set_sources<<<(nsrc + 255) / 256, 256>>>(t->dist, t->sources, nsrc);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) {
    uint32_t one = 1;
    e = cudaMemcpy(t->ctl + kRound, &one, 4, cudaMemcpyHostToDevice);
  }
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    mk_traversal_destroy(t);
    return cuda_fail(e, "traversal create");
  }
  *out = t;
  return MK_OK;
}

// Issues one traversal launch (sources: t's own, or the given device list).
static void free_repair(mk_traversal *t) {
  for (unsigned long long **p : {&t->tseeds, &t->titems0, &t->titems1, &t->tchild, &t->treseed}) {
    cudaFree(*p);
    *p = nullptr;
  }
  for (uint32_t **p : {&t->tcand0, &t->tcand1, &t->tpar}) {
    cudaFree(*p);
    *p = nullptr;
  }
  t->rcap = 0;
}

static int recover_grid(const mk_graph *g) {
  return (int)std::min<uint64_t>((uint64_t)g->V / 256 + 1, (uint64_t)device_sm_count(g->device) * 4);
}

static mk_status trav_issue(mk_traversal *t, uint32_t mode, const uint32_t *bs, const uint32_t *bd,
                            uint32_t n, cudaStream_t s, const uint32_t *srcs, uint32_t nsrc) {
  mk_graph *g = t->g;
  if (mode == kStatic) MK_CUDA(cudaMemsetAsync(t->dist, 0xFF, (size_t)g->V * 8, s));
  const uint32_t delta = (t->sssp && mode != kIncremental && t->far0) ? g->tuning.sssp_delta : 0u;
  if (delta) MK_CUDA(cudaMemsetAsync(t->fbits, 0, ((size_t)g->V + 31) / 32 * 4, s));
  k_trav_recover<<<recover_grid(g), 256, 0, s>>>(t->ctl, t->stamp, t->inval, t->tpar, g->V);
  // clear everything but the persistent round counter
  MK_CUDA(cudaMemsetAsync(t->ctl, 0, kRound * 4, s));
  MK_CUDA(cudaMemsetAsync(t->ctl + kTrimN, 0, (kCtlWords - kTrimN) * 4, s));
  MK_CUDA(cudaMemsetAsync(t->ctl + kTrimLo, 0xFF, 4, s));
  MK_CUDA(cudaMemsetAsync(t->pushed, 0, 8, s));
  TravArgs a;
  a.g = g->view();
  a.dist = t->dist;
  a.stamp = t->stamp;
  a.inval = t->inval;
  a.fr0 = t->fr0;
  a.fr1 = t->fr1;
  a.inv_list = t->inv_list;
  a.ctl = t->ctl;
  a.pushed = t->pushed;
  a.bsrc = bs;
  a.bdst = bd;
  a.bn = n;
  a.sources = srcs ? srcs : t->sources;
  a.nsources = srcs ? nsrc : t->nsources;
  a.chunk = g->tuning.frontier_chunk ? g->tuning.frontier_chunk : kDefaultChunk;
  a.delta = delta;
  a.rg = t->rev ? t->rev->view() : GraphView{};
  if (!t->rev) a.rg.V = 0;
  a.pull_items = (t->rev && g->tuning.pull_permille)
                     ? (uint32_t)std::max<uint64_t>(1, (uint64_t)g->V * g->tuning.pull_permille / 1000)
                     : 0u;
  a.recompute_inv = g->tuning.recompute_permille
                        ? (uint32_t)std::max<uint64_t>(1, (uint64_t)g->V * g->tuning.recompute_permille / 1000)
                        : 0u;
  a.far0 = t->far0;
  a.far1 = t->far1;
  a.fbits = t->fbits;
  a.mode = mode;
  a.limit_ns = g->wait_limit_ns();
  a.trim = (mode == kDecremental && !t->sssp && t->rev && t->tseeds) ? 1u : 0u;
  a.tseeds = t->tseeds;
  a.tcand0 = t->tcand0;
  a.tcand1 = t->tcand1;
  a.tpar = t->tpar;
  a.titems0 = t->titems0;
  a.titems1 = t->titems1;
  a.tchild = t->tchild;
  a.treseed = t->rev ? t->treseed : nullptr;
  const void *fn;
  if (g->weighted)
    fn = t->sssp ? (const void *)k_traverse<true, true> : (const void *)k_traverse<true, false>;
  else
    fn = (const void *)k_traverse<false, false>;
  if (t->nblocks == 0) t->nblocks = persistent_blocks(fn, kTravBlock, 0, g->device);
  void *args[] = {&a};
  MK_CUDA(cudaLaunchCooperativeKernel(fn, dim3(t->nblocks), dim3(kTravBlock), args, 0, s));
  return MK_OK;
}

static mk_status trav_launch(mk_traversal *t, uint32_t mode, const uint32_t *bs,
                             const uint32_t *bd, uint32_t n, void *stream,
                             float *ms_out) {
  DeviceGuard dg(t->g->device);
  cudaStream_t s = as_stream(stream);
  if (n && (!bs || !bd)) return fail(MK_ERR_INVALID, "traversal: null batch");
  MK_CHECK(t->timer.start(s, ms_out != nullptr));
  MK_CHECK(trav_issue(t, mode, bs, bd, n, s, nullptr, 0));
  MK_CHECK(t->timer.stop(ms_out));
  if (ms_out) {  // the call has synchronised: report a barrier that gave up
    uint32_t err = 0;
    MK_CUDA(cudaMemcpy(&err, t->ctl + kErr, 4, cudaMemcpyDeviceToHost));
    if (err & kErrTimeout) return fail(MK_ERR_TIMEOUT, "traversal: grid barrier timed out");
  }
  if (mode == kStatic) t->has_static = true;
  return MK_OK;
}

namespace mk {
mk_status trav_member_bufs(mk_traversal *t, TravMemberBufs *out) {
  if (!t || !out) return fail(MK_ERR_INVALID, "trav_member_bufs: null argument");
  out->dist = t->dist;
  out->items = reinterpret_cast<uint32_t *>(t->fr0);
  out->found = t->inv_list;
  return MK_OK;
}
}  // namespace mk

extern "C" {

mk_status mk_bfs_create(mk_graph *g, uint32_t source, mk_traversal **out) {
  return trav_create(g, &source, 1, false, out);
}

mk_status mk_sssp_create(mk_graph *g, uint32_t source, mk_traversal **out) {
  return trav_create(g, &source, 1, true, out);
}

mk_status mk_bfs_create_multi(mk_graph *g, const uint32_t *h_sources, uint32_t n,
                              mk_traversal **out) {
  return trav_create(g, h_sources, n, false, out);
}

mk_status mk_sssp_create_multi(mk_graph *g, const uint32_t *h_sources, uint32_t n,
                               mk_traversal **out) {
  return trav_create(g, h_sources, n, true, out);
}

mk_status mk_traversal_set_sources(mk_traversal *t, const uint32_t *h_sources, uint32_t n) {
  if (!t || !h_sources) return fail(MK_ERR_INVALID, "mk_traversal_set_sources: null argument");
  if (n == 0) return fail(MK_ERR_INVALID, "mk_traversal_set_sources: no source");
  MK_CHECK(check_sources(t->g, h_sources, n, "mk_traversal_set_sources"));
  DeviceGuard dg(t->g->device);
  if (n > t->src_cap) {
    uint32_t *p = nullptr;
    MK_CUDA(cudaMalloc(&p, (size_t)n * 4));
    cudaFree(t->sources);
    t->sources = p;
    t->src_cap = n;
  }
  // ordered after every earlier launch of this traversal on any stream
  MK_CUDA(cudaDeviceSynchronize());
  MK_CUDA(cudaMemcpy(t->sources, h_sources, (size_t)n * 4, cudaMemcpyHostToDevice));
  t->nsources = n;
  t->h_sources.assign(h_sources, h_sources + n);
  t->has_static = false;
  t->members_prepared = false;
  return MK_OK;
}

mk_status mk_traversal_set_sources_async(mk_traversal *t, const uint32_t *h_sources, uint32_t n,
                                         void *stream) {
  if (!t || !h_sources) return fail(MK_ERR_INVALID, "mk_traversal_set_sources_async: null argument");
  if (n == 0) return fail(MK_ERR_INVALID, "mk_traversal_set_sources_async: no source");
  MK_CHECK(check_sources(t->g, h_sources, n, "mk_traversal_set_sources_async"));
  DeviceGuard dg(t->g->device);
  if (n > t->src_cap) {  // growing synchronises the device, as cudaFree does
    MK_CUDA(cudaDeviceSynchronize());
    uint32_t *p = nullptr;
    MK_CUDA(cudaMalloc(&p, (size_t)n * 4));
    cudaFree(t->sources);
    t->sources = p;
    t->src_cap = n;
  }
  MK_CHECK(t->staging.upload(t->sources, h_sources, (size_t)n * 4, as_stream(stream)));
  t->nsources = n;
  t->h_sources.assign(h_sources, h_sources + n);
  t->has_static = false;
  t->members_prepared = false;
  return MK_OK;
}

mk_status mk_traversal_set_reverse(mk_traversal *t, mk_graph *g_rev) {
  if (!t) return fail(MK_ERR_INVALID, "mk_traversal_set_reverse: null handle");
  if (g_rev) {
    if (t->sssp && !g_rev->weighted)
      return fail(MK_ERR_INVALID, "mk_traversal_set_reverse: SSSP needs a weighted reverse graph");
    if (!g_rev->reverse || g_rev->V != t->g->V || g_rev->device != t->g->device)
      return fail(MK_ERR_INVALID,
                  "mk_traversal_set_reverse: needs a reverse graph of the same size on the same device");
  }
  DeviceGuard dg(t->g->device);
  if (g_rev) {
    // Sized once per handle for the largest reverse graph attached.  A vertex
    // is a seed, a candidate, affected or re-seeded at most once per call, and
    // pushes at most (its buckets / kRepairChunk + 1) items to a list.
    const size_t V = t->g->V;
    const size_t rin = (size_t)g_rev->num_buckets / kRepairChunk + V + 64;
    const size_t fout = (size_t)t->g->num_buckets / kRepairChunk + V + 64;
    if (t->treseed && rin > t->rcap) {
      MK_CUDA(cudaDeviceSynchronize());
      free_repair(t);
    }
    if (!t->treseed) {
      MK_CUDA(cudaDeviceSynchronize());
      cudaError_t e = cudaMalloc(&t->treseed, rin * 8);
      if (e == cudaSuccess && !t->sssp) {
        e = cudaMalloc(&t->tseeds, (V + 16) * 8);
        if (e == cudaSuccess) e = cudaMalloc(&t->tcand0, (V + 16) * 4);
        if (e == cudaSuccess) e = cudaMalloc(&t->tcand1, (V + 16) * 4);
        if (e == cudaSuccess) e = cudaMalloc(&t->tpar, V * 4 + 4);
        if (e == cudaSuccess) e = cudaMalloc(&t->titems0, rin * 8);
        if (e == cudaSuccess) e = cudaMalloc(&t->titems1, rin * 8);
        if (e == cudaSuccess) e = cudaMalloc(&t->tchild, fout * 8);
        if (e == cudaSuccess) e = cudaMemset(t->tpar, 0xFF, V * 4 + 4);
      }
      if (e != cudaSuccess) {
        free_repair(t);
        return cuda_fail(e, "mk_traversal_set_reverse: repair lists");
      }
      t->rcap = rin;
    }
  }
  t->rev = g_rev;
  return MK_OK;
}

mk_status mk_traversal_static(mk_traversal *t, void *stream, float *ms_out) {
  if (!t) return fail(MK_ERR_INVALID, "mk_traversal_static: null handle");
  return trav_launch(t, kStatic, nullptr, nullptr, 0, stream, ms_out);
}

mk_status mk_bfs_prepare_members(mk_traversal *t, const uint32_t *h_vertex_ranges,
                                 uint32_t nranges) {
  const char *what = "mk_bfs_prepare_members";
  if (!t || (nranges && !h_vertex_ranges)) return fail(MK_ERR_INVALID, std::string(what) + ": null argument");
  if (t->sssp) return fail(MK_ERR_INVALID, std::string(what) + ": BFS only");
  if (nranges != t->nsources)
    return fail(MK_ERR_INVALID, std::string(what) + ": need one range per source");
  mk_graph *g = t->g;
  std::vector<uint32_t> small_ids, large_src;
  std::vector<std::pair<uint32_t, uint32_t>> spans;
  for (uint32_t r = 0; r < nranges; ++r) {
    const uint32_t b = h_vertex_ranges[2 * r], e = h_vertex_ranges[2 * r + 1];
    if (b >= e || e > g->V) return fail(MK_ERR_INVALID, std::string(what) + ": bad vertex range");
    if (t->h_sources[r] < b || t->h_sources[r] >= e)
      return fail(MK_ERR_INVALID, std::string(what) + ": source outside its range");
    spans.emplace_back(b, e);
    if (e - b <= kMemLocalMax)
      small_ids.push_back(r);
    else
      large_src.push_back(t->h_sources[r]);
  }
  std::sort(spans.begin(), spans.end());
  for (size_t i = 1; i < spans.size(); ++i)
    if (spans[i].first < spans[i - 1].second)
      return fail(MK_ERR_INVALID, std::string(what) + ": overlapping ranges");
  auto len = [&](uint32_t r) { return h_vertex_ranges[2 * r + 1] - h_vertex_ranges[2 * r]; };
  std::stable_sort(small_ids.begin(), small_ids.end(),
                   [&](uint32_t a, uint32_t b) { return len(a) > len(b); });
  const size_t ns = small_ids.size(), nl = large_src.size();
  std::vector<uint32_t> host(4 + 5 * ns + nl, 0u);
  uint32_t *tab = host.data() + 4, *ssrc = tab + 4 * ns, *lsrc = ssrc + ns;
  for (size_t i = 0; i < ns; ++i) {
    const uint32_t r = small_ids[i], b = h_vertex_ranges[2 * r], e = h_vertex_ranges[2 * r + 1];
    tab[4 * i + 0] = b;
    tab[4 * i + 1] = e;
    tab[4 * i + 2] = g->h_boff[b];
    tab[4 * i + 3] = g->h_boff[e];
    ssrc[i] = t->h_sources[r];
  }
  std::copy(large_src.begin(), large_src.end(), lsrc);
  DeviceGuard dg(g->device);
  // queued work may still read the previous table
  MK_CUDA(cudaDeviceSynchronize());
  t->members_prepared = false;
  MK_CHECK(t->members.reserve(host.size(), &g->device_bytes));
  MK_CUDA(cudaMemcpy(t->members.ptr, host.data(), host.size() * 4, cudaMemcpyHostToDevice));
  t->n_small = (uint32_t)ns;
  t->n_large = (uint32_t)nl;
  t->small_max = ns ? len(small_ids[0]) : 0;
  t->small_grid = 0;
  if (ns) {
    const size_t smem = bfs_member_smem(t->small_max);
    auto kern = g->weighted ? k_bfs_members<true> : k_bfs_members<false>;
    const int most = (int)bfs_member_smem(kMemLocalMax);
    MK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, most));
    int per_sm = 0;
    MK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kMemThreads, smem));
    t->small_grid = (int)std::min<uint64_t>(ns, (uint64_t)device_sm_count(g->device) * std::max(per_sm, 1));
  }
  t->members_prepared = true;
  return MK_OK;
}

mk_status mk_bfs_static_members(mk_traversal *t, void *stream, float *ms_out) {
  if (!t) return fail(MK_ERR_INVALID, "mk_bfs_static_members: null handle");
  if (!t->members_prepared) return fail(MK_ERR_INVALID, "mk_bfs_static_members: no prepared ranges");
  mk_graph *g = t->g;
  DeviceGuard dg(g->device);
  cudaStream_t s = as_stream(stream);
  MK_CHECK(t->timer.start(s, ms_out != nullptr));
  const uint32_t ns = t->n_small, nl = t->n_large;
  uint32_t *counter = t->members.ptr;
  const uint4 *tab = reinterpret_cast<const uint4 *>(counter + 4);
  const uint32_t *ssrc = counter + 4 + 4 * (size_t)ns, *lsrc = ssrc + ns;
  if (nl) {
    // ranges too large for shared memory: the device-wide kernel from their
    // sources (it also resets every distance)
    MK_CHECK(trav_issue(t, kStatic, nullptr, nullptr, 0, s, lsrc, nl));
  } else {
    MK_CUDA(cudaMemsetAsync(t->dist, 0xFF, (size_t)g->V * 8, s));
    k_trav_recover<<<recover_grid(g), 256, 0, s>>>(t->ctl, t->stamp, t->inval, t->tpar, g->V);
    MK_CUDA(cudaMemsetAsync(t->ctl, 0, kRound * 4, s));
  }
  if (ns) {
    const size_t smem = bfs_member_smem(t->small_max);
    MK_CUDA(cudaMemsetAsync(counter, 0, 4, s));
    uint32_t *items = reinterpret_cast<uint32_t *>(t->fr0);
    if (g->weighted)
      k_bfs_members<true><<<t->small_grid, kMemThreads, smem, s>>>(g->view(), tab, ssrc, ns, counter, t->dist,
                                                                   items, t->inv_list, g->err_word());
    else
      k_bfs_members<false><<<t->small_grid, kMemThreads, smem, s>>>(g->view(), tab, ssrc, ns, counter, t->dist,
                                                                    items, t->inv_list, g->err_word());
    MK_CUDA(cudaGetLastError());
  }
  MK_CHECK(t->timer.stop(ms_out));
  t->has_static = true;
  return MK_OK;
}

mk_status mk_traversal_incremental(mk_traversal *t, const uint32_t *d_src,
                                   const uint32_t *d_dst, const uint32_t *d_w,
                                   uint32_t n, void *stream, float *ms_out) {
  (void)d_w;
  if (!t) return fail(MK_ERR_INVALID, "mk_traversal_incremental: null handle");
  return trav_launch(t, kIncremental, d_src, d_dst, n, stream, ms_out);
}

mk_status mk_traversal_decremental(mk_traversal *t, const uint32_t *d_src,
                                   const uint32_t *d_dst, const uint32_t *d_w,
                                   uint32_t n, void *stream, float *ms_out) {
  (void)d_w;
  if (!t) return fail(MK_ERR_INVALID, "mk_traversal_decremental: null handle");
  return trav_launch(t, kDecremental, d_src, d_dst, n, stream, ms_out);
}

mk_status mk_traversal_distances(mk_traversal *t, uint32_t *h_out) {
  if (!t || !h_out) return fail(MK_ERR_INVALID, "mk_traversal_distances: null argument");
  DeviceGuard dg(t->g->device);
  const size_t V = t->g->V;
  std::vector<unsigned long long> tmp(V);
  MK_CUDA(cudaDeviceSynchronize());
  uint32_t err = 0;
  MK_CUDA(cudaMemcpy(&err, t->ctl + kErr, 4, cudaMemcpyDeviceToHost));
  MK_CUDA(cudaMemcpy(tmp.data(), t->dist, V * 8, cudaMemcpyDeviceToHost));
  for (size_t i = 0; i < V; ++i) h_out[i] = pack_hi(tmp[i]);
  if (err & kErrTimeout) return fail(MK_ERR_TIMEOUT, "traversal: grid barrier timed out");
  return MK_OK;
}

mk_status mk_traversal_packed(mk_traversal *t, const uint64_t **d_packed) {
  if (!t || !d_packed) return fail(MK_ERR_INVALID, "mk_traversal_packed: null argument");
  *d_packed = reinterpret_cast<const uint64_t *>(t->dist);
  return MK_OK;
}

mk_status mk_traversal_packed_host(mk_traversal *t, uint64_t *h_out) {
  if (!t || !h_out) return fail(MK_ERR_INVALID, "mk_traversal_packed_host: null argument");
  DeviceGuard dg(t->g->device);
  MK_CUDA(cudaDeviceSynchronize());
  MK_CUDA(cudaMemcpy(h_out, t->dist, (size_t)t->g->V * 8, cudaMemcpyDeviceToHost));
  return MK_OK;
}

mk_status mk_traversal_stats(mk_traversal *t, uint32_t *h_levels, uint64_t *h_pushed) {
  if (!t) return fail(MK_ERR_INVALID, "mk_traversal_stats: null handle");
  DeviceGuard dg(t->g->device);
  MK_CUDA(cudaDeviceSynchronize());
  uint32_t ctl[kCtlWords];
  unsigned long long p = 0;
  MK_CUDA(cudaMemcpy(ctl, t->ctl, sizeof(ctl), cudaMemcpyDeviceToHost));
  MK_CUDA(cudaMemcpy(&p, t->pushed, 8, cudaMemcpyDeviceToHost));
  if (h_levels) *h_levels = ctl[kLevels];
  if (h_pushed) *h_pushed = p;
  if (ctl[kErr] & kErrTimeout) return fail(MK_ERR_TIMEOUT, "traversal: grid barrier timed out");
  return MK_OK;
}

mk_status mk_traversal_decremental_stats(mk_traversal *t, uint64_t *h_invalidated,
                                         uint32_t *h_recomputed) {
  if (!t) return fail(MK_ERR_INVALID, "mk_traversal_decremental_stats: null handle");
  DeviceGuard dg(t->g->device);
  MK_CUDA(cudaDeviceSynchronize());
  uint32_t ctl[kCtlWords];
  MK_CUDA(cudaMemcpy(ctl, t->ctl, sizeof(ctl), cudaMemcpyDeviceToHost));
  if (h_invalidated) *h_invalidated = ctl[kInvCount] + ctl[kEarly];
  if (h_recomputed) *h_recomputed = ctl[kRestart];
  if (ctl[kErr] & kErrTimeout) return fail(MK_ERR_TIMEOUT, "traversal: grid barrier timed out");
  return MK_OK;
}

mk_status mk_traversal_destroy(mk_traversal *t) {
  if (!t) return MK_OK;
  DeviceGuard dg(t->g->device);
  t->staging.release();
  cudaFree(t->dist);
  cudaFree(t->stamp);
  cudaFree(t->inval);
  cudaFree(t->fr0);
  cudaFree(t->fr1);
  cudaFree(t->inv_list);
  cudaFree(t->ctl);
  cudaFree(t->pushed);
  cudaFree(t->sources);
  free_repair(t);
  cudaFree(t->far0);
  cudaFree(t->far1);
  cudaFree(t->fbits);
  t->members.release();
  delete t;
  return MK_OK;
}

}  // extern "C"
