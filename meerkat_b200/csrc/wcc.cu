// Weakly connected components by lock-free union-find.
//
// The reference ships the device primitives only
// (include/Util/UnionFind.cuh:24-254): find with path splitting/halving, and
// union that hooks the larger root under the smaller one with a CAS
// (UnionAsync, :194-215), so every root is the minimum vertex id of its tree.
// This build adds the entry points:
//   static       every vertex is its own parent; two sampled out-edges per
//                vertex are unions, then every live edge whose endpoints do
//                not share a parent yet; then every vertex is compressed to
//                its root;
//   incremental  union of the edges the last insert applied, then compress;
//   decremental  see below.
// Labels are the minimum vertex id of each weakly connected component.
//
// Spanning forest.  Every union whose CAS hooks a root records the graph edge
// that caused it in the hooked root's slot (fe[root] = a << 32 | b, "a's slab
// table holds b").  Each hook joins two different trees, so the recorded
// edges form a spanning forest F of the graph: exactly the edges whose loss
// can split a component.  The decremental call uses F:
//   1. a forest edge whose directed edge the batch deleted stays in F,
//      turned around, when the reverse edge b -> a still exists; otherwise it
//      is dead and its component is affected.  No dead edge: nothing changed.
//   2. the affected components' parents are reset and their surviving forest
//      edges are unioned again: each component falls apart into the pieces
//      of F minus the dead edges (min-id roots);
//   3. one piece of each affected component is its main piece (the largest
//      of a sample for the most sampled component, else the piece holding
//      the old label); every edge that can join two pieces touches a vertex
//      outside the main piece, so only those vertices' out-edges and
//      (through the attached reverse graph) in-edges are scanned and unioned,
//      then the affected vertices are compressed (min-id roots: the labels
//      come out the same whichever piece is main).
// Without a reverse graph, or when the vertices outside the main pieces hold
// more than half of the graph's edge ends, the affected components are reset
// and rebuilt from their vertices' out-edges instead (an edge into an affected
// vertex comes from the same old component, so those out-edges are all its
// edges).  Every rebuild records its hooks, so F stays a spanning forest.
//
// Every retry loop is bounded; on expiry the kernel sets MK_DEVERR_TIMEOUT.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "mk_internal.h"
#include "mk_slab.cuh"
#include "mk_members.cuh"
#include "mk_update.cuh"

namespace mk {

// find with path halving; parent words are read through L2 because other
// SMs hook and halve concurrently.
__device__ __forceinline__ uint32_t uf_find(uint32_t *p, uint32_t x) {
  for (uint32_t it = 0; it < kUfLimit; ++it) {
    uint32_t px = __ldcg(p + x);
    if (px == x) return x;
    uint32_t gx = __ldcg(p + px);
    if (px != gx) p[x] = gx;  // x is not a root: only halving writes it
    x = gx;
  }
  return x;
}

// Root of x without writing: the compress pass uses it, because there a
// halving store from one thread (p[x] = grandparent) could land after
// another thread's final p[x] = root and leave x below a non-root.
__device__ __forceinline__ uint32_t uf_root(const uint32_t *p, uint32_t x) {
  for (uint32_t it = 0; it < kUfLimit; ++it) {
    const uint32_t px = __ldcg(p + x);
    if (px == x) return x;
    x = px;
  }
  return x;
}

constexpr unsigned long long kNoForest = ~0ull;  // empty forest slot

__device__ __forceinline__ unsigned long long fedge(uint32_t a, uint32_t b) {
  return ((unsigned long long)a << 32) | b;
}

// Union of the sets of a and b for the graph edge a -> b (a's slab table
// holds b).  With fe, the hook that joins two sets records that edge in the
// hooked root's forest slot (empty: a root has never been hooked since its
// reset).
__device__ __forceinline__ void uf_union(uint32_t *p, uint32_t a, uint32_t b, uint32_t *err,
                                         unsigned long long *fe = nullptr) {
  for (uint32_t it = 0; it < kUfLimit; ++it) {
    uint32_t ra = uf_find(p, a), rb = uf_find(p, b);
    if (ra == rb) return;
    uint32_t hi = ra > rb ? ra : rb, lo = ra > rb ? rb : ra;
    if (atomicCAS(p + hi, hi, lo) == hi) {
      if (fe) fe[hi] = fedge(a, b);
      return;
    }
  }
  atomicOr(err, kErrTimeout);
}

// uf_union that returns a vertex of the joined set which was its root during
// the call (kEmptyKey when the retry limit ran out).  An edge pass keeps it
// as the owner's parent for the owner's next keys: a key whose parent equals
// it is in the same set, so the hook just made is not tried again key by key.
__device__ __forceinline__ uint32_t uf_union_root(uint32_t *p, uint32_t a, uint32_t b,
                                                  uint32_t *err, unsigned long long *fe) {
  for (uint32_t it = 0; it < kUfLimit; ++it) {
    const uint32_t ra = uf_find(p, a), rb = uf_find(p, b);
    if (ra == rb) return ra;
    const uint32_t hi = ra > rb ? ra : rb, lo = ra > rb ? rb : ra;
    if (atomicCAS(p + hi, hi, lo) == hi) {
      if (fe) fe[hi] = fedge(a, b);
      return lo;
    }
  }
  atomicOr(err, kErrTimeout);
  return kEmptyKey;
}

// Resets the selected vertices (all if sel_bits is null) to their own set
// and, with fe, empties their forest slots.
__global__ void k_uf_init(uint32_t *p, uint32_t V, const uint32_t *sel_bits = nullptr,
                          unsigned long long *fe = nullptr) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < V; i += gridDim.x * blockDim.x) {
    if (sel_bits && !((sel_bits[i >> 5] >> (i & 31)) & 1u)) continue;
    p[i] = i;
    if (fe) fe[i] = kNoForest;
  }
}

// Unions of the edges the last insert applied (rev: the graph stores each
// batch edge turned around, so the recorded slab edge is dst -> src).
__global__ void k_uf_batch(const uint32_t *__restrict__ src, const uint32_t *__restrict__ dst,
                           const uint8_t *__restrict__ applied, uint32_t n, uint32_t V,
                           uint32_t rev, uint32_t *p, uint32_t *err, unsigned long long *fe) {
  uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n || !applied[e]) return;
  uint32_t a = src[e], b = dst[e];
  if (rev) {
    const uint32_t t = a;
    a = b;
    b = t;
  }
  if (a != b && a < V && b < V) uf_union(p, a, b, err, fe);
}

__global__ void k_uf_compress(uint32_t *p, uint32_t V, const uint32_t *sel_bits) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < V; i += gridDim.x * blockDim.x) {
    if (sel_bits && !((sel_bits[i >> 5] >> (i & 31)) & 1u)) continue;
    p[i] = uf_root(p, i);
  }
}

// Resets the vertices of affected components (their forest slots too) and
// records them.
__global__ void k_uf_reset(uint32_t *p, uint32_t V, const uint32_t *aff_labels, uint32_t *aff_vertices,
                           unsigned long long *fe) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < V; i += gridDim.x * blockDim.x) {
    uint32_t r = p[i];
    if ((aff_labels[r >> 5] >> (r & 31)) & 1u) {
      p[i] = i;
      fe[i] = kNoForest;
      atomicOr(aff_vertices + (i >> 5), 1u << (i & 31));
    }
  }
}

// ---- sampled linking, then a pass that skips already-connected edges ----
// Each vertex is first linked to up to two out-neighbours from its first head
// slab; after compression most vertices of every large component point at its
// root.  The full pass then skips every edge whose endpoints already have the
// same parent (they are connected), so on graphs with big components most
// edges cost two reads instead of two finds and a CAS.  Skipping only edges
// between vertices already connected keeps the result exact, and it works for
// every component at once (the members of a graph set included).
// Sampled linking: each selected vertex (all if sel_bits is null) unions
// with the first two live keys among the key slots of the first 32-byte
// sector of its first head slab (4 keys weighted, 8 unweighted; deleted
// edges leave tombstones there, so the first two slots alone link fewer
// vertices on a graph that has seen deletions).  A thread takes 4 vertices
// a stride apart per round, so their degree, offset and slab reads are in
// flight together before the unions.
template <bool kW>
__global__ void k_uf_sample(GraphView g, uint32_t *p, const uint32_t *sel_bits, uint32_t *err,
                            unsigned long long *fe) {
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint64_t u0 = blockIdx.x * blockDim.x + threadIdx.x; u0 < g.V; u0 += 4ull * stride) {
    uint32_t uu[4], k0[4], k1[4];
    bool ok[4];
#pragma unroll
    for (uint32_t j = 0; j < 4; ++j) {
      const uint64_t u = u0 + (uint64_t)j * stride;
      uu[j] = (uint32_t)u;
      ok[j] = u < g.V && g.deg[u] != 0 &&
              (!sel_bits || ((sel_bits[uu[j] >> 5] >> (uu[j] & 31)) & 1u));
    }
    uint4 qa[4], qb[4];
#pragma unroll
    for (uint32_t j = 0; j < 4; ++j) {
      if (ok[j]) {
        const uint4 *q = g.slabs + 8ull * g.boff[uu[j]];
        qa[j] = q[0];
        qb[j] = q[1];
      }
    }
#pragma unroll
    for (uint32_t j = 0; j < 4; ++j) {
      k0[j] = k1[j] = kEmptyKey;
      if (!ok[j]) continue;
      constexpr int kN = kW ? 4 : 8;
      const uint32_t keys[8] = {qa[j].x, kW ? qa[j].z : qa[j].y, kW ? qb[j].x : qa[j].z,
                                kW ? qb[j].z : qa[j].w, qb[j].x, qb[j].y, qb[j].z, qb[j].w};
#pragma unroll
      for (int t = 0; t < kN; ++t) {
        const uint32_t k = keys[t];
        if (k >= kTombKey || k == uu[j]) continue;
        if (k0[j] == kEmptyKey)
          k0[j] = k;
        else if (k1[j] == kEmptyKey)
          k1[j] = k;
      }
    }
#pragma unroll
    for (uint32_t j = 0; j < 4; ++j) {
      if (k0[j] < kTombKey) uf_union(p, uu[j], k0[j], err, fe);
      if (k1[j] < kTombKey) uf_union(p, uu[j], k1[j], err, fe);
    }
  }
}

// Unions of the out-edges of bucket b (owner u) whose endpoints do not share
// a parent yet.
template <bool kW>
__device__ __forceinline__ void link_bucket_skip(const GraphView &g, const Lanes &L, uint32_t *p,
                                                 uint32_t b, uint32_t u, uint32_t *err,
                                                 unsigned long long *fe) {
  const uint32_t pu = __ldcg(p + u);
  walk_bucket(g, L, b, [&](const uint4 &q) {
    uint32_t k[4], w[4];
    lane_keys<kW>(q, L.gl, k, w);
#pragma unroll
    for (int j = 0; j < keys_per_lane<kW>(); ++j) {
      const uint32_t v = k[j];
      if (v >= kTombKey || v == u) continue;
      if (__ldcg(p + v) == pu) continue;
      uf_union(p, u, v, err, fe);
    }
  });
}

// Every selected bucket (owner's bit set, all if sel_bits is null): unions of
// the out-edges whose endpoints do not share a parent yet (nothing when
// skip_if is given and holds a non-zero word).  A group takes 4
// consecutive buckets at a time: their owners' parents and head slabs are
// loaded together, chains are followed level by level, and a lane loads the
// parents of all its keys before comparing, so one group keeps several
// reads in flight instead of one dependent read per key.
template <bool kW>
__global__ void k_uf_edges_skip(GraphView g, uint32_t *p, const uint32_t *sel_bits, uint32_t *err,
                                unsigned long long *fe, const unsigned long long *skip_if = nullptr) {
  if (skip_if && *skip_if) return;
  const Lanes L = lanes();
  const uint32_t group = (blockIdx.x * blockDim.x + threadIdx.x) >> 3;
  const uint32_t ngroups = (gridDim.x * blockDim.x) >> 3;
  for (uint64_t b0 = (uint64_t)group * 4; b0 < g.nbuckets; b0 += (uint64_t)ngroups * 4) {
    const uint32_t b = (uint32_t)b0, m = min(4u, g.nbuckets - b);
    uint32_t own[4], pu[4], live = 0;
#pragma unroll
    for (uint32_t j = 0; j < 4; ++j) {
      own[j] = j < m ? __ldg(g.bowner + b + j) : 0u;
      const bool ok = j < m && g.deg[own[j]] != 0 &&
                      (!sel_bits || ((sel_bits[own[j] >> 5] >> (own[j] & 31)) & 1u));
      live |= (ok ? 1u : 0u) << j;
    }
    if (!live) continue;
#pragma unroll
    for (uint32_t j = 0; j < 4; ++j) pu[j] = ((live >> j) & 1u) ? __ldcg(p + own[j]) : 0u;
    walk4_levels(g, L, b, m, [&](uint32_t j, const uint4 q) {
      if (!((live >> j) & 1u)) return;
      const uint32_t u = own[0] * (j == 0) + own[1] * (j == 1) + own[2] * (j == 2) + own[3] * (j == 3);
      uint32_t pj = pu[0] * (j == 0) + pu[1] * (j == 1) + pu[2] * (j == 2) + pu[3] * (j == 3);
      uint32_t k[4], w[4];
      lane_keys<kW>(q, L.gl, k, w);
      uint32_t pv[4];
      bool ok[4];
#pragma unroll
      for (int t = 0; t < keys_per_lane<kW>(); ++t) {
        ok[t] = k[t] < kTombKey && k[t] != u;
        pv[t] = ok[t] ? __ldcg(p + k[t]) : 0u;
      }
#pragma unroll
      for (int t = 0; t < keys_per_lane<kW>(); ++t)
        if (ok[t] && pv[t] != pj) pj = uf_union_root(p, u, k[t], err, fe);
#pragma unroll
      for (uint32_t i = 0; i < 4; ++i)
        if (i == j) pu[i] = pj;
    });
  }
}

// ---- decremental repair over the spanning forest ----
// ctl words (u64) of one decremental call.
enum : int {
  kFDead = 0,       // forest edges the batch removed for good
  kFNmCount = 1,    // vertices outside their component's main piece
  kFNmEnds = 2,     // their out- plus in-degrees
  kFEdges = 3,      // live edges of the graph
  kFMainLabel = 4,  // old label + 1 of the component whose main piece was sampled (0: none)
  kFMainPiece = 5,  // that main piece's root + 1
  kFAffected = 6,   // vertices of the affected components
  kFGiant = 7,      // static passes: the most sampled set's root + 1 (0: none)
  kFItemsOut = 8,   // scan items listed for the graph (out-edges)
  kFItemsIn = 9,    // scan items listed for the reverse graph (in-edges)
  kFCtlWords = 10
};

// A scan item is the first of up to kItemBuckets consecutive buckets of one
// vertex (its owner is bowner[item]), so a hub's buckets spread over many
// groups.  A vertex with nb buckets takes ceil(nb / kItemBuckets) items: a
// list never holds more than V + nbuckets / kItemBuckets of them.
constexpr uint32_t kItemBuckets = 4;

// Vertices per lane of the list-building passes: a warp takes 256 at a time
// and appends their items with one atomic (one per warp and 32 vertices
// queued tens of thousands of atomics on the same word).
constexpr int kPerLane = 8;

// Appends the items of buckets [b0[i], b1[i]) of every lane (empty ranges
// add none), one atomic per warp; any order.  All 32 lanes of the warp call
// it together.
__device__ __forceinline__ void append_items(const uint32_t (&b0)[kPerLane],
                                             const uint32_t (&b1)[kPerLane], uint32_t *items,
                                             unsigned long long *count) {
  const uint32_t lane = threadIdx.x & 31u;
  uint32_t n = 0;
#pragma unroll
  for (int i = 0; i < kPerLane; ++i)
    n += b1[i] > b0[i] ? (b1[i] - b0[i] + kItemBuckets - 1) / kItemBuckets : 0u;
  uint32_t incl = n;
#pragma unroll
  for (uint32_t o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(0xFFFFFFFFu, incl, o);
    if (lane >= o) incl += t;
  }
  const uint32_t total = __shfl_sync(0xFFFFFFFFu, incl, 31);
  if (total == 0) return;
  uint32_t at = 0;
  if (lane == 0) at = (uint32_t)atomicAdd(count, (unsigned long long)total);
  at = __shfl_sync(0xFFFFFFFFu, at, 0) + incl - n;
#pragma unroll
  for (int i = 0; i < kPerLane; ++i)
    for (uint32_t b = b0[i]; b < b1[i]; b += kItemBuckets) items[at++] = b;
}

// Adds v summed over the block to *dst with one atomic.  Every thread of the
// block calls it (blockDim.x a multiple of 32).
__device__ __forceinline__ void block_add(unsigned long long v, unsigned long long *dst) {
  __shared__ unsigned long long part[32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
  if ((threadIdx.x & 31u) == 0) part[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    unsigned long long t = threadIdx.x < (blockDim.x >> 5) ? part[threadIdx.x] : 0ull;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xFFFFFFFFu, t, o);
    if (threadIdx.x == 0 && t) atomicAdd(dst, t);
  }
  __syncthreads();  // part is reused by the next call
}

// Set of the batch's deleted edges (slab orientation a << 32 | b): open
// addressing over a power-of-two table (mask + 1 slots, at least twice the
// batch), linear probing, EMPTY = ~0.
__device__ __forceinline__ uint32_t dh_slot(unsigned long long key, uint32_t mask) {
  key ^= key >> 33;
  key *= 0xff51afd7ed558ccdull;
  key ^= key >> 33;
  return (uint32_t)key & mask;
}

__global__ void k_dh_insert(const uint32_t *__restrict__ src, const uint32_t *__restrict__ dst,
                            const uint8_t *__restrict__ applied, uint32_t n, uint32_t rev,
                            unsigned long long *tab, uint32_t mask) {
  const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n || !applied[e]) return;
  uint32_t a = src[e], b = dst[e];
  if (rev) {
    const uint32_t t = a;
    a = b;
    b = t;
  }
  const unsigned long long key = fedge(a, b);
  uint32_t s = dh_slot(key, mask);
  for (uint32_t it = 0; it <= mask; ++it) {
    const unsigned long long old = atomicCAS(tab + s, kNoForest, key);
    if (old == kNoForest || old == key) return;
    s = (s + 1) & mask;
  }
}

__device__ __forceinline__ bool dh_has(const unsigned long long *tab, uint32_t mask,
                                       unsigned long long key) {
  uint32_t s = dh_slot(key, mask);
  for (uint32_t it = 0; it <= mask; ++it) {
    const unsigned long long k = __ldg(tab + s);
    if (k == key) return true;
    if (k == kNoForest) return false;
    s = (s + 1) & mask;
  }
  return false;
}

// True when u's slab table holds key (one thread, whole slabs).
template <bool kW>
__device__ __forceinline__ bool lane_has_key(const GraphView &g, uint32_t u, uint32_t key) {
  const uint32_t b0 = __ldg(g.boff + u), nb = __ldg(g.boff + u + 1) - b0;
  if (nb == 0) return false;
  uint32_t s = b0 + bucket_of(key, nb);
  for (uint32_t it = 0; it < kProbeLimit; ++it) {
    uint4 q[8];
    lane_load_slab(g, s, q);
    const LaneProbe pr = lane_probe<kW>(q, key);
    if (pr.found_word < 32) return true;
    if (pr.next == kNoSlab) return false;
    s = pr.next;
  }
  return false;
}

// Step 1: forest edges the batch deleted.  A deleted a -> b whose reverse
// b -> a still exists stays in the forest turned around; otherwise the slot
// empties and the component (its label, the compressed parent of a) is
// affected.
template <bool kW>
__global__ void k_fe_dead(GraphView g, unsigned long long *fe, const unsigned long long *tab,
                          uint32_t mask, const uint32_t *p, uint32_t *aff_labels,
                          unsigned long long *ctl) {
  for (uint32_t x = blockIdx.x * blockDim.x + threadIdx.x; x < g.V; x += gridDim.x * blockDim.x) {
    const unsigned long long e = fe[x];
    if (e == kNoForest || !dh_has(tab, mask, e)) continue;
    const uint32_t a = (uint32_t)(e >> 32), b = (uint32_t)e;
    if (lane_has_key<kW>(g, b, a)) {
      fe[x] = fedge(b, a);
      continue;
    }
    fe[x] = kNoForest;
    const uint32_t r = p[a];
    atomicOr(aff_labels + (r >> 5), 1u << (r & 31));
    atomicAdd(ctl + kFDead, 1ull);
  }
}

// Step 1b: vertices of the affected components (labels still compressed),
// one atomic per block.
__global__ void k_fe_count_aff(const uint32_t *p, uint32_t V, const uint32_t *aff_labels,
                               unsigned long long *ctl) {
  unsigned long long n = 0;
  for (uint32_t x = blockIdx.x * blockDim.x + threadIdx.x; x < V; x += gridDim.x * blockDim.x) {
    const uint32_t r = p[x];
    n += (aff_labels[r >> 5] >> (r & 31)) & 1u;
  }
  block_add(n, ctl + kFAffected);
}

// Step 2a: every vertex of an affected component keeps its old label, is
// reset to its own set and hands its forest edge over to fe2; aff_vertices
// gets the affected-vertex bitmap (whole words, one ballot each).
__global__ void k_fe_collect(uint32_t *p, unsigned long long *fe, unsigned long long *fe2, uint32_t V,
                             const uint32_t *aff_labels, uint32_t *oldlab, uint32_t *aff_vertices) {
  const uint32_t words = (V + 31) / 32, lane = threadIdx.x & 31u;
  const uint32_t stride = gridDim.x * blockDim.x;  // a multiple of 32
  for (uint32_t base = (blockIdx.x * blockDim.x + threadIdx.x) & ~31u; base < words * 32u;
       base += stride) {
    const uint32_t x = base + lane;
    bool aff = false;
    if (x < V) {
      const uint32_t r = p[x];
      aff = (aff_labels[r >> 5] >> (r & 31)) & 1u;
      if (aff) {
        oldlab[x] = r;
        p[x] = x;
        fe2[x] = fe[x];
        fe[x] = kNoForest;
      }
    }
    const uint32_t word = __ballot_sync(0xFFFFFFFFu, aff);
    if (lane == 0) aff_vertices[base >> 5] = word;
  }
}

// Step 2b: the surviving forest edges of the affected vertices, unioned again
// (every one joins two sets: they form a forest), recorded at their new hooks.
__global__ void k_fe_union(uint32_t *p, unsigned long long *fe, const unsigned long long *fe2,
                           uint32_t V, const uint32_t *aff_vertices, uint32_t *err) {
  for (uint32_t x = blockIdx.x * blockDim.x + threadIdx.x; x < V; x += gridDim.x * blockDim.x) {
    if (!((aff_vertices[x >> 5] >> (x & 31)) & 1u)) continue;
    const unsigned long long e = fe2[x];
    if (e == kNoForest) continue;
    uf_union(p, (uint32_t)(e >> 32), (uint32_t)e, err, fe);
  }
}

// Step 3a: the main piece of the most sampled component.  Any one piece per
// component may be its main piece (every edge between two pieces touches a
// vertex outside it, and min-id unions give the same labels); the largest
// leaves the least to rescan.  One CTA draws kMainSamples vertices, counts
// the affected ones by piece root in shared memory and keeps the most
// frequent piece (at least 32 samples) as the main piece of its component.
// Every other component keeps the piece of its old label.
constexpr int kMainThreads = 1024;
constexpr uint32_t kMainSamples = 2048, kMainSlots = 4096;  // slots: twice the samples

__global__ void __launch_bounds__(kMainThreads)
    k_fe_main_sample(const uint32_t *p, const uint32_t *oldlab, const uint32_t *aff_vertices,
                     uint32_t V, unsigned long long seed, unsigned long long *ctl) {
  __shared__ uint32_t keys[kMainSlots], cnts[kMainSlots];
  __shared__ unsigned long long best;
  for (uint32_t i = threadIdx.x; i < kMainSlots; i += blockDim.x) {
    keys[i] = 0xFFFFFFFFu;
    cnts[i] = 0u;
  }
  if (threadIdx.x == 0) best = 0;
  __syncthreads();
  for (uint32_t j = threadIdx.x; j < kMainSamples; j += blockDim.x) {
    unsigned long long h = seed + 0x9E3779B97F4A7C15ull * (j + 1);
    h ^= h >> 33;
    h *= 0xff51afd7ed558ccdull;
    h ^= h >> 33;
    const uint32_t x = (uint32_t)(h % V);
    if (!((aff_vertices[x >> 5] >> (x & 31)) & 1u)) continue;
    const uint32_t k = __ldcg(p + x);
    uint32_t sl = (k * 2654435761u) & (kMainSlots - 1);
    for (uint32_t it = 0; it < kMainSlots; ++it) {
      const uint32_t old = atomicCAS(keys + sl, 0xFFFFFFFFu, k);
      if (old == 0xFFFFFFFFu || old == k) {
        atomicAdd(cnts + sl, 1u);
        break;
      }
      sl = (sl + 1) & (kMainSlots - 1);
    }
  }
  __syncthreads();
  unsigned long long mine = 0;
  for (uint32_t i = threadIdx.x; i < kMainSlots; i += blockDim.x) {
    const unsigned long long c = ((unsigned long long)cnts[i] << 32) | keys[i];
    if (cnts[i] && c > mine) mine = c;
  }
  atomicMax(&best, mine);
  __syncthreads();
  if (threadIdx.x == 0 && (best >> 32) >= 32) {
    const uint32_t piece = (uint32_t)best;
    ctl[kFMainLabel] = (unsigned long long)oldlab[piece] + 1;
    ctl[kFMainPiece] = (unsigned long long)piece + 1;
  }
}

// Step 3b (after compressing the affected vertices): the affected vertices
// outside their component's main piece, as scan items of their out-buckets
// (graph) and in-buckets (reverse graph); their count and out- plus
// in-degrees, and the graph's live edge count (one atomic per block).
__global__ void k_fe_nonmain(const uint32_t *p, const uint32_t *oldlab, uint32_t V,
                             const uint32_t *aff_vertices, GraphView g, GraphView rg,
                             uint32_t *items_out, uint32_t *items_in, unsigned long long *ctl) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint64_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = (gridDim.x * blockDim.x) >> 5;
  const unsigned long long ml = ctl[kFMainLabel], mp = ctl[kFMainPiece];
  unsigned long long ends = 0, edges = 0, count = 0;
  for (uint64_t base = warp * 32 * kPerLane; base < V; base += nwarps * 32 * kPerLane) {
    uint32_t ob[kPerLane], oe[kPerLane], ib[kPerLane], ie[kPerLane];
#pragma unroll
    for (int i = 0; i < kPerLane; ++i) {
      ob[i] = oe[i] = ib[i] = ie[i] = 0;
      const uint64_t xx = base + (uint64_t)i * 32 + lane;
      if (xx >= V) continue;
      const uint32_t x = (uint32_t)xx;
      const uint32_t d = g.deg[x];
      edges += d;
      if (!((aff_vertices[x >> 5] >> (x & 31)) & 1u)) continue;
      const uint32_t r = oldlab[x];
      const uint32_t main_piece = (ml && r == ml - 1) ? (uint32_t)(mp - 1) : __ldcg(p + r);
      if (__ldcg(p + x) == main_piece) continue;
      const uint32_t rd = rg.deg[x];
      ends += d + rd;
      ++count;
      if (d) {
        ob[i] = g.boff[x];
        oe[i] = g.boff[x + 1];
      }
      if (rd) {
        ib[i] = rg.boff[x];
        ie[i] = rg.boff[x + 1];
      }
    }
    append_items(ob, oe, items_out, ctl + kFItemsOut);
    append_items(ib, ie, items_in, ctl + kFItemsIn);
  }
  block_add(count, ctl + kFNmCount);
  block_add(ends, ctl + kFNmEnds);
  block_add(edges, ctl + kFEdges);
}

// True once x's set holds its component's main piece: its root is the
// main piece's (the sampled piece for the sampled component, else the piece
// of the old label).  The rescan skips such a vertex's remaining buckets:
// any piece still joined through x finds the edge from its own side.
__device__ __forceinline__ bool fe_joined(uint32_t *p, const uint32_t *oldlab, uint32_t x,
                                          unsigned long long ml, unsigned long long mp) {
  const uint32_t r = __ldg(oldlab + x);
  const uint32_t m = (ml && r == ml - 1) ? (uint32_t)(mp - 1) : r;
  return uf_find(p, x) == uf_find(p, m);
}

// ---- static passes with a reverse graph: skip the largest set ----
// After sampled linking (and a compress) most vertices of a large component
// already point at its root.  One CTA draws kMainSamples vertices with
// out-edges and keeps the most frequent root (at least 32 samples) as the
// giant set.  Every edge with both ends in it needs no union; every other
// edge has an end outside it, whose out-edges (graph) or in-edges (reverse
// graph) are then scanned, so the giant set's own edges are never read.  The
// outside vertices are compacted into a list first: a pass over every bucket
// that only skips most of them costs about as much as one that walks them
// when the buckets are short (on a grid, one slab per vertex).
__global__ void __launch_bounds__(kMainThreads)
    k_uf_giant_sample(const uint32_t *p, const uint32_t *deg, uint32_t V, unsigned long long seed,
                      unsigned long long *ctl) {
  __shared__ uint32_t keys[kMainSlots], cnts[kMainSlots];
  __shared__ unsigned long long best;
  __shared__ uint32_t drawn;  // samples with out-edges
  for (uint32_t i = threadIdx.x; i < kMainSlots; i += blockDim.x) {
    keys[i] = 0xFFFFFFFFu;
    cnts[i] = 0u;
  }
  if (threadIdx.x == 0) {
    best = 0;
    drawn = 0;
  }
  __syncthreads();
  for (uint32_t j = threadIdx.x; j < kMainSamples; j += blockDim.x) {
    unsigned long long h = seed + 0x9E3779B97F4A7C15ull * (j + 1);
    h ^= h >> 33;
    h *= 0xff51afd7ed558ccdull;
    h ^= h >> 33;
    const uint32_t x = (uint32_t)(h % V);
    if (deg[x] == 0) continue;
    atomicAdd(&drawn, 1u);
    const uint32_t k = __ldcg(p + x);
    uint32_t sl = (k * 2654435761u) & (kMainSlots - 1);
    for (uint32_t it = 0; it < kMainSlots; ++it) {
      const uint32_t old = atomicCAS(keys + sl, 0xFFFFFFFFu, k);
      if (old == 0xFFFFFFFFu || old == k) {
        atomicAdd(cnts + sl, 1u);
        break;
      }
      sl = (sl + 1) & (kMainSlots - 1);
    }
  }
  __syncthreads();
  unsigned long long mine = 0;
  for (uint32_t i = threadIdx.x; i < kMainSlots; i += blockDim.x) {
    const unsigned long long c = ((unsigned long long)cnts[i] << 32) | keys[i];
    if (cnts[i] && c > mine) mine = c;
  }
  atomicMax(&best, mine);
  __syncthreads();
  // a set holding under three quarters of the samples would leave most
  // edges to scan from both ends: then no giant set (every out-edge once, as
  // without a reverse graph)
  if (threadIdx.x == 0)
    ctl[kFGiant] = ((best >> 32) >= 32 && 4 * (best >> 32) >= 3ull * drawn)
                       ? (unsigned long long)(uint32_t)best + 1 : 0ull;
}

// The vertices outside the giant set, as scan items of their out-buckets
// (graph) and in-buckets (reverse graph).  Nothing without a giant set.
__global__ void k_uf_outside_items(const uint32_t *p, uint32_t V, GraphView g, GraphView rg,
                                   unsigned long long *ctl, uint32_t *items_out,
                                   uint32_t *items_in) {
  const unsigned long long giant = ctl[kFGiant];
  if (giant == 0) return;
  const uint32_t lane = threadIdx.x & 31u;
  const uint64_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = (gridDim.x * blockDim.x) >> 5;
  for (uint64_t base = warp * 32 * kPerLane; base < V; base += nwarps * 32 * kPerLane) {
    uint32_t ob[kPerLane], oe[kPerLane], ib[kPerLane], ie[kPerLane];
#pragma unroll
    for (int i = 0; i < kPerLane; ++i) {
      ob[i] = oe[i] = ib[i] = ie[i] = 0;
      const uint64_t xx = base + (uint64_t)i * 32 + lane;
      if (xx >= V) continue;
      const uint32_t x = (uint32_t)xx;
      const uint32_t d = g.deg[x], rd = rg.deg[x];
      if ((d | rd) == 0 || __ldcg(p + x) == (uint32_t)(giant - 1)) continue;
      if (d) {
        ob[i] = g.boff[x];
        oe[i] = g.boff[x + 1];
      }
      if (rd) {
        ib[i] = rg.boff[x];
        ie[i] = rg.boff[x + 1];
      }
    }
    append_items(ob, oe, items_out, ctl + kFItemsOut);
    append_items(ib, ie, items_in, ctl + kFItemsIn);
  }
}

// The edges of the listed items (ctl[which] of them) of the graph (kIn: of
// the reverse graph, whose key y is the graph edge y -> x): unions of the
// edges whose endpoints do not share a parent yet.  A group takes 4 items at
// a time and walks one bucket of each per round.  With kStop (the
// decremental rescan) an item stops once its owner is joined to its main
// piece: any piece still joined through it finds the edge from its own side.
template <bool kW, bool kIn, bool kStop>
__global__ void k_uf_scan_items(GraphView g, uint32_t *p, const uint32_t *items, int which,
                                const uint32_t *oldlab, const unsigned long long *ctl,
                                uint32_t *err, unsigned long long *fe) {
  const Lanes L = lanes();
  const uint32_t group = (blockIdx.x * blockDim.x + threadIdx.x) >> 3;
  const uint32_t ngroups = (gridDim.x * blockDim.x) >> 3;
  const uint64_t n = ctl[which];
  const unsigned long long ml = kStop ? ctl[kFMainLabel] : 0, mp = kStop ? ctl[kFMainPiece] : 0;
  for (uint64_t i0 = (uint64_t)group * 4; i0 < n; i0 += (uint64_t)ngroups * 4) {
    const uint32_t m = n - i0 < 4 ? (uint32_t)(n - i0) : 4u;
    uint32_t own[4], bk[4], be[4], px[4];
#pragma unroll
    for (uint32_t j = 0; j < 4; ++j) {
      bk[j] = j < m ? __ldcg(items + i0 + j) : 0u;
      own[j] = j < m ? __ldg(g.bowner + bk[j]) : 0u;
      be[j] = j < m ? min(bk[j] + kItemBuckets, __ldg(g.boff + own[j] + 1)) : 0u;
    }
    bool first = true;
    for (;;) {
      uint32_t live = 0;
#pragma unroll
      for (uint32_t j = 0; j < 4; ++j) live |= (bk[j] < be[j] ? 1u : 0u) << j;
      if (kStop) {
        // decided on one lane and broadcast: the walk below shuffles within
        // the group, so every lane must take the same buckets
        uint32_t drop = 0;
        if (L.gl == 0) {
#pragma unroll
          for (uint32_t j = 0; j < 4; ++j)
            if (((live >> j) & 1u) && fe_joined(p, oldlab, own[j], ml, mp)) drop |= 1u << j;
        }
        drop = __shfl_sync(L.gmask, drop, L.gbase);
        live &= ~drop;
#pragma unroll
        for (uint32_t j = 0; j < 4; ++j)
          if ((drop >> j) & 1u) be[j] = bk[j];
      }
      if (!live) break;
      if (first) {
#pragma unroll
        for (uint32_t j = 0; j < 4; ++j) px[j] = ((live >> j) & 1u) ? __ldcg(p + own[j]) : 0u;
        first = false;
      }
      walk4_set(g, L, bk, live, [&](uint32_t j, const uint4 q) {
        const uint32_t x = own[0] * (j == 0) + own[1] * (j == 1) + own[2] * (j == 2) + own[3] * (j == 3);
        uint32_t pj = px[0] * (j == 0) + px[1] * (j == 1) + px[2] * (j == 2) + px[3] * (j == 3);
        uint32_t k[4], w[4];
        lane_keys<kW>(q, L.gl, k, w);
        uint32_t py[4];
        bool ok[4];
#pragma unroll
        for (int t = 0; t < keys_per_lane<kW>(); ++t) {
          ok[t] = k[t] < kTombKey && k[t] != x && k[t] < g.V;
          py[t] = ok[t] ? __ldcg(p + k[t]) : 0u;
        }
#pragma unroll
        for (int t = 0; t < keys_per_lane<kW>(); ++t) {
          if (!ok[t] || py[t] == pj) continue;
          // kIn: the slab edge k -> x of the graph
          pj = kIn ? uf_union_root(p, k[t], x, err, fe) : uf_union_root(p, x, k[t], err, fe);
        }
#pragma unroll
        for (uint32_t i = 0; i < 4; ++i)
          if (i == j) px[i] = pj;
      });
#pragma unroll
      for (uint32_t j = 0; j < 4; ++j) bk[j] += bk[j] < be[j] ? 1u : 0u;
    }
  }
}

// Both item scans over the graph and its reverse graph.
template <bool kStop>
static void launch_item_scans(const GraphView &v, bool vw, const GraphView &rv, bool rw, int blocks,
                              uint32_t *p, const uint32_t *items_out, const uint32_t *items_in,
                              const uint32_t *oldlab, const unsigned long long *ctl, uint32_t *err,
                              unsigned long long *fe, cudaStream_t s) {
  if (vw)
    k_uf_scan_items<true, false, kStop><<<blocks, 256, 0, s>>>(v, p, items_out, kFItemsOut, oldlab,
                                                               ctl, err, fe);
  else
    k_uf_scan_items<false, false, kStop><<<blocks, 256, 0, s>>>(v, p, items_out, kFItemsOut, oldlab,
                                                                ctl, err, fe);
  if (rw)
    k_uf_scan_items<true, true, kStop><<<blocks, 256, 0, s>>>(rv, p, items_in, kFItemsIn, oldlab,
                                                              ctl, err, fe);
  else
    k_uf_scan_items<false, true, kStop><<<blocks, 256, 0, s>>>(rv, p, items_in, kFItemsIn, oldlab,
                                                               ctl, err, fe);
}

// ---- vertex-range variants: only the listed ranges are touched ----
// Ranges are given as prefix sums: range r covers the global indices
// [pre[r], pre[r+1]) of a concatenation, starting at base[r].
__device__ __forceinline__ uint32_t range_at(const uint32_t *pre, uint32_t nr, uint32_t i,
                                             const uint32_t *base) {
  uint32_t lo = 0, hi = nr;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (pre[mid] <= i)
      lo = mid;
    else
      hi = mid;
  }
  return base[lo] + (i - pre[lo]);
}

__global__ void k_uf_init_ranges(uint32_t *p, const uint32_t *vpre, const uint32_t *vbase,
                                 uint32_t nr) {
  const uint32_t total = vpre[nr];
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
    const uint32_t v = range_at(vpre, nr, i, vbase);
    p[v] = v;
  }
}

template <bool kW>
__global__ void k_uf_sample_ranges(GraphView g, uint32_t *p, const uint32_t *vpre,
                                   const uint32_t *vbase, uint32_t nr, uint32_t *err) {
  const uint32_t total = vpre[nr];
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
    const uint32_t u = range_at(vpre, nr, i, vbase);
    if (g.deg[u] == 0) continue;
    const uint32_t *w = reinterpret_cast<const uint32_t *>(g.slabs + 8ull * g.boff[u]);
    const uint32_t k0 = w[0], k1 = kW ? w[2] : w[1];
    if (k0 < kTombKey && k0 != u) uf_union(p, u, k0, err);
    if (k1 < kTombKey && k1 != u) uf_union(p, u, k1, err);
  }
}

template <bool kW>
__global__ void k_uf_edges_ranges(GraphView g, uint32_t *p, const uint32_t *bpre,
                                  const uint32_t *bbase, uint32_t nr, uint32_t *err) {
  const Lanes L = lanes();
  const uint32_t group = (blockIdx.x * blockDim.x + threadIdx.x) >> 3;
  const uint32_t ngroups = (gridDim.x * blockDim.x) >> 3;
  const uint32_t total = bpre[nr];
  for (uint32_t i = group; i < total; i += ngroups) {
    const uint32_t b = range_at(bpre, nr, i, bbase);
    const uint32_t u = g.bowner[b];
    if (g.deg[u] == 0) continue;
    link_bucket_skip<kW>(g, L, p, b, u, err, nullptr);
  }
}

__global__ void k_uf_compress_ranges(uint32_t *p, const uint32_t *vpre, const uint32_t *vbase,
                                     uint32_t nr) {
  const uint32_t total = vpre[nr];
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
    const uint32_t v = range_at(vpre, nr, i, vbase);
    p[v] = uf_root(p, v);
  }
}

// ---- ranges held in shared memory ----
// A range of at most kUfLocalMax vertices (a member of a graph set) is solved
// by one CTA with its union-find in shared memory (uf_member).  CTAs take
// ranges from a counter, largest first.  rng[r] = (first vertex, end vertex,
// first bucket, end bucket).
template <bool kW>
__global__ void __launch_bounds__(kMemThreads, 1)
    k_uf_members(GraphView g, const uint4 *__restrict__ rng, uint32_t nr, uint32_t *counter,
                 uint32_t *__restrict__ labels, uint32_t *err) {
  extern __shared__ uint16_t sp[];
  __shared__ uint32_t s_range;
  const Lanes L = lanes();
  for (;;) {
    if (threadIdx.x == 0) s_range = atomicAdd(counter, 1u);
    __syncthreads();
    const uint32_t r = s_range;
    if (r >= nr) break;
    uf_member<kW, false>(g, L, rng[r], labels, err, sp);
  }
}

}  // namespace mk

using namespace mk;

struct mk_wcc {
  mk_graph *g = nullptr;
  uint32_t *parent = nullptr;
  uint32_t *aff_labels = nullptr;
  uint32_t *aff_vertices = nullptr;
  uint32_t *err = nullptr;  // the graph's sticky device error word
  // spanning forest: fe[v] = the edge (a << 32 | b) whose union hooked root v
  unsigned long long *fe = nullptr;
  bool forest_valid = false;  // fe spans every component (after a full static)
  mk_graph *rev = nullptr;    // reverse graph of the same edges (in-edges), optional
  // decremental scratch: batch edge set, old labels, handed-over forest
  // edges, ctl words
  DevBuf<unsigned long long> dtab;
  DevBuf<unsigned long long> fe2;
  DevBuf<uint32_t> oldlab;
  // scan items (first buckets) of the graph and of the reverse graph
  DevBuf<uint32_t> items_out, items_in;
  unsigned long long *fctl = nullptr;
  // last decremental call: forest edges lost, vertices rescanned, path taken
  uint64_t last_dead = 0, last_rescanned = 0;
  uint32_t last_path = 0;
  uint64_t calls = 0;  // decremental calls (seeds the main-piece sample)
  // after a split whose pieces were too large to rescan, the next calls go
  // straight to the static passes: skip_left of them, doubling (to 8) with
  // every further such split, reset by a rescan that succeeds
  uint32_t skip_left = 0, skip_next = 0;
  // prepared range table: counter word, then uint4 (lo, hi, b0, b1) per small
  // range (largest first), then vpre, vbase, bpre, bbase of the large ranges
  DevBuf<uint32_t> ranges;
  uint32_t n_small = 0, n_large = 0, small_max = 0;
  uint64_t large_vt = 0, large_bt = 0;
  int small_grid = 0;
  bool prepared = false;
  PinnedRing staging;  // stream-ordered range-table uploads
  Timer timer;
};

static int flat_grid(uint64_t n, int device) {
  return (int)std::min<uint64_t>(n / 256 + 1, (uint64_t)device_sm_count(device) * 8);
}

// Room for every scan item of the graph and of the reverse graph.
static mk_status reserve_items(mk_wcc *w) {
  mk_graph *g = w->g;
  MK_CHECK(w->items_out.reserve(g->V + g->num_buckets / kItemBuckets + 1, &g->device_bytes));
  MK_CHECK(w->items_in.reserve(g->V + w->rev->num_buckets / kItemBuckets + 1, &g->device_bytes));
  return MK_OK;
}

// Unions of the out-edges of the selected vertices (all if sel is null), whose
// parents start reset: sample two neighbours each, compress, then every edge
// whose endpoints do not share a parent yet.
static mk_status wcc_link(mk_wcc *w, const uint32_t *sel, cudaStream_t s) {
  mk_graph *g = w->g;
  const int fg = flat_grid(g->V, g->device);
  const GraphView v = g->view();
  if (g->weighted)
    k_uf_sample<true><<<fg, 256, 0, s>>>(v, w->parent, sel, w->err, w->fe);
  else
    k_uf_sample<false><<<fg, 256, 0, s>>>(v, w->parent, sel, w->err, w->fe);
  k_uf_compress<<<fg, 256, 0, s>>>(w->parent, g->V, sel);
  const int blocks = (int)std::min<uint64_t>(g->num_buckets * 8 / 256 + 1,
                                             (uint64_t)device_sm_count(g->device) * 8);
  if (g->weighted)
    k_uf_edges_skip<true><<<blocks, 256, 0, s>>>(v, w->parent, sel, w->err, w->fe);
  else
    k_uf_edges_skip<false><<<blocks, 256, 0, s>>>(v, w->parent, sel, w->err, w->fe);
  k_uf_compress<<<fg, 256, 0, s>>>(w->parent, g->V, sel);
  MK_CUDA(cudaGetLastError());
  return MK_OK;
}

// Static passes.  With a reverse graph attached: sampled linking, then only
// the vertices outside the largest sampled set have their out- and in-edges
// scanned, as lists of bucket items (k_uf_giant_sample; when that set holds
// under 3/4 of the samples, every out-edge once instead: the device decides,
// the host launches both forms and one returns at once); without one, every
// edge through k_uf_edges_skip.
static mk_status wcc_static(mk_wcc *w, cudaStream_t s) {
  mk_graph *g = w->g;
  const uint32_t V = g->V;
  const int fg = flat_grid(V, g->device);
  k_uf_init<<<fg, 256, 0, s>>>(w->parent, V, nullptr, w->fe);
  w->forest_valid = true;
  if (!w->rev) return wcc_link(w, nullptr, s);
  const GraphView v = g->view(), rv = w->rev->view();
  MK_CHECK(reserve_items(w));
  if (g->weighted)
    k_uf_sample<true><<<fg, 256, 0, s>>>(v, w->parent, nullptr, w->err, w->fe);
  else
    k_uf_sample<false><<<fg, 256, 0, s>>>(v, w->parent, nullptr, w->err, w->fe);
  k_uf_compress<<<fg, 256, 0, s>>>(w->parent, V, nullptr);
  MK_CUDA(cudaMemsetAsync(w->fctl, 0, kFCtlWords * 8, s));
  k_uf_giant_sample<<<1, kMainThreads, 0, s>>>(w->parent, g->deg, V, 0x61A0000ull + (++w->calls),
                                               w->fctl);
  k_uf_outside_items<<<fg, 256, 0, s>>>(w->parent, V, v, rv, w->fctl, w->items_out.ptr,
                                        w->items_in.ptr);
  const int ob = (int)std::min<uint64_t>(g->num_buckets * 8 / 256 + 1,
                                         (uint64_t)device_sm_count(g->device) * 8);
  if (g->weighted)
    k_uf_edges_skip<true><<<ob, 256, 0, s>>>(v, w->parent, nullptr, w->err, w->fe, w->fctl + kFGiant);
  else
    k_uf_edges_skip<false><<<ob, 256, 0, s>>>(v, w->parent, nullptr, w->err, w->fe, w->fctl + kFGiant);
  launch_item_scans<false>(v, g->weighted, rv, w->rev->weighted, fg, w->parent, w->items_out.ptr,
                           w->items_in.ptr, nullptr, w->fctl, w->err, w->fe, s);
  k_uf_compress<<<fg, 256, 0, s>>>(w->parent, V, nullptr);
  MK_CUDA(cudaGetLastError());
  return MK_OK;
}

// Decremental repair over the spanning forest (the file header has the
// steps).  Synchronises twice: after finding the lost forest edges and after
// counting the vertices outside the main pieces, to choose the path.
static mk_status wcc_decremental_forest(mk_wcc *w, const uint32_t *d_src, const uint32_t *d_dst,
                                        uint32_t n, cudaStream_t s) {
  mk_graph *g = w->g;
  const uint32_t V = g->V;
  const size_t words = ((size_t)V + 31) / 32;
  const int fg = flat_grid(V, g->device);
  const GraphView v = g->view();
  uint32_t cap = 1024;  // n < 2^30 (checked by the caller): cap <= 2^31
  while (cap < 2ull * n) cap <<= 1;
  MK_CHECK(w->dtab.reserve(cap, &g->device_bytes));
  MK_CUDA(cudaMemsetAsync(w->dtab.ptr, 0xFF, (size_t)cap * 8, s));
  MK_CUDA(cudaMemsetAsync(w->fctl, 0, kFCtlWords * 8, s));
  MK_CUDA(cudaMemsetAsync(w->aff_labels, 0, words * 4, s));
  k_dh_insert<<<(n + 255) / 256, 256, 0, s>>>(d_src, d_dst, g->applied.ptr, n, g->reverse,
                                              w->dtab.ptr, cap - 1);
  if (g->weighted)
    k_fe_dead<true><<<fg, 256, 0, s>>>(v, w->fe, w->dtab.ptr, cap - 1, w->parent, w->aff_labels, w->fctl);
  else
    k_fe_dead<false><<<fg, 256, 0, s>>>(v, w->fe, w->dtab.ptr, cap - 1, w->parent, w->aff_labels, w->fctl);
  k_fe_count_aff<<<fg, 256, 0, s>>>(w->parent, V, w->aff_labels, w->fctl);
  MK_CUDA(cudaGetLastError());
  unsigned long long h[kFCtlWords] = {};
  MK_CUDA(cudaMemcpyAsync(h, w->fctl, sizeof(h), cudaMemcpyDeviceToHost, s));
  MK_CUDA(cudaStreamSynchronize(s));
  w->last_dead = h[kFDead];
  w->last_rescanned = 0;
  if (h[kFDead] == 0) {
    w->last_path = 0;  // the forest still spans every component: labels stand
    return MK_OK;
  }
  const bool most = 2 * h[kFAffected] > V;
  // without a rescan: the affected components rebuilt from their out-edges,
  // or the whole graph when they hold most of it (the same passes without the
  // per-vertex selection)
  auto rebuild = [&]() -> mk_status {
    if (most) {
      w->last_path = 3;
      return wcc_static(w, s);
    }
    MK_CUDA(cudaMemsetAsync(w->aff_vertices, 0, words * 4, s));
    k_uf_reset<<<fg, 256, 0, s>>>(w->parent, V, w->aff_labels, w->aff_vertices, w->fe);
    w->last_path = 2;
    return wcc_link(w, w->aff_vertices, s);
  };
  if (!w->rev) return rebuild();
  MK_CHECK(w->fe2.reserve(V, &g->device_bytes));
  MK_CHECK(w->oldlab.reserve(V, &g->device_bytes));
  MK_CHECK(reserve_items(w));
  k_fe_collect<<<fg, 256, 0, s>>>(w->parent, w->fe, w->fe2.ptr, V, w->aff_labels, w->oldlab.ptr,
                                  w->aff_vertices);
  k_fe_union<<<fg, 256, 0, s>>>(w->parent, w->fe, w->fe2.ptr, V, w->aff_vertices, w->err);
  k_uf_compress<<<fg, 256, 0, s>>>(w->parent, V, w->aff_vertices);
  k_fe_main_sample<<<1, kMainThreads, 0, s>>>(w->parent, w->oldlab.ptr, w->aff_vertices, V,
                                              0x5EED0000ull + (++w->calls), w->fctl);
  const GraphView rv = w->rev->view();
  k_fe_nonmain<<<fg, 256, 0, s>>>(w->parent, w->oldlab.ptr, V, w->aff_vertices, v, rv,
                                  w->items_out.ptr, w->items_in.ptr, w->fctl);
  MK_CUDA(cudaGetLastError());
  MK_CUDA(cudaMemcpyAsync(h, w->fctl, sizeof(h), cudaMemcpyDeviceToHost, s));
  MK_CUDA(cudaStreamSynchronize(s));
  if (2 * h[kFNmEnds] > h[kFEdges]) {
    // the split-off pieces hold most of the graph's edge ends
    w->skip_next = std::min<uint32_t>(w->skip_next ? 2 * w->skip_next : 1, 8);
    w->skip_left = w->skip_next;
    if (!most) k_uf_init<<<fg, 256, 0, s>>>(w->parent, V, w->aff_vertices, w->fe);
    if (most) {
      w->last_path = 3;
      return wcc_static(w, s);
    }
    w->last_path = 2;
    return wcc_link(w, w->aff_vertices, s);
  }
  w->skip_next = 0;
  w->last_path = 1;
  w->last_rescanned = h[kFNmCount];
  if (h[kFNmCount]) {
    // item lists: a hub outside its main piece spreads over many groups
    launch_item_scans<true>(v, g->weighted, rv, w->rev->weighted, fg, w->parent, w->items_out.ptr,
                            w->items_in.ptr, w->oldlab.ptr, w->fctl, w->err, w->fe, s);
    k_uf_compress<<<fg, 256, 0, s>>>(w->parent, V, w->aff_vertices);
  }
  MK_CUDA(cudaGetLastError());
  return MK_OK;
}

static bool batch_matches(const mk_graph *g, const uint32_t *d_src, const uint32_t *d_dst,
                          uint32_t n, int op) {
  return n == g->last_n && d_src == g->last_src && d_dst == g->last_dst && g->last_op == op;
}

namespace mk {
uint32_t *wcc_label_buf(mk_wcc *w) { return w ? w->parent : nullptr; }
}  // namespace mk

extern "C" {

mk_status mk_wcc_create(mk_graph *g, mk_wcc **out) {
  if (!g || !out) return fail(MK_ERR_INVALID, "mk_wcc_create: null argument");
  DeviceGuard dg(g->device);
  mk_wcc *w = new mk_wcc();
  w->g = g;
  const size_t V = g->V, words = (V + 31) / 32;
  cudaError_t e = cudaMalloc(&w->parent, V * 4);
  if (e == cudaSuccess) e = cudaMalloc(&w->aff_labels, words * 4);
  if (e == cudaSuccess) e = cudaMalloc(&w->aff_vertices, words * 4);
  if (e == cudaSuccess) e = cudaMalloc(&w->fe, V * 8);
  if (e == cudaSuccess) e = cudaMalloc(&w->fctl, kFCtlWords * 8);
  w->err = g->err_word();
  if (e != cudaSuccess) {
    mk_wcc_destroy(w);
    return cuda_fail(e, "mk_wcc_create");
  }
  k_uf_init<<<flat_grid(V, g->device), 256>>>(w->parent, (uint32_t)V, nullptr, w->fe);
  e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    mk_wcc_destroy(w);
    return cuda_fail(e, "mk_wcc_create");
  }
  *out = w;
  return MK_OK;
}

mk_status mk_wcc_static(mk_wcc *w, void *stream, float *ms_out) {
  if (!w) return fail(MK_ERR_INVALID, "mk_wcc_static: null handle");
  DeviceGuard dg(w->g->device);
  cudaStream_t s = as_stream(stream);
  MK_CHECK(w->timer.start(s, ms_out != nullptr));
  MK_CHECK(wcc_static(w, s));
  return w->timer.stop(ms_out);
}

mk_status mk_wcc_static_subset(mk_wcc *w, const uint32_t *d_sel_bits, void *stream,
                               float *ms_out) {
  if (!w || !d_sel_bits) return fail(MK_ERR_INVALID, "mk_wcc_static_subset: null argument");
  mk_graph *g = w->g;
  DeviceGuard dg(g->device);
  cudaStream_t s = as_stream(stream);
  MK_CHECK(w->timer.start(s, ms_out != nullptr));
  k_uf_init<<<flat_grid(g->V, g->device), 256, 0, s>>>(w->parent, g->V, d_sel_bits, w->fe);
  MK_CHECK(wcc_link(w, d_sel_bits, s));
  return w->timer.stop(ms_out);
}

// Builds and uploads the range table: blocking (device-wide wait, then a
// plain copy) when async is false, else stream-ordered on `s` through pinned
// staging.
static mk_status wcc_prepare(mk_wcc *w, const uint32_t *h_vertex_ranges, uint32_t nranges,
                             bool async, cudaStream_t s) {
  mk_graph *g = w->g;
  std::vector<uint32_t> small_ids, large_ids;
  for (uint32_t r = 0; r < nranges; ++r) {
    const uint32_t b = h_vertex_ranges[2 * r], e = h_vertex_ranges[2 * r + 1];
    if (b >= e || e > g->V) return fail(MK_ERR_INVALID, "mk_wcc_prepare_ranges: bad vertex range");
    (e - b <= kUfLocalMax ? small_ids : large_ids).push_back(r);
  }
  auto len = [&](uint32_t r) { return h_vertex_ranges[2 * r + 1] - h_vertex_ranges[2 * r]; };
  std::stable_sort(small_ids.begin(), small_ids.end(),
                   [&](uint32_t a, uint32_t b) { return len(a) > len(b); });
  const size_t ns = small_ids.size(), nl = large_ids.size();
  std::vector<uint32_t> host(4 + 4 * ns + 4 * (nl + 1), 0u);
  uint32_t *sm = host.data() + 4;
  for (size_t i = 0; i < ns; ++i) {
    const uint32_t r = small_ids[i], b = h_vertex_ranges[2 * r], e = h_vertex_ranges[2 * r + 1];
    sm[4 * i + 0] = b;
    sm[4 * i + 1] = e;
    sm[4 * i + 2] = g->h_boff[b];
    sm[4 * i + 3] = g->h_boff[e];
  }
  uint32_t *vpre = sm + 4 * ns, *vbase = vpre + nl + 1, *bpre = vbase + nl + 1, *bbase = bpre + nl + 1;
  uint64_t vt = 0, bt = 0;
  for (size_t i = 0; i < nl; ++i) {
    const uint32_t r = large_ids[i], b = h_vertex_ranges[2 * r], e = h_vertex_ranges[2 * r + 1];
    vpre[i] = (uint32_t)vt;
    vbase[i] = b;
    bpre[i] = (uint32_t)bt;
    bbase[i] = g->h_boff[b];
    vt += e - b;
    bt += g->h_boff[e] - g->h_boff[b];
  }
  vpre[nl] = (uint32_t)vt;
  bpre[nl] = (uint32_t)bt;
  DeviceGuard dg(g->device);
  w->prepared = false;
  if (host.size() > w->ranges.cap) MK_CUDA(cudaDeviceSynchronize());  // growth frees the old table
  MK_CHECK(w->ranges.reserve(host.size(), &g->device_bytes));
  if (async) {
    // ordered after the earlier launches on s, which may still read the old table
    MK_CHECK(w->staging.upload(w->ranges.ptr, host.data(), host.size() * 4, s));
  } else {
    // queued work may still read the previous table
    MK_CUDA(cudaDeviceSynchronize());
    MK_CUDA(cudaMemcpy(w->ranges.ptr, host.data(), host.size() * 4, cudaMemcpyHostToDevice));
  }
  w->n_small = (uint32_t)ns;
  w->n_large = (uint32_t)nl;
  w->small_max = ns ? len(small_ids[0]) : 0;
  w->large_vt = vt;
  w->large_bt = bt;
  w->small_grid = 0;
  if (ns) {
    const size_t smem = uf_member_smem(w->small_max);
    auto kern = g->weighted ? k_uf_members<true> : k_uf_members<false>;
    MK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)uf_member_smem(kUfLocalMax)));
    int per_sm = 0;
    MK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kMemThreads, smem));
    w->small_grid = (int)std::min<uint64_t>(ns, (uint64_t)device_sm_count(g->device) * std::max(per_sm, 1));
  }
  w->prepared = true;
  return MK_OK;
}

mk_status mk_wcc_prepare_ranges(mk_wcc *w, const uint32_t *h_vertex_ranges, uint32_t nranges) {
  if (!w || (nranges && !h_vertex_ranges))
    return fail(MK_ERR_INVALID, "mk_wcc_prepare_ranges: null argument");
  return wcc_prepare(w, h_vertex_ranges, nranges, false, nullptr);
}

mk_status mk_wcc_prepare_ranges_async(mk_wcc *w, const uint32_t *h_vertex_ranges,
                                      uint32_t nranges, void *stream) {
  if (!w || (nranges && !h_vertex_ranges))
    return fail(MK_ERR_INVALID, "mk_wcc_prepare_ranges_async: null argument");
  return wcc_prepare(w, h_vertex_ranges, nranges, true, as_stream(stream));
}

mk_status mk_wcc_static_prepared(mk_wcc *w, void *stream, float *ms_out) {
  if (!w) return fail(MK_ERR_INVALID, "mk_wcc_static_prepared: null handle");
  if (!w->prepared) return fail(MK_ERR_INVALID, "mk_wcc_static_prepared: no prepared ranges");
  mk_graph *g = w->g;
  DeviceGuard dg(g->device);
  cudaStream_t s = as_stream(stream);
  MK_CHECK(w->timer.start(s, ms_out != nullptr));
  w->forest_valid = false;  // the range passes record no forest
  const GraphView v = g->view();
  uint32_t *counter = w->ranges.ptr;
  const uint32_t ns = w->n_small, nl = w->n_large;
  if (ns) {
    const size_t smem = uf_member_smem(w->small_max);
    const uint4 *rng = reinterpret_cast<const uint4 *>(w->ranges.ptr + 4);
    MK_CUDA(cudaMemsetAsync(counter, 0, 4, s));
    if (g->weighted)
      k_uf_members<true><<<w->small_grid, kMemThreads, smem, s>>>(v, rng, ns, counter, w->parent, w->err);
    else
      k_uf_members<false><<<w->small_grid, kMemThreads, smem, s>>>(v, rng, ns, counter, w->parent, w->err);
  }
  if (nl) {
    const uint32_t *dv = w->ranges.ptr + 4 + 4 * (size_t)ns, *dvb = dv + nl + 1;
    const uint32_t *db = dvb + nl + 1, *dbb = db + nl + 1;
    const int fg = flat_grid(w->large_vt, g->device);
    k_uf_init_ranges<<<fg, 256, 0, s>>>(w->parent, dv, dvb, nl);
    if (g->weighted)
      k_uf_sample_ranges<true><<<fg, 256, 0, s>>>(v, w->parent, dv, dvb, nl, w->err);
    else
      k_uf_sample_ranges<false><<<fg, 256, 0, s>>>(v, w->parent, dv, dvb, nl, w->err);
    k_uf_compress_ranges<<<fg, 256, 0, s>>>(w->parent, dv, dvb, nl);
    const int blocks = (int)std::min<uint64_t>(w->large_bt * 8 / 256 + 1, (uint64_t)device_sm_count(g->device) * 8);
    if (g->weighted)
      k_uf_edges_ranges<true><<<blocks, 256, 0, s>>>(v, w->parent, db, dbb, nl, w->err);
    else
      k_uf_edges_ranges<false><<<blocks, 256, 0, s>>>(v, w->parent, db, dbb, nl, w->err);
    k_uf_compress_ranges<<<fg, 256, 0, s>>>(w->parent, dv, dvb, nl);
  }
  MK_CUDA(cudaGetLastError());
  return w->timer.stop(ms_out);
}

mk_status mk_wcc_static_ranges(mk_wcc *w, const uint32_t *h_vertex_ranges, uint32_t nranges,
                               void *stream, float *ms_out) {
  if (!w || (nranges && !h_vertex_ranges))
    return fail(MK_ERR_INVALID, "mk_wcc_static_ranges: null argument");
  MK_CHECK(mk_wcc_prepare_ranges(w, h_vertex_ranges, nranges));
  return mk_wcc_static_prepared(w, stream, ms_out);
}

mk_status mk_wcc_incremental(mk_wcc *w, const uint32_t *d_src, const uint32_t *d_dst,
                             uint32_t n, void *stream, float *ms_out) {
  if (!w) return fail(MK_ERR_INVALID, "mk_wcc_incremental: null handle");
  mk_graph *g = w->g;
  DeviceGuard dg(g->device);
  cudaStream_t s = as_stream(stream);
  MK_CHECK(w->timer.start(s, ms_out != nullptr));
  if (!batch_matches(g, d_src, d_dst, n, 1)) {
    MK_CHECK(wcc_static(w, s));
  } else if (n) {
    k_uf_batch<<<(n + 255) / 256, 256, 0, s>>>(d_src, d_dst, g->applied.ptr, n, g->V, g->reverse,
                                                w->parent, w->err, w->fe);
    k_uf_compress<<<flat_grid(g->V, g->device), 256, 0, s>>>(w->parent, g->V, nullptr);
    MK_CUDA(cudaGetLastError());
  }
  return w->timer.stop(ms_out);
}

mk_status mk_wcc_decremental(mk_wcc *w, const uint32_t *d_src, const uint32_t *d_dst,
                             uint32_t n, void *stream, float *ms_out) {
  if (!w) return fail(MK_ERR_INVALID, "mk_wcc_decremental: null handle");
  mk_graph *g = w->g;
  DeviceGuard dg(g->device);
  cudaStream_t s = as_stream(stream);
  MK_CHECK(w->timer.start(s, ms_out != nullptr));
  w->last_dead = w->last_rescanned = 0;
  w->last_path = 0;
  if (!batch_matches(g, d_src, d_dst, n, 2) || !w->forest_valid || (n && w->rev && w->skip_left)) {
    if (w->skip_left) --w->skip_left;
    MK_CHECK(wcc_static(w, s));
    w->last_path = 3;
  } else if (n >= (1u << 30)) {
    MK_CHECK(wcc_static(w, s));  // beyond the batch set's size
    w->last_path = 3;
  } else if (n) {
    MK_CHECK(wcc_decremental_forest(w, d_src, d_dst, n, s));
  }
  return w->timer.stop(ms_out);
}

// Loads the kernels of the static passes and of the decremental repair: with
// lazy module loading the first launch of each would otherwise pay for it
// inside the first (timed) call.
static mk_status preload_kernels() {
  cudaFuncAttributes a;
  const void *fns[] = {
      (const void *)k_uf_init, (const void *)k_uf_compress, (const void *)k_uf_reset,
      (const void *)k_uf_sample<false>, (const void *)k_uf_sample<true>,
      (const void *)k_uf_edges_skip<false>, (const void *)k_uf_edges_skip<true>,
      (const void *)k_uf_giant_sample, (const void *)k_uf_outside_items,
      (const void *)k_uf_scan_items<false, false, false>, (const void *)k_uf_scan_items<true, false, false>,
      (const void *)k_uf_scan_items<false, true, false>, (const void *)k_uf_scan_items<true, true, false>,
      (const void *)k_uf_scan_items<false, false, true>, (const void *)k_uf_scan_items<true, false, true>,
      (const void *)k_uf_scan_items<false, true, true>, (const void *)k_uf_scan_items<true, true, true>,
      (const void *)k_dh_insert, (const void *)k_fe_dead<false>, (const void *)k_fe_dead<true>,
      (const void *)k_fe_count_aff, (const void *)k_fe_collect, (const void *)k_fe_union,
      (const void *)k_fe_main_sample, (const void *)k_fe_nonmain};
  for (const void *f : fns) MK_CUDA(cudaFuncGetAttributes(&a, f));
  return MK_OK;
}

mk_status mk_wcc_set_reverse(mk_wcc *w, mk_graph *g_rev) {
  if (!w) return fail(MK_ERR_INVALID, "mk_wcc_set_reverse: null handle");
  mk_graph *g = w->g;
  if (g_rev && (g_rev->V != g->V || g_rev->device != g->device || g_rev->reverse == g->reverse))
    return fail(MK_ERR_INVALID,
                "mk_wcc_set_reverse: need the reverse graph of the same vertices on the same device");
  w->rev = g_rev;
  if (g_rev) {
    // the piece-rescan scratch, and a batch set sized for the graph's batch
    // scratch, allocated here rather than inside a timed decremental call
    DeviceGuard dg(g->device);
    const size_t V = g->V;
    MK_CHECK(w->fe2.reserve(V, &g->device_bytes));
    MK_CHECK(w->oldlab.reserve(V, &g->device_bytes));
    MK_CHECK(reserve_items(w));
    MK_CHECK(preload_kernels());
    uint64_t cap = 1024;
    while (cap < 2ull * std::min<uint64_t>(g->applied.cap, g->V)) cap <<= 1;
    MK_CHECK(w->dtab.reserve(cap, &g->device_bytes));
  }
  return MK_OK;
}

mk_status mk_wcc_decremental_stats(mk_wcc *w, uint64_t *h_dead_forest_edges,
                                   uint64_t *h_rescanned_vertices, uint32_t *h_path) {
  if (!w) return fail(MK_ERR_INVALID, "mk_wcc_decremental_stats: null handle");
  if (h_dead_forest_edges) *h_dead_forest_edges = w->last_dead;
  if (h_rescanned_vertices) *h_rescanned_vertices = w->last_rescanned;
  if (h_path) *h_path = w->last_path;
  return MK_OK;
}

mk_status mk_wcc_labels(mk_wcc *w, uint32_t *h_out) {
  if (!w || !h_out) return fail(MK_ERR_INVALID, "mk_wcc_labels: null argument");
  DeviceGuard dg(w->g->device);
  MK_CUDA(cudaDeviceSynchronize());
  uint32_t err = 0;
  MK_CUDA(cudaMemcpy(&err, w->err, 4, cudaMemcpyDeviceToHost));
  MK_CUDA(cudaMemcpy(h_out, w->parent, (size_t)w->g->V * 4, cudaMemcpyDeviceToHost));
  if (err & kErrTimeout) return fail(MK_ERR_TIMEOUT, "wcc: union-find retry limit exceeded");
  return MK_OK;
}

mk_status mk_wcc_labels_device(mk_wcc *w, const uint32_t **d_labels) {
  if (!w || !d_labels) return fail(MK_ERR_INVALID, "mk_wcc_labels_device: null argument");
  *d_labels = w->parent;
  return MK_OK;
}

mk_status mk_wcc_destroy(mk_wcc *w) {
  if (!w) return MK_OK;
  DeviceGuard dg(w->g->device);
  cudaFree(w->parent);
  cudaFree(w->aff_labels);
  cudaFree(w->aff_vertices);
  cudaFree(w->fe);
  cudaFree(w->fctl);
  w->dtab.release();
  w->fe2.release();
  w->oldlab.release();
  w->items_out.release();
  w->items_in.release();
  w->staging.release();
  w->ranges.release();
  delete w;
  return MK_OK;
}

}  // extern "C"
