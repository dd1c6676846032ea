// Per-member solvers of a graph set, run by one whole CTA with the member's
// state in shared memory.  The member kernels (one query kind per launch)
// and the one-launch graph-set step (its last phase) both call them.
//
// bfs_member: static BFS of one vertex range from its source.  The member's
// BFS state lives in shared memory -- a 16-bit parent per vertex (0xFFFF:
// not reached) and a visited bitmap -- and its levels are separated by block
// barriers instead of grid barriers.  A level's frontier is a list of work
// items (vertex, chunk of buckets) in the range's slice of a device array, so
// a hub's buckets spread over many 8-lane groups.  A newly reached vertex
// keeps the smallest-id frontier vertex with an edge to it as its parent (a
// 16-bit CAS minimum).  Distances equal the device-wide kernel's; parents
// form a valid BFS tree, as there, where (as in the reference,
// BFSImpl.cuh:311-314) the first of several equal-distance parents stays.
// After each level the newly reached vertices get their packed word in
// device memory, their visited bit and their work items.
//
// uf_member: connected components of one vertex range.  Its union-find parent
// array lives in shared memory as 16-bit local ids, so every find, halving
// store and hooking CAS stays on chip, and device memory sees one pass over
// the range's slabs and one write of its labels.  The union rule is the one
// of the device-wide kernels (larger root under smaller, as the reference's
// UnionAsync, include/Util/UnionFind.cuh:194-215), so labels are the minimum
// vertex id of each component.
//
// kFused: the kernel updated the graph itself earlier in the same launch
// (behind a grid barrier): slabs are read with plain loads, never the
// non-coherent path (ld_slab), and the BFS writes the unreached vertices'
// words itself instead of relying on a reset before the launch.
#pragma once

#include "mk_common.cuh"
#include "mk_slab.cuh"

namespace mk {

constexpr uint32_t kUfLimit = 1u << 26;   // bound on every find / union retry loop
constexpr uint32_t kMemLocalMax = 65535;  // BFS member: 0xFFFF marks "not reached"
constexpr uint32_t kUfLocalMax = 1u << 16;  // WCC member: 16-bit local parents
constexpr int kMemThreads = 1024;         // threads of a member CTA
constexpr uint32_t kMemChunk = 4;         // buckets per BFS work item (head slabs loaded together)
constexpr uint32_t kMemberHeads = 4;      // head slabs a WCC group loads together

// Dynamic shared memory of a BFS member of n vertices: visited bitmap, then
// 16-bit parents (16-byte aligned size).
__host__ __device__ constexpr size_t bfs_member_smem(size_t n) {
  return (n + 31) / 32 * 4 + ((n * 2 + 15) & ~(size_t)15);
}
// Dynamic shared memory of a WCC member of n vertices: 16-bit parents.
__host__ __device__ constexpr size_t uf_member_smem(size_t n) { return (n * 2 + 15) & ~(size_t)15; }

// Buckets per work item of a vertex with nb buckets: the chunk index must fit
// 16 bits.
__device__ __forceinline__ uint32_t mem_chunk(uint32_t nb) {
  return nb > 65536u * kMemChunk ? (nb + 65535u) / 65536u : kMemChunk;
}

// Lowers *p to v if v is smaller; true if this call replaced 0xFFFF.  Every
// failed CAS means another thread lowered *p, so the loop ends within 65,536
// rounds.
__device__ __forceinline__ bool cas_min16_first(uint16_t *p, uint32_t v) {
  volatile unsigned short *vp = p;
  unsigned short cur = *vp;
  for (uint32_t it = 0; it <= 65536u; ++it) {
    if (v >= cur) return false;
    const unsigned short prev =
        atomicCAS(reinterpret_cast<unsigned short *>(p), cur, (unsigned short)v);
    if (prev == cur) return cur == 0xFFFFu;
    cur = prev;
  }
  return false;
}

// R = (first vertex, end vertex, first bucket, end bucket) of a range of at
// most kMemLocalMax vertices, src its source (global id).  The range uses the
// slices [R.z, R.w) of items (one word per bucket: a vertex's items never
// exceed its buckets) and [R.x, R.y) of found (a vertex is reached once).
// Without kFused, dist must already hold kInfInf for the range.  smem holds
// bfs_member_smem(n) bytes; s_nfound / s_nitems are CTA-shared words.  Ends
// with the CTA synchronised.
template <bool kW, bool kFused>
__device__ __forceinline__ void bfs_member(const GraphView &g, const Lanes &L, const uint4 R,
                                           uint32_t src, unsigned long long *__restrict__ dist,
                                           uint32_t *__restrict__ items,
                                           uint32_t *__restrict__ found, uint32_t *err,
                                           uint32_t *smem, uint32_t &s_nfound,
                                           uint32_t &s_nitems) {
  const uint32_t group = threadIdx.x >> 3, ngroups = blockDim.x >> 3;
  const uint32_t lo = R.x, n = R.y - R.x, s0 = src - lo;
  const uint32_t nw = (n + 31) >> 5;
  uint32_t *vis = smem;
  uint16_t *par = reinterpret_cast<uint16_t *>(smem + nw);
  uint32_t *q = items + R.z;
  uint32_t *fl = found + lo;
  for (uint32_t i = threadIdx.x; i < nw; i += blockDim.x) vis[i] = 0u;
  for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) par[i] = 0xFFFFu;
  __syncthreads();
  if (threadIdx.x == 0) {
    par[s0] = (uint16_t)s0;
    fl[0] = s0;
    s_nfound = 1;
    s_nitems = 0;
  }
  __syncthreads();
  uint32_t fbeg = 0, ibeg = 0;
  for (uint32_t level = 0; level <= n; ++level) {
    // vertices reached at `level`: packed word, visited bit, work items
    const uint32_t fend = s_nfound;
    for (uint32_t i = fbeg + threadIdx.x; i < fend; i += blockDim.x) {
      const uint32_t v = fl[i], gv = lo + v;
      dist[gv] = pack(level, lo + par[v]);
      atomicOr(vis + (v >> 5), 1u << (v & 31));
      if (g.deg[gv] == 0) continue;
      const uint32_t nb = g.boff[gv + 1] - g.boff[gv];
      const uint32_t cs = mem_chunk(nb), nc = (nb + cs - 1) / cs;
      const uint32_t pos = atomicAdd(&s_nitems, nc);
      for (uint32_t c = 0; c < nc; ++c) q[pos + c] = v | (c << 16);
    }
    __syncthreads();
    const uint32_t iend = s_nitems;
    if (iend == ibeg) break;
    // expand the items of `level`
    for (uint32_t it = ibeg + group; it < iend; it += ngroups) {
      const uint32_t item = q[it];
      const uint32_t u = item & 0xFFFFu, gu = lo + u;
      const uint32_t ub0 = g.boff[gu], nb = g.boff[gu + 1] - ub0, cs = mem_chunk(nb);
      const uint32_t bb = ub0 + (item >> 16) * cs, be = min(bb + cs, ub0 + nb);
      auto relax = [&](const uint4 x) {
        uint32_t k[4], w[4];
        lane_keys<kW>(x, L.gl, k, w);
#pragma unroll
        for (int t = 0; t < keys_per_lane<kW>(); ++t) {
          if (k[t] >= kTombKey) continue;
          const uint32_t v = k[t] - lo;
          if (v >= n) {
            atomicOr(err, kErrInvalidId);
            continue;
          }
          if ((vis[v >> 5] >> (v & 31)) & 1u) continue;
          if (cas_min16_first(par + v, u)) fl[atomicAdd(&s_nfound, 1u)] = v;
        }
      };
      for (uint32_t b = bb; b < be; b += kMemChunk)
        walk4_levels<kFused>(g, L, b, min(kMemChunk, be - b),
                             [&](uint32_t, const uint4 x) { relax(x); });
    }
    fbeg = fend;
    ibeg = iend;
    __syncthreads();
  }
  if (kFused) {
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x)
      if (!((vis[i >> 5] >> (i & 31)) & 1u)) dist[lo + i] = kInfInf;
  }
  __syncthreads();
}

__device__ __forceinline__ uint32_t ls_find(uint16_t *p, uint32_t x) {
  volatile uint16_t *vp = p;
  for (uint32_t it = 0; it < kUfLimit; ++it) {
    const uint32_t px = vp[x];
    if (px == x) return x;
    const uint32_t gx = vp[px];
    if (px != gx) vp[x] = (uint16_t)gx;  // x is not a root: only halving writes it
    x = gx;
  }
  return x;
}

__device__ __forceinline__ uint32_t ls_root(const uint16_t *p, uint32_t x) {
  const volatile uint16_t *vp = p;
  for (uint32_t it = 0; it < kUfLimit; ++it) {
    const uint32_t px = vp[x];
    if (px == x) return x;
    x = px;
  }
  return x;
}

__device__ __forceinline__ void ls_union(uint16_t *p, uint32_t a, uint32_t b, uint32_t *err) {
  for (uint32_t it = 0; it < kUfLimit; ++it) {
    const uint32_t ra = ls_find(p, a), rb = ls_find(p, b);
    if (ra == rb) return;
    const uint32_t hi = ra > rb ? ra : rb, lo = ra > rb ? rb : ra;
    if (atomicCAS(reinterpret_cast<unsigned short *>(p + hi), (unsigned short)hi,
                  (unsigned short)lo) == (unsigned short)hi)
      return;
  }
  atomicOr(err, kErrTimeout);
}

// R = (first vertex, end vertex, first bucket, end bucket), at most
// kUfLocalMax vertices; labels[R.x .. R.y) get the minimum vertex id of each
// component.  A key outside the range (a range that is not closed under
// edges) is skipped and reported as MK_DEVERR_INVALID_ID.  sp holds
// uf_member_smem(n) bytes.  Ends with the CTA synchronised.
template <bool kW, bool kFused>
__device__ __forceinline__ void uf_member(const GraphView &g, const Lanes &L, const uint4 R,
                                          uint32_t *__restrict__ labels, uint32_t *err,
                                          uint16_t *sp) {
  const uint32_t group = threadIdx.x >> 3, ngroups = blockDim.x >> 3;
  const uint32_t lo = R.x, n = R.y - R.x;
  for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) sp[i] = (uint16_t)i;
  __syncthreads();
  for (uint32_t b = R.z + group * kMemberHeads; b < R.w; b += ngroups * kMemberHeads) {
    const uint32_t m = min(kMemberHeads, R.w - b);
    uint32_t own[kMemberHeads];
#pragma unroll
    for (uint32_t j = 0; j < kMemberHeads; ++j) own[j] = j < m ? __ldg(g.bowner + b + j) - lo : 0u;
    walk4_levels<kFused>(g, L, b, m, [&](uint32_t j, const uint4 x) {
      const uint32_t u = own[0] * (j == 0) + own[1] * (j == 1) + own[2] * (j == 2) + own[3] * (j == 3);
      uint32_t k[4], w[4];
      lane_keys<kW>(x, L.gl, k, w);
#pragma unroll
      for (int t = 0; t < keys_per_lane<kW>(); ++t) {
        if (k[t] >= kTombKey) continue;
        const uint32_t v = k[t] - lo;
        if (v >= n || u >= n) {
          atomicOr(err, kErrInvalidId);
          continue;
        }
        if (v != u) ls_union(sp, u, v, err);
      }
    });
  }
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) labels[lo + i] = lo + ls_root(sp, i);
  __syncthreads();
}

}  // namespace mk
