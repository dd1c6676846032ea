// Group-cooperative slab probes and per-vertex slab walks.
//
// An 8-lane group holds one 128-byte slab as 8 x uint4: lane gl owns words
// 4*gl .. 4*gl+3.  For set slabs every word except 31 is a key slot (lane 7's
// .w is the next-slab id); for map slabs the key slots are words 0,2,..,28
// (.x and .z of lanes 0..6, .x of lane 7) with the value in the following
// word.  This replaces the slab-hash iterator and searchKey that the
// reference calls (include/Algorithms/impl/BFSImpl.cuh:123-139,
// include/Graph/warp/SearchEdge.cuh:23-24).
#pragma once

#include "mk_common.cuh"

namespace mk {

// Probe of one slab for `key`: slot of the key (255 if absent), first EMPTY
// key slot (255 if none) and the next-slab id, all group-uniform.
template <bool kWeighted>
__device__ __forceinline__ void probe_slab(const uint4 &q, uint32_t key,
                                           const Lanes &L, bool &found,
                                           uint32_t &slot_key,
                                           uint32_t &first_empty,
                                           uint32_t &next) {
  uint32_t my_found_slot = 255, my_empty = 255;
  if (!kWeighted) {
    bool k3 = (L.gl != 7);
    if (q.x == key) my_found_slot = L.gl * 4 + 0;
    else if (q.y == key) my_found_slot = L.gl * 4 + 1;
    else if (q.z == key) my_found_slot = L.gl * 4 + 2;
    else if (k3 && q.w == key) my_found_slot = L.gl * 4 + 3;
    if (q.x == kEmptyKey) my_empty = L.gl * 4 + 0;
    else if (q.y == kEmptyKey) my_empty = L.gl * 4 + 1;
    else if (q.z == kEmptyKey) my_empty = L.gl * 4 + 2;
    else if (k3 && q.w == kEmptyKey) my_empty = L.gl * 4 + 3;
  } else {
    bool k1 = (L.gl != 7);
    if (q.x == key) my_found_slot = L.gl * 2 + 0;
    else if (k1 && q.z == key) my_found_slot = L.gl * 2 + 1;
    if (q.x == kEmptyKey) my_empty = L.gl * 2 + 0;
    else if (k1 && q.z == kEmptyKey) my_empty = L.gl * 2 + 1;
  }
  slot_key = __reduce_min_sync(L.gmask, my_found_slot);
  found = slot_key != 255;
  first_empty = __reduce_min_sync(L.gmask, my_empty);
  next = __shfl_sync(L.gmask, q.w, L.gbase + 7);
}

// Group-cooperative membership test of (u, v) (u = the vertex whose table is
// probed).  Returns found; *val gets the stored value for map slabs.
template <bool kWeighted>
__device__ __forceinline__ bool find_edge(const GraphView &g, const Lanes &L,
                                          uint32_t u, uint32_t v,
                                          uint32_t *val) {
  const uint32_t b0 = g.boff[u];
  const uint32_t nb = g.boff[u + 1] - b0;
  uint32_t s = b0 + bucket_of(v, nb);
  for (uint32_t it = 0; it < (1u << 24) && s != kNoSlab; ++it) {
    uint4 q = ld_slab_ro(g.slabs + 8ull * s + L.gl);
    bool f;
    uint32_t fslot, eslot, next;
    probe_slab<kWeighted>(q, v, L, f, fslot, eslot, next);
    if (f) {
      if (kWeighted && val) {
        uint32_t owner = fslot >> 1;
        uint32_t cand = (fslot & 1) ? q.w : q.y;
        *val = __shfl_sync(L.gmask, cand, L.gbase + owner);
      }
      return true;
    }
    s = next;
  }
  return false;
}

// Keys (and values) held by one lane of a slab.  n = number of key slots
// (4/3 for set slabs, 2/1 for map slabs); invalid slots are returned as
// EMPTY so callers just test k < kTombKey.
template <bool kWeighted>
__device__ __forceinline__ void lane_keys(const uint4 &q, uint32_t gl,
                                          uint32_t (&k)[4], uint32_t (&w)[4]) {
  if (!kWeighted) {
    k[0] = q.x;
    k[1] = q.y;
    k[2] = q.z;
    k[3] = (gl != 7) ? q.w : kEmptyKey;
    w[0] = w[1] = w[2] = w[3] = 1u;
  } else {
    k[0] = q.x;
    w[0] = q.y;
    k[1] = (gl != 7) ? q.z : kEmptyKey;
    w[1] = q.w;
    k[2] = k[3] = kEmptyKey;
    w[2] = w[3] = 0u;
  }
}

template <bool kWeighted>
__host__ __device__ constexpr int keys_per_lane() {
  return kWeighted ? 2 : 4;
}

// Visits every slab of vertex u with the group; f(q) is called by all 8
// lanes with their quarter of the slab.  Chains are followed bucket by
// bucket; head slabs are contiguous.
template <class F>
__device__ __forceinline__ void walk_vertex(const GraphView &g, const Lanes &L,
                                            uint32_t u, F &&f) {
  const uint32_t b1 = g.boff[u + 1];
  for (uint32_t b = g.boff[u]; b < b1; ++b) {
    uint32_t s = b;
    while (s != kNoSlab) {
      uint4 q = ld_slab_ro(g.slabs + 8ull * s + L.gl);
      f(q);
      s = __shfl_sync(L.gmask, q.w, L.gbase + 7);
    }
  }
}

// Visits the slab chain of one bucket (head slab id = bucket index).
template <class F>
__device__ __forceinline__ void walk_bucket(const GraphView &g, const Lanes &L, uint32_t b,
                                            F &&f) {
  uint32_t s = b;
  while (s != kNoSlab) {
    uint4 q = ld_slab_ro(g.slabs + 8ull * s + L.gl);
    f(q);
    s = __shfl_sync(L.gmask, q.w, L.gbase + 7);
  }
}

// Visits buckets [b0, b1) with the head slabs of up to 4 buckets loaded
// together (independent loads in flight), then follows overflow chains.
template <class F>
__device__ __forceinline__ void walk_buckets(const GraphView &g, const Lanes &L, uint32_t b0,
                                             uint32_t b1, F &&f) {
  for (uint32_t b = b0; b < b1; b += 4) {
    uint4 q[4];
    const uint32_t n = min(4u, b1 - b);
#pragma unroll
    for (int j = 0; j < 4; ++j)
      if ((uint32_t)j < n) q[j] = ld_slab_ro(g.slabs + 8ull * (b + j) + L.gl);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      if ((uint32_t)j < n) {
        f(q[j]);
        uint32_t s = __shfl_sync(L.gmask, q[j].w, L.gbase + 7);
        while (s != kNoSlab) {
          uint4 r = ld_slab_ro(g.slabs + 8ull * s + L.gl);
          f(r);
          s = __shfl_sync(L.gmask, r.w, L.gbase + 7);
        }
      }
    }
  }
}

// Visits buckets [b, b + m), m <= 4: the head slabs are loaded together,
// then the overflow chains level by level, the next slabs of every chain
// still running loaded together.  f(j, q) gets the bucket's index j in
// [0, m) and the lane's quarter of one slab.  kCg: the kernel wrote slabs
// earlier in the same launch (ld_slab).
template <bool kCg = false, class F>
__device__ __forceinline__ void walk4_levels(const GraphView &g, const Lanes &L, uint32_t b,
                                             uint32_t m, F &&f) {
  uint4 q[4];
  uint32_t nx[4];
#pragma unroll
  for (uint32_t j = 0; j < 4; ++j)
    if (j < m) q[j] = ld_slab<kCg>(g.slabs + 8ull * (b + j) + L.gl);
#pragma unroll
  for (uint32_t j = 0; j < 4; ++j) {
    nx[j] = kNoSlab;
    if (j < m) {
      f(j, q[j]);
      nx[j] = __shfl_sync(L.gmask, q[j].w, L.gbase + 7);
    }
  }
  while ((nx[0] & nx[1] & nx[2] & nx[3]) != kNoSlab) {  // some chain still running
#pragma unroll
    for (uint32_t j = 0; j < 4; ++j)
      if (nx[j] != kNoSlab) q[j] = ld_slab<kCg>(g.slabs + 8ull * nx[j] + L.gl);
#pragma unroll
    for (uint32_t j = 0; j < 4; ++j)
      if (nx[j] != kNoSlab) {
        f(j, q[j]);
        nx[j] = __shfl_sync(L.gmask, q[j].w, L.gbase + 7);
      }
  }
}

// walk4_levels over 4 arbitrary buckets bk[j] (those with bit j of live
// set), chains followed level by level.  Every lane of the group must pass
// the same bk and live.
template <class F>
__device__ __forceinline__ void walk4_set(const GraphView &g, const Lanes &L, const uint32_t (&bk)[4],
                                          uint32_t live, F &&f) {
  uint4 q[4];
  uint32_t nx[4];
#pragma unroll
  for (uint32_t j = 0; j < 4; ++j)
    if ((live >> j) & 1u) q[j] = ld_slab<false>(g.slabs + 8ull * bk[j] + L.gl);
#pragma unroll
  for (uint32_t j = 0; j < 4; ++j) {
    nx[j] = kNoSlab;
    if ((live >> j) & 1u) {
      f(j, q[j]);
      nx[j] = __shfl_sync(L.gmask, q[j].w, L.gbase + 7);
    }
  }
  while ((nx[0] & nx[1] & nx[2] & nx[3]) != kNoSlab) {
#pragma unroll
    for (uint32_t j = 0; j < 4; ++j)
      if (nx[j] != kNoSlab) q[j] = ld_slab<false>(g.slabs + 8ull * nx[j] + L.gl);
#pragma unroll
    for (uint32_t j = 0; j < 4; ++j)
      if (nx[j] != kNoSlab) {
        f(j, q[j]);
        nx[j] = __shfl_sync(L.gmask, q[j].w, L.gbase + 7);
      }
  }
}

}  // namespace mk
