// Thread-per-edge slab probes and updates, shared by the update kernels and
// the connected-components edge probe.  A lane loads its edge's whole head slab with 8
// independent 16-byte loads (through L2: other SMs write the same slabs),
// decides alone (no cross-lane synchronisation) and commits with one CAS;
// a chain that continues, a lost race or a full slab is walked by the same
// lane.  Key and sentinel words are those of mk_common.cuh; weighted slabs
// hold (key, value) pairs with the key word even.
#pragma once

#include "mk_common.cuh"

namespace mk {

constexpr uint32_t kProbeLimit = 1u << 24;  // slab steps per edge before giving up

struct LaneProbe {
  uint32_t found_word;  // word index of the key, 32 if absent
  uint32_t empty_word;  // first EMPTY key word, 32 if none
  uint32_t next;        // next-slab id
};

template <bool kWeighted>
__device__ __forceinline__ LaneProbe lane_probe(const uint4 (&q)[8], uint32_t key) {
  LaneProbe r{32u, 32u, q[7].w};
#pragma unroll
  for (int j = 7; j >= 0; --j) {
    const uint32_t wv[4] = {q[j].x, q[j].y, q[j].z, q[j].w};
#pragma unroll
    for (int c = 3; c >= 0; --c) {
      const uint32_t word = 4 * j + c;
      const bool is_key = kWeighted ? ((word & 1u) == 0 && word < 30) : (word < 31);
      if (!is_key) continue;
      if (wv[c] == key) r.found_word = word;
      if (wv[c] == kEmptyKey) r.empty_word = word;
    }
  }
  return r;
}

__device__ __forceinline__ void lane_load_slab(const GraphView &g, uint32_t s, uint4 (&q)[8]) {
  const uint4 *p = g.slabs + 8ull * s;
#pragma unroll
  for (int j = 0; j < 8; ++j) q[j] = __ldcg(p + j);
}

// Single-lane insert into the chain at s (first slab already in q).
template <bool kWeighted>
__device__ uint32_t lane_insert_chain(const GraphView &g, uint32_t s, uint4 (&q)[8], uint32_t v,
                                      uint32_t wt) {
  for (uint32_t it = 0; it < kProbeLimit; ++it) {
    if (it) lane_load_slab(g, s, q);
    const LaneProbe p = lane_probe<kWeighted>(q, v);
    if (p.found_word < 32) {
      // live edge: weighted graphs keep the smaller weight (upsert-min)
      if (kWeighted) atomicMin(reinterpret_cast<uint32_t *>(g.slabs + 8ull * s) + p.found_word + 1, wt);
      return 0;
    }
    if (p.empty_word < 32) {
      uint32_t *wp = reinterpret_cast<uint32_t *>(g.slabs + 8ull * s) + p.empty_word;
      // weighted: one 64-bit CAS installs key and weight together (the pair
      // of a never-used slot is EMPTY in both words)
      const uint32_t old =
          kWeighted ? (uint32_t)atomicCAS(reinterpret_cast<unsigned long long *>(wp), ~0ull,
                                          ((unsigned long long)wt << 32) | v)
                    : atomicCAS(wp, kEmptyKey, v);
      if (old == kEmptyKey || old == v) {
        // a copy that found its key already placed keeps the minimum weight
        // (the value word of a never-used slot is EMPTY, so atomicMin is
        // exact under any interleaving)
        if (kWeighted && old == v) atomicMin(wp + 1, wt);
        return old == kEmptyKey ? 1u : 0u;
      }
      continue;
    }
    if (p.next == kLinkBusy) {
      __nanosleep(64);
      continue;
    }
    if (p.next != kNoSlab) {
      s = p.next;
      continue;
    }
    uint32_t *nextp = reinterpret_cast<uint32_t *>(g.slabs + 8ull * s) + 31;
    if (atomicCAS(nextp, kNoSlab, kLinkBusy) == kNoSlab) {
      const uint32_t ns = atomicAdd(g.pool_top, 1u);
      if (ns >= g.pool_cap) {
        atomicOr(g.err, kErrOom);
        atomicExch(nextp, kNoSlab);
        return 0;
      }
      uint32_t *np = reinterpret_cast<uint32_t *>(g.slabs + 8ull * ns);
      np[0] = v;
      if (kWeighted) np[1] = wt;
      __threadfence();
      atomicExch(nextp, ns);
      return 1;
    }
  }
  atomicOr(g.err, kErrTimeout);
  return 0;
}

template <bool kWeighted>
__device__ uint32_t lane_delete_chain(const GraphView &g, uint32_t s, uint4 (&q)[8], uint32_t v) {
  for (uint32_t it = 0; it < kProbeLimit; ++it) {
    if (it) lane_load_slab(g, s, q);
    const LaneProbe p = lane_probe<kWeighted>(q, v);
    if (p.found_word < 32) {
      uint32_t *wp = reinterpret_cast<uint32_t *>(g.slabs + 8ull * s) + p.found_word;
      return atomicCAS(wp, v, kTombKey) == v ? 1u : 0u;
    }
    if (p.next == kNoSlab) return 0;
    s = p.next;
  }
  atomicOr(g.err, kErrTimeout);
  return 0;
}

}  // namespace mk
