// Slab-hash dynamic graph: construction, batched insert / delete / search,
// CSR export and structural counters.
//
// Reference behaviour followed:
//   bucket count per vertex  max(1, ceil(hint / (slots * LoadFactor)))
//                            (include/Graph/SlabGraph.cuh:403-407; the
//                            reference divides by 32 for both slab kinds, this
//                            build divides by the slots a slab really holds:
//                            31 keys, or 15 pairs for weighted graphs)
//   head slabs               one contiguous 128-B slab per bucket, 0xFF filled
//                            (SlabGraph.cuh:417-423)
//   insert                   skip self loops (InsertEdgeKernel.cuh:21-26),
//                            key already present -> unchanged, otherwise take
//                            the first EMPTY key word of the bucket's slab chain,
//                            growing the chain with a pool slab when it is full
//                            (the slab-hash insertKey semantics used at
//                            include/Graph/warp/InsertEdge.cuh:86-88)
//   delete                   live key -> TOMBSTONE, degree - 1
//                            (include/Graph/warp/DeleteEdge.cuh:7-39)
//   search                   (include/Graph/warp/SearchEdge.cuh:8-63)
//
// B200 design: a warp takes 32 batch edges; every lane resolves its edge to
// the bucket's head slab and issues a 128-B TMA bulk copy of it (L2
// evict_last) into the warp's shared-memory stage, double-buffered so the next
// 32 edges' copies are in flight while these are decided.  Each lane then
// decides alone from its staged slab and commits with one CAS.  No sort, no
// locks: a key can only be placed in the first EMPTY word of the chain, which
// makes concurrent inserts of the same key collide on one word, so duplicates
// are impossible.  On weighted graphs the stored weight of an edge is the
// minimum over its live value and every inserted copy (atomicMin on the value
// word), so the result does not depend on the order of concurrent inserts.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <atomic>
#include <mutex>
#include <string>

#include "mk_internal.h"
#include "mk_slab.cuh"
#include "mk_update.cuh"

namespace mk {

static thread_local std::string g_last_error;

void set_error(const std::string &msg) { g_last_error = msg; }

mk_status fail(mk_status st, const std::string &msg) {
  g_last_error = msg;
  return st;
}

mk_status cuda_fail(cudaError_t e, const char *what) {
  g_last_error = std::string(what) + ": " + cudaGetErrorString(e);
  return e == cudaErrorMemoryAllocation ? MK_ERR_OOM : MK_ERR_CUDA;
}

int device_sm_count(int device) {
  int n = 0;
  cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, device);
  return n > 0 ? n : 1;
}

int persistent_blocks(const void *kernel, int block, size_t smem, int device) {
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, smem);
  if (per_sm < 1) per_sm = 1;
  return per_sm * device_sm_count(device);
}

mk_status Timer::start(cudaStream_t st, bool enable) {
  on = enable;
  s = st;
  if (!on) return MK_OK;
  if (!a) MK_CUDA(cudaEventCreate(&a));
  if (!b) MK_CUDA(cudaEventCreate(&b));
  MK_CUDA(cudaEventRecord(a, s));
  return MK_OK;
}

mk_status Timer::stop(float *ms_out) {
  if (!on) return MK_OK;
  MK_CUDA(cudaEventRecord(b, s));
  MK_CUDA(cudaEventSynchronize(b));
  float ms = 0.f;
  MK_CUDA(cudaEventElapsedTime(&ms, a, b));
  if (ms_out) *ms_out = ms;
  return MK_OK;
}

mk_status PinnedRing::upload(void *d_dst, const void *src, size_t bytes, cudaStream_t s) {
  Slot &sl = slots[next++ % kSlots];
  if (sl.used) MK_CUDA(cudaEventSynchronize(sl.done));  // the copy that last read this slot
  if (sl.cap < bytes) {
    if (sl.host) cudaFreeHost(sl.host);
    sl.host = nullptr;
    sl.cap = 0;
    const size_t want = std::max<size_t>(bytes, 64 * 1024);
    MK_CUDA(cudaMallocHost(&sl.host, want));
    sl.cap = want;
  }
  if (!sl.done) MK_CUDA(cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming));
  std::memcpy(sl.host, src, bytes);
  MK_CUDA(cudaMemcpyAsync(d_dst, sl.host, bytes, cudaMemcpyHostToDevice, s));
  MK_CUDA(cudaEventRecord(sl.done, s));
  sl.used = true;
  return MK_OK;
}

void PinnedRing::release() {
  for (Slot &sl : slots) {
    if (sl.used) cudaEventSynchronize(sl.done);
    if (sl.done) cudaEventDestroy(sl.done);
    if (sl.host) cudaFreeHost(sl.host);
    sl = Slot();
  }
}

Timer::~Timer() {
  if (a) cudaEventDestroy(a);
  if (b) cudaEventDestroy(b);
}

// ---------------------------------------------------------------------------
// Exclusive scan u32 -> u64 (three passes: tile sums, scan of sums, tiles).
// ---------------------------------------------------------------------------
constexpr int kScanBlock = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanBlock * kScanItems;

__device__ __forceinline__ unsigned long long block_excl_scan(unsigned long long v,
                                                              unsigned long long *sm,
                                                              unsigned long long *total) {
  // sm has blockDim.x/32 + 1 entries
  uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  unsigned long long x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    unsigned long long y = __shfl_up_sync(0xFFFFFFFFu, x, o);
    if (lane >= (uint32_t)o) x += y;
  }
  if (lane == 31) sm[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint32_t nw = blockDim.x >> 5;
    unsigned long long s = lane < nw ? sm[lane] : 0ull;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      unsigned long long y = __shfl_up_sync(0xFFFFFFFFu, s, o);
      if (lane >= (uint32_t)o) s += y;
    }
    if (lane < nw) sm[lane] = s;  // inclusive warp totals
  }
  __syncthreads();
  unsigned long long warp_off = warp ? sm[warp - 1] : 0ull;
  if (total) *total = sm[(blockDim.x >> 5) - 1];
  __syncthreads();
  return warp_off + x - v;
}

__global__ void k_scan_tiles(const uint32_t *__restrict__ in, uint32_t n,
                             unsigned long long *__restrict__ tile_sums) {
  __shared__ unsigned long long sm[kScanBlock / 32 + 1];
  uint64_t base = (uint64_t)blockIdx.x * kScanTile;
  unsigned long long s = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    uint64_t idx = base + (uint64_t)i * kScanBlock + threadIdx.x;
    if (idx < n) s += in[idx];
  }
  unsigned long long tot;
  block_excl_scan(s, sm, &tot);
  if (threadIdx.x == 0) tile_sums[blockIdx.x] = tot;
}

__global__ void k_scan_sums(unsigned long long *sums, uint32_t m) {
  __shared__ unsigned long long sm[kScanBlock / 32 + 1];
  unsigned long long carry = 0;
  for (uint32_t base = 0; base < m; base += kScanBlock) {
    uint32_t idx = base + threadIdx.x;
    unsigned long long v = idx < m ? sums[idx] : 0ull;
    unsigned long long tot;
    unsigned long long ex = block_excl_scan(v, sm, &tot);
    if (idx < m) sums[idx] = carry + ex;
    carry += tot;
    __syncthreads();
  }
}

__global__ void k_scan_apply(const uint32_t *__restrict__ in, uint32_t n,
                             const unsigned long long *__restrict__ tile_off,
                             unsigned long long *__restrict__ out) {
  __shared__ unsigned long long sm[kScanBlock / 32 + 1];
  uint64_t base = (uint64_t)blockIdx.x * kScanTile + (uint64_t)threadIdx.x * kScanItems;
  uint32_t v[kScanItems];
  unsigned long long s = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    uint64_t idx = base + i;
    v[i] = idx < n ? in[idx] : 0u;
    s += v[i];
  }
  unsigned long long tot;
  unsigned long long ex = block_excl_scan(s, sm, &tot) + tile_off[blockIdx.x];
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    uint64_t idx = base + i;
    if (idx < n) out[idx] = ex;
    ex += v[i];
  }
  if (blockIdx.x == gridDim.x - 1 && threadIdx.x == blockDim.x - 1) out[n] = ex;
}

mk_status scan_u32_to_u64(const uint32_t *d_in, unsigned long long *d_out,
                          uint32_t n, DevBuf<unsigned long long> &tmp,
                          cudaStream_t s) {
  uint32_t tiles = (n + kScanTile - 1) / kScanTile;
  if (tiles == 0) {
    MK_CUDA(cudaMemsetAsync(d_out, 0, sizeof(unsigned long long), s));
    return MK_OK;
  }
  MK_CHECK(tmp.reserve(tiles));
  k_scan_tiles<<<tiles, kScanBlock, 0, s>>>(d_in, n, tmp.ptr);
  k_scan_sums<<<1, kScanBlock, 0, s>>>(tmp.ptr, tiles);
  k_scan_apply<<<tiles, kScanBlock, 0, s>>>(d_in, n, tmp.ptr, d_out);
  MK_CUDA(cudaGetLastError());
  return MK_OK;
}

// ---------------------------------------------------------------------------
// Update kernels
// ---------------------------------------------------------------------------
constexpr int kUpdBlock = 256;

__device__ __forceinline__ unsigned long long mix64(unsigned long long x) {
  x ^= x >> 33;
  x *= 0xff51afd7ed558ccdull;
  x ^= x >> 33;
  x *= 0xc4ceb9fe1a85ec53ull;
  x ^= x >> 33;
  return x;
}


// Update kernels.  A warp takes 32 batch edges at a time:
//   1. every lane resolves its edge to the bucket's head slab;
//   2. every lane issues one 128-byte TMA bulk copy of that slab into the
//      warp's shared-memory stage (completion on the stage's mbarrier), and
//      the warp moves on to resolve its next 32 edges into the other stage
//      while the copies are in flight (double buffering);
//   3. each lane decides from its staged slab (144-B stride: conflict-free
//      reads) and commits with one CAS;
//   4. a lane whose CAS lost a race, whose chain continues or that needs a
//      new slab walks the chain itself from global memory.
// A staged slab that went stale only costs step 4: inside one insert call key
// words only move EMPTY -> key, inside one delete call only key -> TOMBSTONE.
constexpr int kUpdWarps = 4;  // warps per block
constexpr int kCoopBlock = 256;  // threads per block of the warp-cooperative kernel
constexpr size_t kStageStride = 9;  // uint4 per staged slab: 128 B + 16 B pad
constexpr size_t kUpdSmem = (size_t)kUpdWarps * 2 * 32 * kStageStride * 16;  // 2 stages x 32 slabs per warp

struct UpdEdge {
  uint32_t u, v, wt, head;
};

template <bool kWeighted, bool kInsert>
__device__ __forceinline__ UpdEdge upd_resolve(const GraphView &g, const uint32_t *__restrict__ src,
                                               const uint32_t *__restrict__ dst,
                                               const uint32_t *__restrict__ w, uint32_t n, uint64_t e,
                                               uint8_t *__restrict__ applied) {
  UpdEdge E{0u, 0u, 0u, kNoSlab};
  if (e < n) {
    uint32_t u = src[e], v = dst[e];
    if (kWeighted && kInsert && w) E.wt = w[e];
    if (g.reverse) {
      uint32_t t = u;
      u = v;
      v = t;
    }
    E.u = u;
    E.v = v;
    bool ok = (u != v);
    if (u >= g.V || v >= g.V) {
      ok = false;
      atomicOr(g.err, kErrInvalidId);
    }
    if (ok) {
      const uint32_t b0 = g.boff[u];
      const uint32_t b1 = g.boff[u + 1];
      if (ok) E.head = b0 + bucket_of(v, b1 - b0);
    }
    if (!ok) applied[e] = 0;
  }
  return E;
}

// Batch record of one edge, loaded ahead of use.
struct UpdRaw {
  uint32_t u, v, wt;
  uint32_t present;  // e < n
};
// Bucket offsets of a record's source, loaded ahead of use.
struct UpdOff {
  uint32_t b0, b1;
  uint32_t ok;  // in range and not a self-loop
};

template <bool kWeighted, bool kInsert>
__device__ __forceinline__ UpdRaw upd_load(const uint32_t *__restrict__ src,
                                           const uint32_t *__restrict__ dst,
                                           const uint32_t *__restrict__ w, uint32_t n, uint64_t e,
                                           unsigned long long stream_pol) {
  UpdRaw r{0u, 0u, 0u, 0u};
  if (e < n) {
    r.u = ld_stream_u32(src + e, stream_pol);
    r.v = ld_stream_u32(dst + e, stream_pol);
    if (kWeighted && kInsert && w) r.wt = ld_stream_u32(w + e, stream_pol);
    r.present = 1u;
  }
  return r;
}

__device__ __forceinline__ UpdOff upd_offsets(const GraphView &g, UpdRaw &r,
                                              unsigned long long keep_pol) {
  UpdOff o{0u, 0u, 0u};
  if (!r.present) return o;
  if (g.reverse) {
    const uint32_t t = r.u;
    r.u = r.v;
    r.v = t;
  }
  if (r.u >= g.V || r.v >= g.V) {
    atomicOr(g.err, kErrInvalidId);
    return o;
  }
  if (r.u == r.v) return o;
  o.b0 = ld_hint_u32(g.boff + r.u, keep_pol);
  o.b1 = ld_hint_u32(g.boff + r.u + 1, keep_pol);
  o.ok = 1u;
  return o;
}

// A lane's decision for its edge, committed one iteration later.
struct UpdPending {
  uint32_t head, u, v, wt;
  uint32_t word;  // slot word the CAS targets
  uint32_t old;   // value the CAS returned
  uint32_t kind;  // 0 done (not applied), 1 CAS issued, 2 walk the chain
};

// Decides from the staged head slab and issues the one CAS of the fast path
// without waiting for its result.
template <bool kWeighted, bool kInsert>
__device__ __forceinline__ UpdPending upd_decide_probe(const GraphView &g, const LaneProbe &pr,
                                                       uint32_t head, const UpdRaw &r) {
  UpdPending p{head, r.u, r.v, r.wt, 0u, 0u, 0u};
  uint32_t *slab = reinterpret_cast<uint32_t *>(g.slabs + 8ull * head);
  if (kInsert) {
    if (pr.found_word < 32) {
      if (kWeighted) atomicMin(slab + pr.found_word + 1, r.wt);  // live edge: upsert-min
    } else if (pr.empty_word < 32) {
      p.word = pr.empty_word;
      if (kWeighted) {
        // key and weight share one 8-byte pair (key word even): one 64-bit
        // CAS installs both.  A never-used slot is EMPTY in both words; a key
        // placed by the two-step chain walk (key CAS, then atomicMin) makes
        // this CAS fail and return that key.
        unsigned long long *pw = reinterpret_cast<unsigned long long *>(slab + pr.empty_word);
        p.old = (uint32_t)atomicCAS(pw, ~0ull, ((unsigned long long)r.wt << 32) | r.v);
      } else {
        p.old = atomicCAS(slab + pr.empty_word, kEmptyKey, r.v);
      }
      p.kind = 1;
    } else {
      p.kind = 2;
    }
  } else {
    if (pr.found_word < 32) {
      p.word = pr.found_word;
      p.old = atomicCAS(slab + pr.found_word, r.v, kTombKey);
      p.kind = 1;
    } else if (pr.next != kNoSlab) {
      p.kind = 2;
    }
  }
  return p;
}

template <bool kWeighted, bool kInsert>
__device__ __forceinline__ UpdPending upd_decide(const GraphView &g, const uint4 (&q)[8],
                                                 uint32_t head, const UpdRaw &r) {
  return upd_decide_probe<kWeighted, kInsert>(g, lane_probe<kWeighted>(q, r.v), head, r);
}

// Reads the CAS result (or walks the chain) and returns whether the edge
// was applied.
template <bool kWeighted, bool kInsert>
__device__ __forceinline__ uint32_t upd_finish(const GraphView &g, const UpdPending &p) {
  if (p.kind == 0) return 0u;
  uint32_t *slab = reinterpret_cast<uint32_t *>(g.slabs + 8ull * p.head);
  if (p.kind == 1) {
    if (!kInsert) return p.old == p.v ? 1u : 0u;
    if (p.old == kEmptyKey || p.old == p.v) {
      // the pair CAS wrote the weight with the key; a copy that found the key
      // already placed keeps the minimum (the value word of a never-used
      // slot is EMPTY, so atomicMin is exact under any interleaving)
      if (kWeighted && p.old == p.v) atomicMin(slab + p.word + 1, p.wt);
      return p.old == kEmptyKey ? 1u : 0u;
    }
  }
  // lost the slot to another key, or the chain continues: walk it
  uint4 q[8];
  lane_load_slab(g, p.head, q);
  return kInsert ? lane_insert_chain<kWeighted>(g, p.head, q, p.v, p.wt)
                 : lane_delete_chain<kWeighted>(g, p.head, q, p.v);
}

// Warp-staged update kernel.  Each warp walks groups of 32 edges through a
// software pipeline, one group per step per iteration:
//   load    the batch records of group i+3 (streamed, evict-first);
//   offsets the bucket offsets of group i+2's sources (evict-last: the
//           per-vertex arrays stay in L2 under the slab traffic);
//   stage   group i+1's head slabs: one 128-byte cp.async.bulk per lane into
//           the warp's shared-memory stage, completing on its mbarrier;
//   decide  group i: each lane decides from its staged slab and issues its
//           one CAS without waiting for the result;
//   finish  group i-1: the CAS results are read (a weighted insert that
//           met its own key placed concurrently atomicMins the value word;
//           a lost race walks the chain).
// Every result a step consumes was requested one iteration earlier, so a
// warp waits about one memory latency per group.
template <bool kWeighted, bool kInsert>
__global__ void __launch_bounds__(kUpdWarps * 32)
    k_update(GraphView g, const uint32_t *__restrict__ src, const uint32_t *__restrict__ dst,
             const uint32_t *__restrict__ w, uint32_t n, uint8_t *__restrict__ applied,
             unsigned long long *count) {
  extern __shared__ __align__(128) uint4 stage_smem[];
  __shared__ __align__(8) uint64_t bars[kUpdWarps][2];
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t wib = threadIdx.x >> 5;
  const uint64_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = (gridDim.x * blockDim.x) >> 5;
  const uint64_t ngroups = ((uint64_t)n + 31) / 32;
  if (warp >= ngroups) return;
  // [stage][lane] slabs of kStageStride uint4 (144 B: conflict-free lane reads)
  uint4 *wst = stage_smem + (size_t)wib * 2 * 32 * kStageStride;
  if (lane == 0) {
    mbar_init(&bars[wib][0], 1);
    mbar_init(&bars[wib][1], 1);
    mbar_init_fence();
  }
  __syncwarp();
  const unsigned long long keep = l2_policy_evict_last();
  const unsigned long long once = l2_policy_evict_first();
  uint32_t parity[2] = {0u, 0u};
  uint32_t mine = 0;
  // Staging stops for good once a wait gives up (warp-uniform): the rest of
  // the warp's groups read their slabs from global memory, so no copy is
  // issued into a stage whose state is unknown; inflight[s] marks a stage
  // whose copy was issued and not yet seen complete, drained before exit.
  bool staging = true;
  uint32_t inflight[2] = {0u, 0u};

  auto edge_of = [&](uint64_t k) { return (warp + k * nwarps) * 32 + lane; };
  auto group_ok = [&](uint64_t k) { return warp + k * nwarps < ngroups; };
  // stage the head slab of this lane's edge (head == kNoSlab: nothing)
  auto stage = [&](uint32_t head, uint32_t st) {
    if (!staging) return;
    inflight[st] = 1u;
    const uint32_t valid = __ballot_sync(0xFFFFFFFFu, head != kNoSlab);
    fence_proxy_async_smem();  // this warp's earlier reads of the buffer come first
    __syncwarp();
    if (lane == 0) mbar_arrive_expect_tx(&bars[wib][st], 128u * __popc(valid));
    __syncwarp();
    if (head != kNoSlab)
      bulk_load(wst + ((size_t)st * 32 + lane) * kStageStride, g.slabs + 8ull * head, 128u,
                &bars[wib][st]);
  };
  auto head_of = [&](const UpdRaw &r, const UpdOff &o) {
    return o.ok ? o.b0 + bucket_of(r.v, o.b1 - o.b0) : kNoSlab;
  };
  auto finish = [&](const UpdPending &p, uint64_t e) {
    const uint32_t app = upd_finish<kWeighted, kInsert>(g, p);
    if (app) {
      red_add_hint_u32(g.deg + p.u, kInsert ? 1u : 0xFFFFFFFFu, keep);
      ++mine;
    }
    if (e < n) applied[e] = (uint8_t)app;
  };

  // prologue: group 0 staged, group 1's offsets and group 2's records in flight
  UpdRaw r0 = upd_load<kWeighted, kInsert>(src, dst, w, n, edge_of(0), once);
  UpdRaw r1 = group_ok(1) ? upd_load<kWeighted, kInsert>(src, dst, w, n, edge_of(1), once)
                          : UpdRaw{0u, 0u, 0u, 0u};
  UpdRaw r2 = group_ok(2) ? upd_load<kWeighted, kInsert>(src, dst, w, n, edge_of(2), once)
                          : UpdRaw{0u, 0u, 0u, 0u};
  UpdOff o0 = upd_offsets(g, r0, keep);
  UpdOff o1 = upd_offsets(g, r1, keep);
  uint32_t head0 = head_of(r0, o0);
  stage(head0, 0);
  uint32_t st = 0;
  UpdPending prev{kNoSlab, 0u, 0u, 0u, 0u, 0u, 0u};
  uint64_t prev_e = ~0ull;
  for (uint64_t k = 0;; ++k) {
    const bool has1 = group_ok(k + 1);
    uint32_t head1 = kNoSlab;
    if (has1) {
      head1 = head_of(r1, o1);
      stage(head1, st ^ 1u);
    }
    UpdOff o2{0u, 0u, 0u};
    if (group_ok(k + 2)) o2 = upd_offsets(g, r2, keep);
    UpdRaw r3{0u, 0u, 0u, 0u};
    if (group_ok(k + 3)) r3 = upd_load<kWeighted, kInsert>(src, dst, w, n, edge_of(k + 3), once);
    if (k) finish(prev, prev_e);

    // decide group k from its staged slab
    bool ready = false;
    if (staging) {
      ready = __all_sync(0xFFFFFFFFu, mbar_wait(&bars[wib][st], parity[st], g.err));
      if (ready) {
        parity[st] ^= 1u;
        inflight[st] = 0u;
      } else {
        staging = false;  // inflight[st] stays set: its copy may still land
      }
    }
    UpdPending cur{kNoSlab, 0u, 0u, 0u, 0u, 0u, 0u};
    if (head0 != kNoSlab) {
      uint4 q[8];
      const uint4 *sp = wst + ((size_t)st * 32 + lane) * kStageStride;
      if (ready) {
#pragma unroll
        for (int j = 0; j < 8; ++j) q[j] = sp[j];
      } else {
        lane_load_slab(g, head0, q);
      }
      cur = upd_decide<kWeighted, kInsert>(g, q, head0, r0);
    }
    prev = cur;
    prev_e = edge_of(k);
    if (!has1) break;
    __syncwarp();
    r0 = r1;
    head0 = head1;
    r1 = r2;
    o1 = o2;
    r2 = r3;
    st ^= 1u;
  }
  finish(prev, prev_e);
  mine = __reduce_add_sync(0xFFFFFFFFu, mine);
  if (lane == 0 && mine) atomicAdd(count, (unsigned long long)mine);
  // after a wait gave up: give the copies still in flight a bounded time to
  // land before the block's shared memory is released
#pragma unroll
  for (int sidx = 0; sidx < 2; ++sidx)
    if (inflight[sidx]) mbar_wait(&bars[wib][sidx], parity[sidx], g.err);
}

// Warp-cooperative update kernel (no shared memory, no bulk copies): a warp
// loads the head slabs of its 32 edges as 32 coalesced 128-byte loads (lane
// l holds word l of every slab), then decides edge j from slab j with two
// ballots (key found / first EMPTY word) and one shuffle (next-slab word);
// lane j commits its own edge with one CAS.  Batch records and bucket
// offsets are prefetched one group ahead, CAS results read one group later.
template <bool kWeighted, bool kInsert>
__global__ void __launch_bounds__(kCoopBlock, 3)
    k_update_coop(GraphView g, const uint32_t *__restrict__ src, const uint32_t *__restrict__ dst,
                  const uint32_t *__restrict__ w, uint32_t n, uint8_t *__restrict__ applied,
                  unsigned long long *count) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint64_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = (gridDim.x * blockDim.x) >> 5;
  const uint64_t ngroups = ((uint64_t)n + 31) / 32;
  if (warp >= ngroups) return;
  const unsigned long long keep = l2_policy_evict_last();
  const unsigned long long once = l2_policy_evict_first();
  const uint32_t *words = reinterpret_cast<const uint32_t *>(g.slabs);
  // key words: set slabs 0..30, map slabs the even words 0..28
  const bool keylane = kWeighted ? ((lane & 1u) == 0 && lane < 30) : (lane < 31);
  uint32_t mine = 0;
  auto edge_of = [&](uint64_t k) { return (warp + k * nwarps) * 32 + lane; };
  auto group_ok = [&](uint64_t k) { return warp + k * nwarps < ngroups; };
  auto finish = [&](const UpdPending &p, uint64_t e) {
    const uint32_t app = upd_finish<kWeighted, kInsert>(g, p);
    if (app) {
      red_add_hint_u32(g.deg + p.u, kInsert ? 1u : 0xFFFFFFFFu, keep);
      ++mine;
    }
    if (e < n) applied[e] = (uint8_t)app;
  };

  UpdRaw r0 = upd_load<kWeighted, kInsert>(src, dst, w, n, edge_of(0), once);
  UpdRaw r1 = group_ok(1) ? upd_load<kWeighted, kInsert>(src, dst, w, n, edge_of(1), once)
                          : UpdRaw{0u, 0u, 0u, 0u};
  UpdOff o0 = upd_offsets(g, r0, keep);
  UpdPending prev{kNoSlab, 0u, 0u, 0u, 0u, 0u, 0u};
  uint64_t prev_e = ~0ull;
  for (uint64_t k = 0;; ++k) {
    const bool has1 = group_ok(k + 1);
    UpdOff o1{0u, 0u, 0u};
    if (has1) o1 = upd_offsets(g, r1, keep);
    UpdRaw r2{0u, 0u, 0u, 0u};
    if (group_ok(k + 2)) r2 = upd_load<kWeighted, kInsert>(src, dst, w, n, edge_of(k + 2), once);
    const uint32_t head0 = o0.ok ? o0.b0 + bucket_of(r0.v, o0.b1 - o0.b0) : kNoSlab;
    uint32_t wv[32];
#pragma unroll
    for (int j = 0; j < 32; ++j) {
      const uint32_t h = __shfl_sync(0xFFFFFFFFu, head0, j);
      wv[j] = h != kNoSlab ? __ldcg(words + (size_t)h * 32 + lane) : kEmptyKey;
    }
    if (k) finish(prev, prev_e);
    LaneProbe pr{32u, 32u, kNoSlab};
#pragma unroll
    for (int j = 0; j < 32; ++j) {
      const uint32_t vj = __shfl_sync(0xFFFFFFFFu, r0.v, j);
      const uint32_t hit = __ballot_sync(0xFFFFFFFFu, keylane && wv[j] == vj);
      const uint32_t emp = __ballot_sync(0xFFFFFFFFu, keylane && wv[j] == kEmptyKey);
      const uint32_t nx = __shfl_sync(0xFFFFFFFFu, wv[j], 31);
      if (lane == (uint32_t)j) {
        pr.found_word = hit ? (uint32_t)__ffs(hit) - 1u : 32u;
        pr.empty_word = emp ? (uint32_t)__ffs(emp) - 1u : 32u;
        pr.next = nx;
      }
    }
    UpdPending cur{kNoSlab, 0u, 0u, 0u, 0u, 0u, 0u};
    if (head0 != kNoSlab) cur = upd_decide_probe<kWeighted, kInsert>(g, pr, head0, r0);
    prev = cur;
    prev_e = edge_of(k);
    if (!has1) break;
    r0 = r1;
    o0 = o1;
    r1 = r2;
  }
  finish(prev, prev_e);
  mine = __reduce_add_sync(0xFFFFFFFFu, mine);
  if (lane == 0 && mine) atomicAdd(count, (unsigned long long)mine);
}

// ---------------------------------------------------------------------------
// Thread-per-edge variant: a lane loads its edge's whole head slab with 8
// independent 16-byte loads, decides alone (no cross-lane synchronisation),
// and commits with one CAS.  Chains and lost races are walked by the same
// lane.  Selected by the tuner when it beats the warp-staged kernel.
// ---------------------------------------------------------------------------
template <bool kWeighted, bool kInsert>
__global__ void __launch_bounds__(256)
    k_update_lane(GraphView g, const uint32_t *__restrict__ src, const uint32_t *__restrict__ dst,
                  const uint32_t *__restrict__ w, uint32_t n, uint8_t *__restrict__ applied,
                  unsigned long long *count) {
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t nthreads = gridDim.x * blockDim.x;
  uint32_t mine = 0;
  for (uint64_t e = tid; e < n; e += nthreads) {
    const UpdEdge E = upd_resolve<kWeighted, kInsert>(g, src, dst, w, n, e, applied);
    if (E.head == kNoSlab) continue;
    uint4 q[8];
    lane_load_slab(g, E.head, q);
    const uint32_t app = kInsert ? lane_insert_chain<kWeighted>(g, E.head, q, E.v, E.wt)
                                 : lane_delete_chain<kWeighted>(g, E.head, q, E.v);
    applied[e] = (uint8_t)app;
    if (app) {
      if (kInsert)
        atomicAdd(g.deg + E.u, 1u);
      else
        atomicSub(g.deg + E.u, 1u);
      ++mine;
    }
  }
  mine = __reduce_add_sync(0xFFFFFFFFu, mine);
  if ((threadIdx.x & 31) == 0 && mine) atomicAdd(count, (unsigned long long)mine);
}

template <bool kWeighted>
__global__ void __launch_bounds__(kUpdBlock)
    k_search(GraphView g, const uint32_t *__restrict__ src,
             const uint32_t *__restrict__ dst, uint32_t n,
             uint8_t *__restrict__ found_out, uint32_t *__restrict__ w_out) {
  const Lanes L = lanes();
  const uint32_t group = (blockIdx.x * blockDim.x + threadIdx.x) >> 3;
  const uint32_t ngroups = (gridDim.x * blockDim.x) >> 3;
  for (uint32_t e = group; e < n; e += ngroups) {
    uint32_t u = src[e], v = dst[e];
    if (g.reverse) {
      uint32_t t = u;
      u = v;
      v = t;
    }
    bool hit = false;
    uint32_t val = 0;
    if (u < g.V && v < g.V && u != v) {
      const uint32_t b0 = g.boff[u];
      const uint32_t nb = g.boff[u + 1] - b0;
      uint32_t s = b0 + bucket_of(v, nb);
      for (uint32_t it = 0; it < kProbeLimit && s != kNoSlab; ++it) {
        uint4 q = ld_slab_ro(g.slabs + 8ull * s + L.gl);
        bool f;
        uint32_t fslot, eslot, next;
        probe_slab<kWeighted>(q, v, L, f, fslot, eslot, next);
        if (f) {
          hit = true;
          if (kWeighted) {
            // value word 2*fslot+1 lives in lane fslot/2, component y or w
            uint32_t owner = fslot >> 1;
            uint32_t cand = (fslot & 1) ? q.w : q.y;
            val = __shfl_sync(L.gmask, cand, L.gbase + owner);
          }
          break;
        }
        s = next;
      }
    }
    if (L.gl == 0) {
      if (found_out) found_out[e] = hit ? 1 : 0;
      if (w_out) w_out[e] = val;
    }
  }
}

// Per-vertex walk helpers ----------------------------------------------------

// Number of live keys and tombstones held by one lane's 16-byte quarter.
template <bool kWeighted>
__device__ __forceinline__ void lane_counts(const uint4 &q, uint32_t gl,
                                            uint32_t &live, uint32_t &tomb) {
  live = 0;
  tomb = 0;
  auto acc = [&](uint32_t k) {
    live += (k < kTombKey);
    tomb += (k == kTombKey);
  };
  if (!kWeighted) {
    acc(q.x);
    acc(q.y);
    acc(q.z);
    if (gl != 7) acc(q.w);
  } else {
    acc(q.x);
    if (gl != 7) acc(q.z);
  }
}

// Live keys per bucket (group per bucket: balanced under degree skew).
template <bool kWeighted>
__global__ void k_bucket_live(GraphView g, uint32_t *__restrict__ bcnt) {
  const Lanes L = lanes();
  const uint32_t group = (blockIdx.x * blockDim.x + threadIdx.x) >> 3;
  const uint32_t ngroups = (gridDim.x * blockDim.x) >> 3;
  for (uint32_t b = group; b < g.nbuckets; b += ngroups) {
    uint32_t c = 0;
    walk_bucket(g, L, b, [&](const uint4 &q) {
      uint32_t live, tomb;
      lane_counts<kWeighted>(q, L.gl, live, tomb);
      c += live;
    });
    c = __reduce_add_sync(L.gmask, c);
    if (L.gl == 0) bcnt[b] = c;
  }
}

template <bool kWeighted>
__global__ void k_count_tombstones(GraphView g, uint32_t *__restrict__ out) {
  const Lanes L = lanes();
  const uint32_t group = (blockIdx.x * blockDim.x + threadIdx.x) >> 3;
  const uint32_t ngroups = (gridDim.x * blockDim.x) >> 3;
  for (uint32_t b = group; b < g.nbuckets; b += ngroups) {
    uint32_t t = 0;
    walk_bucket(g, L, b, [&](const uint4 &q) {
      uint32_t live, tomb;
      lane_counts<kWeighted>(q, L.gl, live, tomb);
      t += tomb;
    });
    t = __reduce_add_sync(L.gmask, t);
    if (L.gl == 0 && t) atomicAdd(out + g.bowner[b], t);
  }
}

// row_ptr[u] = bucket position of u's first bucket.
__global__ void k_rows_from_buckets(const uint32_t *__restrict__ boff, uint32_t V, uint32_t nb,
                                    const unsigned long long *__restrict__ bpos,
                                    unsigned long long *__restrict__ row_ptr) {
  for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u <= V; u += gridDim.x * blockDim.x)
    row_ptr[u] = bpos[u < V ? boff[u] : nb];
}

// Writes the live keys of every bucket at its scanned position.
template <bool kWeighted>
__global__ void k_bucket_fill(GraphView g, const unsigned long long *__restrict__ bpos,
                              uint32_t *__restrict__ col, uint32_t *__restrict__ wout) {
  const Lanes L = lanes();
  const uint32_t group = (blockIdx.x * blockDim.x + threadIdx.x) >> 3;
  const uint32_t ngroups = (gridDim.x * blockDim.x) >> 3;
  for (uint32_t b = group; b < g.nbuckets; b += ngroups) {
    unsigned long long pos = bpos[b];
    const unsigned long long end = bpos[b + 1];
    walk_bucket(g, L, b, [&](const uint4 &q) {
      uint32_t live, tomb;
      lane_counts<kWeighted>(q, L.gl, live, tomb);
      uint32_t incl = live;
#pragma unroll
      for (int o = 1; o < 8; o <<= 1) {
        uint32_t y = __shfl_up_sync(L.gmask, incl, o, 8);
        if (L.gl >= (uint32_t)o) incl += y;
      }
      uint32_t total = __shfl_sync(L.gmask, incl, L.gbase + 7);
      unsigned long long p = pos + (incl - live);
      auto put = [&](uint32_t k, uint32_t val) {
        if (k < kTombKey) {
          if (p < end) {
            col[p] = k;
            if (wout) wout[p] = val;
          }
          ++p;
        }
      };
      if (!kWeighted) {
        put(q.x, 0);
        put(q.y, 0);
        put(q.z, 0);
        if (L.gl != 7) put(q.w, 0);
      } else {
        put(q.x, q.y);
        if (L.gl != 7) put(q.z, q.w);
      }
      pos += total;
    });
  }
}

// Sum of deg[vb .. ve) into *out (zeroed by the caller).
__global__ void k_sum_degrees(const uint32_t *__restrict__ deg, uint32_t vb, uint32_t ve,
                              unsigned long long *out) {
  unsigned long long acc = 0;
  for (uint32_t u = vb + blockIdx.x * blockDim.x + threadIdx.x; u < ve; u += gridDim.x * blockDim.x)
    acc += deg[u];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xFFFFFFFFu, acc, o);
  if ((threadIdx.x & 31) == 0 && acc) atomicAdd(out, acc);
}

// Range export: live keys per bucket of the buckets [b0, b0 + nbr), written
// at bcnt[b - b0].
template <bool kWeighted>
__global__ void k_bucket_live_range(GraphView g, uint32_t b0, uint32_t nbr,
                                    uint32_t *__restrict__ bcnt) {
  const Lanes L = lanes();
  const uint32_t group = (blockIdx.x * blockDim.x + threadIdx.x) >> 3;
  const uint32_t ngroups = (gridDim.x * blockDim.x) >> 3;
  for (uint32_t i = group; i < nbr; i += ngroups) {
    uint32_t c = 0;
    walk_bucket(g, L, b0 + i, [&](const uint4 &q) {
      uint32_t live, tomb;
      lane_counts<kWeighted>(q, L.gl, live, tomb);
      c += live;
    });
    c = __reduce_add_sync(L.gmask, c);
    if (L.gl == 0) bcnt[i] = c;
  }
}

// row_ptr[u - vb] = position of u's first bucket, relative to the range.
__global__ void k_rows_from_buckets_range(const uint32_t *__restrict__ boff, uint32_t vb,
                                          uint32_t nv, uint32_t b0, uint32_t nbr,
                                          const unsigned long long *__restrict__ bpos,
                                          unsigned long long *__restrict__ row_ptr) {
  for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u <= nv; u += gridDim.x * blockDim.x)
    row_ptr[u] = bpos[u < nv ? boff[vb + u] - b0 : nbr];
}

// Writes the live keys of the buckets [b0, b0 + nbr) at their positions.
template <bool kWeighted>
__global__ void k_bucket_fill_range(GraphView g, uint32_t b0, uint32_t nbr,
                                    const unsigned long long *__restrict__ bpos,
                                    uint32_t *__restrict__ col, uint32_t *__restrict__ wout) {
  const Lanes L = lanes();
  const uint32_t group = (blockIdx.x * blockDim.x + threadIdx.x) >> 3;
  const uint32_t ngroups = (gridDim.x * blockDim.x) >> 3;
  for (uint32_t i = group; i < nbr; i += ngroups) {
    unsigned long long pos = bpos[i];
    const unsigned long long end = bpos[i + 1];
    walk_bucket(g, L, b0 + i, [&](const uint4 &q) {
      uint32_t live, tomb;
      lane_counts<kWeighted>(q, L.gl, live, tomb);
      uint32_t incl = live;
#pragma unroll
      for (int o = 1; o < 8; o <<= 1) {
        uint32_t y = __shfl_up_sync(L.gmask, incl, o, 8);
        if (L.gl >= (uint32_t)o) incl += y;
      }
      uint32_t total = __shfl_sync(L.gmask, incl, L.gbase + 7);
      unsigned long long p = pos + (incl - live);
      auto put = [&](uint32_t k, uint32_t val) {
        if (k < kTombKey) {
          if (p < end) {
            col[p] = k;
            if (wout) wout[p] = val;
          }
          ++p;
        }
      };
      if (!kWeighted) {
        put(q.x, 0);
        put(q.y, 0);
        put(q.z, 0);
        if (L.gl != 7) put(q.w, 0);
      } else {
        put(q.x, q.y);
        if (L.gl != 7) put(q.z, q.w);
      }
      pos += total;
    });
  }
}

static int update_grid(uint32_t n, int device) {
  // one warp per 32 edges, at most the resident blocks (each warp loops)
  uint64_t blocks = ((uint64_t)n + kUpdWarps * 32 - 1) / (kUpdWarps * 32);
  uint64_t cap = (uint64_t)device_sm_count(device) * 6;  // 6 x 32 KB stages per SM
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  return (int)blocks;
}

static int lane_grid(uint32_t n, const mk_graph *g) {
  // one lane per edge; 256-thread blocks, capped at the resident count
  uint64_t blocks = ((uint64_t)n + 255) / 256;
  uint32_t per_sm = g->tuning.update_blocks_per_sm ? g->tuning.update_blocks_per_sm : 6;
  uint64_t cap = (uint64_t)device_sm_count(g->device) * per_sm;
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  return (int)blocks;
}

// Warp-cooperative kernel: one warp per group of 32 edges, capped at the
// resident count (or update_blocks_per_sm blocks per SM when set).
template <class K>
static int coop_grid(uint32_t n, const mk_graph *g, K kernel) {
  const uint64_t groups = ((uint64_t)n + 31) / 32;
  uint64_t blocks = (groups + kCoopBlock / 32 - 1) / (kCoopBlock / 32);
  uint32_t per_sm = g->tuning.update_blocks_per_sm;
  if (per_sm == 0) {
    int occ = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, kCoopBlock, 0);
    per_sm = occ > 0 ? (uint32_t)occ : 1u;
  }
  const uint64_t cap = (uint64_t)device_sm_count(g->device) * per_sm;
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  return (int)blocks;
}

// Opts a kernel into kUpdSmem of dynamic shared memory, once per device.
template <class K>
static mk_status set_update_smem(K kernel) {
  static std::atomic<uint64_t> done{0};  // bit per device ordinal
  int dev = 0;
  cudaGetDevice(&dev);
  const uint64_t bit = 1ull << (dev & 63);
  if (done.load(std::memory_order_acquire) & bit) return MK_OK;
  MK_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kUpdSmem));
  done.fetch_or(bit, std::memory_order_acq_rel);
  return MK_OK;
}

static int group_grid(uint32_t n, int device) {
  // 8 lanes per item
  uint64_t blocks = ((uint64_t)n * 8 + kUpdBlock - 1) / kUpdBlock;
  uint64_t cap = (uint64_t)device_sm_count(device) * 8;
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  return (int)blocks;
}

}  // namespace mk

using namespace mk;

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

const char *mk_last_error_string(void) { return g_last_error.c_str(); }
const char *mk_version(void) { return "meerkat_b200 0.1 sm_100a"; }

mk_status mk_graph_create(const mk_graph_desc *desc, mk_graph **out) {
  if (!desc || !out) return fail(MK_ERR_INVALID, "mk_graph_create: null argument");
  *out = nullptr;
  if (desc->num_vertices == 0 || desc->num_vertices >= kTombKey)
    return fail(MK_ERR_INVALID, "mk_graph_create: num_vertices out of range");
  if (!(desc->load_factor > 0.0) || !std::isfinite(desc->load_factor))
    return fail(MK_ERR_INVALID, "mk_graph_create: load_factor must be > 0");
  if (desc->flags != 0) return fail(MK_ERR_INVALID, "mk_graph_create: flags must be 0");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return fail(MK_ERR_CUDA, "mk_graph_create: no CUDA device");
  if (desc->device < 0 || desc->device >= ndev)
    return fail(MK_ERR_INVALID, "mk_graph_create: bad device index");
  DeviceGuard dg(desc->device);

  mk_graph *g = new mk_graph();
  g->device = desc->device;
  g->V = desc->num_vertices;
  g->weighted = desc->weighted ? 1u : 0u;
  g->reverse = desc->reverse ? 1u : 0u;
  g->keys_per_slab = g->weighted ? 15u : 31u;
  g->load_factor = desc->load_factor;

  const uint32_t V = g->V;
  g->h_boff.resize((size_t)V + 1);
  uint64_t total = 0, hint_sum = 0;
  const double per_bucket = (double)g->keys_per_slab * desc->load_factor;
  for (uint32_t i = 0; i < V; ++i) {
    uint32_t hint = desc->h_degree_hints ? desc->h_degree_hints[i] : 1u;
    hint_sum += hint;
    double x = std::ceil((double)hint / per_bucket);
    uint64_t nb = x < 1.0 ? 1 : (uint64_t)x;
    g->h_boff[i] = (uint32_t)total;
    total += nb;
    if (total >= 0xF0000000ull) {
      delete g;
      return fail(MK_ERR_INVALID, "mk_graph_create: too many buckets");
    }
  }
  g->h_boff[V] = (uint32_t)total;
  g->num_buckets = total;
  uint64_t overflow = desc->pool_slabs;
  if (overflow == 0) {
    overflow = std::max<uint64_t>(65536, 2 * total + hint_sum / g->keys_per_slab);
  }
  g->pool_cap = total + overflow;
  if (g->pool_cap >= 0xFFFFFFF0ull) g->pool_cap = 0xFFFFFFF0ull;

  auto cleanup = [&](mk_status st, const char *what, cudaError_t e) {
    mk_graph_destroy(g);
    return cuda_fail(e, what), st;
  };
  cudaError_t e;
  if ((e = cudaMalloc(&g->slabs, g->pool_cap * 128ull)) != cudaSuccess)
    return cleanup(MK_ERR_OOM, "cudaMalloc(slab pool)", e);
  if ((e = cudaMalloc(&g->boff, ((size_t)V + 1) * 4)) != cudaSuccess)
    return cleanup(MK_ERR_OOM, "cudaMalloc(bucket offsets)", e);
  if ((e = cudaMalloc(&g->deg, (size_t)V * 4)) != cudaSuccess)
    return cleanup(MK_ERR_OOM, "cudaMalloc(degrees)", e);
  if ((e = cudaMalloc(&g->bowner, total * 4)) != cudaSuccess)
    return cleanup(MK_ERR_OOM, "cudaMalloc(bucket owners)", e);
  if ((e = cudaMalloc(&g->pool_top, 4 * sizeof(uint32_t))) != cudaSuccess)
    return cleanup(MK_ERR_OOM, "cudaMalloc(pool counter)", e);
  if ((e = cudaMalloc(&g->counters, 4 * sizeof(unsigned long long))) != cudaSuccess)
    return cleanup(MK_ERR_OOM, "cudaMalloc(counters)", e);
  g->device_bytes = g->pool_cap * 128ull + ((size_t)V + 1) * 4 + (size_t)V * 4 + total * 4 + 48;
  if ((e = cudaMemset(g->slabs, 0xFF, g->pool_cap * 128ull)) != cudaSuccess)
    return cleanup(MK_ERR_CUDA, "cudaMemset(slabs)", e);
  if ((e = cudaMemcpy(g->boff, g->h_boff.data(), ((size_t)V + 1) * 4,
                      cudaMemcpyHostToDevice)) != cudaSuccess)
    return cleanup(MK_ERR_CUDA, "cudaMemcpy(bucket offsets)", e);
  if ((e = cudaMemset(g->deg, 0, (size_t)V * 4)) != cudaSuccess)
    return cleanup(MK_ERR_CUDA, "cudaMemset(degrees)", e);
  {
    std::vector<uint32_t> owner(total);
    for (uint32_t i = 0; i < V; ++i)
      for (uint32_t b = g->h_boff[i]; b < g->h_boff[i + 1]; ++b) owner[b] = i;
    if ((e = cudaMemcpy(g->bowner, owner.data(), total * 4, cudaMemcpyHostToDevice)) != cudaSuccess)
      return cleanup(MK_ERR_CUDA, "cudaMemcpy(bucket owners)", e);
  }
  uint32_t init[4] = {(uint32_t)total, 0u, 0u, 0u};
  if ((e = cudaMemcpy(g->pool_top, init, sizeof(init), cudaMemcpyHostToDevice)) != cudaSuccess)
    return cleanup(MK_ERR_CUDA, "cudaMemcpy(pool counter)", e);
  if ((e = cudaMemset(g->counters, 0, 4 * sizeof(unsigned long long))) != cudaSuccess)
    return cleanup(MK_ERR_CUDA, "cudaMemset(counters)", e);
  if ((e = cudaDeviceSynchronize()) != cudaSuccess)
    return cleanup(MK_ERR_CUDA, "cudaDeviceSynchronize(create)", e);
  *out = g;
  return MK_OK;
}

mk_status mk_graph_destroy(mk_graph *g) {
  if (!g) return MK_OK;
  DeviceGuard dg(g->device);
  if (g->slabs) cudaFree(g->slabs);
  if (g->boff) cudaFree(g->boff);
  if (g->deg) cudaFree(g->deg);
  if (g->bowner) cudaFree(g->bowner);
  if (g->pool_top) cudaFree(g->pool_top);
  if (g->counters) cudaFree(g->counters);
  g->applied.release();
  g->scan_tmp.release();
  g->bucket_cnt.release();
  g->bucket_pos.release();
  delete g;
  return MK_OK;
}

mk_status mk_graph_reserve_batch(mk_graph *g, uint32_t n) {
  if (!g) return fail(MK_ERR_INVALID, "mk_graph_reserve_batch: null graph");
  DeviceGuard dg(g->device);
  MK_CHECK(g->applied.reserve(std::max<uint32_t>(n, 1), &g->device_bytes));
  return MK_OK;
}

static mk_status begin_update(mk_graph *g, const uint32_t *d_src,
                              const uint32_t *d_dst, uint32_t n, int op,
                              cudaStream_t s) {
  MK_CHECK(g->applied.reserve(std::max<uint32_t>(n, 1), &g->device_bytes));
  MK_CUDA(cudaMemsetAsync(g->counters, 0, sizeof(unsigned long long), s));
  g->last_n = n;
  g->last_src = d_src;
  g->last_dst = d_dst;
  g->last_op = op;
  return MK_OK;
}

mk_status mk_graph_insert_edges(mk_graph *g, const uint32_t *d_src,
                                const uint32_t *d_dst, const uint32_t *d_w,
                                uint32_t n, void *stream) {
  if (!g) return fail(MK_ERR_INVALID, "mk_graph_insert_edges: null graph");
  if (n && (!d_src || !d_dst)) return fail(MK_ERR_INVALID, "mk_graph_insert_edges: null batch");
  DeviceGuard dg(g->device);
  cudaStream_t s = as_stream(stream);
  MK_CHECK(begin_update(g, d_src, d_dst, n, 1, s));
  if (n == 0) return MK_OK;
  GraphView v = g->view();
  int blocks = update_grid(n, g->device);
  if (g->tuning.update_kernel == 2) {
    if (g->weighted)
      k_update_coop<true, true><<<coop_grid(n, g, k_update_coop<true, true>), kCoopBlock, 0, s>>>(
          v, d_src, d_dst, d_w, n, g->applied.ptr, g->counters);
    else
      k_update_coop<false, true><<<coop_grid(n, g, k_update_coop<false, true>), kCoopBlock, 0, s>>>(
          v, d_src, d_dst, nullptr, n, g->applied.ptr, g->counters);
  } else if (g->tuning.update_kernel == 1) {
    if (g->weighted)
      k_update_lane<true, true><<<lane_grid(n, g), 256, 0, s>>>(v, d_src, d_dst, d_w, n,
                                                                g->applied.ptr, g->counters);
    else
      k_update_lane<false, true><<<lane_grid(n, g), 256, 0, s>>>(v, d_src, d_dst, nullptr, n,
                                                                 g->applied.ptr, g->counters);
  } else if (g->weighted) {
    MK_CHECK(set_update_smem(k_update<true, true>));
    k_update<true, true><<<blocks, kUpdWarps * 32, kUpdSmem, s>>>(v, d_src, d_dst, d_w, n,
                                                                  g->applied.ptr, g->counters);
  } else {
    MK_CHECK(set_update_smem(k_update<false, true>));
    k_update<false, true><<<blocks, kUpdWarps * 32, kUpdSmem, s>>>(v, d_src, d_dst, nullptr, n,
                                                                   g->applied.ptr, g->counters);
  }
  MK_CUDA(cudaGetLastError());
  return MK_OK;
}

mk_status mk_graph_delete_edges(mk_graph *g, const uint32_t *d_src,
                                const uint32_t *d_dst, uint32_t n,
                                void *stream) {
  if (!g) return fail(MK_ERR_INVALID, "mk_graph_delete_edges: null graph");
  if (n && (!d_src || !d_dst)) return fail(MK_ERR_INVALID, "mk_graph_delete_edges: null batch");
  DeviceGuard dg(g->device);
  cudaStream_t s = as_stream(stream);
  MK_CHECK(begin_update(g, d_src, d_dst, n, 2, s));
  if (n == 0) return MK_OK;
  GraphView v = g->view();
  int blocks = update_grid(n, g->device);
  if (g->tuning.update_kernel == 2) {
    if (g->weighted)
      k_update_coop<true, false><<<coop_grid(n, g, k_update_coop<true, false>), kCoopBlock, 0, s>>>(
          v, d_src, d_dst, nullptr, n, g->applied.ptr, g->counters);
    else
      k_update_coop<false, false><<<coop_grid(n, g, k_update_coop<false, false>), kCoopBlock, 0, s>>>(
          v, d_src, d_dst, nullptr, n, g->applied.ptr, g->counters);
  } else if (g->tuning.update_kernel == 1) {
    if (g->weighted)
      k_update_lane<true, false><<<lane_grid(n, g), 256, 0, s>>>(v, d_src, d_dst, nullptr, n,
                                                                 g->applied.ptr, g->counters);
    else
      k_update_lane<false, false><<<lane_grid(n, g), 256, 0, s>>>(v, d_src, d_dst, nullptr, n,
                                                                  g->applied.ptr, g->counters);
  } else if (g->weighted) {
    MK_CHECK(set_update_smem(k_update<true, false>));
    k_update<true, false><<<blocks, kUpdWarps * 32, kUpdSmem, s>>>(v, d_src, d_dst, nullptr, n,
                                                                   g->applied.ptr, g->counters);
  } else {
    MK_CHECK(set_update_smem(k_update<false, false>));
    k_update<false, false><<<blocks, kUpdWarps * 32, kUpdSmem, s>>>(v, d_src, d_dst, nullptr, n,
                                                                    g->applied.ptr, g->counters);
  }
  MK_CUDA(cudaGetLastError());
  return MK_OK;
}

mk_status mk_graph_search_edges(mk_graph *g, const uint32_t *d_src,
                                const uint32_t *d_dst, uint32_t n,
                                uint8_t *d_found, uint32_t *d_w, void *stream) {
  if (!g) return fail(MK_ERR_INVALID, "mk_graph_search_edges: null graph");
  if (n == 0) return MK_OK;
  if (!d_src || !d_dst) return fail(MK_ERR_INVALID, "mk_graph_search_edges: null batch");
  DeviceGuard dg(g->device);
  cudaStream_t s = as_stream(stream);
  GraphView v = g->view();
  int blocks = group_grid(n, g->device);
  if (g->weighted)
    k_search<true><<<blocks, kUpdBlock, 0, s>>>(v, d_src, d_dst, n, d_found, d_w);
  else
    k_search<false><<<blocks, kUpdBlock, 0, s>>>(v, d_src, d_dst, n, d_found, d_w);
  MK_CUDA(cudaGetLastError());
  return MK_OK;
}

mk_status mk_graph_set_tuning(mk_graph *g, const mk_tuning *t) {
  if (!g || !t) return fail(MK_ERR_INVALID, "mk_graph_set_tuning: null argument");
  if (t->update_kernel > 2) return fail(MK_ERR_INVALID, "mk_graph_set_tuning: update_kernel must be 0, 1 or 2");
  if (t->update_blocks_per_sm > 32) return fail(MK_ERR_INVALID, "mk_graph_set_tuning: update_blocks_per_sm > 32");
  if (t->frontier_chunk > 1024) return fail(MK_ERR_INVALID, "mk_graph_set_tuning: frontier_chunk > 1024");
  if (t->recompute_permille > 1000) return fail(MK_ERR_INVALID, "mk_graph_set_tuning: recompute_permille > 1000");
  if (t->pull_permille > 1000) return fail(MK_ERR_INVALID, "mk_graph_set_tuning: pull_permille > 1000");
  g->tuning = *t;
  return MK_OK;
}

mk_status mk_graph_get_tuning(mk_graph *g, mk_tuning *t) {
  if (!g || !t) return fail(MK_ERR_INVALID, "mk_graph_get_tuning: null argument");
  *t = g->tuning;
  return MK_OK;
}

mk_status mk_graph_sync(mk_graph *g, void *stream, uint32_t *h_deverr) {
  if (!g) return fail(MK_ERR_INVALID, "mk_graph_sync: null graph");
  DeviceGuard dg(g->device);
  cudaStream_t s = as_stream(stream);
  uint32_t err = 0;
  MK_CUDA(cudaMemcpyAsync(&err, g->err_word(), 4, cudaMemcpyDeviceToHost, s));
  MK_CUDA(cudaStreamSynchronize(s));
  if (h_deverr) *h_deverr = err;
  if (err & kErrTimeout) return fail(MK_ERR_TIMEOUT, "device wait or probe limit exceeded");
  if (err & kErrOom) return fail(MK_ERR_OOM, "slab pool exhausted");
  if (err & kErrInvalidId)
    return fail(MK_ERR_INVALID,
                "vertex id out of range: a batch id >= num_vertices, or an edge leaving the "
                "vertex range of a range call");
  return MK_OK;
}

mk_status mk_graph_slabs_used_async(mk_graph *g, uint32_t *h_slabs_used, void *stream) {
  if (!g || !h_slabs_used) return fail(MK_ERR_INVALID, "mk_graph_slabs_used_async: null argument");
  DeviceGuard dg(g->device);
  MK_CUDA(cudaMemcpyAsync(h_slabs_used, g->pool_top, 4, cudaMemcpyDeviceToHost, as_stream(stream)));
  return MK_OK;
}

mk_status mk_graph_last_applied(mk_graph *g, uint64_t *h_count) {
  if (!g || !h_count) return fail(MK_ERR_INVALID, "mk_graph_last_applied: null argument");
  DeviceGuard dg(g->device);
  unsigned long long c = 0;
  MK_CUDA(cudaMemcpy(&c, g->counters, 8, cudaMemcpyDeviceToHost));
  *h_count = c;
  return MK_OK;
}

mk_status mk_graph_last_applied_async(mk_graph *g, uint64_t *h_count, void *stream) {
  if (!g || !h_count) return fail(MK_ERR_INVALID, "mk_graph_last_applied_async: null argument");
  DeviceGuard dg(g->device);
  MK_CUDA(cudaMemcpyAsync(h_count, g->counters, 8, cudaMemcpyDeviceToHost, as_stream(stream)));
  return MK_OK;
}

mk_status mk_graph_last_applied_flags(mk_graph *g, const uint8_t **d_flags,
                                      uint32_t *n) {
  if (!g) return fail(MK_ERR_INVALID, "mk_graph_last_applied_flags: null graph");
  if (d_flags) *d_flags = g->applied.ptr;
  if (n) *n = g->last_n;
  return MK_OK;
}

mk_status mk_graph_degrees(mk_graph *g, uint32_t *d_out, void *stream) {
  if (!g || !d_out) return fail(MK_ERR_INVALID, "mk_graph_degrees: null argument");
  DeviceGuard dg(g->device);
  MK_CUDA(cudaMemcpyAsync(d_out, g->deg, (size_t)g->V * 4, cudaMemcpyDeviceToDevice,
                          as_stream(stream)));
  return MK_OK;
}

mk_status mk_graph_bucket_layout(mk_graph *g, uint32_t *h_offsets,
                                 uint32_t *h_buckets_per_vertex) {
  if (!g) return fail(MK_ERR_INVALID, "mk_graph_bucket_layout: null graph");
  for (uint32_t i = 0; i < g->V; ++i) {
    if (h_offsets) h_offsets[i] = g->h_boff[i];
    if (h_buckets_per_vertex) h_buckets_per_vertex[i] = g->h_boff[i + 1] - g->h_boff[i];
  }
  return MK_OK;
}

mk_status mk_graph_get_info(mk_graph *g, mk_graph_info *out) {
  if (!g || !out) return fail(MK_ERR_INVALID, "mk_graph_get_info: null argument");
  DeviceGuard dg(g->device);
  uint32_t top = 0;
  MK_CUDA(cudaMemcpy(&top, g->pool_top, 4, cudaMemcpyDeviceToHost));
  // live edges: sum of degrees
  uint64_t e = 0;
  MK_CHECK(mk_graph_count_edges_range(g, 0, g->V, nullptr, &e));
  out->num_vertices = g->V;
  out->weighted = g->weighted;
  out->reverse = g->reverse;
  out->keys_per_slab = g->keys_per_slab;
  out->num_buckets = g->num_buckets;
  out->pool_capacity = g->pool_cap;
  out->slabs_used = std::min<uint64_t>(top, g->pool_cap);
  out->num_edges = e;
  out->device_bytes = g->device_bytes;
  return MK_OK;
}

mk_status mk_graph_count_edges_range(mk_graph *g, uint32_t v_begin, uint32_t v_end, void *stream,
                                     uint64_t *h_count) {
  if (!g || !h_count) return fail(MK_ERR_INVALID, "mk_graph_count_edges_range: null argument");
  if (v_begin > v_end || v_end > g->V)
    return fail(MK_ERR_INVALID, "mk_graph_count_edges_range: bad vertex range");
  DeviceGuard dg(g->device);
  cudaStream_t s = as_stream(stream);
  unsigned long long *acc = g->counters + 1;
  MK_CUDA(cudaMemsetAsync(acc, 0, 8, s));
  if (v_end > v_begin) {
    const uint32_t n = v_end - v_begin;
    const int blocks = (int)std::min<uint64_t>((n + 255) / 256, (uint64_t)device_sm_count(g->device) * 8);
    k_sum_degrees<<<blocks, 256, 0, s>>>(g->deg, v_begin, v_end, acc);
    MK_CUDA(cudaGetLastError());
  }
  unsigned long long c = 0;
  MK_CUDA(cudaMemcpyAsync(&c, acc, 8, cudaMemcpyDeviceToHost, s));
  MK_CUDA(cudaStreamSynchronize(s));
  *h_count = c;
  return MK_OK;
}

mk_status mk_graph_export_csr_range(mk_graph *g, uint32_t v_begin, uint32_t v_end,
                                    uint64_t *d_row_ptr, uint32_t *d_col, uint32_t *d_w,
                                    void *stream) {
  if (!g || !d_row_ptr || !d_col)
    return fail(MK_ERR_INVALID, "mk_graph_export_csr_range: null argument");
  if (v_begin >= v_end || v_end > g->V)
    return fail(MK_ERR_INVALID, "mk_graph_export_csr_range: bad vertex range");
  DeviceGuard dg(g->device);
  cudaStream_t s = as_stream(stream);
  const uint32_t b0 = g->h_boff[v_begin];
  const uint32_t nbr = g->h_boff[v_end] - b0;
  MK_CHECK(g->bucket_cnt.reserve(nbr, &g->device_bytes));
  MK_CHECK(g->bucket_pos.reserve((size_t)nbr + 1, &g->device_bytes));
  GraphView v = g->view();
  const int blocks = group_grid(nbr, g->device);
  if (g->weighted)
    k_bucket_live_range<true><<<blocks, 256, 0, s>>>(v, b0, nbr, g->bucket_cnt.ptr);
  else
    k_bucket_live_range<false><<<blocks, 256, 0, s>>>(v, b0, nbr, g->bucket_cnt.ptr);
  MK_CHECK(scan_u32_to_u64(g->bucket_cnt.ptr, g->bucket_pos.ptr, nbr, g->scan_tmp, s));
  const uint32_t nv = v_end - v_begin;
  unsigned long long *rp = reinterpret_cast<unsigned long long *>(d_row_ptr);
  k_rows_from_buckets_range<<<(nv + 256) / 256, 256, 0, s>>>(g->boff, v_begin, nv, b0, nbr,
                                                             g->bucket_pos.ptr, rp);
  if (g->weighted)
    k_bucket_fill_range<true><<<blocks, 256, 0, s>>>(v, b0, nbr, g->bucket_pos.ptr, d_col, d_w);
  else
    k_bucket_fill_range<false><<<blocks, 256, 0, s>>>(v, b0, nbr, g->bucket_pos.ptr, d_col, nullptr);
  MK_CUDA(cudaGetLastError());
  return MK_OK;
}

}  // extern "C"

namespace mk {

mk_status export_csr_grow(mk_graph *g, DevBuf<unsigned long long> &row_ptr, DevBuf<uint32_t> &col,
                          cudaStream_t s, uint64_t *h_edges, size_t *bytes_acc) {
  const uint32_t nb = (uint32_t)g->num_buckets;
  MK_CHECK(g->bucket_cnt.reserve(nb, &g->device_bytes));
  MK_CHECK(g->bucket_pos.reserve((size_t)nb + 1, &g->device_bytes));
  MK_CHECK(row_ptr.reserve((size_t)g->V + 1, bytes_acc));
  GraphView v = g->view();
  const int blocks = group_grid(nb, g->device);
  if (g->weighted)
    k_bucket_live<true><<<blocks, 256, 0, s>>>(v, g->bucket_cnt.ptr);
  else
    k_bucket_live<false><<<blocks, 256, 0, s>>>(v, g->bucket_cnt.ptr);
  MK_CHECK(scan_u32_to_u64(g->bucket_cnt.ptr, g->bucket_pos.ptr, nb, g->scan_tmp, s));
  unsigned long long total = 0;
  MK_CUDA(cudaMemcpyAsync(&total, g->bucket_pos.ptr + nb, 8, cudaMemcpyDeviceToHost, s));
  MK_CUDA(cudaStreamSynchronize(s));
  MK_CHECK(col.reserve(std::max<unsigned long long>(total, 1), bytes_acc));
  k_rows_from_buckets<<<(g->V + 256) / 256, 256, 0, s>>>(g->boff, g->V, nb, g->bucket_pos.ptr, row_ptr.ptr);
  if (g->weighted)
    k_bucket_fill<true><<<blocks, 256, 0, s>>>(v, g->bucket_pos.ptr, col.ptr, nullptr);
  else
    k_bucket_fill<false><<<blocks, 256, 0, s>>>(v, g->bucket_pos.ptr, col.ptr, nullptr);
  MK_CUDA(cudaGetLastError());
  *h_edges = total;
  return MK_OK;
}

}  // namespace mk

extern "C" {

mk_status mk_graph_export_csr(mk_graph *g, uint64_t *d_row_ptr, uint32_t *d_col,
                              uint32_t *d_w, void *stream) {
  if (!g || !d_row_ptr || !d_col) return fail(MK_ERR_INVALID, "mk_graph_export_csr: null argument");
  DeviceGuard dg(g->device);
  cudaStream_t s = as_stream(stream);
  const uint32_t nb = (uint32_t)g->num_buckets;
  MK_CHECK(g->bucket_cnt.reserve(nb, &g->device_bytes));
  MK_CHECK(g->bucket_pos.reserve((size_t)nb + 1, &g->device_bytes));
  GraphView v = g->view();
  int blocks = group_grid(nb, g->device);
  if (g->weighted)
    k_bucket_live<true><<<blocks, 256, 0, s>>>(v, g->bucket_cnt.ptr);
  else
    k_bucket_live<false><<<blocks, 256, 0, s>>>(v, g->bucket_cnt.ptr);
  MK_CHECK(scan_u32_to_u64(g->bucket_cnt.ptr, g->bucket_pos.ptr, nb, g->scan_tmp, s));
  unsigned long long *rp = reinterpret_cast<unsigned long long *>(d_row_ptr);
  k_rows_from_buckets<<<(g->V + 256) / 256, 256, 0, s>>>(g->boff, g->V, nb, g->bucket_pos.ptr, rp);
  if (g->weighted)
    k_bucket_fill<true><<<blocks, 256, 0, s>>>(v, g->bucket_pos.ptr, d_col, d_w);
  else
    k_bucket_fill<false><<<blocks, 256, 0, s>>>(v, g->bucket_pos.ptr, d_col, nullptr);
  MK_CUDA(cudaGetLastError());
  return MK_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// CSR export that allocates nothing.  mk_graph_export_csr keeps its per-bucket
// counts and positions in buffers it grows on demand with cudaMalloc, which
// synchronises the whole device and can fail once the memory is spoken for.
// Callers that must not allocate after start-up -- a serving process that
// handed all free memory to its own pool, or a loop whose concurrent streams
// must not be stalled by an implicit device synchronisation -- use this
// variant instead: its scratch is a fixed file-scope device array, sized for
// graphs of up to kNoAllocMaxBuckets buckets.
// ---------------------------------------------------------------------------
namespace mk {

constexpr uint32_t kNoAllocMaxBuckets = 1u << 18;  // 262,144 buckets
constexpr size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }
constexpr uint32_t kNaMaxTiles = (kNoAllocMaxBuckets + kScanTile - 1) / kScanTile;
constexpr size_t kNaCntOff = 0;  // uint32 live count per bucket
constexpr size_t kNaPosOff = align256(kNaCntOff + (size_t)kNoAllocMaxBuckets * 4);  // uint64[nb + 1]
constexpr size_t kNaTileOff = align256(kNaPosOff + ((size_t)kNoAllocMaxBuckets + 1) * 8);  // uint64 per scan tile
constexpr size_t kNaBytes = align256(kNaTileOff + (size_t)kNaMaxTiles * 8);  // about 3 MiB

// Shared by every call on a device.  Nothing in it has to start at zero:
// each word a call reads was written earlier in the same call.
static __device__ __align__(256) unsigned char g_export_scratch[kNaBytes];

constexpr int kNaMaxDevices = 64;
static std::mutex g_na_mu;
static unsigned char *g_na_ptr[kNaMaxDevices] = {};

// Device address of the scratch array, looked up once per device (the
// calling thread has that device current).
static mk_status export_scratch(int device, unsigned char **out) {
  if (device < 0 || device >= kNaMaxDevices)
    return fail(MK_ERR_INVALID, "mk_graph_export_csr_noalloc: device index out of range");
  std::lock_guard<std::mutex> lock(g_na_mu);
  if (!g_na_ptr[device]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_export_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "mk_graph_export_csr_noalloc: cudaGetSymbolAddress");
    g_na_ptr[device] = static_cast<unsigned char *>(p);
  }
  *out = g_na_ptr[device];
  return MK_OK;
}

}  // namespace mk

extern "C" {

mk_status mk_graph_export_csr_noalloc(mk_graph *g, uint64_t *d_row_ptr, uint32_t *d_col,
                                      uint32_t *d_w, void *stream) {
  if (!g || !d_row_ptr || !d_col)
    return fail(MK_ERR_INVALID, "mk_graph_export_csr_noalloc: null argument");
  if (g->num_buckets > kNoAllocMaxBuckets)
    return fail(MK_ERR_INVALID,
                "mk_graph_export_csr_noalloc: the graph has " + std::to_string(g->num_buckets) +
                    " buckets, more than the " + std::to_string(kNoAllocMaxBuckets) +
                    " its fixed scratch holds; use mk_graph_export_csr");
  DeviceGuard dg(g->device);
  unsigned char *base = nullptr;
  MK_CHECK(export_scratch(g->device, &base));
  uint32_t *cnt = reinterpret_cast<uint32_t *>(base + kNaCntOff);
  unsigned long long *pos = reinterpret_cast<unsigned long long *>(base + kNaPosOff);
  unsigned long long *tiles = reinterpret_cast<unsigned long long *>(base + kNaTileOff);
  cudaStream_t s = as_stream(stream);
  const uint32_t nb = (uint32_t)g->num_buckets;  // >= 1: every vertex owns a bucket
  const uint32_t nt = (nb + kScanTile - 1) / kScanTile;
  GraphView v = g->view();
  const int blocks = group_grid(nb, g->device);
  if (g->weighted)
    k_bucket_live<true><<<blocks, 256, 0, s>>>(v, cnt);
  else
    k_bucket_live<false><<<blocks, 256, 0, s>>>(v, cnt);
  k_scan_tiles<<<nt, kScanBlock, 0, s>>>(cnt, nb, tiles);
  k_scan_sums<<<1, kScanBlock, 0, s>>>(tiles, nt);
  k_scan_apply<<<nt, kScanBlock, 0, s>>>(cnt, nb, tiles, pos);
  unsigned long long *rp = reinterpret_cast<unsigned long long *>(d_row_ptr);
  k_rows_from_buckets<<<(g->V + 256) / 256, 256, 0, s>>>(g->boff, g->V, nb, pos, rp);
  if (g->weighted)
    k_bucket_fill<true><<<blocks, 256, 0, s>>>(v, pos, d_col, d_w);
  else
    k_bucket_fill<false><<<blocks, 256, 0, s>>>(v, pos, d_col, nullptr);
  MK_CUDA(cudaGetLastError());
  return MK_OK;
}

mk_status mk_graph_count_tombstones(mk_graph *g, uint32_t *d_out, void *stream) {
  if (!g || !d_out) return fail(MK_ERR_INVALID, "mk_graph_count_tombstones: null argument");
  DeviceGuard dg(g->device);
  cudaStream_t s = as_stream(stream);
  MK_CUDA(cudaMemsetAsync(d_out, 0, (size_t)g->V * 4, s));
  GraphView v = g->view();
  int blocks = group_grid((uint32_t)g->num_buckets, g->device);
  if (g->weighted)
    k_count_tombstones<true><<<blocks, 256, 0, s>>>(v, d_out);
  else
    k_count_tombstones<false><<<blocks, 256, 0, s>>>(v, d_out);
  MK_CUDA(cudaGetLastError());
  return MK_OK;
}

}  // extern "C"
