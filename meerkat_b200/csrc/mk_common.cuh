// Shared device-side definitions of the slab-hash dynamic graph.
//
// Slab format (128 bytes = 32 x u32 words), kept from the reference's slab
// hash so the per-vertex edge containers read the same way:
//   set slab  (unweighted):  words 0..30 hold keys, word 31 is the next-slab
//                            id  (REGULAR_NODE_KEY_MASK 0x7FFFFFFF,
//                            NEXT_PTR_LANE 31; used at
//                            include/Graph/device/UpdateSlablistPointers.cuh:25-85)
//   map slab  (weighted):    (key, value) pairs in words (2i, 2i+1), i < 15,
//                            word 30 unused, word 31 next (the value sits in
//                            lane+1, include/Algorithms/impl/SSSPImpl.cuh:134)
// Unused key words hold EMPTY (0xFFFFFFFF); a deleted key becomes TOMBSTONE
// (0xFFFFFFFE) and is never reused, so tombstones per vertex after deleting
// every edge equal the original degree (test/GraphTest.cu:958-1007).
//
// B200 layout: all slabs (the per-bucket head slabs first, then the overflow
// pool) live in one 128-byte aligned array addressed by a 32-bit slab id.  A
// group of 8 lanes reads one slab with one 16-byte load per lane, so a warp
// probes 4 slabs per instruction.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace mk {

constexpr uint32_t kEmptyKey = 0xFFFFFFFFu;
constexpr uint32_t kTombKey = 0xFFFFFFFEu;
constexpr uint32_t kNoSlab = 0xFFFFFFFFu;
// Next-slab word while one insert group is linking a new slab (transient,
// only ever seen inside the insert kernel).
constexpr uint32_t kLinkBusy = 0xFFFFFFFEu;
constexpr uint32_t kInf = 0xFFFFFFFFu;
constexpr unsigned long long kInfInf = 0xFFFFFFFFFFFFFFFFull;

constexpr uint32_t kErrInvalidId = 0x1u;
constexpr uint32_t kErrOom = 0x2u;
constexpr uint32_t kErrTimeout = 0x4u;
constexpr uint32_t kErrOverflow = 0x8u;


// Device view of one dynamic graph.  Passed by value to kernels.
struct GraphView {
  uint4 *slabs;           // slab s = slabs[8*s .. 8*s+7]
  const uint32_t *boff;   // bucket offsets, V+1 entries; head slab id = bucket
  const uint32_t *bowner; // owning vertex of each bucket (nbuckets entries)
  uint32_t nbuckets;
  uint32_t *deg;          // live out-degree (in-degree for reverse graphs)
  uint32_t *pool_top;     // next free overflow slab id (bump pointer)
  uint32_t *err;          // sticky MK_DEVERR_* bits
  uint32_t V;
  uint32_t pool_cap;      // total slabs (heads + overflow)
  uint32_t weighted;
  uint32_t reverse;
};

__host__ __device__ __forceinline__ uint32_t pack_hi(unsigned long long x) {
  return static_cast<uint32_t>(x >> 32);
}
__host__ __device__ __forceinline__ uint32_t pack_lo(unsigned long long x) {
  return static_cast<uint32_t>(x & 0xFFFFFFFFull);
}
__host__ __device__ __forceinline__ unsigned long long pack(uint32_t dist,
                                                            uint32_t parent) {
  return (static_cast<unsigned long long>(dist) << 32) | parent;
}

// Integer finaliser (a published 32-bit avalanche mix: xor-shift / multiply
// rounds).  Spreads consecutive vertex ids over the buckets of a vertex.
__host__ __device__ __forceinline__ uint32_t mix32(uint32_t x) {
  x ^= x >> 16;
  x *= 0x7feb352dU;
  x ^= x >> 15;
  x *= 0x846ca68bU;
  x ^= x >> 16;
  return x;
}

// Bucket of `key` among `nb` buckets (multiply-shift range reduction).
__device__ __forceinline__ uint32_t bucket_of(uint32_t key, uint32_t nb) {
  return __umulhi(mix32(key), nb);
}

// Read-only slab load for traversals (graph is not mutated during them).
__device__ __forceinline__ uint4 ld_slab_ro(const uint4 *p) { return __ldg(p); }

// Slab load of a walk (kWritten: in a kernel that wrote slabs earlier in
// the same launch, the one-launch graph-set step).  A walk of a graph no
// kernel phase writes uses the read-only path; otherwise a plain load,
// never the non-coherent one: the grid barrier before the walk (release
// fence, then an acquire load) orders it after every SM's writes and drops
// this SM's stale L1 lines, and a plain load still allocates in L1 (loads
// through L2 only measured 2.5x slower for these walks).
template <bool kWritten>
__device__ __forceinline__ uint4 ld_slab(const uint4 *p) {
  return kWritten ? *p : __ldg(p);
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ uint32_t ld_acquire_u32(const uint32_t *p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ uint32_t ld_relaxed_u32(const uint32_t *p) {
  uint32_t v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Grid-wide barrier for persistent kernels launched cooperatively (all
// blocks co-resident).  bar[0] = arrival count, bar[1] = generation.  The
// wait is bounded by `limit_ns`; on expiry the kernel's error word gets
// kErrTimeout and the barrier returns false so every block can leave.
__device__ __forceinline__ bool grid_barrier(uint32_t *bar, uint32_t *err,
                                             unsigned long long limit_ns) {
  __shared__ uint32_t ok_s;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t ok = 1;
    uint32_t gen = ld_acquire_u32(bar + 1);
    __threadfence();
    uint32_t nblocks = gridDim.x * gridDim.y * gridDim.z;
    uint32_t arrived = atomicAdd(bar, 1u);
    if (arrived == nblocks - 1) {
      atomicExch(bar, 0u);
      __threadfence();
      atomicAdd(bar + 1, 1u);
    } else {
      // the clock is read on every spin, so even a limit of a microsecond
      // is honoured; another block's timeout is noticed within 16 spins
      const unsigned long long t0 = global_ns();
      uint32_t spins = 0;
      while (ld_acquire_u32(bar + 1) == gen) {
        if (global_ns() - t0 > limit_ns) {
          atomicOr(err, kErrTimeout);
          ok = 0;
          break;
        }
        if ((++spins & 15u) == 0 && (ld_relaxed_u32(err) & kErrTimeout)) {
          ok = 0;
          break;
        }
        __nanosleep(32);
      }
    }
    __threadfence();
    ok_s = ok;
  }
  __syncthreads();
  return ok_s != 0;
}

// ---- TMA bulk copies and mbarriers (sm_90+ PTX, used on sm_100a) ----------
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}
// Makes mbarrier initialisation visible to the async (TMA) proxy.
__device__ __forceinline__ void mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait for phase `parity` of an mbarrier; false (and kErrTimeout in
// *err) if it did not complete within `limit` polls.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, uint32_t *err,
                                          uint32_t limit = 1u << 22) {
  for (uint32_t i = 0; i < limit; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  atomicOr(err, kErrTimeout);
  return false;
}
// One bulk copy global -> shared (no multicast), completing on `bar`.
// Addresses 16-byte aligned, size a multiple of 16.
__device__ __forceinline__ void bulk_load(void *dst_smem, const void *src_gmem, uint32_t bytes,
                                          uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_u32(dst_smem)),
      "l"(src_gmem), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
// L2 policies: evict_last for small arrays read on every edge (bucket
// offsets, degrees), evict_first for data streamed once (batch arrays).
__device__ __forceinline__ unsigned long long l2_policy_evict_last() {
  unsigned long long pol;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}
__device__ __forceinline__ unsigned long long l2_policy_evict_first() {
  unsigned long long pol;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}
// Loads issued where they stand (volatile: the compiler keeps their order
// against the other asm, so a prefetch is not sunk to its use).
__device__ __forceinline__ uint32_t ld_hint_u32(const uint32_t *p, unsigned long long pol) {
  uint32_t v;
  asm volatile("ld.global.L2::cache_hint.u32 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ uint32_t ld_stream_u32(const uint32_t *p, unsigned long long pol) {
  uint32_t v;
  asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.u32 %0, [%1], %2;"
               : "=r"(v)
               : "l"(p), "l"(pol));
  return v;
}
// Fire-and-forget add with an L2 policy (degree counters).
__device__ __forceinline__ void red_add_hint_u32(uint32_t *p, uint32_t v, unsigned long long pol) {
  asm volatile("red.global.add.L2::cache_hint.u32 [%0], %1, %2;" ::"l"(p), "r"(v), "l"(pol)
               : "memory");
}
// Orders this thread's earlier generic-proxy shared accesses before later
// async-proxy (TMA) writes to the same buffer.
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Lane bookkeeping for 8-lane slab groups.
struct Lanes {
  uint32_t lane;   // 0..31
  uint32_t gl;     // lane within group 0..7
  uint32_t grp;    // group within warp 0..3
  uint32_t gmask;  // the group's 8 lanes
  uint32_t gbase;  // first lane of the group
};

__device__ __forceinline__ Lanes lanes() {
  Lanes l;
  l.lane = threadIdx.x & 31u;
  l.gl = l.lane & 7u;
  l.grp = l.lane >> 3;
  l.gbase = l.grp << 3;
  l.gmask = 0xFFu << l.gbase;
  return l;
}

}  // namespace mk
