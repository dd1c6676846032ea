// PageRank by pull sweeps over a reverse (in-edge) slab graph.
//
// Reference semantics (include/Algorithms/impl/PageRankImpl.cuh):
//   contribution  c[v] = PR[v] / outdeg[v], 0 for dangling v     (:133-144)
//   update        PR'[u] = (1-d)/N + d * sum_{v in in(u)} c[v]
//                          + d * sum_{outdeg[v]=0} PR[v] / N     (:41-52, :89-115)
//   delta         sum_u |PR'[u] - PR[u]|                          (:117-131)
//   start         PR = 1/N (PageRank.cuh:42-43); dynamic calls warm-start
//                 from the previous ranks after adjusting out-degrees
//                 (PageRankImpl.cuh:222-251).
//
// B200 design: a solve first compacts the reverse graph into CSR (column ids
// in slab order; the graph does not change during a solve), then runs as one
// cooperative launch.  Slab buckets of low-degree vertices are mostly empty
// 128-byte lines, so a pull straight over the slabs reads several times the
// edge bytes and is latency bound; over CSR every iteration streams 4 bytes
// per edge (evict-first, so c[] and the ranks stay in L2) plus 4-byte gathers
// of c[].  An iteration is one pull pass that also writes the next
// contributions and accumulates |delta| and the dangling mass:
//   * vertices of in-degree <= kPrFlat: a warp takes 32 consecutive ones and
//     walks the concatenation of their rows 32 edges per step (coalesced
//     column loads, several steps in flight), a segmented warp scan giving
//     each vertex its share of every step; each warp owns a contiguous run
//     of these 32-vertex groups holding an equal share of the flat edges
//     (a prefix sum per solve, one binary search per warp), so no warp
//     waits at the iteration's barrier for a neighbour with heavier rows;
//   * hubs (in-degree > kPrFlat) are split into work items of kPrChunk
//     in-edges, one warp per item, and combine their item partials in a
//     second, fixed-order pass.
// Item and multi-item lists are built per solve by scans, not atomics.
// Bounded grid barriers separate the passes.  All sums are Kahan-compensated
// FP32 in a fixed order (segmented warp scans, per-lane, warp butterfly,
// per-block tree, per-grid fixed order), so a solve is deterministic for a
// given slab layout.
//
// Stopping rule: `tol` is read as the L1 error target.  The iteration is a
// d-contraction in L1, so after a step with change delta the remaining error
// is at most delta * d / (1 - d); the solve stops once that bound is <= tol/2
// (or after max_iter iterations).  The reference stops at delta <= tol, which
// can leave up to ~5.7 tol of error at d = 0.85.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "mk_internal.h"
#include "mk_slab.cuh"

namespace mk {

struct Kahan {
  float s = 0.f, c = 0.f;
  __device__ __forceinline__ void add(float x) {
    float y = x - c;
    float t = s + y;
    c = (t - s) - y;
    s = t;
  }
  __device__ __forceinline__ void merge(const Kahan &o) {
    add(o.s);
    add(-o.c);
  }
  __device__ __forceinline__ float value() const { return s - c; }
};

__device__ __forceinline__ Kahan shfl_xor_kahan(const Kahan &k, uint32_t mask, int o) {
  Kahan r;
  r.s = __shfl_xor_sync(mask, k.s, o);
  r.c = __shfl_xor_sync(mask, k.c, o);
  return r;
}

enum PrCtl : int { kPBar0 = 0, kPBar1 = 1, kPErr = 2, kPIters = 3, kPCur = 4, kPCtlWords = 8 };

struct PrArgs {
  uint32_t V;
  const unsigned long long *rp;    // V+1 CSR row offsets of the reverse graph
  const uint32_t *col;             // in-neighbours, row by row
  const unsigned long long *ioff;  // V+1: items of vertex u are [ioff[u], ioff[u+1]); ioff[V] = items
  const uint32_t *item_v;          // vertex of each item (items of a vertex are contiguous)
  const unsigned long long *moff;  // V+1: moff[V] = vertices with several items
  const uint32_t *multi;           // those vertices, in increasing id order
  const unsigned long long *gpre;  // ngroups+1: prefix sums of the flat work of the 32-vertex groups
  uint32_t ngroups;
  float *ipart;      // per-item Kahan partials (s, c) = 2 * items
  float *pr0, *pr1;
  float *c0, *c1;
  const uint32_t *outdeg;
  float *part;       // [2 parity][2 kind][2 (s,c)][nblocks]
  float *delta_out;
  uint32_t *ctl;
  float damping;
  float stop_delta;
  uint32_t max_iter;
  uint32_t cur;      // buffer holding the starting ranks
  unsigned long long limit_ns;
};

constexpr int kPrBlock = 256;

// Block reduction of two Kahan accumulators into part[..][blockIdx].
__device__ __forceinline__ void block_reduce2(Kahan a, Kahan b, float *pa, float *pb) {
  __shared__ float sh[4][kPrBlock / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a.merge(shfl_xor_kahan(a, 0xFFFFFFFFu, o));
    b.merge(shfl_xor_kahan(b, 0xFFFFFFFFu, o));
  }
  uint32_t w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) {
    sh[0][w] = a.s;
    sh[1][w] = a.c;
    sh[2][w] = b.s;
    sh[3][w] = b.c;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    Kahan ra, rb;
    for (int i = 0; i < kPrBlock / 32; ++i) {
      Kahan t;
      t.s = sh[0][i];
      t.c = sh[1][i];
      ra.merge(t);
      t.s = sh[2][i];
      t.c = sh[3][i];
      rb.merge(t);
    }
    uint32_t nb = gridDim.x;
    pa[blockIdx.x] = ra.s;
    pa[nb + blockIdx.x] = ra.c;
    pb[blockIdx.x] = rb.s;
    pb[nb + blockIdx.x] = rb.c;
  }
  __syncthreads();
}

// Fixed-order grid reductions of two partial arrays at once (done
// redundantly by every block's warp 0, so every block sees the same values);
// each lane has four blocks' partials in flight at a time.
__device__ __forceinline__ void grid_totals(const float *p, const float *q, float &tp, float &tq) {
  __shared__ float res[2];
  const uint32_t nb = gridDim.x;
  if (threadIdx.x < 32) {
    Kahan kp, kq;
    for (uint32_t i0 = threadIdx.x; i0 < nb; i0 += 128) {
      float ps[4], pc[4], qs[4], qc[4];
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const uint32_t i = i0 + 32u * r;
        const bool ok = i < nb;
        ps[r] = ok ? __ldcg(p + i) : 0.f;
        pc[r] = ok ? __ldcg(p + nb + i) : 0.f;
        qs[r] = ok ? __ldcg(q + i) : 0.f;
        qc[r] = ok ? __ldcg(q + nb + i) : 0.f;
      }
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        if (i0 + 32u * r >= nb) continue;
        Kahan t;
        t.s = ps[r];
        t.c = pc[r];
        kp.merge(t);
        t.s = qs[r];
        t.c = qc[r];
        kq.merge(t);
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      kp.merge(shfl_xor_kahan(kp, 0xFFFFFFFFu, o));
      kq.merge(shfl_xor_kahan(kq, 0xFFFFFFFFu, o));
    }
    if (threadIdx.x == 0) {
      res[0] = kp.value();
      res[1] = kq.value();
    }
  }
  __syncthreads();
  tp = res[0];
  tq = res[1];
  __syncthreads();
}

constexpr uint32_t kPrFlat = 256;   // in-degree up to which the flat pass sums a vertex
constexpr uint32_t kPrChunk = 256;  // in-edges per work item of a hub (in-degree > kPrFlat)
constexpr int kPrSteps = 4;         // 32-edge steps of the flat pass whose loads are in flight together

// Segmented inclusive sum across the warp: lanes with equal keys form
// contiguous runs, and each lane ends with the sum of its run up to itself
// (a fixed tree order).
__device__ __forceinline__ float seg_scan(float v, uint32_t key, uint32_t lane) {
#pragma unroll
  for (int s = 1; s < 32; s <<= 1) {
    const float y = __shfl_up_sync(0xFFFFFFFFu, v, s);
    const uint32_t ky = __shfl_up_sync(0xFFFFFFFFu, key, s);
    if (lane >= (uint32_t)s && ky == key) v += y;
  }
  return v;
}

__global__ void __launch_bounds__(kPrBlock) k_pagerank(PrArgs a) {
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t nthreads = gridDim.x * blockDim.x;
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t wid = tid >> 5, nwarps = nthreads >> 5;
  const uint32_t V = a.V;
  const uint32_t nb = gridDim.x;
  auto pr = [&](uint32_t k) { return k ? a.pr1 : a.pr0; };
  auto cb = [&](uint32_t k) { return k ? a.c1 : a.c0; };
  auto part = [&](uint32_t parity, uint32_t kind) { return a.part + ((parity * 2 + kind) * 2) * nb; };
  uint32_t cur = a.cur;
  const unsigned long long nitems = a.ioff[V], nmulti = a.moff[V];
  // this warp's run of 32-vertex groups: [glo, ghi), an equal share of the
  // flat work (lane 0 searches, the warp shares the result)
  uint32_t glo = 0, ghi = 0;
  if (lane == 0) {
    const unsigned long long total = a.gpre[a.ngroups];
    auto first_at = [&](unsigned long long t) {  // first group g with gpre[g + 1] > t
      uint32_t lo = 0, hi = a.ngroups;
      while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (a.gpre[mid + 1] > t)
          hi = mid;
        else
          lo = mid + 1;
      }
      return lo;
    };
    glo = first_at(total * wid / nwarps);
    ghi = wid + 1 == nwarps ? a.ngroups : first_at(total * (wid + 1) / nwarps);
  }
  glo = __shfl_sync(0xFFFFFFFFu, glo, 0);
  ghi = __shfl_sync(0xFFFFFFFFu, ghi, 0);
  const float d = a.damping;
  const float invV = 1.0f / (float)V;

  // prologue: contributions and dangling mass of the starting ranks
  {
    Kahan dang, zero;
    for (uint32_t u = tid; u < V; u += nthreads) {
      uint32_t od = a.outdeg[u];
      float p = pr(cur)[u];
      cb(cur)[u] = od ? p / (float)od : 0.0f;
      if (!od) dang.add(p);
    }
    block_reduce2(dang, zero, part(0, 0), part(0, 1));
    if (!grid_barrier(a.ctl + kPBar0, a.ctl + kPErr, a.limit_ns)) return;
  }
  uint32_t it = 0;
  float delta = 0.f, dangling = 0.f, unused = 0.f;
  grid_totals(part(0, 0), part(0, 1), dangling, unused);
  while (it < a.max_iter) {
    const uint32_t rp = it & 1u, wp = rp ^ 1u;
    const float base = (1.0f - d) * invV + d * (dangling * invV);
    const float *c = cb(cur);
    const float *pold = pr(cur);
    float *pnew = pr(cur ^ 1);
    float *cnew = cb(cur ^ 1);
    Kahan kd, kdang;
    auto finalize = [&](uint32_t u, float sum) {
      float nv = base + d * sum;
      pnew[u] = nv;
      kd.add(fabsf(nv - __ldcg(pold + u)));
      uint32_t od = a.outdeg[u];
      cnew[u] = od ? nv / (float)od : 0.0f;
      if (!od) kdang.add(nv);
    };
    // pass A, flat: a warp takes 32 consecutive vertices and walks the
    // concatenation of their in-edge rows (hubs excluded) 32 edges per step,
    // kPrSteps steps with their loads in flight together; a segmented scan
    // hands every vertex the sum of its part of each step
    for (uint32_t grp = glo; grp < ghi; ++grp) {
      const uint32_t u = grp * 32u + lane;
      unsigned long long j0 = 0;
      uint32_t dl = 0;
      bool mine = false;
      if (u < V) {
        j0 = a.rp[u];
        const unsigned long long dd = a.rp[u + 1] - j0;
        mine = dd <= kPrFlat;
        dl = mine ? (uint32_t)dd : 0u;
      }
      uint32_t incl = dl;
#pragma unroll
      for (int s2 = 1; s2 < 32; s2 <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, s2);
        if (lane >= (uint32_t)s2) incl += y;
      }
      const uint32_t off = incl - dl;
      const uint32_t T = __shfl_sync(0xFFFFFFFFu, incl, 31);
      const unsigned long long basej = j0 - off;  // edge x of the run of lane l is col[basej(l) + x]
      Kahan acc;
      for (uint32_t t0 = 0; t0 < T; t0 += 32u * kPrSteps) {
        uint32_t own[kPrSteps], kc[kPrSteps];
        float val[kPrSteps];
#pragma unroll
        for (int q = 0; q < kPrSteps; ++q) {
          const uint32_t x = t0 + 32u * q + lane;
          uint32_t lo = 0;  // last lane whose run starts at or before x
#pragma unroll
          for (int st = 16; st > 0; st >>= 1) {
            const uint32_t cand = lo + (uint32_t)st;
            if (__shfl_sync(0xFFFFFFFFu, off, cand) <= x) lo = cand;
          }
          const unsigned long long bj = __shfl_sync(0xFFFFFFFFu, basej, lo);
          own[q] = x < T ? lo : 32u;
          kc[q] = x < T ? __ldcs(a.col + (bj + x)) : 0u;
        }
#pragma unroll
        for (int q = 0; q < kPrSteps; ++q) val[q] = own[q] < 32u ? __ldca(c + kc[q]) : 0.0f;
#pragma unroll
        for (int q = 0; q < kPrSteps; ++q) {
          const float sv = seg_scan(val[q], own[q], lane);
          const uint32_t sb = t0 + 32u * q;
          const bool hit = dl && off < sb + 32u && off + dl > sb;
          const uint32_t last = hit ? min(off + dl, sb + 32u) - 1u - sb : 0u;
          const float tot = __shfl_sync(0xFFFFFFFFu, sv, last);
          if (hit) acc.add(tot);
        }
      }
      if (mine) finalize(u, acc.value());
    }
    // pass A, hubs: one warp per work item of kPrChunk in-edges
    for (unsigned long long i = wid; i < nitems; i += nwarps) {
      const uint32_t u = a.item_v[i];
      const unsigned long long j0 = a.rp[u] + (i - a.ioff[u]) * kPrChunk;
      const unsigned long long j1 = min(j0 + kPrChunk, a.rp[u + 1]);
      constexpr int kPer = (int)(kPrChunk / 32);
      uint32_t kc[kPer];
      float x[kPer];
#pragma unroll
      for (int q = 0; q < kPer; ++q) {
        const unsigned long long j = j0 + 32u * q + lane;
        kc[q] = j < j1 ? __ldcs(a.col + j) : 0u;
      }
#pragma unroll
      for (int q = 0; q < kPer; ++q) x[q] = (j0 + 32u * q + lane < j1) ? __ldca(c + kc[q]) : 0.0f;
      Kahan acc;
#pragma unroll
      for (int q = 0; q < kPer; ++q)
        if (j0 + 32u * q + lane < j1) acc.add(x[q]);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) acc.merge(shfl_xor_kahan(acc, 0xFFFFFFFFu, o));
      if (lane == 0) {
        a.ipart[2 * i] = acc.s;
        a.ipart[2 * i + 1] = acc.c;
      }
    }
    if (nmulti) {
      if (!grid_barrier(a.ctl + kPBar0, a.ctl + kPErr, a.limit_ns)) return;
      // pass B: every hub combines its item partials in order
      for (unsigned long long m = wid; m < nmulti; m += nwarps) {
        const uint32_t u = a.multi[m];
        const unsigned long long i0 = a.ioff[u], i1 = a.ioff[u + 1];
        Kahan acc;
        for (unsigned long long i = i0 + lane; i < i1; i += 32) {
          Kahan t;
          t.s = __ldcg(a.ipart + 2 * i);
          t.c = __ldcg(a.ipart + 2 * i + 1);
          acc.merge(t);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc.merge(shfl_xor_kahan(acc, 0xFFFFFFFFu, o));
        if (lane == 0) finalize(u, acc.value());
      }
    }
    block_reduce2(kdang, kd, part(wp, 0), part(wp, 1));
    if (!grid_barrier(a.ctl + kPBar0, a.ctl + kPErr, a.limit_ns)) return;
    // this iteration's |delta| and the next one's dangling mass in one pass
    grid_totals(part(wp, 1), part(wp, 0), delta, dangling);
    cur ^= 1u;
    ++it;
    if (delta <= a.stop_delta) break;
  }
  if (tid == 0) {
    a.ctl[kPIters] = it;
    a.ctl[kPCur] = cur;
    *a.delta_out = delta;
  }
}

// out-degree +-1 for every batch edge the last graph update applied
__global__ void k_outdeg_adjust(const uint32_t *__restrict__ src, const uint8_t *__restrict__ applied,
                                uint32_t n, uint32_t *outdeg, int sign) {
  uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e < n && applied[e]) atomicAdd(outdeg + src[e], (uint32_t)sign);
}

// out-degree from scratch: count every key of the reverse graph (one group
// per bucket, balanced whatever the degree skew)
template <bool kW>
__global__ void k_outdeg_count(GraphView g, uint32_t *outdeg) {
  const Lanes L = lanes();
  const uint32_t group = (blockIdx.x * blockDim.x + threadIdx.x) >> 3;
  const uint32_t ngroups = (gridDim.x * blockDim.x) >> 3;
  for (uint32_t b = group; b < g.nbuckets; b += ngroups) {
    walk_bucket(g, L, b, [&](const uint4 &q) {
      uint32_t k[4], w[4];
      lane_keys<kW>(q, L.gl, k, w);
#pragma unroll
      for (int i = 0; i < keys_per_lane<kW>(); ++i)
        if (k[i] < kTombKey) atomicAdd(outdeg + k[i], 1u);
    });
  }
}

// work items per vertex: ceil(in-degree / kPrChunk) for a hub (in-degree
// above kPrFlat, so at least two items), else 0; flag = hub
__global__ void k_pr_item_counts(const unsigned long long *__restrict__ rp, uint32_t V,
                                 uint32_t *__restrict__ cnt, uint32_t *__restrict__ mflag) {
  for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < V; u += gridDim.x * blockDim.x) {
    const unsigned long long d = rp[u + 1] - rp[u];
    const uint32_t c = d > kPrFlat ? (uint32_t)((d + kPrChunk - 1) / kPrChunk) : 0u;
    cnt[u] = c;
    mflag[u] = c > 1 ? 1u : 0u;
  }
}

// flat work of each 32-vertex group: in-edges of its vertices of in-degree
// <= kPrFlat, plus 2 per vertex for the per-vertex finish
__global__ void k_pr_group_counts(const unsigned long long *__restrict__ rp, uint32_t V,
                                  uint32_t *__restrict__ gcnt) {
  const uint32_t G = (V + 31) / 32;
  for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < G; g += gridDim.x * blockDim.x) {
    uint32_t c = 0;
    const uint32_t u1 = min(V, g * 32u + 32u);
    for (uint32_t u = g * 32u; u < u1; ++u) {
      const unsigned long long d = rp[u + 1] - rp[u];
      c += (d <= kPrFlat ? (uint32_t)d : 0u) + 2u;
    }
    gcnt[g] = c;
  }
}

__global__ void k_pr_item_fill(const uint32_t *__restrict__ cnt, const unsigned long long *__restrict__ ioff,
                               const unsigned long long *__restrict__ moff, uint32_t V,
                               uint32_t *__restrict__ item_v, uint32_t *__restrict__ multi) {
  for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < V; u += gridDim.x * blockDim.x) {
    const uint32_t c = cnt[u];
    if (!c) continue;
    const unsigned long long o = ioff[u];
    for (uint32_t j = 0; j < c; ++j) item_v[o + j] = u;
    if (c > 1) multi[moff[u]] = u;
  }
}

__global__ void k_fill(float *p, uint32_t n, float v) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i] = v;
}

}  // namespace mk

using namespace mk;

struct mk_pagerank {
  mk_graph *g = nullptr;
  float damping = 0.85f, tol = 1e-6f;
  uint32_t max_iter = 100;
  float *pr0 = nullptr, *pr1 = nullptr, *c0 = nullptr, *c1 = nullptr;
  uint32_t *outdeg = nullptr;
  float *part = nullptr;
  float *delta = nullptr;
  // per-solve CSR of the reverse graph and its work items
  DevBuf<unsigned long long> rp, ioff, moff, gpre, scan_tmp;
  DevBuf<uint32_t> col, cnt, mflag, item_v, multi, gcnt;
  DevBuf<float> ipart;
  uint32_t *ctl = nullptr;
  uint32_t cur = 0;  // host mirror of the buffer with the latest ranks
  int nblocks = 0;
  Timer timer;
};

static mk_status pr_recount_outdeg(mk_pagerank *p, cudaStream_t s) {
  mk_graph *g = p->g;
  MK_CUDA(cudaMemsetAsync(p->outdeg, 0, (size_t)g->V * 4, s));
  int blocks = std::min<uint64_t>(g->num_buckets * 8 / 256 + 1, (uint64_t)device_sm_count(g->device) * 8);
  if (g->weighted)
    k_outdeg_count<true><<<blocks, 256, 0, s>>>(g->view(), p->outdeg);
  else
    k_outdeg_count<false><<<blocks, 256, 0, s>>>(g->view(), p->outdeg);
  MK_CUDA(cudaGetLastError());
  return MK_OK;
}

// CSR of the reverse graph and the work items of this solve.
static mk_status pr_prepare(mk_pagerank *p, cudaStream_t s) {
  mk_graph *g = p->g;
  const uint32_t V = g->V;
  uint64_t E = 0;
  MK_CHECK(export_csr_grow(g, p->rp, p->col, s, &E, nullptr));
  MK_CHECK(p->cnt.reserve(V));
  MK_CHECK(p->mflag.reserve(V));
  MK_CHECK(p->ioff.reserve((size_t)V + 1));
  MK_CHECK(p->moff.reserve((size_t)V + 1));
  // a vertex with items has more than kPrFlat in-edges, and
  // ceil(d / kPrChunk) <= d / kPrChunk + 1
  const size_t heavy_cap = E / (kPrFlat + 1) + 1;
  const size_t item_cap = E / kPrChunk + heavy_cap;
  MK_CHECK(p->item_v.reserve(item_cap));
  MK_CHECK(p->multi.reserve(heavy_cap));
  MK_CHECK(p->ipart.reserve(2 * item_cap));
  const int fb = (int)std::min<uint64_t>((uint64_t)V / 256 + 1, (uint64_t)device_sm_count(g->device) * 8);
  k_pr_item_counts<<<fb, 256, 0, s>>>(p->rp.ptr, V, p->cnt.ptr, p->mflag.ptr);
  MK_CHECK(scan_u32_to_u64(p->cnt.ptr, p->ioff.ptr, V, p->scan_tmp, s));
  MK_CHECK(scan_u32_to_u64(p->mflag.ptr, p->moff.ptr, V, p->scan_tmp, s));
  k_pr_item_fill<<<fb, 256, 0, s>>>(p->cnt.ptr, p->ioff.ptr, p->moff.ptr, V, p->item_v.ptr, p->multi.ptr);
  const uint32_t G = (V + 31) / 32;
  MK_CHECK(p->gcnt.reserve(G));
  MK_CHECK(p->gpre.reserve((size_t)G + 1));
  k_pr_group_counts<<<(int)std::min<uint64_t>(G / 256 + 1, (uint64_t)device_sm_count(g->device) * 8), 256, 0, s>>>(
      p->rp.ptr, V, p->gcnt.ptr);
  MK_CHECK(scan_u32_to_u64(p->gcnt.ptr, p->gpre.ptr, G, p->scan_tmp, s));
  MK_CUDA(cudaGetLastError());
  return MK_OK;
}

// Grid size of the persistent solve and its per-block partial sums.  The
// occupancy query loads the kernel's module; create does this once, so no
// solve pays for it inside its timed window.
static mk_status pr_setup_launch(mk_pagerank *p) {
  if (p->nblocks) return MK_OK;
  const int nb = persistent_blocks((const void *)k_pagerank, kPrBlock, 0, p->g->device);
  cudaError_t e = cudaMalloc(&p->part, (size_t)nb * 8 * sizeof(float));
  if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(pagerank partials)");
  p->nblocks = nb;
  return MK_OK;
}

static mk_status pr_solve(mk_pagerank *p, cudaStream_t s) {
  mk_graph *g = p->g;
  MK_CHECK(pr_prepare(p, s));
  const void *fn = (const void *)k_pagerank;
  MK_CHECK(pr_setup_launch(p));
  MK_CUDA(cudaMemsetAsync(p->ctl, 0, kPCtlWords * 4, s));
  PrArgs a;
  a.V = g->V;
  a.rp = p->rp.ptr;
  a.col = p->col.ptr;
  a.ioff = p->ioff.ptr;
  a.item_v = p->item_v.ptr;
  a.moff = p->moff.ptr;
  a.multi = p->multi.ptr;
  a.gpre = p->gpre.ptr;
  a.ngroups = (g->V + 31) / 32;
  a.ipart = p->ipart.ptr;
  a.pr0 = p->pr0;
  a.pr1 = p->pr1;
  a.c0 = p->c0;
  a.c1 = p->c1;
  a.outdeg = p->outdeg;
  a.part = p->part;
  a.delta_out = p->delta;
  a.ctl = p->ctl;
  a.damping = p->damping;
  a.stop_delta = p->tol * 0.5f * (1.0f - p->damping) / p->damping;
  a.max_iter = p->max_iter;
  a.cur = p->cur;
  a.limit_ns = g->wait_limit_ns();
  void *args[] = {&a};
  MK_CUDA(cudaLaunchCooperativeKernel(fn, dim3(p->nblocks), dim3(kPrBlock), args, 0, s));
  // the solve waits for its launch: the buffer holding the final ranks and
  // the error word of the bounded grid barriers come back here
  uint32_t ctl[kPCtlWords];
  MK_CUDA(cudaMemcpyAsync(ctl, p->ctl, sizeof(ctl), cudaMemcpyDeviceToHost, s));
  MK_CUDA(cudaStreamSynchronize(s));
  if (ctl[kPErr] & kErrTimeout) {  // the ranks of this solve are undefined
    p->cur = 0;
    return fail(MK_ERR_TIMEOUT, "pagerank: grid barrier timed out");
  }
  p->cur = ctl[kPCur];
  return MK_OK;
}

extern "C" {

mk_status mk_pagerank_create(mk_graph *g_rev, float damping, float tol,
                             uint32_t max_iter, const uint32_t *h_out_degree,
                             mk_pagerank **out) {
  if (!g_rev || !out) return fail(MK_ERR_INVALID, "mk_pagerank_create: null argument");
  *out = nullptr;
  if (!(damping > 0.f && damping < 1.f)) return fail(MK_ERR_INVALID, "mk_pagerank_create: damping must be in (0,1)");
  if (!(tol > 0.f)) return fail(MK_ERR_INVALID, "mk_pagerank_create: tol must be > 0");
  DeviceGuard dg(g_rev->device);
  mk_pagerank *p = new mk_pagerank();
  p->g = g_rev;
  p->damping = damping;
  p->tol = tol;
  p->max_iter = max_iter;
  const size_t V = g_rev->V;
  cudaError_t e = cudaSuccess;
  auto A = [&](void **ptr, size_t bytes) {
    if (e == cudaSuccess) e = cudaMalloc(ptr, bytes);
  };
  A((void **)&p->pr0, V * 4);
  A((void **)&p->pr1, V * 4);
  A((void **)&p->c0, V * 4);
  A((void **)&p->c1, V * 4);
  A((void **)&p->outdeg, V * 4);
  A((void **)&p->delta, 4);
  A((void **)&p->ctl, kPCtlWords * 4);
  if (e != cudaSuccess) {
    mk_pagerank_destroy(p);
    return cuda_fail(e, "mk_pagerank_create");
  }
  k_fill<<<256, 256>>>(p->pr0, (uint32_t)V, 1.0f / (float)V);
  if (h_out_degree) {
    e = cudaMemcpy(p->outdeg, h_out_degree, V * 4, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      mk_pagerank_destroy(p);
      return cuda_fail(e, "mk_pagerank_create: out-degree copy");
    }
  } else {
    mk_status st = pr_recount_outdeg(p, nullptr);
    if (st != MK_OK) {
      mk_pagerank_destroy(p);
      return st;
    }
  }
  e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    mk_pagerank_destroy(p);
    return cuda_fail(e, "mk_pagerank_create");
  }
  // Size every per-solve buffer for the graph as it is now and set up the
  // launch, so the first solve allocates nothing and loads no module (its
  // timed window holds only the solve; later solves grow the buffers only
  // if the graph grows past them).
  mk_status st = pr_prepare(p, nullptr);
  if (st == MK_OK) st = pr_setup_launch(p);
  if (st == MK_OK) {
    e = cudaDeviceSynchronize();
    if (e != cudaSuccess) st = cuda_fail(e, "mk_pagerank_create");
  }
  if (st != MK_OK) {
    mk_pagerank_destroy(p);
    return st;
  }
  *out = p;
  return MK_OK;
}

mk_status mk_pagerank_static(mk_pagerank *p, void *stream, float *ms_out) {
  if (!p) return fail(MK_ERR_INVALID, "mk_pagerank_static: null handle");
  DeviceGuard dg(p->g->device);
  cudaStream_t s = as_stream(stream);
  MK_CHECK(p->timer.start(s, ms_out != nullptr));
  p->cur = 0;
  k_fill<<<256, 256, 0, s>>>(p->pr0, p->g->V, 1.0f / (float)p->g->V);
  MK_CHECK(pr_solve(p, s));
  return p->timer.stop(ms_out);
}

mk_status mk_pagerank_static_recount(mk_pagerank *p, void *stream, float *ms_out) {
  if (!p) return fail(MK_ERR_INVALID, "mk_pagerank_static_recount: null handle");
  DeviceGuard dg(p->g->device);
  cudaStream_t s = as_stream(stream);
  MK_CHECK(p->timer.start(s, ms_out != nullptr));
  MK_CHECK(pr_recount_outdeg(p, s));
  p->cur = 0;
  k_fill<<<256, 256, 0, s>>>(p->pr0, p->g->V, 1.0f / (float)p->g->V);
  MK_CHECK(pr_solve(p, s));
  return p->timer.stop(ms_out);
}

static mk_status pr_dynamic(mk_pagerank *p, const uint32_t *d_src, const uint32_t *d_dst,
                            uint32_t n, bool inc, void *stream, float *ms_out) {
  if (!p) return fail(MK_ERR_INVALID, "pagerank dynamic: null handle");
  mk_graph *g = p->g;
  DeviceGuard dg(g->device);
  cudaStream_t s = as_stream(stream);
  MK_CHECK(p->timer.start(s, ms_out != nullptr));
  const bool matches = n == g->last_n && d_src == g->last_src && d_dst == g->last_dst &&
                       g->last_op == (inc ? 1 : 2);
  if (n) {
    if (matches) {
      k_outdeg_adjust<<<(n + 255) / 256, 256, 0, s>>>(d_src, g->applied.ptr, n, p->outdeg, inc ? 1 : -1);
      MK_CUDA(cudaGetLastError());
    } else {
      MK_CHECK(pr_recount_outdeg(p, s));
    }
  }
  MK_CHECK(pr_solve(p, s));
  return p->timer.stop(ms_out);
}

mk_status mk_pagerank_incremental(mk_pagerank *p, const uint32_t *d_src,
                                  const uint32_t *d_dst, uint32_t n, void *stream,
                                  float *ms_out) {
  return pr_dynamic(p, d_src, d_dst, n, true, stream, ms_out);
}

mk_status mk_pagerank_decremental(mk_pagerank *p, const uint32_t *d_src,
                                  const uint32_t *d_dst, uint32_t n, void *stream,
                                  float *ms_out) {
  return pr_dynamic(p, d_src, d_dst, n, false, stream, ms_out);
}

mk_status mk_pagerank_values(mk_pagerank *p, float *h_out) {
  if (!p || !h_out) return fail(MK_ERR_INVALID, "mk_pagerank_values: null argument");
  DeviceGuard dg(p->g->device);
  MK_CUDA(cudaDeviceSynchronize());
  uint32_t err = 0;
  MK_CUDA(cudaMemcpy(&err, p->ctl + kPErr, 4, cudaMemcpyDeviceToHost));
  MK_CUDA(cudaMemcpy(h_out, p->cur ? p->pr1 : p->pr0, (size_t)p->g->V * 4, cudaMemcpyDeviceToHost));
  if (err & kErrTimeout) return fail(MK_ERR_TIMEOUT, "pagerank: grid barrier timed out");
  return MK_OK;
}

mk_status mk_pagerank_values_device(mk_pagerank *p, const float **d_values) {
  if (!p || !d_values) return fail(MK_ERR_INVALID, "mk_pagerank_values_device: null argument");
  *d_values = p->cur ? p->pr1 : p->pr0;
  return MK_OK;
}

mk_status mk_pagerank_stats(mk_pagerank *p, uint32_t *h_iters, float *h_delta) {
  if (!p) return fail(MK_ERR_INVALID, "mk_pagerank_stats: null handle");
  DeviceGuard dg(p->g->device);
  MK_CUDA(cudaDeviceSynchronize());
  uint32_t ctl[kPCtlWords];
  float dl = 0.f;
  MK_CUDA(cudaMemcpy(ctl, p->ctl, sizeof(ctl), cudaMemcpyDeviceToHost));
  MK_CUDA(cudaMemcpy(&dl, p->delta, 4, cudaMemcpyDeviceToHost));
  if (h_iters) *h_iters = ctl[kPIters];
  if (h_delta) *h_delta = dl;
  return MK_OK;
}

mk_status mk_pagerank_destroy(mk_pagerank *p) {
  if (!p) return MK_OK;
  DeviceGuard dg(p->g->device);
  cudaFree(p->pr0);
  cudaFree(p->pr1);
  cudaFree(p->c0);
  cudaFree(p->c1);
  cudaFree(p->outdeg);
  cudaFree(p->part);
  cudaFree(p->delta);
  cudaFree(p->ctl);
  p->rp.release();
  p->ioff.release();
  p->moff.release();
  p->scan_tmp.release();
  p->col.release();
  p->cnt.release();
  p->mflag.release();
  p->item_v.release();
  p->multi.release();
  p->gcnt.release();
  p->gpre.release();
  p->ipart.release();
  delete p;
  return MK_OK;
}

}  // extern "C"
