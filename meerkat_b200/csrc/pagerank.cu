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
// B200 design: the whole solve is one cooperative launch.  Each iteration
// is one pull pass over fixed work items (chunks of up to 32 buckets of one
// vertex, 8-lane group per item, 16-byte slab loads, 4-byte gathers of c[]
// which stays L2 resident) that also writes the next contributions and
// accumulates |delta| and the dangling mass.  A vertex with one item is
// finished in that pass; hubs with several items combine the item partials
// in a second, fixed-order pass.  Bounded grid barriers separate the passes.  All sums are Kahan-compensated FP32 in
// a fixed order (per-lane, 8-lane butterfly, per-block tree, per-grid fixed
// order), so a solve is deterministic for a given slab layout.
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
  GraphView g;       // reverse graph
  const uint32_t *item_b0;   // first bucket of each work item (items of a vertex are contiguous)
  const uint32_t *item_off;  // V+1: items of vertex u are [item_off[u], item_off[u+1])
  const uint32_t *multi;     // vertices with more than one item
  uint32_t nitems;
  uint32_t nmulti;
  float *ipart;      // per-item Kahan partials (s, c) = 2 * nitems
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

// Fixed-order grid reduction of one partial array (done redundantly by every
// block's warp 0, so every block sees the same value).
__device__ __forceinline__ float grid_total(const float *p) {
  __shared__ float res;
  uint32_t nb = gridDim.x;
  if (threadIdx.x < 32) {
    Kahan k;
    for (uint32_t i = threadIdx.x; i < nb; i += 32) {
      Kahan t;
      t.s = __ldcg(p + i);
      t.c = __ldcg(p + nb + i);
      k.merge(t);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) k.merge(shfl_xor_kahan(k, 0xFFFFFFFFu, o));
    if (threadIdx.x == 0) res = k.value();
  }
  __syncthreads();
  float r = res;
  __syncthreads();
  return r;
}

constexpr uint32_t kPrChunk = 32;  // buckets per work item

// Kahan sum of contributions over buckets [b0, b1) (group-cooperative).
template <bool kW>
__device__ __forceinline__ Kahan pull_range(const GraphView &g, const Lanes &L, uint32_t b0,
                                            uint32_t b1, const float *__restrict__ c) {
  Kahan acc;
  walk_buckets(g, L, b0, b1, [&](const uint4 &q) {
    uint32_t k[4], w[4];
    lane_keys<kW>(q, L.gl, k, w);
#pragma unroll
    for (int i = 0; i < keys_per_lane<kW>(); ++i)
      if (k[i] < kTombKey) acc.add(__ldcg(c + k[i]));  // c is rewritten every iteration
  });
#pragma unroll
  for (int o = 4; o > 0; o >>= 1) acc.merge(shfl_xor_kahan(acc, L.gmask, o));
  return acc;
}

template <bool kW>
__global__ void __launch_bounds__(kPrBlock) k_pagerank(PrArgs a) {
  const Lanes L = lanes();
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t nthreads = gridDim.x * blockDim.x;
  const uint32_t group = tid >> 3;
  const uint32_t ngroups = nthreads >> 3;
  const uint32_t V = a.g.V;
  const uint32_t nb = gridDim.x;
  float *pr[2] = {a.pr0, a.pr1};
  float *cb[2] = {a.c0, a.c1};
  auto part = [&](uint32_t parity, uint32_t kind) { return a.part + ((parity * 2 + kind) * 2) * nb; };
  uint32_t cur = a.cur;
  const float d = a.damping;
  const float invV = 1.0f / (float)V;

  // prologue: contributions and dangling mass of the starting ranks
  {
    Kahan dang, zero;
    for (uint32_t u = tid; u < V; u += nthreads) {
      uint32_t od = a.outdeg[u];
      float p = pr[cur][u];
      cb[cur][u] = od ? p / (float)od : 0.0f;
      if (!od) dang.add(p);
    }
    block_reduce2(dang, zero, part(0, 0), part(0, 1));
    if (!grid_barrier(a.ctl + kPBar0, a.ctl + kPErr, a.limit_ns)) return;
  }
  uint32_t it = 0;
  float delta = 0.f;
  while (it < a.max_iter) {
    const uint32_t rp = it & 1u, wp = rp ^ 1u;
    const float dangling = grid_total(part(rp, 0));
    const float base = (1.0f - d) * invV + d * (dangling * invV);
    const float *c = cb[cur];
    const float *pold = pr[cur];
    float *pnew = pr[cur ^ 1];
    float *cnew = cb[cur ^ 1];
    Kahan kd, kdang;
    auto finalize = [&](uint32_t u, float sum) {  // lane 0 of a group
      float nv = base + d * sum;
      pnew[u] = nv;
      kd.add(fabsf(nv - __ldcg(pold + u)));
      uint32_t od = a.outdeg[u];
      cnew[u] = od ? nv / (float)od : 0.0f;
      if (!od) kdang.add(nv);
    };
    // pass A: every work item; a vertex with a single item is finished here
    for (uint32_t i = group; i < a.nitems; i += ngroups) {
      const uint32_t b0 = a.item_b0[i];
      const uint32_t u = a.g.bowner[b0];
      const uint32_t b1 = min(a.g.boff[u + 1], b0 + kPrChunk);
      Kahan acc = pull_range<kW>(a.g, L, b0, b1, c);
      if (L.gl == 0) {
        if (a.item_off[u + 1] - a.item_off[u] == 1) {
          finalize(u, acc.value());
        } else {
          a.ipart[2 * i] = acc.s;
          a.ipart[2 * i + 1] = acc.c;
        }
      }
    }
    if (a.nmulti) {
      if (!grid_barrier(a.ctl + kPBar0, a.ctl + kPErr, a.limit_ns)) return;
      // pass B: vertices with several items combine their partials in order
      for (uint32_t m = group; m < a.nmulti; m += ngroups) {
        const uint32_t u = a.multi[m];
        const uint32_t i0 = a.item_off[u], i1 = a.item_off[u + 1];
        Kahan acc;
        for (uint32_t i = i0 + L.gl; i < i1; i += 8) {
          Kahan t;
          t.s = __ldcg(a.ipart + 2 * i);
          t.c = __ldcg(a.ipart + 2 * i + 1);
          acc.merge(t);
        }
#pragma unroll
        for (int o = 4; o > 0; o >>= 1) acc.merge(shfl_xor_kahan(acc, L.gmask, o));
        if (L.gl == 0) finalize(u, acc.value());
      }
    }
    block_reduce2(kdang, kd, part(wp, 0), part(wp, 1));
    if (!grid_barrier(a.ctl + kPBar0, a.ctl + kPErr, a.limit_ns)) return;
    delta = grid_total(part(wp, 1));
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
  uint32_t *item_b0 = nullptr, *item_off = nullptr, *multi = nullptr;
  float *ipart = nullptr;
  uint32_t nitems = 0, nmulti = 0;
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

static mk_status pr_solve(mk_pagerank *p, cudaStream_t s) {
  mk_graph *g = p->g;
  const void *fn = g->weighted ? (const void *)k_pagerank<true> : (const void *)k_pagerank<false>;
  if (p->nblocks == 0) {
    p->nblocks = persistent_blocks(fn, kPrBlock, 0, g->device);
    cudaError_t e = cudaMalloc(&p->part, (size_t)p->nblocks * 8 * sizeof(float));
    if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(pagerank partials)");
  }
  MK_CUDA(cudaMemsetAsync(p->ctl, 0, kPCtlWords * 4, s));
  PrArgs a;
  a.g = g->view();
  a.item_b0 = p->item_b0;
  a.item_off = p->item_off;
  a.multi = p->multi;
  a.nitems = p->nitems;
  a.nmulti = p->nmulti;
  a.ipart = p->ipart;
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
  a.limit_ns = 4000000000ull;
  void *args[] = {&a};
  MK_CUDA(cudaLaunchCooperativeKernel(fn, dim3(p->nblocks), dim3(kPrBlock), args, 0, s));
  // the final buffer index is read back lazily (values / next solve)
  uint32_t curv = 0;
  MK_CUDA(cudaMemcpyAsync(&curv, p->ctl + kPCur, 4, cudaMemcpyDeviceToHost, s));
  MK_CUDA(cudaStreamSynchronize(s));
  p->cur = curv;
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
  // fixed work items: chunks of kPrChunk buckets, contiguous per vertex
  std::vector<uint32_t> ib0, ioff(V + 1), mul;
  for (uint32_t u = 0; u < V; ++u) {
    ioff[u] = (uint32_t)ib0.size();
    const uint32_t lo = g_rev->h_boff[u], hi = g_rev->h_boff[u + 1];
    for (uint32_t b = lo; b < hi; b += kPrChunk) ib0.push_back(b);
    if (hi - lo > kPrChunk) mul.push_back(u);
  }
  ioff[V] = (uint32_t)ib0.size();
  p->nitems = (uint32_t)ib0.size();
  p->nmulti = (uint32_t)mul.size();
  A((void **)&p->item_b0, ib0.size() * 4);
  A((void **)&p->item_off, ioff.size() * 4);
  A((void **)&p->multi, std::max<size_t>(mul.size(), 1) * 4);
  A((void **)&p->ipart, ib0.size() * 8);
  if (e == cudaSuccess) e = cudaMemcpy(p->item_b0, ib0.data(), ib0.size() * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(p->item_off, ioff.data(), ioff.size() * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && !mul.empty()) e = cudaMemcpy(p->multi, mul.data(), mul.size() * 4, cudaMemcpyHostToDevice);
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
  cudaFree(p->item_b0);
  cudaFree(p->item_off);
  cudaFree(p->multi);
  cudaFree(p->ipart);
  delete p;
  return MK_OK;
}

}  // extern "C"
