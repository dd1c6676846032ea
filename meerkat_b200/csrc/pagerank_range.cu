// PageRank of one vertex range of an out-edge graph (a member of a graph
// set), by push sweeps: no reverse graph needed.
//
// Same formula as the pull solver (reference: PageRankImpl.cuh:41-52,
// :89-144, PageRank.cuh:42-43) restricted to the range [lo, hi), N = hi - lo:
//   PR'[v] = (1-d)/N + d * sum_{u -> v} PR[u] / outdeg[u]
//                    + d * sum_{outdeg[u] = 0} PR[u] / N
// starting from PR = 1/N, stopping once delta * d / (1 - d) <= tol / 2 (the
// L1 error bound of the contraction) or after max_iter iterations.  The
// range must be closed under out-edges.  Out-degrees are the graph's live
// degrees, so a graph updated between calls needs no recount.
//
// One iteration: a dangling-mass reduction, a base fill of PR', a push pass
// (one 8-lane group per bucket of the range, each live edge u -> v adds
// PR[u] / outdeg[u] to PR'[v] with an FP64 atomic), and an |delta|
// reduction read back by the host.  FP64 accumulation keeps the result
// within the same L1 tolerance as the pull solver although the atomic order
// varies from run to run.
#include <cuda_runtime.h>

#include <algorithm>

#include "mk_internal.h"
#include "mk_slab.cuh"

namespace mk {
namespace {

__device__ __forceinline__ double warp_sum(double x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xFFFFFFFFu, x, o);
  return x;
}

// Block-reduced sum of per-thread values into *out.
__device__ __forceinline__ void block_add(double x, double *out) {
  __shared__ double part[32];
  x = warp_sum(x);
  const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
  if (lane == 0) part[w] = x;
  __syncthreads();
  if (w == 0) {
    double y = lane < (blockDim.x >> 5) ? part[lane] : 0.0;
    y = warp_sum(y);
    if (lane == 0 && y != 0.0) atomicAdd(out, y);
  }
  __syncthreads();
}

__global__ void k_prr_fill(double *__restrict__ pr, uint32_t n, double x) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    pr[i] = x;
}

// acc[0] += dangling mass of pr
__global__ void k_prr_dangling(const double *__restrict__ pr, const uint32_t *__restrict__ deg,
                               uint32_t n, double *acc) {
  double x = 0.0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    if (deg[i] == 0) x += pr[i];
  block_add(x, acc);
}

__global__ void k_prr_base(double *__restrict__ nx, uint32_t n, const double *acc, double d) {
  const double base = (1.0 - d) / n + d * acc[0] / n;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    nx[i] = base;
}

template <bool kW>
__global__ void k_prr_push(GraphView g, uint32_t lo, uint32_t b0, uint32_t nb,
                           const double *__restrict__ pr, double *nx, double d) {
  const Lanes L = lanes();
  const uint32_t group = (blockIdx.x * blockDim.x + threadIdx.x) >> 3;
  const uint32_t ngroups = (gridDim.x * blockDim.x) >> 3;
  for (uint32_t i = group; i < nb; i += ngroups) {
    const uint32_t b = b0 + i;
    const uint32_t u = g.bowner[b];
    const uint32_t du = g.deg[u];
    if (du == 0) continue;
    const double c = d * pr[u - lo] / (double)du;
    walk_bucket(g, L, b, [&](const uint4 &q) {
      uint32_t k[4], w[4];
      lane_keys<kW>(q, L.gl, k, w);
#pragma unroll
      for (int j = 0; j < keys_per_lane<kW>(); ++j)
        if (k[j] < kTombKey) atomicAdd(nx + (k[j] - lo), c);
    });
  }
}

// acc[1] += sum |nx - pr|
__global__ void k_prr_delta(const double *__restrict__ pr, const double *__restrict__ nx,
                            uint32_t n, double *acc) {
  double x = 0.0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    x += fabs(nx[i] - pr[i]);
  block_add(x, acc + 1);
}

__global__ void k_prr_out(const double *__restrict__ pr, uint32_t n, float *__restrict__ out) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    out[i] = (float)pr[i];
}

int flat_blocks(uint64_t n, int device) {
  return (int)std::max<uint64_t>(1, std::min<uint64_t>(n / 256 + 1, (uint64_t)device_sm_count(device) * 8));
}

}  // namespace
}  // namespace mk

using namespace mk;

struct mk_pagerank_range {
  mk_graph *g = nullptr;
  uint32_t cap = 0;  // vertices
  double *a = nullptr, *b = nullptr;
  double *acc = nullptr;  // [0] dangling, [1] delta
  float *out = nullptr;
  uint32_t n = 0;  // vertices of the last run
  uint32_t iters = 0;
  float delta = 0.f;
  Timer timer;
};

extern "C" {

mk_status mk_pagerank_range_create(mk_graph *g, uint32_t max_vertices, mk_pagerank_range **out) {
  if (!g || !out || max_vertices == 0)
    return fail(MK_ERR_INVALID, "mk_pagerank_range_create: bad argument");
  if (g->reverse) return fail(MK_ERR_INVALID, "mk_pagerank_range_create: needs an out-edge graph");
  *out = nullptr;
  DeviceGuard dg(g->device);
  mk_pagerank_range *p = new mk_pagerank_range();
  p->g = g;
  p->cap = max_vertices;
  cudaError_t e = cudaMalloc(&p->a, (size_t)max_vertices * 8);
  if (e == cudaSuccess) e = cudaMalloc(&p->b, (size_t)max_vertices * 8);
  if (e == cudaSuccess) e = cudaMalloc(&p->acc, 16);
  if (e == cudaSuccess) e = cudaMalloc(&p->out, (size_t)max_vertices * 4);
  if (e != cudaSuccess) {
    mk_pagerank_range_destroy(p);
    return cuda_fail(e, "mk_pagerank_range_create");
  }
  *out = p;
  return MK_OK;
}

mk_status mk_pagerank_range_run(mk_pagerank_range *p, uint32_t v_begin, uint32_t v_end,
                                float damping, float tol, uint32_t max_iter, void *stream,
                                float *ms_out) {
  if (!p) return fail(MK_ERR_INVALID, "mk_pagerank_range_run: null handle");
  mk_graph *g = p->g;
  if (v_begin >= v_end || v_end > g->V)
    return fail(MK_ERR_INVALID, "mk_pagerank_range_run: bad vertex range");
  if (v_end - v_begin > p->cap)
    return fail(MK_ERR_INVALID, "mk_pagerank_range_run: range larger than max_vertices");
  if (!(damping > 0.f && damping < 1.f) || !(tol > 0.f))
    return fail(MK_ERR_INVALID, "mk_pagerank_range_run: damping must be in (0,1), tol > 0");
  DeviceGuard dg(g->device);
  cudaStream_t s = as_stream(stream);
  MK_CHECK(p->timer.start(s, ms_out != nullptr));
  const uint32_t n = v_end - v_begin;
  const uint32_t b0 = g->h_boff[v_begin], nb = g->h_boff[v_end] - b0;
  const double d = damping;
  const int fb = flat_blocks(n, g->device);
  const int gb = (int)std::min<uint64_t>((uint64_t)nb * 8 / 256 + 1, (uint64_t)device_sm_count(g->device) * 8);
  const GraphView v = g->view();
  double *pr = p->a, *nx = p->b;
  k_prr_fill<<<fb, 256, 0, s>>>(pr, n, 1.0 / n);
  uint32_t it = 0;
  double delta = 0.0;
  while (it < max_iter) {
    MK_CUDA(cudaMemsetAsync(p->acc, 0, 16, s));
    k_prr_dangling<<<fb, 256, 0, s>>>(pr, g->deg + v_begin, n, p->acc);
    k_prr_base<<<fb, 256, 0, s>>>(nx, n, p->acc, d);
    if (g->weighted)
      k_prr_push<true><<<gb, 256, 0, s>>>(v, v_begin, b0, nb, pr, nx, d);
    else
      k_prr_push<false><<<gb, 256, 0, s>>>(v, v_begin, b0, nb, pr, nx, d);
    k_prr_delta<<<fb, 256, 0, s>>>(pr, nx, n, p->acc);
    MK_CUDA(cudaGetLastError());
    MK_CUDA(cudaMemcpyAsync(&delta, p->acc + 1, 8, cudaMemcpyDeviceToHost, s));
    MK_CUDA(cudaStreamSynchronize(s));
    std::swap(pr, nx);
    ++it;
    if (delta * d / (1.0 - d) <= 0.5 * tol) break;
  }
  k_prr_out<<<fb, 256, 0, s>>>(pr, n, p->out);
  MK_CUDA(cudaGetLastError());
  p->n = n;
  p->iters = it;
  p->delta = (float)delta;
  return p->timer.stop(ms_out);
}

mk_status mk_pagerank_range_values(mk_pagerank_range *p, float *h_out) {
  if (!p || !h_out) return fail(MK_ERR_INVALID, "mk_pagerank_range_values: null argument");
  DeviceGuard dg(p->g->device);
  MK_CUDA(cudaDeviceSynchronize());
  MK_CUDA(cudaMemcpy(h_out, p->out, (size_t)p->n * 4, cudaMemcpyDeviceToHost));
  return MK_OK;
}

mk_status mk_pagerank_range_stats(mk_pagerank_range *p, uint32_t *h_iters, float *h_delta) {
  if (!p) return fail(MK_ERR_INVALID, "mk_pagerank_range_stats: null handle");
  if (h_iters) *h_iters = p->iters;
  if (h_delta) *h_delta = p->delta;
  return MK_OK;
}

mk_status mk_pagerank_range_destroy(mk_pagerank_range *p) {
  if (!p) return MK_OK;
  DeviceGuard dg(p->g->device);
  cudaFree(p->a);
  cudaFree(p->b);
  cudaFree(p->acc);
  cudaFree(p->out);
  delete p;
  return MK_OK;
}

}  // extern "C"
