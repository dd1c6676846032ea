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
//   decremental  union-find cannot split, so every component that lost an
//                edge is reset and rebuilt from its vertices' out-edges (an
//                edge into an affected vertex comes from the same old
//                component, so those out-edges are all its edges).
// Labels are the minimum vertex id of each weakly connected component.
//
// Every retry loop is bounded; on expiry the kernel sets MK_DEVERR_TIMEOUT.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "mk_internal.h"
#include "mk_slab.cuh"
#include "mk_members.cuh"

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

__device__ __forceinline__ void uf_union(uint32_t *p, uint32_t a, uint32_t b, uint32_t *err) {
  for (uint32_t it = 0; it < kUfLimit; ++it) {
    uint32_t ra = uf_find(p, a), rb = uf_find(p, b);
    if (ra == rb) return;
    uint32_t hi = ra > rb ? ra : rb, lo = ra > rb ? rb : ra;
    if (atomicCAS(p + hi, hi, lo) == hi) return;
  }
  atomicOr(err, kErrTimeout);
}

__global__ void k_uf_init(uint32_t *p, uint32_t V, const uint32_t *sel_bits = nullptr) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < V; i += gridDim.x * blockDim.x) {
    if (sel_bits && !((sel_bits[i >> 5] >> (i & 31)) & 1u)) continue;
    p[i] = i;
  }
}

__global__ void k_uf_batch(const uint32_t *__restrict__ src, const uint32_t *__restrict__ dst,
                           const uint8_t *__restrict__ applied, uint32_t n, uint32_t V,
                           uint32_t *p, uint32_t *err) {
  uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n || !applied[e]) return;
  uint32_t a = src[e], b = dst[e];
  if (a != b && a < V && b < V) uf_union(p, a, b, err);
}

__global__ void k_uf_compress(uint32_t *p, uint32_t V, const uint32_t *sel_bits) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < V; i += gridDim.x * blockDim.x) {
    if (sel_bits && !((sel_bits[i >> 5] >> (i & 31)) & 1u)) continue;
    p[i] = uf_root(p, i);
  }
}

// Marks the label (root) of every endpoint of an applied deletion.
__global__ void k_uf_mark(const uint32_t *__restrict__ src, const uint8_t *__restrict__ applied,
                          uint32_t n, uint32_t V, const uint32_t *p, uint32_t *aff_labels) {
  uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n || !applied[e]) return;
  uint32_t a = src[e];
  if (a >= V) return;
  uint32_t r = p[a];
  atomicOr(aff_labels + (r >> 5), 1u << (r & 31));
}

// Resets the vertices of affected components and records them.
__global__ void k_uf_reset(uint32_t *p, uint32_t V, const uint32_t *aff_labels, uint32_t *aff_vertices) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < V; i += gridDim.x * blockDim.x) {
    uint32_t r = p[i];
    if ((aff_labels[r >> 5] >> (r & 31)) & 1u) {
      p[i] = i;
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
template <bool kW>
__global__ void k_uf_sample(GraphView g, uint32_t *p, const uint32_t *sel_bits, uint32_t *err) {
  for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < g.V; u += gridDim.x * blockDim.x) {
    if (g.deg[u] == 0) continue;
    if (sel_bits && !((sel_bits[u >> 5] >> (u & 31)) & 1u)) continue;
    const uint32_t *w = reinterpret_cast<const uint32_t *>(g.slabs + 8ull * g.boff[u]);
    const uint32_t k0 = w[0], k1 = kW ? w[2] : w[1];
    if (k0 < kTombKey && k0 != u) uf_union(p, u, k0, err);
    if (k1 < kTombKey && k1 != u) uf_union(p, u, k1, err);
  }
}

// Unions of the out-edges of bucket b (owner u) whose endpoints do not share
// a parent yet.
template <bool kW>
__device__ __forceinline__ void link_bucket_skip(const GraphView &g, const Lanes &L, uint32_t *p,
                                                 uint32_t b, uint32_t u, uint32_t *err) {
  const uint32_t pu = __ldcg(p + u);
  walk_bucket(g, L, b, [&](const uint4 &q) {
    uint32_t k[4], w[4];
    lane_keys<kW>(q, L.gl, k, w);
#pragma unroll
    for (int j = 0; j < keys_per_lane<kW>(); ++j) {
      const uint32_t v = k[j];
      if (v >= kTombKey || v == u) continue;
      if (__ldcg(p + v) == pu) continue;
      uf_union(p, u, v, err);
    }
  });
}

template <bool kW>
__global__ void k_uf_edges_skip(GraphView g, uint32_t *p, const uint32_t *sel_bits, uint32_t *err) {
  const Lanes L = lanes();
  const uint32_t group = (blockIdx.x * blockDim.x + threadIdx.x) >> 3;
  const uint32_t ngroups = (gridDim.x * blockDim.x) >> 3;
  for (uint32_t b = group; b < g.nbuckets; b += ngroups) {
    const uint32_t u = g.bowner[b];
    if (g.deg[u] == 0) continue;
    if (sel_bits && !((sel_bits[u >> 5] >> (u & 31)) & 1u)) continue;
    link_bucket_skip<kW>(g, L, p, b, u, err);
  }
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
    link_bucket_skip<kW>(g, L, p, b, u, err);
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

// Unions of the out-edges of the selected vertices (all if sel is null), whose
// parents start reset: sample two neighbours each, compress, then every edge
// whose endpoints do not share a parent yet.
static mk_status wcc_link(mk_wcc *w, const uint32_t *sel, cudaStream_t s) {
  mk_graph *g = w->g;
  const int fg = flat_grid(g->V, g->device);
  const GraphView v = g->view();
  if (g->weighted)
    k_uf_sample<true><<<fg, 256, 0, s>>>(v, w->parent, sel, w->err);
  else
    k_uf_sample<false><<<fg, 256, 0, s>>>(v, w->parent, sel, w->err);
  k_uf_compress<<<fg, 256, 0, s>>>(w->parent, g->V, sel);
  const int blocks = (int)std::min<uint64_t>(g->num_buckets * 8 / 256 + 1,
                                             (uint64_t)device_sm_count(g->device) * 8);
  if (g->weighted)
    k_uf_edges_skip<true><<<blocks, 256, 0, s>>>(v, w->parent, sel, w->err);
  else
    k_uf_edges_skip<false><<<blocks, 256, 0, s>>>(v, w->parent, sel, w->err);
  k_uf_compress<<<fg, 256, 0, s>>>(w->parent, g->V, sel);
  MK_CUDA(cudaGetLastError());
  return MK_OK;
}

static mk_status wcc_static(mk_wcc *w, cudaStream_t s) {
  mk_graph *g = w->g;
  k_uf_init<<<flat_grid(g->V, g->device), 256, 0, s>>>(w->parent, g->V);
  return wcc_link(w, nullptr, s);
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
  w->err = g->err_word();
  if (e != cudaSuccess) {
    mk_wcc_destroy(w);
    return cuda_fail(e, "mk_wcc_create");
  }
  k_uf_init<<<flat_grid(V, g->device), 256>>>(w->parent, (uint32_t)V);
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
  k_uf_init<<<flat_grid(g->V, g->device), 256, 0, s>>>(w->parent, g->V, d_sel_bits);
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
    k_uf_batch<<<(n + 255) / 256, 256, 0, s>>>(d_src, d_dst, g->applied.ptr, n, g->V, w->parent, w->err);
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
  if (!batch_matches(g, d_src, d_dst, n, 2)) {
    MK_CHECK(wcc_static(w, s));
  } else if (n) {
    const size_t words = ((size_t)g->V + 31) / 32;
    MK_CUDA(cudaMemsetAsync(w->aff_labels, 0, words * 4, s));
    MK_CUDA(cudaMemsetAsync(w->aff_vertices, 0, words * 4, s));
    k_uf_mark<<<(n + 255) / 256, 256, 0, s>>>(d_src, g->applied.ptr, n, g->V, w->parent, w->aff_labels);
    k_uf_reset<<<flat_grid(g->V, g->device), 256, 0, s>>>(w->parent, g->V, w->aff_labels, w->aff_vertices);
    MK_CHECK(wcc_link(w, w->aff_vertices, s));
  }
  return w->timer.stop(ms_out);
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
  w->staging.release();
  w->ranges.release();
  delete w;
  return MK_OK;
}

}  // extern "C"
