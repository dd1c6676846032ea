// The batched many-graph step behind the C ABI: a graph set, one query kind
// per member (BFS from a source, or components), and a step that applies
// every member's update batch and answers every member's query.
//
// No counterpart in the reference, whose drivers hold one graph and one
// algorithm object per process (src/BFS.cu:11-131); this is the path a C++
// caller of the drop-in uses for thousands of small graphs.  Two forms:
//
//   sequence  four stream-ordered launches, those of the Python batched
//             runner: one delete and one insert kernel over all members'
//             batches, one shared-memory member BFS over the BFS members,
//             one member WCC over the WCC members;
//   fused     one persistent launch (every member of at most 65,535
//             vertices): a CTA takes a member from a counter, largest
//             first, finds the member's slices of the delete and insert
//             batches (a 256-way search per bound over the member-grouped
//             arrays), applies its deletes, then its inserts (a thread per
//             edge), then answers its query with the member's state in
//             shared memory.  Members are disjoint, so a member's order
//             (deletes, inserts, query) needs only block barriers; no grid
//             barrier and no phase counter.  The last CTA out publishes the
//             insert count and resets the member counter for the next step.
//
// Everything a step issues is asynchronous and allocation-free once the
// batch scratch is reserved, so a step can be captured into a CUDA graph and
// replayed.
#include <cuda_runtime.h>

#include <algorithm>
#include <numeric>
#include <vector>

#include "mk_internal.h"
#include "mk_members.cuh"
#include "mk_slab.cuh"
#include "mk_update.cuh"

using namespace mk;

namespace mk {
namespace {

constexpr uint32_t kStepNone = 0, kStepBfs = 1, kStepWcc = 2;

struct StepBatch {
  const uint32_t *ds, *dd;
  const uint32_t *is, *id, *iw;
  uint32_t nd, ni;
};

// Bounds of a member's slices: bound j of (delete lo, delete hi, insert lo,
// insert hi) is the first index i of its array with a[i] >= x (x = the
// member's first or end vertex).  Over an array grouped by member in
// ascending member order that predicate is monotone, so each bound is found
// by 256 threads narrowing the interval 256-fold per round (at most five
// rounds for 2^32 entries).  Results in s_l[0..3]; ends synchronised.
__device__ __forceinline__ void slice_bounds(const StepBatch &B, uint32_t lo, uint32_t hi,
                                             uint32_t *s_l, uint32_t *s_r, uint32_t *s_cnt) {
  const uint32_t j = threadIdx.x >> 8, t = threadIdx.x & 255u;
  const uint32_t *a = j < 2 ? B.ds : B.is;
  const uint32_t x = (j & 1u) ? hi : lo;
  if (t == 0) {
    s_l[j] = 0;
    s_r[j] = j < 2 ? B.nd : B.ni;
    s_cnt[j] = 0;
  }
  __syncthreads();
  for (uint32_t round = 0; round < 8; ++round) {
    const uint32_t l = s_l[j], r = s_r[j];
    const bool active = l < r;
    if (!__syncthreads_or(active)) break;
    const uint32_t step = active ? (r - l + 255u) / 256u : 0u;
    const uint32_t pos = l + t * step;
    const bool below = active && pos < r && __ldg(a + pos) < x;
    const uint32_t bal = __ballot_sync(0xFFFFFFFFu, below);
    if ((threadIdx.x & 31u) == 0 && bal) atomicAdd(s_cnt + j, (uint32_t)__popc(bal));
    __syncthreads();
    if (t == 0) {
      const uint32_t k = s_cnt[j];
      if (active) {
        if (k == 0) {
          s_r[j] = l;  // a[l] >= x already
        } else {
          s_l[j] = l + (k - 1) * step + 1;  // the k-th sample is below x
          s_r[j] = min(l + k * step, r);
        }
      }
      s_cnt[j] = 0;
    }
    __syncthreads();
  }
}

// tab[m] = (first vertex, end vertex, first bucket, end bucket) of member m
// (members sorted by bucket count, largest first), meta[m] = query kind << 16
// | local BFS source.  ctl[0] = member counter, ctl[1] = CTAs done (both 0
// between launches); acc[0] = insert count being gathered (0 between
// launches), published to count_out.
template <bool kW>
__global__ void __launch_bounds__(kMemThreads, 1)
    k_set_step(GraphView g, const uint4 *__restrict__ tab, const uint32_t *__restrict__ meta,
               uint32_t nm, uint32_t *ctl, unsigned long long *acc,
               unsigned long long *count_out, StepBatch B, uint8_t *__restrict__ applied,
               unsigned long long *__restrict__ dist, uint32_t *__restrict__ items,
               uint32_t *__restrict__ found, uint32_t *__restrict__ labels) {
  extern __shared__ uint32_t smem[];
  __shared__ uint32_t s_member, s_nfound, s_nitems;
  __shared__ uint32_t s_l[4], s_r[4], s_cnt[4];
  const Lanes L = lanes();
  uint32_t inserted = 0;
  for (;;) {
    if (threadIdx.x == 0) s_member = atomicAdd(ctl, 1u);
    __syncthreads();
    const uint32_t m = s_member;
    if (m >= nm) break;
    const uint4 R = tab[m];
    const uint32_t lo = R.x, n = R.y - R.x, mt = meta[m];
    slice_bounds(B, lo, R.y, s_l, s_r, s_cnt);
    uint32_t d0 = s_l[0], d1 = s_l[1], i0 = s_l[2], i1 = s_l[3];
    // bounds that do not partition the batch: the arrays are not grouped
    // by member (the last member also closes both arrays)
    if (threadIdx.x == 0 && (d1 < d0 || i1 < i0 || (R.y == g.V && (d1 != B.nd || i1 != B.ni))))
      atomicOr(g.err, kErrInvalidId);
    d1 = max(d1, d0);
    i1 = max(i1, i0);
    for (uint32_t e = d0 + threadIdx.x; e < d1; e += blockDim.x) {
      const uint32_t u = __ldg(B.ds + e), v = __ldg(B.dd + e);
      if (u - lo >= n || v - lo >= n) {
        atomicOr(g.err, kErrInvalidId);  // outside the member's slice
        continue;
      }
      if (u == v) continue;
      const uint32_t b0 = __ldg(g.boff + u);
      const uint32_t head = b0 + bucket_of(v, __ldg(g.boff + u + 1) - b0);
      uint4 q[8];
      lane_load_slab(g, head, q);
      if (lane_delete_chain<kW>(g, head, q, v)) atomicSub(g.deg + u, 1u);
    }
    __syncthreads();
    for (uint32_t e = i0 + threadIdx.x; e < i1; e += blockDim.x) {
      const uint32_t u = __ldg(B.is + e), v = __ldg(B.id + e);
      uint32_t app = 0;
      if (u - lo >= n || v - lo >= n) {
        atomicOr(g.err, kErrInvalidId);
      } else if (u != v) {
        const uint32_t wt = (kW && B.iw) ? __ldg(B.iw + e) : 0u;
        const uint32_t b0 = __ldg(g.boff + u);
        const uint32_t head = b0 + bucket_of(v, __ldg(g.boff + u + 1) - b0);
        uint4 q[8];
        lane_load_slab(g, head, q);
        app = lane_insert_chain<kW>(g, head, q, v, wt);
        if (app) {
          atomicAdd(g.deg + u, 1u);
          ++inserted;
        }
      }
      applied[e] = (uint8_t)app;
    }
    __syncthreads();
    const uint32_t kind = mt >> 16;
    if (kind == kStepBfs)
      bfs_member<kW, true>(g, L, R, lo + (mt & 0xFFFFu), dist, items, found, g.err, smem,
                           s_nfound, s_nitems);
    else if (kind == kStepWcc)
      uf_member<kW, true>(g, L, R, labels, g.err, reinterpret_cast<uint16_t *>(smem));
  }
  inserted = __reduce_add_sync(0xFFFFFFFFu, inserted);
  if ((threadIdx.x & 31u) == 0 && inserted) atomicAdd(acc, (unsigned long long)inserted);
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(ctl + 1, 1u) == gridDim.x - 1) {
      // every CTA has drawn its last member and added its count
      __threadfence();
      *count_out = atomicExch(acc, 0ull);
      atomicExch(ctl, 0u);
      atomicExch(ctl + 1, 0u);
    }
  }
}

}  // namespace
}  // namespace mk

struct mk_set_runner {
  mk_graphset *set = nullptr;
  mk_graph *g = nullptr;
  mk_traversal *bfs = nullptr;
  mk_wcc *wcc = nullptr;
  uint32_t num_graphs = 0, n_bfs = 0, n_wcc = 0;
  uint32_t max_members = 0;  // vertices of the largest member
  // fused step
  bool fused = false;
  DevBuf<uint32_t> ftab;   // uint4 per member, then one meta word per member
  uint32_t *fctl = nullptr;  // [0] member counter, [1] CTAs done, [2..3] u64 insert count
  size_t fsmem = 0;
  int fgrid = 0;
};

namespace {

mk_status build_fused(mk_set_runner *r, const std::vector<uint32_t> &off, const uint8_t *h_query,
                      const uint32_t *h_src_local) {
  mk_graph *g = r->g;
  const uint32_t G = r->num_graphs;
  std::vector<uint32_t> order(G);
  std::iota(order.begin(), order.end(), 0u);
  auto buckets = [&](uint32_t m) { return g->h_boff[off[m + 1]] - g->h_boff[off[m]]; };
  std::stable_sort(order.begin(), order.end(),
                   [&](uint32_t a, uint32_t b) { return buckets(a) > buckets(b); });
  std::vector<uint32_t> host((size_t)G * 5);
  uint32_t *tab = host.data(), *meta = tab + 4 * (size_t)G;
  size_t smem = 0;
  for (uint32_t i = 0; i < G; ++i) {
    const uint32_t m = order[i], lo = off[m], hi = off[m + 1];
    tab[4 * i + 0] = lo;
    tab[4 * i + 1] = hi;
    tab[4 * i + 2] = g->h_boff[lo];
    tab[4 * i + 3] = g->h_boff[hi];
    uint32_t kind = kStepNone, src = 0;
    if (h_query[m] == MK_QUERY_BFS) {
      kind = kStepBfs;
      src = h_src_local[m];
      smem = std::max(smem, bfs_member_smem(hi - lo));
    } else if (h_query[m] == MK_QUERY_WCC) {
      kind = kStepWcc;
      smem = std::max(smem, uf_member_smem(hi - lo));
    }
    meta[i] = (kind << 16) | src;
  }
  MK_CHECK(r->ftab.reserve(host.size(), &g->device_bytes));
  MK_CUDA(cudaMemcpy(r->ftab.ptr, host.data(), host.size() * 4, cudaMemcpyHostToDevice));
  if (!r->fctl) {
    MK_CUDA(cudaMalloc(&r->fctl, 16));
    g->device_bytes += 16;
  }
  MK_CUDA(cudaMemset(r->fctl, 0, 16));
  auto kern = g->weighted ? k_set_step<true> : k_set_step<false>;
  MK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)bfs_member_smem(kMemLocalMax)));
  int per_sm = 0;
  MK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kMemThreads, smem));
  r->fsmem = smem;
  r->fgrid = (int)std::min<uint64_t>(G, (uint64_t)device_sm_count(g->device) * std::max(per_sm, 1));
  if (r->bfs) {
    // a member that asks no BFS keeps the packed words this writes
    TravMemberBufs tb{};
    MK_CHECK(trav_member_bufs(r->bfs, &tb));
    MK_CUDA(cudaMemset(tb.dist, 0xFF, (size_t)g->V * 8));
  }
  return MK_OK;
}

}  // namespace

extern "C" {

mk_status mk_set_runner_create(mk_graphset *s, const uint8_t *h_query,
                               const uint32_t *h_bfs_source_local, mk_set_runner **out) {
  if (!s || !h_query || !out) return fail(MK_ERR_INVALID, "mk_set_runner_create: null argument");
  *out = nullptr;
  mk_graph *g = nullptr;
  MK_CHECK(mk_graphset_union(s, &g));
  uint32_t ng = 0;
  MK_CHECK(mk_graphset_num_graphs(s, &ng));
  std::vector<uint32_t> off((size_t)ng + 1);
  MK_CHECK(mk_graphset_offsets(s, off.data()));
  const uint32_t G = (uint32_t)off.size() - 1;
  std::vector<uint32_t> sources, bfs_ranges, wcc_ranges;
  uint32_t max_members = 0;
  for (uint32_t m = 0; m < G; ++m) {
    max_members = std::max(max_members, off[m + 1] - off[m]);
    if (h_query[m] == MK_QUERY_BFS) {
      if (!h_bfs_source_local) return fail(MK_ERR_INVALID, "mk_set_runner_create: BFS members need sources");
      const uint64_t src = (uint64_t)off[m] + h_bfs_source_local[m];
      if (src >= off[m + 1]) return fail(MK_ERR_INVALID, "mk_set_runner_create: source outside its member");
      sources.push_back((uint32_t)src);
      bfs_ranges.push_back(off[m]);
      bfs_ranges.push_back(off[m + 1]);
    } else if (h_query[m] == MK_QUERY_WCC) {
      wcc_ranges.push_back(off[m]);
      wcc_ranges.push_back(off[m + 1]);
    } else if (h_query[m] != MK_QUERY_NONE) {
      return fail(MK_ERR_INVALID, "mk_set_runner_create: unknown query kind");
    }
  }
  mk_set_runner *r = new mk_set_runner();
  r->set = s;
  r->g = g;
  r->num_graphs = G;
  r->max_members = max_members;
  r->n_bfs = (uint32_t)sources.size();
  r->n_wcc = (uint32_t)wcc_ranges.size() / 2;
  mk_status st = MK_OK;
  if (r->n_bfs) {
    st = mk_bfs_create_multi(g, sources.data(), r->n_bfs, &r->bfs);
    if (st == MK_OK) st = mk_bfs_prepare_members(r->bfs, bfs_ranges.data(), r->n_bfs);
  }
  if (st == MK_OK && r->n_wcc) {
    st = mk_wcc_create(g, &r->wcc);
    if (st == MK_OK) st = mk_wcc_prepare_ranges(r->wcc, wcc_ranges.data(), r->n_wcc);
  }
  if (st == MK_OK && max_members <= kMemLocalMax && !g->reverse) {
    DeviceGuard dg(g->device);
    st = build_fused(r, off, h_query, h_bfs_source_local);
  }
  if (st != MK_OK) {
    mk_set_runner_destroy(r);
    return st;
  }
  *out = r;
  return MK_OK;
}

mk_status mk_set_runner_set_fused(mk_set_runner *r, uint32_t on) {
  if (!r) return fail(MK_ERR_INVALID, "mk_set_runner_set_fused: null handle");
  if (on && !r->ftab.ptr)
    return fail(MK_ERR_INVALID, "mk_set_runner_set_fused: a member has more than 65535 vertices");
  r->fused = on != 0;
  return MK_OK;
}

mk_status mk_set_runner_launches(mk_set_runner *r, uint32_t *h_launches) {
  if (!r || !h_launches) return fail(MK_ERR_INVALID, "mk_set_runner_launches: null argument");
  *h_launches = r->fused ? 1u : 2u + (r->bfs ? 1u : 0u) + (r->wcc ? 1u : 0u);
  return MK_OK;
}

mk_status mk_set_runner_handles(mk_set_runner *r, mk_traversal **bfs, mk_wcc **wcc) {
  if (!r) return fail(MK_ERR_INVALID, "mk_set_runner_handles: null handle");
  if (bfs) *bfs = r->bfs;
  if (wcc) *wcc = r->wcc;
  return MK_OK;
}

mk_status mk_set_runner_step(mk_set_runner *r, const uint32_t *d_del_src,
                             const uint32_t *d_del_dst, uint32_t n_del,
                             const uint32_t *d_ins_src, const uint32_t *d_ins_dst,
                             const uint32_t *d_ins_w, uint32_t n_ins, void *stream) {
  if (!r) return fail(MK_ERR_INVALID, "mk_set_runner_step: null handle");
  if ((n_del && (!d_del_src || !d_del_dst)) || (n_ins && (!d_ins_src || !d_ins_dst)))
    return fail(MK_ERR_INVALID, "mk_set_runner_step: null batch");
  if (!r->fused) {
    MK_CHECK(mk_graph_delete_edges(r->g, d_del_src, d_del_dst, n_del, stream));
    MK_CHECK(mk_graph_insert_edges(r->g, d_ins_src, d_ins_dst, d_ins_w, n_ins, stream));
    if (r->bfs) MK_CHECK(mk_bfs_static_members(r->bfs, stream, nullptr));
    if (r->wcc) MK_CHECK(mk_wcc_static_prepared(r->wcc, stream, nullptr));
    return MK_OK;
  }
  mk_graph *g = r->g;
  DeviceGuard dg(g->device);
  cudaStream_t s = as_stream(stream);
  MK_CHECK(g->applied.reserve(std::max<uint32_t>(n_ins, 1), &g->device_bytes));
  // the graph's last update is the insert batch, as after the sequence
  g->last_n = n_ins;
  g->last_src = d_ins_src;
  g->last_dst = d_ins_dst;
  g->last_op = 1;
  TravMemberBufs tb{};
  if (r->bfs) MK_CHECK(trav_member_bufs(r->bfs, &tb));
  uint32_t *labels = r->wcc ? wcc_label_buf(r->wcc) : nullptr;
  const uint32_t G = r->num_graphs;
  const uint4 *tab = reinterpret_cast<const uint4 *>(r->ftab.ptr);
  const uint32_t *meta = r->ftab.ptr + 4 * (size_t)G;
  unsigned long long *acc = reinterpret_cast<unsigned long long *>(r->fctl + 2);
  StepBatch B{d_del_src, d_del_dst, d_ins_src, d_ins_dst, d_ins_w, n_del, n_ins};
  if (g->weighted)
    k_set_step<true><<<r->fgrid, kMemThreads, r->fsmem, s>>>(g->view(), tab, meta, G, r->fctl, acc,
                                                            g->counters, B, g->applied.ptr, tb.dist,
                                                            tb.items, tb.found, labels);
  else
    k_set_step<false><<<r->fgrid, kMemThreads, r->fsmem, s>>>(g->view(), tab, meta, G, r->fctl, acc,
                                                             g->counters, B, g->applied.ptr, tb.dist,
                                                             tb.items, tb.found, labels);
  MK_CUDA(cudaGetLastError());
  return MK_OK;
}

mk_status mk_set_runner_results(mk_set_runner *r, const uint64_t **d_bfs_packed,
                                const uint32_t **d_wcc_labels) {
  if (!r) return fail(MK_ERR_INVALID, "mk_set_runner_results: null handle");
  if (d_bfs_packed) {
    *d_bfs_packed = nullptr;
    if (r->bfs) MK_CHECK(mk_traversal_packed(r->bfs, d_bfs_packed));
  }
  if (d_wcc_labels) {
    *d_wcc_labels = nullptr;
    if (r->wcc) MK_CHECK(mk_wcc_labels_device(r->wcc, d_wcc_labels));
  }
  return MK_OK;
}

mk_status mk_set_runner_destroy(mk_set_runner *r) {
  if (!r) return MK_OK;
  if (r->bfs) mk_traversal_destroy(r->bfs);
  if (r->wcc) mk_wcc_destroy(r->wcc);
  r->ftab.release();
  if (r->fctl) cudaFree(r->fctl);
  delete r;
  return MK_OK;
}

}  // extern "C"
