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
//   one launch  (mk_set_runner_set_single, every member of at most 65,535
//             vertices) a cooperative kernel, one 1,024-thread CTA per SM,
//             in three phases separated by bounded grid barriers: every
//             delete of the batch (a thread per edge), every insert, then
//             the members' queries, a CTA taking members from a counter,
//             largest first, BFS and WCC members mixed, each solved with
//             its state in shared memory.
//
// Everything a step issues is asynchronous and allocation-free once the
// batch scratch is reserved, so a step can be captured into a CUDA graph and
// replayed.
//
// The one-launch form is correct and capturable but not the faster one:
// measured on 4,096 members it takes 13.6-18.3 ms per step against
// 10.3-13.2 ms for the four launches.  Its update phases run at one
// 1,024-thread CTA per SM (the member phase's shared memory allows no more),
// about 1.5x the update kernels' own time at their tuned occupancy, and
// merging the two query kernels gains less than that.  Loads matter in the
// member phase: through L2 only (ld.global.cg) it was 2.5x slower again;
// plain loads behind the grid barrier are both correct and as fast as the
// read-only path.  An earlier design that handed each CTA a whole member
// (its deletes, inserts and query between block barriers) was slower still.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "mk_internal.h"
#include "mk_members.cuh"
#include "mk_slab.cuh"
#include "mk_update.cuh"

namespace mk {
namespace {

constexpr uint32_t kStepNone = 0, kStepBfs = 1, kStepWcc = 2;
// ctl words of the one-launch step: grid barrier (count, generation), the
// member counter; zeroed before every launch (a barrier that timed out
// leaves its count behind)
enum : int { kSBar0 = 0, kSMember = 2, kSCtlWords = 4 };

// Thread-per-edge deletes (kIns false) or inserts over the whole batch; an
// insert records its applied flag and the count of applied inserts.
template <bool kW, bool kIns>
__device__ __forceinline__ void step_updates(const GraphView &g, const uint32_t *__restrict__ src,
                                             const uint32_t *__restrict__ dst,
                                             const uint32_t *__restrict__ w, uint32_t n,
                                             uint8_t *__restrict__ applied,
                                             unsigned long long *count) {
  const uint64_t nthreads = (uint64_t)gridDim.x * blockDim.x;
  uint32_t mine = 0;
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < n; e += nthreads) {
    const uint32_t u = __ldg(src + e), v = __ldg(dst + e);
    uint32_t app = 0;
    if (u >= g.V || v >= g.V) {
      atomicOr(g.err, kErrInvalidId);
    } else if (u != v) {
      const uint32_t b0 = __ldg(g.boff + u);
      const uint32_t head = b0 + bucket_of(v, __ldg(g.boff + u + 1) - b0);
      uint4 q[8];
      lane_load_slab(g, head, q);
      if (kIns) {
        app = lane_insert_chain<kW>(g, head, q, v, (kW && w) ? __ldg(w + e) : 0u);
        if (app) atomicAdd(g.deg + u, 1u);
      } else {
        app = lane_delete_chain<kW>(g, head, q, v);
        if (app) atomicSub(g.deg + u, 1u);
      }
    }
    if (kIns) applied[e] = (uint8_t)app;
    mine += app;
  }
  if (kIns) {
    mine = __reduce_add_sync(0xFFFFFFFFu, mine);
    if ((threadIdx.x & 31u) == 0 && mine) atomicAdd(count, (unsigned long long)mine);
  }
}

struct StepArgs {
  const uint32_t *ds, *dd;
  const uint32_t *is, *id, *iw;
  uint32_t nd, ni;
  const uint4 *tab;       // per queried member (largest first): first vertex, end, first bucket, end bucket
  const uint32_t *meta;   // kind << 16 | local BFS source
  uint32_t nm;
  uint32_t *ctl;
  uint8_t *applied;
  unsigned long long *count;  // applied inserts (the graph's last-update count)
  unsigned long long *dist;
  uint32_t *items, *found, *labels;
  unsigned long long limit_ns;
};

template <bool kW>
__global__ void __launch_bounds__(kMemThreads, 1) k_set_step(GraphView g, StepArgs a) {
  extern __shared__ uint32_t smem[];
  __shared__ uint32_t s_member, s_nfound, s_nitems;
  if (blockIdx.x == 0 && threadIdx.x == 0) *a.count = 0;
  step_updates<kW, false>(g, a.ds, a.dd, nullptr, a.nd, nullptr, nullptr);
  if (!grid_barrier(a.ctl + kSBar0, g.err, a.limit_ns)) return;
  step_updates<kW, true>(g, a.is, a.id, a.iw, a.ni, a.applied, a.count);
  if (!grid_barrier(a.ctl + kSBar0, g.err, a.limit_ns)) return;
  const Lanes L = lanes();
  for (;;) {
    if (threadIdx.x == 0) s_member = atomicAdd(a.ctl + kSMember, 1u);
    __syncthreads();
    const uint32_t m = s_member;
    if (m >= a.nm) break;
    const uint4 R = a.tab[m];
    const uint32_t mt = a.meta[m];
    if ((mt >> 16) == kStepBfs)
      bfs_member<kW, true>(g, L, R, R.x + (mt & 0xFFFFu), a.dist, a.items, a.found, g.err, smem,
                           s_nfound, s_nitems);
    else
      uf_member<kW, true>(g, L, R, a.labels, g.err, reinterpret_cast<uint16_t *>(smem));
  }
}

}  // namespace
}  // namespace mk

using namespace mk;

struct mk_set_runner {
  mk_graphset *set = nullptr;
  mk_graph *g = nullptr;
  mk_traversal *bfs = nullptr;
  mk_wcc *wcc = nullptr;
  uint32_t num_graphs = 0, n_bfs = 0, n_wcc = 0;
  uint32_t max_member = 0;  // vertices of the largest member
  // one-launch step: queried-member table, ctl words, launch shape
  bool single = false;
  DevBuf<uint32_t> stab;  // uint4 per queried member, then one meta word each
  uint32_t nq = 0;
  uint32_t *sctl = nullptr;
  size_t ssmem = 0;
  int sgrid = 0;
};

namespace {

mk_status build_single(mk_set_runner *r, const std::vector<uint32_t> &off, const uint8_t *h_query,
                       const uint32_t *h_src_local) {
  mk_graph *g = r->g;
  const uint32_t G = r->num_graphs;
  std::vector<uint32_t> order;
  for (uint32_t m = 0; m < G; ++m)
    if (h_query[m] == MK_QUERY_BFS || h_query[m] == MK_QUERY_WCC) order.push_back(m);
  auto buckets = [&](uint32_t m) { return g->h_boff[off[m + 1]] - g->h_boff[off[m]]; };
  std::stable_sort(order.begin(), order.end(),
                   [&](uint32_t a, uint32_t b) { return buckets(a) > buckets(b); });
  const size_t nq = order.size();
  std::vector<uint32_t> host(std::max<size_t>(nq, 1) * 5, 0u);
  uint32_t *tab = host.data(), *meta = tab + 4 * nq;
  size_t smem = 0;
  for (size_t i = 0; i < nq; ++i) {
    const uint32_t m = order[i], lo = off[m], hi = off[m + 1];
    tab[4 * i + 0] = lo;
    tab[4 * i + 1] = hi;
    tab[4 * i + 2] = g->h_boff[lo];
    tab[4 * i + 3] = g->h_boff[hi];
    if (h_query[m] == MK_QUERY_BFS) {
      meta[i] = (kStepBfs << 16) | h_src_local[m];
      smem = std::max(smem, bfs_member_smem(hi - lo));
    } else {
      meta[i] = kStepWcc << 16;
      smem = std::max(smem, uf_member_smem(hi - lo));
    }
  }
  MK_CHECK(r->stab.reserve(host.size(), &g->device_bytes));
  MK_CUDA(cudaMemcpy(r->stab.ptr, host.data(), host.size() * 4, cudaMemcpyHostToDevice));
  if (!r->sctl) {
    MK_CUDA(cudaMalloc(&r->sctl, kSCtlWords * 4));
    g->device_bytes += kSCtlWords * 4;
  }
  MK_CUDA(cudaMemset(r->sctl, 0, kSCtlWords * 4));
  auto kern = g->weighted ? k_set_step<true> : k_set_step<false>;
  MK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)bfs_member_smem(kMemLocalMax)));
  r->nq = (uint32_t)nq;
  r->ssmem = smem;
  r->sgrid = persistent_blocks((const void *)kern, kMemThreads, smem, g->device);
  if (r->bfs) {
    // the vertices of members that ask no BFS keep these words
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
  uint32_t max_member = 0;
  for (uint32_t m = 0; m < G; ++m) {
    max_member = std::max(max_member, off[m + 1] - off[m]);
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
  r->max_member = max_member;
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
  if (st == MK_OK && max_member <= kMemLocalMax && !g->reverse) {
    DeviceGuard dg(g->device);
    st = build_single(r, off, h_query, h_bfs_source_local);
  }
  if (st != MK_OK) {
    mk_set_runner_destroy(r);
    return st;
  }
  *out = r;
  return MK_OK;
}

mk_status mk_set_runner_set_single(mk_set_runner *r, uint32_t on) {
  if (!r) return fail(MK_ERR_INVALID, "mk_set_runner_set_single: null handle");
  if (on && !r->sctl)
    return fail(MK_ERR_INVALID, "mk_set_runner_set_single: a member has more than 65535 vertices");
  r->single = on != 0;
  return MK_OK;
}

mk_status mk_set_runner_launches(mk_set_runner *r, uint32_t *h_launches) {
  if (!r || !h_launches) return fail(MK_ERR_INVALID, "mk_set_runner_launches: null argument");
  *h_launches = r->single ? 1u : 2u + (r->bfs ? 1u : 0u) + (r->wcc ? 1u : 0u);
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
  if (r->single) {
    mk_graph *g = r->g;
    DeviceGuard dg(g->device);
    MK_CHECK(g->applied.reserve(std::max<uint32_t>(n_ins, 1), &g->device_bytes));
    // the graph's last update is the insert batch, as after the sequence
    g->last_n = n_ins;
    g->last_src = d_ins_src;
    g->last_dst = d_ins_dst;
    g->last_op = 1;
    TravMemberBufs tb{};
    if (r->bfs) MK_CHECK(trav_member_bufs(r->bfs, &tb));
    StepArgs a;
    a.ds = d_del_src;
    a.dd = d_del_dst;
    a.is = d_ins_src;
    a.id = d_ins_dst;
    a.iw = d_ins_w;
    a.nd = n_del;
    a.ni = n_ins;
    a.tab = reinterpret_cast<const uint4 *>(r->stab.ptr);
    a.meta = r->stab.ptr + 4 * (size_t)r->nq;
    a.nm = r->nq;
    a.ctl = r->sctl;
    a.applied = g->applied.ptr;
    a.count = g->counters;
    a.dist = tb.dist;
    a.items = tb.items;
    a.found = tb.found;
    a.labels = r->wcc ? wcc_label_buf(r->wcc) : nullptr;
    a.limit_ns = g->wait_limit_ns();
    GraphView v = g->view();
    void *args[] = {&v, &a};
    MK_CUDA(cudaMemsetAsync(r->sctl, 0, kSCtlWords * 4, as_stream(stream)));
    const void *fn = g->weighted ? (const void *)k_set_step<true> : (const void *)k_set_step<false>;
    MK_CUDA(cudaLaunchCooperativeKernel(fn, dim3(r->sgrid), dim3(kMemThreads), args, r->ssmem,
                                        as_stream(stream)));
    return MK_OK;
  }
  MK_CHECK(mk_graph_delete_edges(r->g, d_del_src, d_del_dst, n_del, stream));
  MK_CHECK(mk_graph_insert_edges(r->g, d_ins_src, d_ins_dst, d_ins_w, n_ins, stream));
  if (r->bfs) MK_CHECK(mk_bfs_static_members(r->bfs, stream, nullptr));
  if (r->wcc) MK_CHECK(mk_wcc_static_prepared(r->wcc, stream, nullptr));
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
  r->stab.release();
  if (r->sctl) cudaFree(r->sctl);
  delete r;
  return MK_OK;
}

}  // extern "C"
