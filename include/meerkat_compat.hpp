// meerkat_compat.hpp -- header-only C++17 drop-in for the reference's class
// templates (meerkat-pkd/Meerkat include/Graph/SlabGraph.cuh and
// include/Algorithms/*.cuh) on top of the C ABI in meerkat_b200.h.
//
// A reference call site such as src/BFS.cu keeps compiling with only its
// include line changed:
//
//   using AllocPolicy = FullAllocatorPolicy<9, 48, 1>;      // src/BFS.cu:53
//   std::unique_ptr<Allocator> Alloc{new Allocator};
//   DynGraph Graph{VertexN, *Alloc, 0.7, hints.data(), 0};  // src/BFS.cu:58
//   Graph.InsertEdges(SrcDev, DstDev, EdgeN);
//   BFS<AllocPolicy> B(Graph, TheSrc, VertexN);
//   float ms = B.Static(EdgeN);
//   ms = B.Incremental(BatchSrcDev, BatchDstDev, BatchN);
//
// Differences a caller can observe (all deliberate):
//   * errors throw meerkat::Error instead of printing through CHECK_ERROR;
//   * Distances() returns the true uint32 distances (the reference copies
//     4*N bytes of its u64 array, BFS.cuh:55-60);
//   * TC needs a symmetric graph and its Incremental/Decremental return the
//     exact triangle count of the updated graph;
//   * WCC is new (the reference has only the union-find primitives).
#ifndef MEERKAT_COMPAT_HPP_
#define MEERKAT_COMPAT_HPP_

#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "meerkat_b200.h"

namespace meerkat {

struct Error : std::runtime_error {
  mk_status status;
  Error(mk_status s, const std::string &what)
      : std::runtime_error(what + ": " + mk_last_error_string()), status(s) {}
};

inline void check(mk_status s, const char *what) {
  if (s != MK_OK) throw Error(s, what);
}

// Allocator policies (SlabHash's SlabAlloc template parameters, used at
// src/BFS.cu:53 and src/PageRank.cu:32).  Here they only size the overflow
// slab pool: super blocks x 2^LogMemBlocks memory blocks x 1024 slabs.
template <uint32_t LogNumMemBlocks, uint32_t NumSuperBlocks, uint32_t NumReplicas = 1>
struct FullAllocatorPolicy {
  static constexpr uint64_t kPoolSlabs = (uint64_t)NumSuperBlocks << (LogNumMemBlocks + 10);
  struct DynamicAllocatorT {};
  using AllocatorContextT = DynamicAllocatorT;
};
template <uint32_t LogNumMemBlocks, uint32_t NumSuperBlocks, uint32_t NumReplicas = 1>
struct LightAllocatorPolicy {
  static constexpr uint64_t kPoolSlabs = (uint64_t)NumSuperBlocks << (LogNumMemBlocks + 10);
  struct DynamicAllocatorT {};
  using AllocatorContextT = DynamicAllocatorT;
};

// Edge policies (SlabGraph.cuh:92-240): weighted/unweighted x forward/reverse.
template <class AllocPolicy, bool Weighted, bool Reverse>
struct EdgePolicyTag {
  using AllocPolicyT = AllocPolicy;
  using VertexT = uint32_t;
  using EdgeValueT = uint32_t;
  using CountT = uint32_t;
  static constexpr bool IsWeightedEdge = Weighted;
  static constexpr bool IsReverse = Reverse;
};
template <class AP, class V = uint32_t, class C = uint32_t>
using UnweightedEdgePolicyT = EdgePolicyTag<AP, false, false>;
template <class AP, class V = uint32_t, class C = uint32_t>
using RevUnweightedEdgePolicyT = EdgePolicyTag<AP, false, true>;
template <class AP, class V = uint32_t, class E = uint32_t, class C = uint32_t>
using WeightedEdgePolicyMapT = EdgePolicyTag<AP, true, false>;
template <class AP, class V = uint32_t, class E = uint32_t, class C = uint32_t>
using RevWeightedEdgePolicyMapT = EdgePolicyTag<AP, true, true>;
template <class AP, class V = uint32_t, class E = uint32_t, class C = uint32_t>
using WeightedEdgePolicyPCMapT = EdgePolicyTag<AP, true, false>;

// DynamicGraph<EdgePolicy, IsWeighted> (SlabGraph.cuh:343-506, :508-752).
template <class EdgePolicy, bool IsWeighted = EdgePolicy::IsWeightedEdge>
class DynamicGraph {
 public:
  using EdgePolicyT = EdgePolicy;
  using VertexT = uint32_t;
  using EdgeValueT = uint32_t;
  using CountT = uint32_t;
  using EdgeDynAllocator = typename EdgePolicy::AllocPolicyT::DynamicAllocatorT;

  DynamicGraph(uint32_t N, EdgeDynAllocator &, double LoadFactor, uint32_t *VertexDegreeHints,
               uint32_t DeviceIdx = 0)
      : N_(N) {
    mk_graph_desc d{};
    d.num_vertices = N;
    d.weighted = IsWeighted ? 1u : 0u;
    d.reverse = EdgePolicy::IsReverse ? 1u : 0u;
    d.load_factor = LoadFactor;
    d.h_degree_hints = VertexDegreeHints;
    d.device = (int32_t)DeviceIdx;
    d.pool_slabs = EdgePolicy::AllocPolicyT::kPoolSlabs;
    check(mk_graph_create(&d, &g_), "DynamicGraph");
    offsets_.resize(N);
    buckets_.resize(N);
    check(mk_graph_bucket_layout(g_, offsets_.data(), buckets_.data()), "DynamicGraph");
  }
  DynamicGraph(const DynamicGraph &) = delete;
  DynamicGraph &operator=(const DynamicGraph &) = delete;
  ~DynamicGraph() { mk_graph_destroy(g_); }

  // InsertEdges(src*, dst*, n[, vals*]) -- asynchronous on the default stream.
  void InsertEdges(VertexT *Src, VertexT *Dst, CountT N, EdgeValueT *Vals = nullptr) {
    check(mk_graph_insert_edges(g_, Src, Dst, Vals, N, nullptr), "InsertEdges");
  }
  void DeleteEdges(VertexT *Src, VertexT *Dst, CountT N) {
    check(mk_graph_delete_edges(g_, Src, Dst, N, nullptr), "DeleteEdges");
  }
  // UpdateSlabPointers (SlabGraph.cuh:493): the reference never calls it and
  // this layout keeps no per-bucket update cursor, so it is a no-op.
  void UpdateSlabPointers() {}

  uint32_t *GetVertexBucketsOffsets() { return offsets_.data(); }
  uint32_t *GetBucketsPerVertex() { return buckets_.data(); }
  uint32_t NumVertices() const { return N_; }
  mk_graph *handle() const { return g_; }
  // Waits for queued updates and raises on a device-side error.
  void Sync() { check(mk_graph_sync(g_, nullptr, nullptr), "Sync"); }

 private:
  uint32_t N_;
  mk_graph *g_ = nullptr;
  std::vector<uint32_t> offsets_, buckets_;
};

template <class EdgePolicy>
using DynGraph = DynamicGraph<EdgePolicy, EdgePolicy::IsWeightedEdge>;

namespace detail {
class Traversal {
 public:
  Traversal(mk_graph *g, uint32_t src, uint32_t N, bool sssp) : N_(N) {
    check(sssp ? mk_sssp_create(g, src, &t_) : mk_bfs_create(g, src, &t_),
          sssp ? "SSSP" : "BFS");
  }
  Traversal(const Traversal &) = delete;
  ~Traversal() { mk_traversal_destroy(t_); }
  float Static(uint32_t) {
    float ms = 0;
    check(mk_traversal_static(t_, nullptr, &ms), "Static");
    return ms;
  }
  float Incremental(uint32_t *S, uint32_t *D, uint32_t *W, uint32_t n) {
    float ms = 0;
    check(mk_traversal_incremental(t_, S, D, W, n, nullptr, &ms), "Incremental");
    return ms;
  }
  float Decremental(uint32_t *S, uint32_t *D, uint32_t *W, uint32_t n) {
    float ms = 0;
    check(mk_traversal_decremental(t_, S, D, W, n, nullptr, &ms), "Decremental");
    return ms;
  }
  std::vector<uint32_t> Distances() {
    std::vector<uint32_t> out(N_);
    check(mk_traversal_distances(t_, out.data()), "Distances");
    return out;
  }
  // Extension (no counterpart in the reference): attaches the reverse graph
  // of the same edges (a DynGraph with a Rev*EdgePolicy, weighted for SSSP),
  // which the caller updates with every batch; decremental calls then repair
  // from in-edges (mk_traversal_set_reverse).
  template <class RevGraph>
  void SetReverse(RevGraph &Gr) {
    check(mk_traversal_set_reverse(t_, Gr.handle()), "SetReverse");
  }

 private:
  uint32_t N_;
  mk_traversal *t_ = nullptr;
};
}  // namespace detail

// BFS<AllocPolicy> (include/Algorithms/BFS.cuh:13-69).
template <class AllocPolicy>
struct BFS : detail::Traversal {
  using GraphT = DynGraph<UnweightedEdgePolicyT<AllocPolicy>>;
  BFS(GraphT &G, uint32_t Src, uint32_t N) : detail::Traversal(G.handle(), Src, N, false) {}
  float Incremental(uint32_t *S, uint32_t *D, uint32_t n) {
    return detail::Traversal::Incremental(S, D, nullptr, n);
  }
  float Decremental(uint32_t *S, uint32_t *D, uint32_t n) {
    return detail::Traversal::Decremental(S, D, nullptr, n);
  }
};

// SSSP<AllocPolicy> (include/Algorithms/SSSP.cuh:11-69).
template <class AllocPolicy>
struct SSSP : detail::Traversal {
  using GraphT = DynGraph<WeightedEdgePolicyMapT<AllocPolicy>>;
  SSSP(GraphT &G, uint32_t Src, uint32_t N) : detail::Traversal(G.handle(), Src, N, true) {}
};

// PageRank<AllocPolicy> (include/Algorithms/PageRank.cuh:9-67).
template <class AllocPolicy>
class PageRank {
 public:
  using GraphT = DynGraph<RevUnweightedEdgePolicyT<AllocPolicy>>;
  PageRank(GraphT &G, float DampingFactor, float ErrorMargin, uint32_t VertexN,
           uint32_t *VertexOutDegree, uint32_t MaxIter = 100)
      : N_(VertexN) {
    check(mk_pagerank_create(G.handle(), DampingFactor, ErrorMargin, MaxIter, VertexOutDegree,
                             &p_),
          "PageRank");
  }
  PageRank(const PageRank &) = delete;
  ~PageRank() { mk_pagerank_destroy(p_); }
  float Static() {
    float ms = 0;
    check(mk_pagerank_static(p_, nullptr, &ms), "Static");
    return ms;
  }
  float Incremental(uint32_t *S, uint32_t *D, uint32_t n) {
    float ms = 0;
    check(mk_pagerank_incremental(p_, S, D, n, nullptr, &ms), "Incremental");
    return ms;
  }
  float Decremental(uint32_t *S, uint32_t *D, uint32_t n) {
    float ms = 0;
    check(mk_pagerank_decremental(p_, S, D, n, nullptr, &ms), "Decremental");
    return ms;
  }
  std::vector<float> Values() {
    std::vector<float> out(N_);
    check(mk_pagerank_values(p_, out.data()), "Values");
    return out;
  }

 private:
  uint32_t N_;
  mk_pagerank *p_ = nullptr;
};

// TC<AllocPolicy> (include/Algorithms/TC.cuh:9-40).
template <class AllocPolicy>
class TC {
 public:
  using GraphT = DynGraph<UnweightedEdgePolicyT<AllocPolicy>>;
  using Allocator = typename AllocPolicy::DynamicAllocatorT;
  TC(GraphT &G, uint32_t) { check(mk_tc_create(G.handle(), &t_), "TC"); }
  TC(const TC &) = delete;
  ~TC() { mk_tc_destroy(t_); }
  unsigned long long GetCount() const {
    uint64_t c = 0;
    check(mk_tc_count(t_, &c), "GetCount");
    return c;
  }
  float Static(uint32_t) {
    float ms = 0;
    check(mk_tc_static(t_, nullptr, &ms), "Static");
    return ms;
  }
  float Incremental(uint32_t *S, uint32_t *D, uint32_t n, std::unique_ptr<Allocator> &) {
    float ms = 0;
    check(mk_tc_incremental(t_, S, D, n, nullptr, &ms), "Incremental");
    return ms;
  }
  float Decremental(uint32_t *S, uint32_t *D, uint32_t n, std::unique_ptr<Allocator> &) {
    float ms = 0;
    check(mk_tc_decremental(t_, S, D, n, nullptr, &ms), "Decremental");
    return ms;
  }

 private:
  mk_tc *t_ = nullptr;
};

// Connected components (new; union-find semantics of include/Util/UnionFind.cuh).
template <class AllocPolicy, class EdgePolicy = UnweightedEdgePolicyT<AllocPolicy>>
class WCC {
 public:
  using GraphT = DynGraph<EdgePolicy>;
  WCC(GraphT &G, uint32_t N) : N_(N) { check(mk_wcc_create(G.handle(), &w_), "WCC"); }
  WCC(const WCC &) = delete;
  ~WCC() { mk_wcc_destroy(w_); }
  float Static() {
    float ms = 0;
    check(mk_wcc_static(w_, nullptr, &ms), "Static");
    return ms;
  }
  float Incremental(uint32_t *S, uint32_t *D, uint32_t n) {
    float ms = 0;
    check(mk_wcc_incremental(w_, S, D, n, nullptr, &ms), "Incremental");
    return ms;
  }
  float Decremental(uint32_t *S, uint32_t *D, uint32_t n) {
    float ms = 0;
    check(mk_wcc_decremental(w_, S, D, n, nullptr, &ms), "Decremental");
    return ms;
  }
  std::vector<uint32_t> Labels() {
    std::vector<uint32_t> out(N_);
    check(mk_wcc_labels(w_, out.data()), "Labels");
    return out;
  }
  // Extension: attaches the reverse graph of the same edges, which the
  // caller updates with every batch; static calls then scan only the edges
  // of the vertices outside the largest sampled set, decremental calls only
  // the pieces a deletion split off (mk_wcc_set_reverse).
  template <class RevGraph>
  void SetReverse(RevGraph &Gr) {
    check(mk_wcc_set_reverse(w_, Gr.handle()), "SetReverse");
  }

 private:
  uint32_t N_;
  mk_wcc *w_ = nullptr;
};

// Many small dynamic graphs stored and updated as one (mk_graphset_*), and
// the batched step over them (mk_set_runner_*): no counterpart in the
// reference, whose drivers hold one graph per process.  Member m owns the
// union vertex ids [Offsets()[m], Offsets()[m + 1]).
class GraphSet {
 public:
  GraphSet(const std::vector<uint32_t> &num_vertices, bool weighted, int device = 0,
           double load_factor = 0.7, const std::vector<const uint32_t *> *hints = nullptr,
           uint64_t pool_slabs = 0) {
    check(mk_graphset_create((uint32_t)num_vertices.size(), num_vertices.data(),
                             hints ? hints->data() : nullptr, load_factor, weighted ? 1u : 0u,
                             device, pool_slabs, &s_),
          "GraphSet");
  }
  GraphSet(const GraphSet &) = delete;
  ~GraphSet() { mk_graphset_destroy(s_); }
  mk_graphset *handle() const { return s_; }
  mk_graph *Union() const {
    mk_graph *g = nullptr;
    check(mk_graphset_union(s_, &g), "Union");
    return g;
  }
  std::vector<uint32_t> Offsets() const {
    uint32_t n = 0;
    check(mk_graphset_num_graphs(s_, &n), "Offsets");
    std::vector<uint32_t> off(n + 1);
    check(mk_graphset_offsets(s_, off.data()), "Offsets");
    return off;
  }
  // Device batches with union vertex ids, stream-ordered.
  void InsertEdges(const uint32_t *S, const uint32_t *D, uint32_t n, const uint32_t *W = nullptr,
                   void *stream = nullptr) {
    check(mk_graph_insert_edges(Union(), S, D, W, n, stream), "InsertEdges");
  }
  void DeleteEdges(const uint32_t *S, const uint32_t *D, uint32_t n, void *stream = nullptr) {
    check(mk_graph_delete_edges(Union(), S, D, n, stream), "DeleteEdges");
  }

 private:
  mk_graphset *s_ = nullptr;
};

class GraphSetRunner {
 public:
  // query[m]: MK_QUERY_BFS / MK_QUERY_WCC / MK_QUERY_NONE; bfs_source[m]:
  // local source of a BFS member.
  GraphSetRunner(GraphSet &set, const std::vector<uint8_t> &query,
                 const std::vector<uint32_t> &bfs_source) {
    check(mk_set_runner_create(set.handle(), query.data(),
                               bfs_source.empty() ? nullptr : bfs_source.data(), &r_),
          "GraphSetRunner");
  }
  GraphSetRunner(const GraphSetRunner &) = delete;
  ~GraphSetRunner() { mk_set_runner_destroy(r_); }
  uint32_t LaunchesPerStep() const {
    uint32_t n = 0;
    check(mk_set_runner_launches(r_, &n), "LaunchesPerStep");
    return n;
  }
  // One cooperative launch per step from now on (members of at most 65,535
  // vertices); false: four launches.
  void SetSingle(bool on) { check(mk_set_runner_set_single(r_, on ? 1u : 0u), "SetSingle"); }
  // One step: the deletes, the inserts, every member's query (asynchronous).
  void Step(const uint32_t *dS, const uint32_t *dD, uint32_t nDel, const uint32_t *iS,
            const uint32_t *iD, const uint32_t *iW, uint32_t nIns, void *stream = nullptr) {
    check(mk_set_runner_step(r_, dS, dD, nDel, iS, iD, iW, nIns, stream), "Step");
  }
  const uint64_t *BfsPacked() const {
    const uint64_t *p = nullptr;
    check(mk_set_runner_results(r_, &p, nullptr), "BfsPacked");
    return p;
  }
  const uint32_t *WccLabels() const {
    const uint32_t *p = nullptr;
    check(mk_set_runner_results(r_, nullptr, &p), "WccLabels");
    return p;
  }

 private:
  mk_set_runner *r_ = nullptr;
};

// The reference drivers' input files (src/BFS.cu:27-36, :76-91): a graph
// file "V E" + E pairs, and update batches "<prefix>.batch.<i>".
struct EdgeList {
  uint32_t num_vertices = 0;
  std::vector<uint32_t> src, dst;
};

inline EdgeList ReadGraphFile(const std::string &path) {
  EdgeList e;
  uint64_t n = 0;
  check(mk_read_edge_list(path.c_str(), &e.num_vertices, &n, nullptr, nullptr), "ReadGraphFile");
  e.src.resize(n);
  e.dst.resize(n);
  check(mk_read_edge_list(path.c_str(), &e.num_vertices, &n, e.src.data(), e.dst.data()),
        "ReadGraphFile");
  return e;
}

inline EdgeList ReadBatchFile(const std::string &prefix, uint32_t index) {
  const std::string path = prefix + ".batch." + std::to_string(index);
  EdgeList e;
  uint64_t n = 0;
  check(mk_read_batch_file(path.c_str(), &n, nullptr, nullptr), "ReadBatchFile");
  e.src.resize(n);
  e.dst.resize(n);
  check(mk_read_batch_file(path.c_str(), &n, e.src.data(), e.dst.data()), "ReadBatchFile");
  return e;
}

}  // namespace meerkat

#ifndef MEERKAT_COMPAT_NO_GLOBAL_NAMES
// The reference declares these at global scope.
using meerkat::BFS;
using meerkat::DynamicGraph;
using meerkat::DynGraph;
using meerkat::FullAllocatorPolicy;
using meerkat::LightAllocatorPolicy;
using meerkat::PageRank;
using meerkat::RevUnweightedEdgePolicyT;
using meerkat::RevWeightedEdgePolicyMapT;
using meerkat::SSSP;
using meerkat::TC;
using meerkat::UnweightedEdgePolicyT;
using meerkat::WCC;
using meerkat::WeightedEdgePolicyMapT;
using meerkat::WeightedEdgePolicyPCMapT;
#endif

#endif  // MEERKAT_COMPAT_HPP_
