/*
 * meerkat_b200.h -- C ABI of the B200-native dynamic-graph engine.
 *
 * Every entry point takes plain pointers and sizes.  Pointers named d_* are
 * device pointers, h_* are host pointers.  `stream` is a cudaStream_t passed
 * as void* (NULL = legacy default stream) so this header needs no CUDA
 * include.  Calls are stream-ordered and asynchronous unless they take a
 * `float *ms_out`: when ms_out is non-NULL the call synchronises and writes
 * the elapsed device time of its kernels in milliseconds (the reference's
 * algorithm calls return that float).
 *
 * Each declaration cites the reference interface it replaces
 * (path:line inside meerkat-pkd/Meerkat).
 */
#ifndef MEERKAT_B200_H_
#define MEERKAT_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Slab word sentinels.  Vertex ids must be < MK_TOMBSTONE_KEY. */
#define MK_EMPTY_KEY 0xFFFFFFFFu
#define MK_TOMBSTONE_KEY 0xFFFFFFFEu
#define MK_EMPTY_SLAB 0xFFFFFFFFu
/* Unreachable distance (reference: INF, include/Algorithms/definitions.cuh:4). */
#define MK_INF 0xFFFFFFFFu
/* Packed distance/parent word: dist << 32 | parent
 * (reference: PACK/DISTANCE/PARENT, include/Algorithms/definitions.cuh:14-17). */
#define MK_INFINF 0xFFFFFFFFFFFFFFFFull

typedef enum mk_status {
  MK_OK = 0,
  MK_ERR_INVALID = 1, /* bad argument or out-of-range vertex id in a batch  */
  MK_ERR_OOM = 2,     /* slab pool or device memory exhausted              */
  MK_ERR_TIMEOUT = 3, /* a bounded device-side wait gave up                */
  MK_ERR_CUDA = 4,    /* a CUDA runtime call failed                        */
  MK_ERR_STATE = 5    /* call made in the wrong state (e.g. before Static) */
} mk_status;

/* Sticky device error bits reported by mk_graph_sync / mk_*_sync. */
#define MK_DEVERR_INVALID_ID 0x1u
#define MK_DEVERR_OOM 0x2u
#define MK_DEVERR_TIMEOUT 0x4u
#define MK_DEVERR_OVERFLOW 0x8u

/* Message of the last failing call on this host thread. */
const char *mk_last_error_string(void);
/* Library version string. */
const char *mk_version(void);

/* ------------------------------------------------------------------------
 * Dynamic graph: per-vertex slab hash tables of 128-byte slabs.
 * Replaces DynamicGraph<EdgePolicy, IsWeighted>
 * (include/Graph/SlabGraph.cuh:343-506 weighted, :508-752 unweighted).
 * ---------------------------------------------------------------------- */
typedef struct mk_graph mk_graph;

typedef struct mk_graph_desc {
  uint32_t num_vertices;  /* N (reference ctor arg, SlabGraph.cuh:382)        */
  uint32_t weighted;      /* 1 = (key, value) slabs: WeightedEdgePolicyMapT    */
  uint32_t reverse;       /* 1 = edges keyed by destination: Rev*EdgePolicyT   */
  uint32_t flags;         /* reserved, must be 0                               */
  double load_factor;     /* LoadFactor (SlabGraph.cuh:403-407), e.g. 0.7      */
  const uint32_t *h_degree_hints; /* VertexDegreeHints[N] or NULL (= all 1)    */
  int32_t device;         /* DeviceIdx                                         */
  uint32_t pad0;
  uint64_t pool_slabs;    /* overflow slab capacity; 0 = automatic             */
} mk_graph_desc;

typedef struct mk_graph_info {
  uint32_t num_vertices;
  uint32_t weighted;
  uint32_t reverse;
  uint32_t keys_per_slab;  /* 31 (set) or 15 (map)                      */
  uint64_t num_buckets;    /* head slabs                                */
  uint64_t pool_capacity;  /* head + overflow slabs                     */
  uint64_t slabs_used;     /* head + allocated overflow slabs           */
  uint64_t num_edges;      /* live edges = sum of degrees               */
  uint64_t device_bytes;   /* bytes of device memory held by the graph  */
} mk_graph_info;

/* DynamicGraph(N, Allocator&, LoadFactor, DegreeHints*, DeviceIdx)
 * (SlabGraph.cuh:382-466, :633-717). */
mk_status mk_graph_create(const mk_graph_desc *desc, mk_graph **out);
/* ~DynamicGraph (SlabGraph.cuh:470-480). */
mk_status mk_graph_destroy(mk_graph *g);

/* InsertEdges(src*, dst*, n, vals*) (SlabGraph.cuh:486-488, impl
 * SlabGraphImpl.cuh:6-34).  Self-loops are skipped (InsertEdgeKernel.cuh:25).
 * Set semantics: a live edge is never duplicated; on weighted graphs its
 * stored weight becomes the minimum of the live weight and every inserted copy
 * (upsert-min), which is independent of the order of concurrent inserts.  An
 * entry counts as applied only when it adds a new edge.  d_w may be NULL
 * (weight 0) and is ignored for unweighted graphs. */
mk_status mk_graph_insert_edges(mk_graph *g, const uint32_t *d_src,
                                const uint32_t *d_dst, const uint32_t *d_w,
                                uint32_t n, void *stream);
/* DeleteEdges(src*, dst*, n) (SlabGraph.cuh:490-491, SlabGraphImpl.cuh:36-62).
 * A live edge becomes a tombstone; absent edges and self-loops are no-ops. */
mk_status mk_graph_delete_edges(mk_graph *g, const uint32_t *d_src,
                                const uint32_t *d_dst, uint32_t n,
                                void *stream);
/* Batched SearchEdge (include/Graph/warp/SearchEdge.cuh:8-63, :118-142):
 * d_found[i] = 1 if (src[i], dst[i]) is live; d_w[i] = its value (may be NULL). */
mk_status mk_graph_search_edges(mk_graph *g, const uint32_t *d_src,
                                const uint32_t *d_dst, uint32_t n,
                                uint8_t *d_found, uint32_t *d_w, void *stream);
/* Waits for the graph's work on `stream`, returns MK_OK or the first error and
 * writes the sticky device error bits (MK_DEVERR_*) to *h_deverr if given. */
mk_status mk_graph_sync(mk_graph *g, void *stream, uint32_t *h_deverr);
/* Stream-ordered copy of the slabs in use (head + allocated overflow slabs,
 * mk_graph_info.slabs_used; capacity: pool_capacity) into *h_slabs_used
 * (pinned host memory for an asynchronous copy).  A server admits inserts
 * against it: an insert of n edges needs at most n new slabs.  No
 * counterpart in the reference, which has no OOM reporting. */
mk_status mk_graph_slabs_used_async(mk_graph *g, uint32_t *h_slabs_used, void *stream);
/* Number of batch edges the last insert/delete actually applied (synchronises). */
mk_status mk_graph_last_applied(mk_graph *g, uint64_t *h_count);
/* Stream-ordered copy of the same count into h_count (pinned host memory for
 * a truly asynchronous copy): it lands once the update before it on `stream`
 * has finished.  No counterpart in the reference. */
mk_status mk_graph_last_applied_async(mk_graph *g, uint64_t *h_count, void *stream);
/* Device pointer to the per-edge applied flags (uint8, one per batch entry)
 * of the last insert/delete; valid until the next update call. */
mk_status mk_graph_last_applied_flags(mk_graph *g, const uint8_t **d_flags,
                                      uint32_t *n);
/* Vertex degrees: GetVertexDegrees (SlabGraph.cuh:303-305). */
mk_status mk_graph_degrees(mk_graph *g, uint32_t *d_out, void *stream);
/* GetVertexBucketsOffsets / GetBucketsPerVertex (SlabGraph.cuh:483-484):
 * host copies, N entries each (either pointer may be NULL). */
mk_status mk_graph_bucket_layout(mk_graph *g, uint32_t *h_offsets,
                                 uint32_t *h_buckets_per_vertex);
mk_status mk_graph_get_info(mk_graph *g, mk_graph_info *out);
/* Compacts live edges into CSR (row_ptr has N+1 entries; rows in slab order).
 * Mirrors CollectEdges (include/Algorithms/impl/TCImpl.cuh:110-147) and the
 * test kernels CollectEdges (test/GraphTest.cu:285-346).  d_col and d_w need
 * room for num_edges entries; d_w may be NULL. */
mk_status mk_graph_export_csr(mk_graph *g, uint64_t *d_row_ptr,
                              uint32_t *d_col, uint32_t *d_w, void *stream);
/* Live edges of the vertices [v_begin, v_end) (sum of their degrees);
 * synchronises the stream.  No counterpart in the reference. */
mk_status mk_graph_count_edges_range(mk_graph *g, uint32_t v_begin, uint32_t v_end,
                                     void *stream, uint64_t *h_count);
/* CSR of the rows [v_begin, v_end) only: d_row_ptr gets v_end - v_begin + 1
 * offsets starting at 0, d_col / d_w (may be NULL) the edges of those rows
 * (room for mk_graph_count_edges_range of the range).  Column ids stay
 * global.  Exports one member of a graph set without touching the others;
 * no counterpart in the reference. */
mk_status mk_graph_export_csr_range(mk_graph *g, uint32_t v_begin, uint32_t v_end,
                                    uint64_t *d_row_ptr, uint32_t *d_col,
                                    uint32_t *d_w, void *stream);
/* Same output as mk_graph_export_csr, for callers that must not allocate
 * device memory after start-up (no counterpart in the reference).  The
 * plain export grows its scratch with cudaMalloc, which synchronises the
 * whole device and fails once a pool has taken the free memory; this one
 * calls no allocator: its scratch is one fixed array of about 3 MiB inside
 * the library, shared by every call on a device.
 *   - Limit: graphs of at most 262,144 buckets (num_buckets of
 *     mk_graph_get_info); larger graphs get MK_ERR_INVALID.
 *   - The first call on each device looks the array up and may load the
 *     library's device code; make that first call before any stream capture.
 *   - Calls that overlap in time on one device (different streams, or
 *     host threads) race on the shared scratch: order them on one stream.
 *   - The array's device address is looked up once per device and kept; a
 *     cudaDeviceReset of that device invalidates it, so do not call this
 *     entry point on a device after resetting it in the same process.
 *   - Like the plain export it does not read the graph's sticky error word:
 *     an update that ran out of slab pool drops edges, so check
 *     mk_graph_sync before exporting. */
mk_status mk_graph_export_csr_noalloc(mk_graph *g, uint64_t *d_row_ptr,
                                      uint32_t *d_col, uint32_t *d_w,
                                      void *stream);
/* Per-vertex tombstone count (test/GraphTest.cu:58-95 CountTombstones). */
mk_status mk_graph_count_tombstones(mk_graph *g, uint32_t *d_out,
                                    void *stream);
/* Pre-sizes the per-batch scratch for batches of up to n edges so later
 * updates of that size allocate nothing. */
mk_status mk_graph_reserve_batch(mk_graph *g, uint32_t n);

/* Kernel choices of the update path (no counterpart in the reference, which
 * has a single insert/delete kernel).  The autotuner in
 * meerkat_b200/autotune.py measures the variants on live batches. */
typedef struct mk_tuning {
  uint32_t update_kernel;        /* 0 = warp-staged (TMA bulk copies into shared
                                    memory), 1 = one lane per edge,
                                    2 = warp-cooperative coalesced slab loads  */
  uint32_t update_blocks_per_sm; /* resident blocks per SM, 0 = automatic     */
  uint32_t frontier_chunk;       /* buckets per BFS/SSSP frontier work item,
                                    1..1024, 0 = 4                            */
  uint32_t sssp_delta;           /* static SSSP near-far step: relaxations to
                                    distances >= threshold wait on a far list
                                    until the near frontier drains; 0 = off
                                    (plain level-synchronous)                  */
  uint32_t recompute_permille;   /* decremental BFS/SSSP: once this share of
                                    the vertices (per mille) is invalidated,
                                    recompute from the sources instead of
                                    repairing; 0 = never                       */
  uint32_t pull_permille;        /* static BFS with a reverse graph attached
                                    (mk_traversal_set_reverse): a level whose
                                    frontier holds this share of the vertices
                                    (per mille) is pulled bottom-up; 0 = never */
  uint32_t wait_limit_us;        /* limit of every grid-barrier wait of the
                                    persistent kernels launched on this graph
                                    (BFS/SSSP traversals; PageRank on this
                                    reverse graph), microseconds; 0 = 4 s.  A
                                    wait past it ends the launch: every block
                                    leaves and MK_ERR_TIMEOUT is reported (by
                                    a timed call or a PageRank solve at once,
                                    else by mk_traversal_distances / _stats);
                                    that call's results stay undefined until
                                    the next Static.  Replaces the reference's
                                    unbounded spins
                                    (include/Util/Lock.cuh:43-56).             */
  uint32_t reserved;
} mk_tuning;
mk_status mk_graph_set_tuning(mk_graph *g, const mk_tuning *t);
mk_status mk_graph_get_tuning(mk_graph *g, mk_tuning *t);

/* ------------------------------------------------------------------------
 * BFS and SSSP (replace BFS<AllocPolicy>, include/Algorithms/BFS.cuh:13-69,
 * and SSSP<AllocPolicy>, include/Algorithms/SSSP.cuh:11-69).  A BFS may run
 * on a weighted graph (weights ignored).  SSSP needs a weighted graph.
 * Call protocol as in the reference drivers (src/BFS.cu:111-121): update the
 * graph first, then call Incremental/Decremental with the same batch.
 * ---------------------------------------------------------------------- */
typedef struct mk_traversal mk_traversal;

/* BFS(G, SourceVertex, VertexN) (BFS.cuh:34-53); sets dist[src] = 0. */
mk_status mk_bfs_create(mk_graph *g, uint32_t source, mk_traversal **out);
/* SSSP(G, SourceVertex, VertexN) (SSSP.cuh:33-52). */
mk_status mk_sssp_create(mk_graph *g, uint32_t source, mk_traversal **out);
/* One traversal from several distinct sources at once (no counterpart in the
 * reference): every vertex gets its distance from the nearest source.  On a
 * graph set (below) with one source per member graph this runs one query per
 * member in a single launch.  h_sources is host memory; repeated or
 * out-of-range sources are rejected. */
mk_status mk_bfs_create_multi(mk_graph *g, const uint32_t *h_sources, uint32_t n,
                              mk_traversal **out);
mk_status mk_sssp_create_multi(mk_graph *g, const uint32_t *h_sources, uint32_t n,
                               mk_traversal **out);
/* Replaces the source set (h_sources: n distinct vertices, host memory) of a
 * BFS or SSSP; the next call must be mk_traversal_static.  Lets a server run
 * one multi-source query per round with one resident traversal.  No
 * counterpart in the reference. */
mk_status mk_traversal_set_sources(mk_traversal *t, const uint32_t *h_sources, uint32_t n);
/* Stream-ordered form of mk_traversal_set_sources: the new sources reach the
 * device on `stream`, after the launches queued there before the call, and
 * the call waits for no other device work (a server issues its rounds
 * without stalling on another stream).  The traversal must not have work in
 * flight on any other stream.  Growing past the largest source count seen
 * synchronises the device once. */
mk_status mk_traversal_set_sources_async(mk_traversal *t, const uint32_t *h_sources, uint32_t n,
                                         void *stream);
/* Attaches the reverse graph (in-edges) of the same edge set (for SSSP:
 * weighted, with the same weights): static BFS pulls large levels
 * (tuning.pull_permille), and decremental BFS/SSSP re-seed invalidated
 * vertices from their own in-edges instead of sweeping every bucket.  The
 * caller keeps both graphs updated with the same batches.  NULL detaches.
 * No counterpart in the reference. */
mk_status mk_traversal_set_reverse(mk_traversal *t, mk_graph *g_rev);
/* float Static(EdgesN) (BFSImpl.cuh:590-662, SSSPImpl.cuh:607-690). */
mk_status mk_traversal_static(mk_traversal *t, void *stream, float *ms_out);
/* Static BFS of a multi-source traversal whose sources each lie in their own
 * vertex range, each range closed under edges (members of a graph set):
 * range i = [r[2i], r[2i+1]) holds source i.  prepare uploads the table
 * (blocking; it waits for the device, since queued work may read the
 * previous table); static_members runs it and issues only asynchronous work
 * on `stream`, so it can be captured into a CUDA graph.  A range of at most
 * 65,535 vertices is solved by one CTA with its BFS state in shared memory;
 * larger ones by the device-wide kernel.  The distances of every vertex are
 * those mk_traversal_static gives and the parents form a valid BFS tree
 * (parents are not unique: of several equal-distance parents, the device-wide
 * kernel keeps the first to arrive, the member kernel the smallest id); an
 * edge leaving its range sets MK_DEVERR_INVALID_ID on the graph.  BFS only.
 * No counterpart in the reference. */
mk_status mk_bfs_prepare_members(mk_traversal *t, const uint32_t *h_vertex_ranges,
                                 uint32_t nranges);
mk_status mk_bfs_static_members(mk_traversal *t, void *stream, float *ms_out);
/* float Incremental(src*, dst*, n) (BFSImpl.cuh:664-753, SSSPImpl.cuh:692-785).
 * d_w is accepted for the SSSP signature and ignored: the stored weight of
 * each edge is used. */
mk_status mk_traversal_incremental(mk_traversal *t, const uint32_t *d_src,
                                   const uint32_t *d_dst, const uint32_t *d_w,
                                   uint32_t n, void *stream, float *ms_out);
/* float Decremental(src*, dst*, n) (BFSImpl.cuh:755-846, SSSPImpl.cuh:787-876). */
mk_status mk_traversal_decremental(mk_traversal *t, const uint32_t *d_src,
                                   const uint32_t *d_dst, const uint32_t *d_w,
                                   uint32_t n, void *stream, float *ms_out);
/* Distances() (BFS.cuh:55-60): N distances, MK_INF = unreachable (host). */
mk_status mk_traversal_distances(mk_traversal *t, uint32_t *h_out);
/* Device pointer to the packed dist<<32|parent array (N entries). */
mk_status mk_traversal_packed(mk_traversal *t, const uint64_t **d_packed);
/* Host copy of the packed array (N entries). */
mk_status mk_traversal_packed_host(mk_traversal *t, uint64_t *h_out);
/* Work counters of the last call: levels run and vertices pushed. */
mk_status mk_traversal_stats(mk_traversal *t, uint32_t *h_levels,
                             uint64_t *h_pushed);
/* Repair counters of the last call when it was a Decremental: vertices whose
 * subtree was invalidated (when the call recomputed, the count at which the
 * invalidation walk stopped, tuning.recompute_permille of V) and whether it
 * recomputed from the sources (1) instead of repairing (0).  No counterpart
 * in the reference, whose Decremental (BFSImpl.cuh:755-846) always repairs. */
mk_status mk_traversal_decremental_stats(mk_traversal *t, uint64_t *h_invalidated,
                                         uint32_t *h_recomputed);
mk_status mk_traversal_destroy(mk_traversal *t);

/* ------------------------------------------------------------------------
 * PageRank (replaces PageRank<AllocPolicy>, include/Algorithms/PageRank.cuh:9-67).
 * g must be a reverse graph (in-edges), as RevUnweightedEdgePolicyT in the
 * reference.  h_out_degree (N entries) may be NULL: out-degrees are then
 * counted from the graph.
 * ---------------------------------------------------------------------- */
typedef struct mk_pagerank mk_pagerank;

/* PageRank(G, DampingFactor, ErrorMargin, VertexN, OutDeg*, MaxIter)
 * (PageRank.cuh:32-46). */
mk_status mk_pagerank_create(mk_graph *g_rev, float damping, float tol,
                             uint32_t max_iter, const uint32_t *h_out_degree,
                             mk_pagerank **out);
/* float Static() (PageRankImpl.cuh:218-220). */
mk_status mk_pagerank_static(mk_pagerank *p, void *stream, float *ms_out);
/* Static after out-degrees are recounted from the graph: for a graph that
 * was updated without passing the batches to Incremental/Decremental (a
 * server's cached view).  No counterpart in the reference. */
mk_status mk_pagerank_static_recount(mk_pagerank *p, void *stream, float *ms_out);
/* float Incremental/Decremental(src*, dst*, n) (PageRankImpl.cuh:222-251):
 * out-degrees follow the edges the last graph update applied, then the
 * ranks are re-solved warm-started from the previous ranks. */
mk_status mk_pagerank_incremental(mk_pagerank *p, const uint32_t *d_src,
                                  const uint32_t *d_dst, uint32_t n,
                                  void *stream, float *ms_out);
mk_status mk_pagerank_decremental(mk_pagerank *p, const uint32_t *d_src,
                                  const uint32_t *d_dst, uint32_t n,
                                  void *stream, float *ms_out);
/* Values() (PageRank.cuh:48-53), host. */
mk_status mk_pagerank_values(mk_pagerank *p, float *h_out);
mk_status mk_pagerank_values_device(mk_pagerank *p, const float **d_values);
/* Iterations run and the final L1 change of the last solve. */
mk_status mk_pagerank_stats(mk_pagerank *p, uint32_t *h_iters,
                            float *h_delta);
mk_status mk_pagerank_destroy(mk_pagerank *p);

/* PageRank of one vertex range of an OUT-edge graph (a graph-set member),
 * push form, FP64 accumulation: no reverse graph needed.  Same formula,
 * start and stopping rule as above with N = v_end - v_begin; out-degrees are
 * the graph's live degrees.  The range must be closed under out-edges.
 * No counterpart in the reference (whose PageRank needs the reverse graph). */
typedef struct mk_pagerank_range mk_pagerank_range;
mk_status mk_pagerank_range_create(mk_graph *g, uint32_t max_vertices,
                                   mk_pagerank_range **out);
mk_status mk_pagerank_range_run(mk_pagerank_range *p, uint32_t v_begin, uint32_t v_end,
                                float damping, float tol, uint32_t max_iter,
                                void *stream, float *ms_out);
/* The last run's v_end - v_begin values (host). */
mk_status mk_pagerank_range_values(mk_pagerank_range *p, float *h_out);
mk_status mk_pagerank_range_stats(mk_pagerank_range *p, uint32_t *h_iters, float *h_delta);
mk_status mk_pagerank_range_destroy(mk_pagerank_range *p);

/* ------------------------------------------------------------------------
 * Triangle counting on a symmetric graph (replaces TC<AllocPolicy>,
 * include/Algorithms/TC.cuh:9-40).
 * ---------------------------------------------------------------------- */
typedef struct mk_tc mk_tc;
mk_status mk_tc_create(mk_graph *g, mk_tc **out);
/* float Static(EdgesN) (TCImpl.cuh:288-380). */
mk_status mk_tc_static(mk_tc *t, void *stream, float *ms_out);
/* float Incremental/Decremental(src*, dst*, n, Alloc)
 * (TCImpl.cuh:431-565).  The batch is read as undirected pairs. */
mk_status mk_tc_incremental(mk_tc *t, const uint32_t *d_src,
                            const uint32_t *d_dst, uint32_t n, void *stream,
                            float *ms_out);
mk_status mk_tc_decremental(mk_tc *t, const uint32_t *d_src,
                            const uint32_t *d_dst, uint32_t n, void *stream,
                            float *ms_out);
/* GetCount() (TC.cuh:31). */
mk_status mk_tc_count(mk_tc *t, uint64_t *h_count);
mk_status mk_tc_destroy(mk_tc *t);

/* Triangles of the symmetrised vertex range [v_begin, v_end) of an OUT-edge
 * graph (a member of a graph set), without a symmetric copy: the member's
 * edges are exported, each edge probes for its reverse, and the undirected
 * edges are oriented by (symmetric degree, id) as in mk_tc_static.  The
 * count equals mk_tc_static's on the member's symmetrised simple graph.
 * The range must be closed under out-edges (an edge leaving it is skipped
 * and sets MK_DEVERR_INVALID_ID on the graph).  run synchronises its stream
 * twice (edge count, work sizes); its scratch grows to the largest range
 * seen and is kept.  No counterpart in the reference, whose TC<> needs the
 * symmetric graph (TC.cuh:9-40). */
typedef struct mk_tc_range mk_tc_range;
mk_status mk_tc_range_create(mk_graph *g, mk_tc_range **out);
mk_status mk_tc_range_run(mk_tc_range *t, uint32_t v_begin, uint32_t v_end, void *stream,
                          float *ms_out);
/* The last run's count (synchronises). */
mk_status mk_tc_range_count(mk_tc_range *t, uint64_t *h_count);
/* Stream-ordered copy of the last run's count into h_count (pinned host
 * memory for a truly asynchronous copy). */
mk_status mk_tc_range_count_async(mk_tc_range *t, uint64_t *h_count, void *stream);
mk_status mk_tc_range_destroy(mk_tc_range *t);

/* ------------------------------------------------------------------------
 * Weakly connected components by lock-free union-find with min-id labels.
 * The reference ships only the device primitives
 * (include/Util/UnionFind.cuh:24-254) and no entry point; these are new.
 * ---------------------------------------------------------------------- */
typedef struct mk_wcc mk_wcc;
mk_status mk_wcc_create(mk_graph *g, mk_wcc **out);
mk_status mk_wcc_static(mk_wcc *w, void *stream, float *ms_out);
/* Recomputes the labels of the selected vertices only (bit v of d_sel_bits,
 * a device bitmap of ceil(V/32) words); the other labels stay as they are.
 * The selection must be closed under edges: whole components, or whole
 * member graphs of a graph set.  No counterpart in the reference. */
mk_status mk_wcc_static_subset(mk_wcc *w, const uint32_t *d_sel_bits, void *stream,
                               float *ms_out);
/* Recomputes the labels of the vertex ranges [r[2i], r[2i+1]) only
 * (h_vertex_ranges: 2 * nranges host words), touching nothing else: the
 * work is proportional to the ranges, not to the graph.  Each range must be
 * closed under edges (a member of a graph set).  No counterpart in the
 * reference. */
mk_status mk_wcc_static_ranges(mk_wcc *w, const uint32_t *h_vertex_ranges,
                               uint32_t nranges, void *stream, float *ms_out);
/* The two halves of mk_wcc_static_ranges.  prepare uploads the range table
 * (blocking: it waits for the device, since queued work may read the
 * previous table); static_prepared runs on it and issues only asynchronous
 * work on `stream`, so it can be captured into a CUDA graph (a later prepare
 * invalidates such a capture).  Ranges of at most 65,536 vertices are each
 * solved by one CTA with the parent array in shared memory; larger ones by
 * the device-wide pass.  A key outside its range sets MK_DEVERR_INVALID_ID
 * on the graph.  No counterpart in the reference. */
mk_status mk_wcc_prepare_ranges(mk_wcc *w, const uint32_t *h_vertex_ranges,
                                uint32_t nranges);
mk_status mk_wcc_static_prepared(mk_wcc *w, void *stream, float *ms_out);
/* Stream-ordered form of mk_wcc_prepare_ranges: the table reaches the device
 * on `stream` after the launches queued there before the call; no other
 * device work is waited for.  The WCC handle must not have work in flight on
 * another stream.  A table larger than any prepared before synchronises the
 * device once. */
mk_status mk_wcc_prepare_ranges_async(mk_wcc *w, const uint32_t *h_vertex_ranges,
                                      uint32_t nranges, void *stream);
mk_status mk_wcc_incremental(mk_wcc *w, const uint32_t *d_src,
                             const uint32_t *d_dst, uint32_t n, void *stream,
                             float *ms_out);
mk_status mk_wcc_decremental(mk_wcc *w, const uint32_t *d_src,
                             const uint32_t *d_dst, uint32_t n, void *stream,
                             float *ms_out);
/* Attaches the reverse graph of the same edges (in-edges; the caller keeps
 * it in step with g, as for mk_traversal_set_reverse), or detaches it with
 * NULL.  Decremental calls use it to rescan the pieces a deletion split off;
 * static calls (mk_wcc_static) use it to scan only the vertices outside the
 * largest set that sampled linking formed, when that set holds at least 3/4
 * of 2,048 sampled vertices: their out-edges and, through it, their
 * in-edges, so the edges inside that set are never read.  Attaching
 * allocates the scratch (about 20 bytes per vertex plus 1 per bucket of
 * either graph), loads the kernels of both paths, and sizes a set for
 * batches of up to min(the graph's batch scratch, V) edges (size the batch
 * scratch first with mk_graph_reserve_batch); a larger batch grows the set
 * on its first decremental call.
 *
 * Every static, incremental and decremental call keeps a spanning forest:
 * the edge of each union that hooked a root.  mk_wcc_decremental then
 *   - changes nothing when the batch removed no forest edge (a deleted
 *     forest edge whose reverse edge still exists stays in the forest);
 *   - otherwise splits the affected components along the forest, keeps one
 *     piece of each as its main piece, and rescans only the out- and (with
 *     a reverse graph) in-edges of the other pieces' vertices;
 *   - rebuilds the affected components from their out-edges when no reverse
 *     graph is attached or the split-off pieces hold more than half of the
 *     graph's edge ends (the whole graph by the static passes when the
 *     affected components hold most of its vertices).  After a split whose
 *     pieces were too large, the next calls run the static passes directly
 *     (1, then 2, 4, up to 8 calls after each further such split; a rescan
 *     that succeeds resets this).
 * After mk_wcc_static_ranges / _prepared (which keep no forest) the next
 * decremental call is a full static pass.  The labels are the same on every
 * path.  The decremental call synchronises its stream (it picks the path on
 * the host). */
mk_status mk_wcc_set_reverse(mk_wcc *w, mk_graph *g_rev);
/* The last decremental call: forest edges it removed, vertices rescanned
 * outside their component's main piece, and its path: 0 no forest edge lost,
 * 1 rescan of the split-off pieces, 2 rebuild of the affected components,
 * 3 full static pass (the affected components hold most of the vertices, or
 * no forest was kept). */
mk_status mk_wcc_decremental_stats(mk_wcc *w, uint64_t *h_dead_forest_edges,
                                   uint64_t *h_rescanned_vertices, uint32_t *h_path);
/* N labels: the minimum vertex id of each vertex's component (host). */
mk_status mk_wcc_labels(mk_wcc *w, uint32_t *h_out);
mk_status mk_wcc_labels_device(mk_wcc *w, const uint32_t **d_labels);
mk_status mk_wcc_destroy(mk_wcc *w);

/* ------------------------------------------------------------------------
 * Graph sets: many small dynamic graphs stored and updated as one (no
 * counterpart in the reference, whose drivers hold one graph per process).
 * Member m owns the global vertex ids [offsets[m], offsets[m+1]); members
 * share no edge, so one batch, one multi-source traversal (one source per
 * member) or one subset WCC pass serves them all, and each member's result
 * equals that of a DynamicGraph holding the member alone.
 * ---------------------------------------------------------------------- */
typedef struct mk_graphset mk_graphset;
/* h_num_vertices[num_graphs] member sizes (each >= 1, sum < 2^32 - 2);
 * h_degree_hints NULL or an array of num_graphs host pointers, each NULL or
 * the member's per-vertex hints.  Bucket sizing follows mk_graph_create. */
mk_status mk_graphset_create(uint32_t num_graphs, const uint32_t *h_num_vertices,
                             const uint32_t *const *h_degree_hints, double load_factor,
                             uint32_t weighted, int32_t device, uint64_t pool_slabs,
                             mk_graphset **out);
mk_status mk_graphset_destroy(mk_graphset *s);
/* The union graph, owned by the set: use it with every mk_graph_*, BFS,
 * SSSP, PageRank, TC and WCC entry point; never destroy it directly. */
mk_status mk_graphset_union(mk_graphset *s, mk_graph **g);
/* Number of member graphs. */
mk_status mk_graphset_num_graphs(mk_graphset *s, uint32_t *h_num_graphs);
/* Copies the num_graphs + 1 vertex offsets to host memory. */
mk_status mk_graphset_offsets(mk_graphset *s, uint32_t *h_offsets);
/* Device copy of the same offsets, owned by the set. */
mk_status mk_graphset_offsets_device(mk_graphset *s, const uint32_t **d_offsets);
/* Vertex bitmap (ceil(V/32) device words) of the members whose byte in
 * d_graph_flags[num_graphs] is non-zero; feeds mk_wcc_static_subset. */
mk_status mk_graphset_select_bits(mk_graphset *s, const uint8_t *d_graph_flags,
                                  uint32_t *d_bits, void *stream);
/* R-MAT edges per member on the current device.  Member m owns the vertex
 * ids [d_vertex_offsets[m], d_vertex_offsets[m+1]) (u32 device array of
 * num_graphs + 1 ascending entries, as a set's offsets) and gets the edges
 * [d_edge_offsets[m], d_edge_offsets[m+1]) (u64 device array), drawn with
 * probabilities a, b, c over its own vertex range; no self-loops (members of
 * one vertex get self-loops, which updates skip); duplicates possible.
 * Edge i depends only on (seed, i).  d_w may be NULL.  Needs no graph, so
 * degree hints can be computed before the set is created. */
mk_status mk_gen_rmat_set(const uint32_t *d_vertex_offsets, uint32_t num_graphs,
                          const uint64_t *d_edge_offsets, double a, double b,
                          double c, uint64_t seed, uint32_t w_lo, uint32_t w_hi,
                          uint32_t *d_src, uint32_t *d_dst, uint32_t *d_w,
                          void *stream);
/* Random update batches per member on the device: deletes of live edges
 * drawn from a CSR export of the union graph (d_row_ptr, d_col as written
 * by mk_graph_export_csr) and inserts of uniform pairs of distinct vertices
 * inside each member, counts per member given by the u64 offset arrays
 * d_del_offsets / d_ins_offsets (num_graphs + 1 entries); vertex offsets
 * as for mk_gen_rmat_set.  A member without live edges gets self-loop
 * deletes (no-ops).  d_ins_w may be NULL. */
mk_status mk_gen_set_batches(const uint32_t *d_vertex_offsets, uint32_t num_graphs,
                             const uint64_t *d_row_ptr,
                             const uint32_t *d_col, const uint64_t *d_del_offsets,
                             const uint64_t *d_ins_offsets, uint64_t seed,
                             uint32_t w_lo, uint32_t w_hi, uint32_t *d_del_src,
                             uint32_t *d_del_dst, uint32_t *d_ins_src,
                             uint32_t *d_ins_dst, uint32_t *d_ins_w, void *stream);

/* ------------------------------------------------------------------------
 * The batched many-graph step (no counterpart in the reference, whose
 * drivers hold one graph and one algorithm object per process,
 * src/BFS.cu:11-131).  A runner holds one query per member of a graph set:
 * MK_QUERY_BFS (levels from the member's source; h_bfs_source_local[m] is a
 * local vertex id, read only for BFS members), MK_QUERY_WCC (the member's
 * components) or MK_QUERY_NONE.  create uploads the query tables (blocking).
 * step applies one update batch covering any members (deletes, then inserts;
 * global vertex ids, device arrays; d_ins_w may be NULL) and then answers
 * every member's query: four launches, all asynchronous on `stream` and
 * allocation-free once mk_graph_reserve_batch has sized the batch scratch,
 * so a step can be captured into a CUDA graph.  A member's answers equal
 * those of a DynamicGraph holding the member alone (an edge leaving its
 * member sets MK_DEVERR_INVALID_ID on the union graph).
 * ---------------------------------------------------------------------- */
#define MK_QUERY_BFS 0u
#define MK_QUERY_WCC 1u
#define MK_QUERY_NONE 2u
typedef struct mk_set_runner mk_set_runner;
mk_status mk_set_runner_create(mk_graphset *s, const uint8_t *h_query,
                               const uint32_t *h_bfs_source_local, mk_set_runner **out);
mk_status mk_set_runner_step(mk_set_runner *r, const uint32_t *d_del_src,
                             const uint32_t *d_del_dst, uint32_t n_del,
                             const uint32_t *d_ins_src, const uint32_t *d_ins_dst,
                             const uint32_t *d_ins_w, uint32_t n_ins, void *stream);
/* One-launch step (opt-in): with on != 0 every later step is ONE
 * cooperative kernel (one 1,024-thread CTA per SM) in three phases
 * separated by bounded grid barriers: every delete of the batch, every
 * insert, then the members' queries, a CTA taking members from a counter
 * (largest first) and solving each in shared memory.  The answers and the
 * graph are those of the four-launch step, the batch arrays need no order,
 * and after a step the graph's last update is the insert batch, as there.
 * A wait that runs out sets MK_DEVERR_TIMEOUT (mk_graph_sync).
 * MK_ERR_INVALID when a member has more than 65,535 vertices (the runner
 * keeps the four-launch step). */
mk_status mk_set_runner_set_single(mk_set_runner *r, uint32_t on);
/* Kernel launches one step issues: 1 in the one-launch form, else 2 plus
 * one per query kind present (members beyond one CTA's shared memory add the
 * device-wide kernels, not counted here). */
mk_status mk_set_runner_launches(mk_set_runner *r, uint32_t *h_launches);
/* The runner's BFS and WCC handles (owned by the runner; NULL when no member
 * asks that query), for mk_traversal_distances / mk_wcc_labels. */
mk_status mk_set_runner_handles(mk_set_runner *r, mk_traversal **bfs, mk_wcc **wcc);
/* Device pointers to the answers of the last step (either may be NULL): the
 * packed dist << 32 | parent words of the BFS members' vertices (union ids;
 * NULL when no member asks BFS) and the WCC labels (union ids, the minimum
 * id of each component; NULL when no member asks WCC). */
mk_status mk_set_runner_results(mk_set_runner *r, const uint64_t **d_bfs_packed,
                                const uint32_t **d_wcc_labels);
mk_status mk_set_runner_destroy(mk_set_runner *r);

/* ------------------------------------------------------------------------
 * The reference drivers' text formats (host only; no GPU needed):
 *   graph file "V E" then E pairs "u v"                 (src/BFS.cu:27-36)
 *   batch file "<prefix>.batch.<i>": "n" then n pairs  (src/BFS.cu:76-91)
 * Whitespace-separated unsigned decimals.  Pass NULL arrays first to read
 * only the header; a short file, a malformed token or (graph files) an id
 * >= V is MK_ERR_INVALID with the line in mk_last_error_string().
 * ---------------------------------------------------------------------- */
mk_status mk_read_edge_list(const char *path, uint32_t *h_num_vertices,
                            uint64_t *h_num_edges, uint32_t *h_src, uint32_t *h_dst);
mk_status mk_read_batch_file(const char *path, uint64_t *h_num_edges,
                             uint32_t *h_src, uint32_t *h_dst);
mk_status mk_write_edge_list(const char *path, uint32_t num_vertices,
                             uint64_t num_edges, const uint32_t *h_src,
                             const uint32_t *h_dst);
mk_status mk_write_batch_file(const char *path, uint64_t num_edges,
                              const uint32_t *h_src, const uint32_t *h_dst);

/* ------------------------------------------------------------------------
 * Synthetic inputs (host only; no GPU needed).  Seeded and deterministic.
 * ---------------------------------------------------------------------- */
/* R-MAT: exactly num_edges distinct directed edges without self-loops over
 * 2^scale vertices, probabilities a, b, c (d = 1-a-b-c).  h_w (may be NULL)
 * gets weights uniform in [w_lo, w_hi]. */
mk_status mk_gen_rmat(uint32_t scale, uint64_t num_edges, double a, double b,
                      double c, uint64_t seed, uint32_t w_lo, uint32_t w_hi,
                      uint32_t *h_src, uint32_t *h_dst, uint32_t *h_w);
/* side x side 4-neighbour grid, both directions, plus `shortcuts` random
 * directed long-range edges.  Returns the edge count in *h_num_edges; pass
 * NULL arrays first to query the count. */
mk_status mk_gen_grid(uint32_t side, uint64_t shortcuts, uint64_t seed,
                      uint32_t w_lo, uint32_t w_hi, uint32_t *h_src,
                      uint32_t *h_dst, uint32_t *h_w, uint64_t *h_num_edges);

/* Host edge-set tracker used to draw valid update batches: absent-edge
 * inserts and present-edge deletes, sampled uniformly. */
typedef struct mk_edgeset mk_edgeset;
mk_status mk_edgeset_create(uint32_t num_vertices, const uint32_t *h_src,
                            const uint32_t *h_dst, uint64_t n,
                            mk_edgeset **out);
mk_status mk_edgeset_destroy(mk_edgeset *s);
uint64_t mk_edgeset_size(const mk_edgeset *s);
/* Draws n distinct absent edges (u != v), adds them to the set. */
mk_status mk_edgeset_sample_absent(mk_edgeset *s, uint64_t n, uint64_t seed,
                                   uint32_t *h_src, uint32_t *h_dst);
/* Draws n distinct present edges uniformly, removes them from the set. */
mk_status mk_edgeset_sample_present(mk_edgeset *s, uint64_t n, uint64_t seed,
                                    uint32_t *h_src, uint32_t *h_dst);

#ifdef __cplusplus
}
#endif

#endif /* MEERKAT_B200_H_ */
