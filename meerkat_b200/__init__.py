"""meerkat_b200: B200-native dynamic-graph engine (slab-hash graph, batched
updates, incremental/decremental BFS, SSSP, PageRank, triangle counting and
connected components) behind a C ABI.

This module is the Python mirror of the reference's C++ classes
(DynamicGraph, BFS, SSSP, PageRank, TC; meerkat-pkd/Meerkat
include/Graph/SlabGraph.cuh and include/Algorithms/*.cuh) over that ABI.
Batch arrays are CUDA tensors (int32 or uint32 storage) or raw device
pointers.  There is no CPU fallback: every call runs the sm_100a kernels of
libmeerkat_b200.so.
"""
from __future__ import annotations

import ctypes as C
import weakref
from typing import Optional

import numpy as np

from ._lib import (DEVERR_INVALID_ID, DEVERR_OOM, DEVERR_OVERFLOW, DEVERR_TIMEOUT, MK_INF,
                   GraphDesc, GraphInfo, MeerkatError, Tuning, check, lib)

__all__ = ["DynamicGraph", "GraphSet", "SetRunner", "BFS", "SSSP", "PageRank", "PageRankRange", "TC", "TCRange",
           "WCC",
           "EdgeSet",
           "gen_rmat", "gen_grid", "gen_rmat_members", "read_edge_list", "read_batch",
           "write_edge_list", "write_batch", "MeerkatError", "MK_INF", "DEVERR_INVALID_ID",
           "DEVERR_OOM", "DEVERR_TIMEOUT", "DEVERR_OVERFLOW", "lib", "version"]


def version() -> str:
    return lib().mk_version().decode()


def _ptr(x) -> Optional[int]:
    if x is None:
        return None
    if isinstance(x, int):
        return x
    if isinstance(x, np.ndarray):
        return x.ctypes.data
    return x.data_ptr()


def _count(x, n):
    if n is not None:
        return int(n)
    return int(x.numel()) if hasattr(x, "numel") else int(len(x))


def _stream(s) -> Optional[int]:
    if s is None:
        return None
    if isinstance(s, int):
        return s
    return s.cuda_stream


class _Timed:
    """Reference algorithm calls return elapsed milliseconds (float)."""

    def _call(self, fn, *args, timed=True):
        ms = C.c_float(0.0)
        check(fn(*args, C.byref(ms) if timed else None), fn.__name__)
        return ms.value if timed else None


class DynamicGraph:
    """DynamicGraph<EdgePolicy, IsWeighted>(N, Allocator&, LoadFactor, hints, dev)
    (include/Graph/SlabGraph.cuh:382-466).  `weighted` selects the map slabs of
    WeightedEdgePolicyMapT, `reverse` the Rev* policies (edges keyed by
    destination)."""

    def __init__(self, num_vertices: int, load_factor: float = 0.7, degree_hints=None,
                 weighted: bool = False, reverse: bool = False, device: int = 0,
                 pool_slabs: int = 0):
        L = lib()
        self.num_vertices = int(num_vertices)
        self.weighted = bool(weighted)
        self.reverse = bool(reverse)
        self._hints = None
        d = GraphDesc()
        d.num_vertices = self.num_vertices
        d.weighted = int(weighted)
        d.reverse = int(reverse)
        d.flags = 0
        d.load_factor = float(load_factor)
        if degree_hints is not None:
            self._hints = np.ascontiguousarray(np.asarray(degree_hints, dtype=np.uint32))
            d.h_degree_hints = self._hints.ctypes.data_as(C.POINTER(C.c_uint32))
        d.device = int(device)
        d.pool_slabs = int(pool_slabs)
        h = C.c_void_p()
        check(L.mk_graph_create(C.byref(d), C.byref(h)), "mk_graph_create")
        self._h = h
        self.device = int(device)

    @property
    def handle(self):
        return self._h

    @classmethod
    def _borrow(cls, handle, num_vertices: int, weighted: bool, device: int, owner):
        """View of a graph owned by another object (a GraphSet's union graph)."""
        g = cls.__new__(cls)
        g.num_vertices = int(num_vertices)
        g.weighted = bool(weighted)
        g.reverse = False
        g._hints = None
        g._h = handle
        g.device = int(device)
        g._owner = owner
        return g

    def close(self):
        if getattr(self, "_owner", None) is not None:
            self._h = None
            return
        if getattr(self, "_h", None):
            lib().mk_graph_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def InsertEdges(self, src, dst, n=None, vals=None, stream=None):
        """InsertEdges(src*, dst*, n, vals*) (SlabGraph.cuh:486-488)."""
        check(lib().mk_graph_insert_edges(self._h, _ptr(src), _ptr(dst), _ptr(vals),
                                          _count(src, n), _stream(stream)),
              "mk_graph_insert_edges")

    def DeleteEdges(self, src, dst, n=None, stream=None):
        """DeleteEdges(src*, dst*, n) (SlabGraph.cuh:490-491)."""
        check(lib().mk_graph_delete_edges(self._h, _ptr(src), _ptr(dst), _count(src, n),
                                          _stream(stream)), "mk_graph_delete_edges")

    def SearchEdges(self, src, dst, found, weights=None, n=None, stream=None):
        check(lib().mk_graph_search_edges(self._h, _ptr(src), _ptr(dst), _count(src, n),
                                          _ptr(found), _ptr(weights), _stream(stream)),
              "mk_graph_search_edges")

    def set_tuning(self, update_kernel: Optional[int] = None,
                   update_blocks_per_sm: Optional[int] = None,
                   frontier_chunk: Optional[int] = None,
                   sssp_delta: Optional[int] = None,
                   recompute_permille: Optional[int] = None,
                   pull_permille: Optional[int] = None,
                   wait_limit_us: Optional[int] = None) -> None:
        """Sets the given kernel knobs; the others keep their values."""
        cur = self.get_tuning()
        for k, v in (("update_kernel", update_kernel), ("update_blocks_per_sm", update_blocks_per_sm),
                     ("frontier_chunk", frontier_chunk), ("sssp_delta", sssp_delta),
                     ("recompute_permille", recompute_permille), ("pull_permille", pull_permille),
                     ("wait_limit_us", wait_limit_us)):
            if v is not None:
                cur[k] = int(v)
        t = Tuning(cur["update_kernel"], cur["update_blocks_per_sm"], cur["frontier_chunk"],
                   cur["sssp_delta"], cur["recompute_permille"], cur["pull_permille"],
                   cur["wait_limit_us"])
        check(lib().mk_graph_set_tuning(self._h, C.byref(t)), "mk_graph_set_tuning")

    def get_tuning(self) -> dict:
        t = Tuning()
        check(lib().mk_graph_get_tuning(self._h, C.byref(t)), "mk_graph_get_tuning")
        return {"update_kernel": t.update_kernel, "update_blocks_per_sm": t.update_blocks_per_sm,
                "frontier_chunk": t.frontier_chunk, "sssp_delta": t.sssp_delta,
                "recompute_permille": t.recompute_permille, "pull_permille": t.pull_permille,
                "wait_limit_us": t.wait_limit_us}

    def reserve_batch(self, n: int) -> None:
        check(lib().mk_graph_reserve_batch(self._h, int(n)), "mk_graph_reserve_batch")

    def sync(self, stream=None) -> int:
        err = C.c_uint32(0)
        check(lib().mk_graph_sync(self._h, _stream(stream), C.byref(err)), "mk_graph_sync")
        return err.value

    def last_applied(self) -> int:
        c = C.c_uint64(0)
        check(lib().mk_graph_last_applied(self._h, C.byref(c)), "mk_graph_last_applied")
        return c.value

    def slabs_used_async(self, host_ptr: int, stream=None) -> None:
        """Stream-ordered copy of the slabs in use to host_ptr (pinned u32)."""
        check(lib().mk_graph_slabs_used_async(self._h, host_ptr, _stream(stream)),
              "mk_graph_slabs_used_async")

    def last_applied_async(self, host_ptr: int, stream=None) -> None:
        """Stream-ordered copy of the applied count to host_ptr (pinned u64)."""
        check(lib().mk_graph_last_applied_async(self._h, host_ptr, _stream(stream)),
              "mk_graph_last_applied_async")

    def degrees_into(self, out, stream=None):
        check(lib().mk_graph_degrees(self._h, _ptr(out), _stream(stream)), "mk_graph_degrees")

    def GetVertexBucketsOffsets(self) -> np.ndarray:
        out = np.zeros(self.num_vertices, dtype=np.uint32)
        check(lib().mk_graph_bucket_layout(self._h, out.ctypes.data, None), "bucket_layout")
        return out

    def GetBucketsPerVertex(self) -> np.ndarray:
        out = np.zeros(self.num_vertices, dtype=np.uint32)
        check(lib().mk_graph_bucket_layout(self._h, None, out.ctypes.data), "bucket_layout")
        return out

    def info(self) -> dict:
        i = GraphInfo()
        check(lib().mk_graph_get_info(self._h, C.byref(i)), "mk_graph_get_info")
        return {f: getattr(i, f) for f, _ in GraphInfo._fields_}

    # --- host-side views used by the tests (need torch for device buffers) ---
    def degrees(self) -> np.ndarray:
        import torch
        out = torch.empty(self.num_vertices, dtype=torch.int32, device=f"cuda:{self.device}")
        self.degrees_into(out)
        torch.cuda.synchronize(self.device)
        return out.cpu().numpy().view(np.uint32)

    def tombstones(self) -> np.ndarray:
        import torch
        out = torch.empty(self.num_vertices, dtype=torch.int32, device=f"cuda:{self.device}")
        check(lib().mk_graph_count_tombstones(self._h, out.data_ptr(), None), "tombstones")
        torch.cuda.synchronize(self.device)
        return out.cpu().numpy().view(np.uint32)

    def count_edges(self, v_begin: int = 0, v_end: Optional[int] = None, stream=None) -> int:
        """Live edges of the vertices [v_begin, v_end)."""
        c = C.c_uint64(0)
        v_end = self.num_vertices if v_end is None else int(v_end)
        check(lib().mk_graph_count_edges_range(self._h, int(v_begin), v_end, _stream(stream),
                                               C.byref(c)), "mk_graph_count_edges_range")
        return c.value

    def export_csr_range_device(self, v_begin: int, v_end: int, weights: bool = False,
                                stream=None):
        """Device CSR of the rows [v_begin, v_end): (row_ptr int64[n+1] from 0,
        col int32[E] with global ids, w int32[E] or None)."""
        import torch
        dev = f"cuda:{self.device}"
        E = self.count_edges(v_begin, v_end, stream=stream)
        rp = torch.empty(int(v_end) - int(v_begin) + 1, dtype=torch.int64, device=dev)
        col = torch.empty(max(E, 1), dtype=torch.int32, device=dev)
        w = torch.empty(max(E, 1), dtype=torch.int32, device=dev) if (weights and self.weighted) else None
        check(lib().mk_graph_export_csr_range(self._h, int(v_begin), int(v_end), rp.data_ptr(),
                                              col.data_ptr(), _ptr(w), _stream(stream)),
              "mk_graph_export_csr_range")
        return rp, col[:E], (w[:E] if w is not None else None)

    def export_csr(self, sort_rows: bool = True):
        """Live edges as CSR (row_ptr u64[N+1], col u32[E], w u32[E] or None)."""
        import torch
        dev = f"cuda:{self.device}"
        E = self.info()["num_edges"]
        rp = torch.empty(self.num_vertices + 1, dtype=torch.int64, device=dev)
        col = torch.empty(max(E, 1), dtype=torch.int32, device=dev)
        w = torch.empty(max(E, 1), dtype=torch.int32, device=dev) if self.weighted else None
        check(lib().mk_graph_export_csr(self._h, rp.data_ptr(), col.data_ptr(), _ptr(w), None),
              "mk_graph_export_csr")
        torch.cuda.synchronize(self.device)
        rp_h = rp.cpu().numpy().view(np.uint64)
        col_h = col.cpu().numpy().view(np.uint32)[:E]
        w_h = w.cpu().numpy().view(np.uint32)[:E] if w is not None else None
        if sort_rows:
            rows = np.repeat(np.arange(self.num_vertices, dtype=np.int64),
                             np.diff(rp_h).astype(np.int64))
            order = np.lexsort((col_h, rows))
            col_h = col_h[order]
            if w_h is not None:
                w_h = w_h[order]
        return rp_h, col_h, w_h


class _Traversal(_Timed):
    _create = None

    def __init__(self, G: DynamicGraph, source, num_vertices: Optional[int] = None):
        """`source` is one vertex, or a sequence of distinct vertices for one
        multi-source traversal (e.g. one source per member of a GraphSet)."""
        if num_vertices is not None and int(num_vertices) != G.num_vertices:
            raise ValueError("VertexN must equal the graph's vertex count")
        self.G = G
        h = C.c_void_p()
        if np.ndim(source) == 0:
            self.source = int(source)
            check(getattr(lib(), self._create)(G.handle, self.source, C.byref(h)), self._create)
        else:
            self.sources = np.ascontiguousarray(np.asarray(source, dtype=np.uint32))
            self.source = self.sources
            name = self._create + "_multi"
            check(getattr(lib(), name)(G.handle, self.sources.ctypes.data_as(C.POINTER(C.c_uint32)),
                                       len(self.sources), C.byref(h)), name)
        self._h = h

    @classmethod
    def _borrow(cls, handle, G: DynamicGraph, sources, owner):
        """View of a traversal handle owned by another object (a SetRunner)."""
        t = cls.__new__(cls)
        t.G = G
        t.sources = np.ascontiguousarray(np.asarray(sources, dtype=np.uint32))
        t.source = t.sources
        t._h = handle
        t._owner = owner
        return t

    def close(self):
        if getattr(self, "_owner", None) is not None:
            self._h = None
            return
        if getattr(self, "_h", None):
            lib().mk_traversal_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_sources(self, sources, stream=None) -> None:
        """Replaces the source set (distinct vertices); call Static next.
        With a stream the upload is stream-ordered on it and waits for no
        other device work (mk_traversal_set_sources_async)."""
        self.sources = np.ascontiguousarray(np.atleast_1d(np.asarray(sources, dtype=np.uint32)))
        self.source = self.sources
        p = self.sources.ctypes.data_as(C.POINTER(C.c_uint32))
        if stream is None:
            check(lib().mk_traversal_set_sources(self._h, p, len(self.sources)),
                  "mk_traversal_set_sources")
        else:
            check(lib().mk_traversal_set_sources_async(self._h, p, len(self.sources),
                                                       _stream(stream)),
                  "mk_traversal_set_sources_async")

    def set_reverse(self, G_rev: Optional[DynamicGraph]) -> None:
        """Attaches the reverse graph of the same edges (BFS pull levels)."""
        self._rev = G_rev
        check(lib().mk_traversal_set_reverse(self._h, G_rev.handle if G_rev is not None else None),
              "mk_traversal_set_reverse")

    def Static(self, edges_n=None, stream=None, timed=True):
        return self._call(lib().mk_traversal_static, self._h, _stream(stream), timed=timed)

    def Incremental(self, src, dst, n=None, wgt=None, stream=None, timed=True):
        return self._call(lib().mk_traversal_incremental, self._h, _ptr(src), _ptr(dst),
                          _ptr(wgt), _count(src, n), _stream(stream), timed=timed)

    def Decremental(self, src, dst, n=None, wgt=None, stream=None, timed=True):
        return self._call(lib().mk_traversal_decremental, self._h, _ptr(src), _ptr(dst),
                          _ptr(wgt), _count(src, n), _stream(stream), timed=timed)

    def Distances(self) -> np.ndarray:
        out = np.zeros(self.G.num_vertices, dtype=np.uint32)
        check(lib().mk_traversal_distances(self._h, out.ctypes.data), "mk_traversal_distances")
        return out

    def packed_ptr(self) -> int:
        p = C.c_void_p()
        check(lib().mk_traversal_packed(self._h, C.byref(p)), "mk_traversal_packed")
        return p.value

    def packed(self) -> np.ndarray:
        """Host copy of the packed dist<<32|parent array."""
        out = np.zeros(self.G.num_vertices, dtype=np.uint64)
        check(lib().mk_traversal_packed_host(self._h, out.ctypes.data), "mk_traversal_packed_host")
        return out

    def stats(self):
        lv = C.c_uint32(0)
        pushed = C.c_uint64(0)
        check(lib().mk_traversal_stats(self._h, C.byref(lv), C.byref(pushed)), "stats")
        return lv.value, pushed.value

    def decremental_stats(self):
        """(vertices invalidated, recomputed from the sources) of the last
        Decremental call."""
        inv = C.c_uint64(0)
        rec = C.c_uint32(0)
        check(lib().mk_traversal_decremental_stats(self._h, C.byref(inv), C.byref(rec)),
              "mk_traversal_decremental_stats")
        return int(inv.value), bool(rec.value)


class BFS(_Traversal):
    """BFS<AllocPolicy>(G, SourceVertex, VertexN) (include/Algorithms/BFS.cuh:13-69)."""
    _create = "mk_bfs_create"

    def PrepareMembers(self, ranges):
        """Uploads one vertex range [(begin, end), ...] per source, in source
        order, for StaticMembers (blocking).  Each range holds its source and
        is closed under edges (a GraphSet member)."""
        r = np.ascontiguousarray(np.asarray(ranges, dtype=np.uint32).reshape(-1))
        check(lib().mk_bfs_prepare_members(self._h, r.ctypes.data_as(C.POINTER(C.c_uint32)),
                                           len(r) // 2), "mk_bfs_prepare_members")

    def StaticMembers(self, stream=None, timed=True):
        """Static BFS over the prepared ranges: the distances of Static (and
        a valid BFS tree), with a range of at most 65,535 vertices solved by
        one CTA in shared memory.  Only asynchronous work on the stream
        (capturable)."""
        return self._call(lib().mk_bfs_static_members, self._h, _stream(stream), timed=timed)


class SSSP(_Traversal):
    """SSSP<AllocPolicy>(G, SourceVertex, VertexN) (include/Algorithms/SSSP.cuh:11-69)."""
    _create = "mk_sssp_create"


class PageRank(_Timed):
    """PageRank<AllocPolicy>(G, d, tol, N, OutDeg*, MaxIter)
    (include/Algorithms/PageRank.cuh:9-67); G must be a reverse graph."""

    def __init__(self, G: DynamicGraph, damping: float, tol: float, num_vertices=None,
                 out_degree=None, max_iter: int = 100):
        if not G.reverse:
            raise ValueError("PageRank pulls over in-edges: build the graph with reverse=True")
        self.G = G
        self._od = None
        if out_degree is not None:
            self._od = np.ascontiguousarray(np.asarray(out_degree, dtype=np.uint32))
        h = C.c_void_p()
        check(lib().mk_pagerank_create(G.handle, float(damping), float(tol), int(max_iter),
                                       _ptr(self._od), C.byref(h)), "mk_pagerank_create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().mk_pagerank_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def Static(self, stream=None, timed=True):
        return self._call(lib().mk_pagerank_static, self._h, _stream(stream), timed=timed)

    def StaticRecount(self, stream=None, timed=True):
        """Static after recounting out-degrees (graph updated behind its back)."""
        return self._call(lib().mk_pagerank_static_recount, self._h, _stream(stream), timed=timed)

    def Incremental(self, src, dst, n=None, stream=None, timed=True):
        return self._call(lib().mk_pagerank_incremental, self._h, _ptr(src), _ptr(dst),
                          _count(src, n), _stream(stream), timed=timed)

    def Decremental(self, src, dst, n=None, stream=None, timed=True):
        return self._call(lib().mk_pagerank_decremental, self._h, _ptr(src), _ptr(dst),
                          _count(src, n), _stream(stream), timed=timed)

    def Values(self) -> np.ndarray:
        out = np.zeros(self.G.num_vertices, dtype=np.float32)
        check(lib().mk_pagerank_values(self._h, out.ctypes.data), "mk_pagerank_values")
        return out

    def stats(self):
        it = C.c_uint32(0)
        dl = C.c_float(0)
        check(lib().mk_pagerank_stats(self._h, C.byref(it), C.byref(dl)), "mk_pagerank_stats")
        return it.value, dl.value


class PageRankRange(_Timed):
    """PageRank of one vertex range (a GraphSet member) of an out-edge graph,
    push form: no reverse graph needed (mk_pagerank_range_*)."""

    def __init__(self, G: DynamicGraph, max_vertices: int):
        self.G = G
        h = C.c_void_p()
        check(lib().mk_pagerank_range_create(G.handle, int(max_vertices), C.byref(h)),
              "mk_pagerank_range_create")
        self._h = h
        self._n = 0

    def close(self):
        if getattr(self, "_h", None):
            lib().mk_pagerank_range_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def Run(self, v_begin: int, v_end: int, damping: float = 0.85, tol: float = 1e-6,
            max_iter: int = 200, stream=None, timed=True):
        self._n = int(v_end) - int(v_begin)
        return self._call(lib().mk_pagerank_range_run, self._h, int(v_begin), int(v_end),
                          float(damping), float(tol), int(max_iter), _stream(stream), timed=timed)

    def Values(self) -> np.ndarray:
        out = np.zeros(self._n, dtype=np.float32)
        check(lib().mk_pagerank_range_values(self._h, out.ctypes.data), "mk_pagerank_range_values")
        return out

    def stats(self):
        it = C.c_uint32(0)
        dl = C.c_float(0)
        check(lib().mk_pagerank_range_stats(self._h, C.byref(it), C.byref(dl)), "stats")
        return it.value, dl.value


class TC(_Timed):
    """TC<AllocPolicy>(G, N) (include/Algorithms/TC.cuh:9-40); G symmetric."""

    def __init__(self, G: DynamicGraph, num_vertices=None):
        self.G = G
        h = C.c_void_p()
        check(lib().mk_tc_create(G.handle, C.byref(h)), "mk_tc_create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().mk_tc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def Static(self, edges_n=None, stream=None, timed=True):
        return self._call(lib().mk_tc_static, self._h, _stream(stream), timed=timed)

    def Incremental(self, src, dst, n=None, alloc=None, stream=None, timed=True):
        return self._call(lib().mk_tc_incremental, self._h, _ptr(src), _ptr(dst), _count(src, n),
                          _stream(stream), timed=timed)

    def Decremental(self, src, dst, n=None, alloc=None, stream=None, timed=True):
        return self._call(lib().mk_tc_decremental, self._h, _ptr(src), _ptr(dst), _count(src, n),
                          _stream(stream), timed=timed)

    def GetCount(self) -> int:
        c = C.c_uint64(0)
        check(lib().mk_tc_count(self._h, C.byref(c)), "mk_tc_count")
        return c.value


class TCRange(_Timed):
    """Triangles of one vertex range of an out-edge graph (a graph-set
    member), symmetrised, without a symmetric copy (mk_tc_range_*)."""

    def __init__(self, G: DynamicGraph):
        self.G = G
        h = C.c_void_p()
        check(lib().mk_tc_range_create(G.handle, C.byref(h)), "mk_tc_range_create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().mk_tc_range_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def Run(self, v_begin: int, v_end: int, stream=None, timed=True):
        return self._call(lib().mk_tc_range_run, self._h, int(v_begin), int(v_end),
                          _stream(stream), timed=timed)

    def GetCount(self) -> int:
        c = C.c_uint64(0)
        check(lib().mk_tc_range_count(self._h, C.byref(c)), "mk_tc_range_count")
        return int(c.value)

    def count_async(self, host_ptr: int, stream=None) -> None:
        """Stream-ordered copy of the count to host_ptr (pinned, 8 bytes)."""
        check(lib().mk_tc_range_count_async(self._h, C.c_void_p(host_ptr), _stream(stream)),
              "mk_tc_range_count_async")


class WCC(_Timed):
    """Connected components (new entry points over include/Util/UnionFind.cuh)."""

    def __init__(self, G: DynamicGraph):
        self.G = G
        h = C.c_void_p()
        check(lib().mk_wcc_create(G.handle, C.byref(h)), "mk_wcc_create")
        self._h = h

    @classmethod
    def _borrow(cls, handle, G: DynamicGraph, owner):
        """View of a WCC handle owned by another object (a SetRunner)."""
        w = cls.__new__(cls)
        w.G = G
        w._h = handle
        w._owner = owner
        return w

    def close(self):
        if getattr(self, "_owner", None) is not None:
            self._h = None
            return
        if getattr(self, "_h", None):
            lib().mk_wcc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def Static(self, stream=None, timed=True):
        return self._call(lib().mk_wcc_static, self._h, _stream(stream), timed=timed)

    def StaticRanges(self, ranges, stream=None, timed=True):
        """Recomputes the labels of the vertex ranges [(begin, end), ...] only
        (each closed under edges, e.g. members of a GraphSet)."""
        r = np.ascontiguousarray(np.asarray(ranges, dtype=np.uint32).reshape(-1))
        return self._call(lib().mk_wcc_static_ranges, self._h,
                          r.ctypes.data_as(C.POINTER(C.c_uint32)), len(r) // 2, _stream(stream),
                          timed=timed)

    def PrepareRanges(self, ranges, stream=None):
        """Uploads a vertex-range table [(begin, end), ...] for StaticPrepared
        (blocking; with a stream, stream-ordered on it instead).  Ranges of at
        most 65,536 vertices are each solved by one CTA in shared memory;
        larger ones by the device-wide pass."""
        r = np.ascontiguousarray(np.asarray(ranges, dtype=np.uint32).reshape(-1))
        p = r.ctypes.data_as(C.POINTER(C.c_uint32))
        if stream is None:
            check(lib().mk_wcc_prepare_ranges(self._h, p, len(r) // 2), "mk_wcc_prepare_ranges")
        else:
            check(lib().mk_wcc_prepare_ranges_async(self._h, p, len(r) // 2, _stream(stream)),
                  "mk_wcc_prepare_ranges_async")

    def StaticPrepared(self, stream=None, timed=True):
        """StaticRanges over the prepared table; only asynchronous work on the
        stream, so it can be captured into a CUDA graph."""
        return self._call(lib().mk_wcc_static_prepared, self._h, _stream(stream), timed=timed)

    def StaticSubset(self, sel_bits, stream=None, timed=True):
        """Recomputes the labels of the vertices whose bit is set in the device
        bitmap `sel_bits` (ceil(V/32) words, closed under edges)."""
        return self._call(lib().mk_wcc_static_subset, self._h, _ptr(sel_bits), _stream(stream),
                          timed=timed)

    def Incremental(self, src, dst, n=None, stream=None, timed=True):
        return self._call(lib().mk_wcc_incremental, self._h, _ptr(src), _ptr(dst), _count(src, n),
                          _stream(stream), timed=timed)

    def Decremental(self, src, dst, n=None, stream=None, timed=True):
        return self._call(lib().mk_wcc_decremental, self._h, _ptr(src), _ptr(dst), _count(src, n),
                          _stream(stream), timed=timed)

    def Labels(self) -> np.ndarray:
        out = np.zeros(self.G.num_vertices, dtype=np.uint32)
        check(lib().mk_wcc_labels(self._h, out.ctypes.data), "mk_wcc_labels")
        return out

    def set_reverse(self, G_rev: Optional[DynamicGraph]) -> None:
        """Attaches the reverse graph of the same edges (kept in step by the
        caller).  Static calls then scan only the out- and in-edges of the
        vertices outside the largest sampled set; decremental calls rescan
        split-off pieces through it.  None detaches it."""
        self._rev = G_rev
        check(lib().mk_wcc_set_reverse(self._h, G_rev.handle if G_rev is not None else None),
              "mk_wcc_set_reverse")

    def decremental_stats(self):
        """(forest edges removed, vertices rescanned, path) of the last
        Decremental call; path 0 no forest edge lost, 1 rescan of the
        split-off pieces, 2 rebuild of the affected components, 3 full static
        pass (the affected components hold most vertices, or no forest)."""
        dead = C.c_uint64(0)
        res = C.c_uint64(0)
        path = C.c_uint32(0)
        check(lib().mk_wcc_decremental_stats(self._h, C.byref(dead), C.byref(res), C.byref(path)),
              "mk_wcc_decremental_stats")
        return int(dead.value), int(res.value), int(path.value)


class GraphSet:
    """Many small dynamic graphs stored, updated and queried as one union
    graph (member m owns vertex ids offsets[m] .. offsets[m+1]-1).  `graph` is
    a DynamicGraph view of the union graph for every update and algorithm
    call; the set owns it."""

    def __init__(self, num_vertices, degree_hints=None, load_factor: float = 0.7,
                 weighted: bool = False, device: int = 0, pool_slabs: int = 0):
        nv = np.ascontiguousarray(np.asarray(num_vertices, dtype=np.uint32))
        G = len(nv)
        self.num_graphs = G
        self.device = int(device)
        self.weighted = bool(weighted)
        self._hint_arrays = None
        hp = None
        if degree_hints is not None:
            self._hint_arrays = [None if h is None else
                                 np.ascontiguousarray(np.asarray(h, dtype=np.uint32))
                                 for h in degree_hints]
            if len(self._hint_arrays) != G:
                raise ValueError("one degree-hint array (or None) per member graph")
            for h, n in zip(self._hint_arrays, nv):
                if h is not None and len(h) != n:
                    raise ValueError("degree hints must have one entry per member vertex")
            hp = (C.POINTER(C.c_uint32) * G)(*[
                C.cast(None, C.POINTER(C.c_uint32)) if h is None
                else h.ctypes.data_as(C.POINTER(C.c_uint32)) for h in self._hint_arrays])
        h = C.c_void_p()
        check(lib().mk_graphset_create(G, nv.ctypes.data_as(C.POINTER(C.c_uint32)), hp,
                                       float(load_factor), int(weighted), int(device),
                                       int(pool_slabs), C.byref(h)), "mk_graphset_create")
        self._h = h
        self.offsets = np.zeros(G + 1, dtype=np.uint32)
        check(lib().mk_graphset_offsets(h, self.offsets.ctypes.data_as(C.POINTER(C.c_uint32))),
              "mk_graphset_offsets")
        gh = C.c_void_p()
        check(lib().mk_graphset_union(h, C.byref(gh)), "mk_graphset_union")
        self.graph = DynamicGraph._borrow(gh, int(self.offsets[-1]), weighted, device, self)

    @property
    def num_vertices(self) -> int:
        return int(self.offsets[-1])

    def close(self):
        if getattr(self, "_h", None):
            self.graph._h = None
            lib().mk_graphset_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _dev(self):
        return f"cuda:{self.device}"

    def select_bits(self, graph_flags, stream=None):
        """Device vertex bitmap of the members whose flag is non-zero."""
        import torch
        flags = graph_flags
        if not hasattr(flags, "data_ptr"):
            flags = torch.from_numpy(np.ascontiguousarray(np.asarray(graph_flags, dtype=np.uint8)))
        flags = flags.to(self._dev(), dtype=torch.uint8)
        bits = torch.empty((self.num_vertices + 31) // 32, dtype=torch.int32, device=self._dev())
        check(lib().mk_graphset_select_bits(self._h, flags.data_ptr(), bits.data_ptr(),
                                            _stream(stream)), "mk_graphset_select_bits")
        return bits

    def offsets_device(self) -> int:
        p = C.c_void_p()
        check(lib().mk_graphset_offsets_device(self._h, C.byref(p)), "mk_graphset_offsets_device")
        return p.value

    def gen_rmat(self, edges_per_graph, a=0.57, b=0.19, c=0.19, seed=0, w_lo=1, w_hi=64,
                 weights=True, stream=None):
        """Device R-MAT edges, edges_per_graph[m] inside member m (int32 tensors
        holding uint32 ids)."""
        return gen_rmat_members(self.offsets, edges_per_graph, a, b, c, seed, w_lo, w_hi, weights,
                                device=self.device, stream=stream,
                                d_vertex_offsets=self.offsets_device())

    def gen_batches(self, deletes_per_graph, inserts_per_graph, seed=0, w_lo=1, w_hi=64,
                    weights=True, stream=None):
        """Device update batches: deletes of live edges and inserts of random
        pairs, per member.  Returns (del_src, del_dst, ins_src, ins_dst, ins_w)."""
        import torch
        dev = self._dev()
        E = self.graph.info()["num_edges"]
        rp = torch.empty(self.num_vertices + 1, dtype=torch.int64, device=dev)
        col = torch.empty(max(E, 1), dtype=torch.int32, device=dev)
        check(lib().mk_graph_export_csr(self.graph.handle, rp.data_ptr(), col.data_ptr(), None,
                                        _stream(stream)), "mk_graph_export_csr")
        offs = []
        for cnt in (deletes_per_graph, inserts_per_graph):
            o = np.zeros(self.num_graphs + 1, dtype=np.uint64)
            np.cumsum(np.asarray(cnt, dtype=np.uint64), out=o[1:])
            offs.append(o)
        nd, ni = int(offs[0][-1]), int(offs[1][-1])
        d_do = torch.from_numpy(offs[0].view(np.int64)).to(dev)
        d_io = torch.from_numpy(offs[1].view(np.int64)).to(dev)
        ds = torch.empty(max(nd, 1), dtype=torch.int32, device=dev)
        dd = torch.empty(max(nd, 1), dtype=torch.int32, device=dev)
        is_ = torch.empty(max(ni, 1), dtype=torch.int32, device=dev)
        id_ = torch.empty(max(ni, 1), dtype=torch.int32, device=dev)
        iw = torch.empty(max(ni, 1), dtype=torch.int32, device=dev) if weights else None
        check(lib().mk_gen_set_batches(self.offsets_device(), self.num_graphs, rp.data_ptr(),
                                       col.data_ptr(), d_do.data_ptr(),
                                       d_io.data_ptr(), seed, w_lo, w_hi, ds.data_ptr(),
                                       dd.data_ptr(), is_.data_ptr(), id_.data_ptr(), _ptr(iw),
                                       _stream(stream)), "mk_gen_set_batches")
        return ds[:nd], dd[:nd], is_[:ni], id_[:ni], (iw[:ni] if iw is not None else None)


class SetRunner:
    """One query per member of a GraphSet (QUERY_BFS from a local source,
    QUERY_WCC, or QUERY_NONE) and a step that applies one update batch to
    every member and answers every query (mk_set_runner_*): four
    asynchronous launches, or one (set_single) when every member has at most
    65,535 vertices; either is capturable into a CUDA graph.  `bfs` / `wcc`
    are views of the runner's own handles for reading the answers."""

    def __init__(self, gs: "GraphSet", query, sources_local=None):
        q = np.ascontiguousarray(np.asarray(query, dtype=np.uint8))
        if len(q) != gs.num_graphs:
            raise ValueError("one query kind per member")
        src = (np.zeros(gs.num_graphs, dtype=np.uint32) if sources_local is None
               else np.ascontiguousarray(np.asarray(sources_local, dtype=np.uint32)))
        if len(src) != gs.num_graphs:
            raise ValueError("one (local) source entry per member")
        self.gs = gs
        h = C.c_void_p()
        check(lib().mk_set_runner_create(gs._h, q.ctypes.data, src.ctypes.data, C.byref(h)),
              "mk_set_runner_create")
        self._h = h
        bh, wh = C.c_void_p(), C.c_void_p()
        check(lib().mk_set_runner_handles(h, C.byref(bh), C.byref(wh)), "mk_set_runner_handles")
        bfs_m = np.flatnonzero(q == 0)
        glob = gs.offsets[bfs_m].astype(np.uint64) + src[bfs_m]
        # the views refer back weakly: no reference cycle, so the runner is
        # released (and its handles destroyed) while the set it holds lives
        me = weakref.ref(self)
        self.bfs = BFS._borrow(bh, gs.graph, glob, me) if bh.value else None
        self.wcc = WCC._borrow(wh, gs.graph, me) if wh.value else None
        self.single = False

    def set_single(self, on: bool) -> None:
        """One cooperative launch per step (deletes, inserts, then the member
        queries, separated by grid barriers) instead of four launches."""
        check(lib().mk_set_runner_set_single(self._h, int(bool(on))), "mk_set_runner_set_single")
        self.single = bool(on)

    def launches_per_step(self) -> int:
        n = C.c_uint32(0)
        check(lib().mk_set_runner_launches(self._h, C.byref(n)), "mk_set_runner_launches")
        return int(n.value)

    def step(self, del_src, del_dst, ins_src, ins_dst, ins_w=None, stream=None) -> None:
        check(lib().mk_set_runner_step(self._h, _ptr(del_src), _ptr(del_dst), _count(del_src, None),
                                       _ptr(ins_src), _ptr(ins_dst), _ptr(ins_w),
                                       _count(ins_src, None), _stream(stream)),
              "mk_set_runner_step")

    def close(self):
        for v in (getattr(self, "bfs", None), getattr(self, "wcc", None)):
            if v is not None:
                v.close()
        if getattr(self, "_h", None):
            lib().mk_set_runner_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def gen_rmat_members(vertex_offsets, edges_per_graph, a=0.57, b=0.19, c=0.19, seed=0, w_lo=1,
                     w_hi=64, weights=True, device: int = 0, stream=None, d_vertex_offsets=None):
    """Device R-MAT edges for the members of a (future) graph set: member m
    owns vertex ids vertex_offsets[m] .. vertex_offsets[m+1]-1 and gets
    edges_per_graph[m] edges.  Returns int32 tensors holding uint32 ids."""
    import torch
    dev = f"cuda:{device}"
    voff = np.ascontiguousarray(np.asarray(vertex_offsets, dtype=np.uint32))
    G = len(voff) - 1
    keep = None
    if d_vertex_offsets is None:
        keep = torch.from_numpy(voff.view(np.int32)).to(dev)
        d_vertex_offsets = keep.data_ptr()
    cnt = np.asarray(edges_per_graph, dtype=np.uint64)
    if len(cnt) != G:
        raise ValueError("one edge count per member")
    off = np.zeros(G + 1, dtype=np.uint64)
    np.cumsum(cnt, out=off[1:])
    E = int(off[-1])
    d_off = torch.from_numpy(off.view(np.int64)).to(dev)
    src = torch.empty(max(E, 1), dtype=torch.int32, device=dev)
    dst = torch.empty(max(E, 1), dtype=torch.int32, device=dev)
    w = torch.empty(max(E, 1), dtype=torch.int32, device=dev) if weights else None
    check(lib().mk_gen_rmat_set(d_vertex_offsets, G, d_off.data_ptr(), a, b, c, seed, w_lo, w_hi,
                                src.data_ptr(), dst.data_ptr(), _ptr(w), _stream(stream)),
          "mk_gen_rmat_set")
    if keep is not None:  # the kernel reads the offsets: keep them until it is done
        torch.cuda.synchronize(dev)
        del keep
    return src[:E], dst[:E], (w[:E] if w is not None else None)


# ---------------------------------------------------------------------------
# the reference drivers' text formats (host only)
# ---------------------------------------------------------------------------
def read_edge_list(path):
    """Graph file "V E" + E pairs (src/BFS.cu:27-36) -> (V, src, dst)."""
    p = str(path).encode()
    V, E = C.c_uint32(0), C.c_uint64(0)
    check(lib().mk_read_edge_list(p, C.byref(V), C.byref(E), None, None), "mk_read_edge_list")
    src = np.empty(E.value, dtype=np.uint32)
    dst = np.empty(E.value, dtype=np.uint32)
    check(lib().mk_read_edge_list(p, C.byref(V), C.byref(E), src.ctypes.data, dst.ctypes.data),
          "mk_read_edge_list")
    return V.value, src, dst


def read_batch(path):
    """Batch file "n" + n pairs (src/BFS.cu:76-91) -> (src, dst)."""
    p = str(path).encode()
    n = C.c_uint64(0)
    check(lib().mk_read_batch_file(p, C.byref(n), None, None), "mk_read_batch_file")
    src = np.empty(n.value, dtype=np.uint32)
    dst = np.empty(n.value, dtype=np.uint32)
    check(lib().mk_read_batch_file(p, C.byref(n), src.ctypes.data, dst.ctypes.data),
          "mk_read_batch_file")
    return src, dst


def write_edge_list(path, num_vertices: int, src, dst) -> None:
    s = np.ascontiguousarray(src, dtype=np.uint32)
    d = np.ascontiguousarray(dst, dtype=np.uint32)
    check(lib().mk_write_edge_list(str(path).encode(), int(num_vertices), len(s), s.ctypes.data,
                                   d.ctypes.data), "mk_write_edge_list")


def write_batch(path, src, dst) -> None:
    s = np.ascontiguousarray(src, dtype=np.uint32)
    d = np.ascontiguousarray(dst, dtype=np.uint32)
    check(lib().mk_write_batch_file(str(path).encode(), len(s), s.ctypes.data, d.ctypes.data),
          "mk_write_batch_file")


# ---------------------------------------------------------------------------
# synthetic inputs (host only)
# ---------------------------------------------------------------------------
def gen_rmat(scale: int, num_edges: int, a=0.57, b=0.19, c=0.19, seed=0, w_lo=1, w_hi=64,
             weights=True):
    src = np.empty(num_edges, dtype=np.uint32)
    dst = np.empty(num_edges, dtype=np.uint32)
    w = np.empty(num_edges, dtype=np.uint32) if weights else None
    check(lib().mk_gen_rmat(scale, num_edges, a, b, c, seed, w_lo, w_hi, src.ctypes.data,
                            dst.ctypes.data, _ptr(w)), "mk_gen_rmat")
    return src, dst, w


def gen_grid(side: int, shortcuts: int, seed=0, w_lo=1, w_hi=1000, weights=True):
    n = C.c_uint64(0)
    check(lib().mk_gen_grid(side, shortcuts, seed, w_lo, w_hi, None, None, None, C.byref(n)),
          "mk_gen_grid")
    src = np.empty(n.value, dtype=np.uint32)
    dst = np.empty(n.value, dtype=np.uint32)
    w = np.empty(n.value, dtype=np.uint32) if weights else None
    check(lib().mk_gen_grid(side, shortcuts, seed, w_lo, w_hi, src.ctypes.data, dst.ctypes.data,
                            _ptr(w), C.byref(n)), "mk_gen_grid")
    return src, dst, w


class EdgeSet:
    """Host edge set for drawing valid batches (absent inserts / present deletes)."""

    def __init__(self, num_vertices: int, src: np.ndarray, dst: np.ndarray):
        h = C.c_void_p()
        src = np.ascontiguousarray(src, dtype=np.uint32)
        dst = np.ascontiguousarray(dst, dtype=np.uint32)
        check(lib().mk_edgeset_create(num_vertices, src.ctypes.data, dst.ctypes.data, len(src),
                                      C.byref(h)), "mk_edgeset_create")
        self._h = h

    def __len__(self):
        return int(lib().mk_edgeset_size(self._h))

    def sample_absent(self, n: int, seed: int):
        s = np.empty(n, dtype=np.uint32)
        d = np.empty(n, dtype=np.uint32)
        check(lib().mk_edgeset_sample_absent(self._h, n, seed, s.ctypes.data, d.ctypes.data),
              "sample_absent")
        return s, d

    def sample_present(self, n: int, seed: int):
        s = np.empty(n, dtype=np.uint32)
        d = np.empty(n, dtype=np.uint32)
        check(lib().mk_edgeset_sample_present(self._h, n, seed, s.ctypes.data, d.ctypes.data),
              "sample_present")
        return s, d

    def close(self):
        if getattr(self, "_h", None):
            lib().mk_edgeset_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
