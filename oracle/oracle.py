"""ctypes loader of the C oracle (oracle/mk_oracle.c).  Test infrastructure."""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "libmk_oracle.so"
_lib = None


SOURCES = ("mk_oracle.c", "mk_gen.c", "mk_cpu.c", "mk_oracle.h")


def build_oracle() -> Path:
    stale = not LIB.exists() or any(LIB.stat().st_mtime < (HERE / f).stat().st_mtime
                                    for f in SOURCES)
    if stale:
        subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def _L():
    global _lib
    if _lib is None:
        build_oracle()
        L = C.CDLL(str(LIB))
        vp = C.c_void_p
        sig = {
            "og_create": (vp, [C.c_uint32, C.c_int]),
            "og_destroy": (None, [vp]),
            "og_insert": (C.c_uint64, [vp, vp, vp, vp, C.c_uint64, vp]),
            "og_delete": (C.c_uint64, [vp, vp, vp, C.c_uint64, vp]),
            "og_has_edge": (C.c_int, [vp, C.c_uint32, C.c_uint32, vp]),
            "og_num_edges": (C.c_uint64, [vp]),
            "og_degrees": (None, [vp, vp]),
            "og_export_csr": (None, [vp, vp, vp, vp]),
            "og_bfs": (None, [vp, C.c_uint32, vp]),
            "og_sssp": (C.c_int, [vp, C.c_uint32, vp]),
            "og_check_parents": (C.c_uint64, [vp, C.c_uint32, vp, C.c_int]),
            "og_pagerank": (C.c_uint32, [vp, C.c_double, C.c_double, C.c_uint32, C.c_int, vp]),
            "og_triangles": (C.c_uint64, [vp]),
            "og_wcc": (None, [vp, vp]),
            # host generators (mk_gen.c)
            "og_gen_rmat": (C.c_int, [C.c_uint32, C.c_uint64, C.c_double, C.c_double, C.c_double,
                                      C.c_uint64, C.c_uint32, C.c_uint32, vp, vp, vp]),
            "oes_create": (vp, [C.c_uint32, vp, vp, C.c_uint64]),
            "oes_destroy": (None, [vp]),
            "oes_size": (C.c_uint64, [vp]),
            "oes_sample_absent": (C.c_int, [vp, C.c_uint64, C.c_uint64, vp, vp]),
            "oes_sample_present": (C.c_int, [vp, C.c_uint64, C.c_uint64, vp, vp]),
            # multithreaded CPU baseline (mk_cpu.c)
            "otrav_create": (vp, [vp, C.c_uint32, C.c_int]),
            "otrav_destroy": (None, [vp]),
            "otrav_static": (None, [vp]),
            "otrav_incremental": (None, [vp, vp, vp, C.c_uint64]),
            "otrav_decremental": (None, [vp, vp, vp, C.c_uint64]),
            "otrav_distances": (None, [vp, vp]),
            "otrav_packed": (None, [vp, vp]),
            "otrav_stats": (None, [vp, vp, vp, vp]),
            "oc_pagerank": (C.c_uint32, [vp, C.c_double, C.c_double, C.c_uint32, C.c_int, vp]),
            "oc_triangles": (C.c_uint64, [vp]),
            "oc_wcc": (None, [vp, vp]),
            "oc_wcc_incremental": (None, [C.c_uint32, vp, vp, vp, C.c_uint64]),
        }
        for k, (r, a) in sig.items():
            f = getattr(L, k)
            f.restype = r
            f.argtypes = a
        _lib = L
    return _lib


def _u32(a):
    return np.ascontiguousarray(a, dtype=np.uint32)


class OracleGraph:
    """Directed simple graph with the reference's batch semantics."""

    def __init__(self, num_vertices: int, threads: int = 1):
        self.V = int(num_vertices)
        self._h = _L().og_create(self.V, int(threads))

    def __del__(self):
        if getattr(self, "_h", None):
            _L().og_destroy(self._h)
            self._h = None

    def insert(self, src, dst, w=None):
        s, d = _u32(src), _u32(dst)
        ww = _u32(w) if w is not None else None
        applied = np.zeros(len(s), dtype=np.uint8)
        n = _L().og_insert(self._h, s.ctypes.data, d.ctypes.data,
                           ww.ctypes.data if ww is not None else None, len(s), applied.ctypes.data)
        return int(n), applied

    def delete(self, src, dst):
        s, d = _u32(src), _u32(dst)
        applied = np.zeros(len(s), dtype=np.uint8)
        n = _L().og_delete(self._h, s.ctypes.data, d.ctypes.data, len(s), applied.ctypes.data)
        return int(n), applied

    def num_edges(self) -> int:
        return int(_L().og_num_edges(self._h))

    def degrees(self):
        out = np.zeros(self.V, dtype=np.uint32)
        _L().og_degrees(self._h, out.ctypes.data)
        return out

    def csr(self, weights=False):
        E = self.num_edges()
        rp = np.zeros(self.V + 1, dtype=np.uint64)
        col = np.zeros(max(E, 1), dtype=np.uint32)
        w = np.zeros(max(E, 1), dtype=np.uint32) if weights else None
        _L().og_export_csr(self._h, rp.ctypes.data, col.ctypes.data,
                           w.ctypes.data if w is not None else None)
        return rp, col[:E], (w[:E] if w is not None else None)

    def bfs(self, src):
        out = np.zeros(self.V, dtype=np.uint32)
        _L().og_bfs(self._h, int(src), out.ctypes.data)
        return out

    def sssp(self, src):
        out = np.zeros(self.V, dtype=np.uint32)
        rc = _L().og_sssp(self._h, int(src), out.ctypes.data)
        if rc != 0:
            raise OverflowError("a shortest distance does not fit in uint32")
        return out

    def check_parents(self, src, packed, weighted):
        p = np.ascontiguousarray(packed, dtype=np.uint64)
        return int(_L().og_check_parents(self._h, int(src), p.ctypes.data, int(bool(weighted))))

    def pagerank(self, d=0.85, tol=1e-13, max_iter=10000, warm=None):
        pr = np.zeros(self.V, dtype=np.float64) if warm is None else np.array(warm, dtype=np.float64)
        it = _L().og_pagerank(self._h, float(d), float(tol), int(max_iter), int(warm is not None),
                              pr.ctypes.data)
        return pr, int(it)

    def triangles(self) -> int:
        return int(_L().og_triangles(self._h))

    def wcc(self):
        out = np.zeros(self.V, dtype=np.uint32)
        _L().og_wcc(self._h, out.ctypes.data)
        return out


# ---------------------------------------------------------------------------
# host generators of the benchmark's inputs (mk_gen.c)
# ---------------------------------------------------------------------------
def gen_rmat(scale, num_edges, a=0.57, b=0.19, c=0.19, seed=0, w_lo=1, w_hi=1):
    """R-MAT edges as the product's generator draws them (same seeds, same
    edges), without loading the product library."""
    E = int(num_edges)
    s = np.empty(E, dtype=np.uint32)
    d = np.empty(E, dtype=np.uint32)
    w = np.empty(E, dtype=np.uint32)
    rc = _L().og_gen_rmat(int(scale), E, float(a), float(b), float(c), int(seed) & (2**64 - 1),
                          int(w_lo), int(w_hi), s.ctypes.data, d.ctypes.data, w.ctypes.data)
    if rc != 0:
        raise ValueError("og_gen_rmat: bad argument or graph too dense")
    return s, d, w


class OracleEdgeSet:
    """Edge-set tracker drawing absent-edge inserts and present-edge deletes,
    the same draws as the product's EdgeSet."""

    def __init__(self, num_vertices, src, dst):
        s, d = _u32(src), _u32(dst)
        self._h = _L().oes_create(int(num_vertices), s.ctypes.data, d.ctypes.data, len(s))

    def __del__(self):
        if getattr(self, "_h", None):
            _L().oes_destroy(self._h)
            self._h = None

    def __len__(self):
        return int(_L().oes_size(self._h))

    def sample_absent(self, n, seed):
        s = np.empty(n, dtype=np.uint32)
        d = np.empty(n, dtype=np.uint32)
        if _L().oes_sample_absent(self._h, int(n), int(seed) & (2**64 - 1), s.ctypes.data,
                                  d.ctypes.data) != 0:
            raise ValueError("oes_sample_absent: graph too dense")
        return s, d

    def sample_present(self, n, seed):
        s = np.empty(n, dtype=np.uint32)
        d = np.empty(n, dtype=np.uint32)
        if _L().oes_sample_present(self._h, int(n), int(seed) & (2**64 - 1), s.ctypes.data,
                                   d.ctypes.data) != 0:
            raise ValueError("oes_sample_present: fewer edges than requested")
        return s, d


# ---------------------------------------------------------------------------
# multithreaded CPU baseline (mk_cpu.c), on an OracleGraph
# ---------------------------------------------------------------------------
class CpuTraversal:
    """BFS (weighted=False) or SSSP (weighted=True) from one source with
    static, incremental and decremental calls, as the GPU traversals."""

    def __init__(self, graph: OracleGraph, source: int, weighted: bool):
        self.graph = graph  # keeps the adjacency alive
        self.V = graph.V
        self._h = _L().otrav_create(graph._h, int(source), int(bool(weighted)))

    def __del__(self):
        if getattr(self, "_h", None):
            _L().otrav_destroy(self._h)
            self._h = None

    def static(self):
        _L().otrav_static(self._h)

    def incremental(self, src, dst):
        s, d = _u32(src), _u32(dst)
        _L().otrav_incremental(self._h, s.ctypes.data, d.ctypes.data, len(s))

    def decremental(self, src, dst):
        s, d = _u32(src), _u32(dst)
        _L().otrav_decremental(self._h, s.ctypes.data, d.ctypes.data, len(s))

    def distances(self):
        out = np.empty(self.V, dtype=np.uint32)
        _L().otrav_distances(self._h, out.ctypes.data)
        return out

    def packed(self):
        out = np.empty(self.V, dtype=np.uint64)
        _L().otrav_packed(self._h, out.ctypes.data)
        return out

    def stats(self):
        lv, inv, rec = C.c_uint32(0), C.c_uint64(0), C.c_int(0)
        _L().otrav_stats(self._h, C.byref(lv), C.byref(inv), C.byref(rec))
        return {"levels": lv.value, "invalidated": inv.value, "recomputed": bool(rec.value)}


def cpu_pagerank(graph: OracleGraph, d=0.85, tol=1e-13, max_iter=10000, warm=None):
    pr = np.full(graph.V, 0.0) if warm is None else np.array(warm, dtype=np.float64)
    it = _L().oc_pagerank(graph._h, float(d), float(tol), int(max_iter), int(warm is not None),
                          pr.ctypes.data)
    return pr, int(it)


def cpu_triangles(graph: OracleGraph) -> int:
    return int(_L().oc_triangles(graph._h))


def cpu_wcc(graph: OracleGraph):
    out = np.empty(graph.V, dtype=np.uint32)
    _L().oc_wcc(graph._h, out.ctypes.data)
    return out


def cpu_wcc_incremental(labels, src, dst):
    """Unions the batch edges into min-id labels (updated in place)."""
    lab = np.ascontiguousarray(labels, dtype=np.uint32)
    s, d = _u32(src), _u32(dst)
    _L().oc_wcc_incremental(len(lab), lab.ctypes.data, s.ctypes.data, d.ctypes.data, len(s))
    return lab
