"""ctypes loader of the C oracle (oracle/mk_oracle.c).  Test infrastructure."""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "libmk_oracle.so"
_lib = None


def build_oracle() -> Path:
    src = HERE / "mk_oracle.c"
    if not LIB.exists() or LIB.stat().st_mtime < src.stat().st_mtime:
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
