"""Batched many-graph execution: thousands of small dynamic graphs advanced
by one coalesced launch sequence per step.

A step over a set of member graphs applies one mixed update batch per member
and answers one query per member (a BFS from a source, or the member's
connected components).  Run per graph, as a user of the reference's classes
would (one DynamicGraph, one BFS/WCC object per graph;
include/Graph/SlabGraph.cuh, include/Algorithms/BFS.cuh), a step costs
about six launches per member and is bound by launch latency, since each
member's work is far too small to fill the GPU.  The batched runner keeps all
members in one GraphSet and issues, per step,

  one delete launch and one insert launch for every member's batch,
  one multi-source BFS (one source per BFS-queried member; a member of at
  most 65,535 vertices is traversed by one CTA with its state in shared
  memory), and
  one WCC launch over the WCC-queried members (a member of at most 65,536
  vertices is solved by one CTA with its union-find in shared memory),

each member's results being those of the member alone.  When every member
fits one CTA the step can also be ONE cooperative launch (set_single):
every delete, every insert, then the member queries, separated by grid
barriers.  Either form can be captured into a CUDA graph and replayed; the
autotuner picks the update kernel and the BFS frontier chunk of the
four-launch form on the live set.  There is no counterpart in the reference.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np

from . import BFS, WCC, DynamicGraph, GraphSet, SetRunner

QUERY_BFS, QUERY_WCC = 0, 1
WCC_LOCAL_MAX = 1 << 16  # vertices of a member that one CTA solves in shared memory
BFS_LOCAL_MAX = (1 << 16) - 1


@dataclass
class SetSpec:
    """Seeded shape of a graph set: sizes, edge counts, update sizes and query
    kinds per member (all host arrays of length num_graphs)."""
    num_vertices: np.ndarray   # int64
    num_edges: np.ndarray      # int64, R-MAT edges drawn per member
    deletes: np.ndarray        # int64, per-step deletes per member
    inserts: np.ndarray        # int64, per-step inserts per member
    query: np.ndarray          # uint8, QUERY_BFS or QUERY_WCC
    seed: int

    @property
    def num_graphs(self) -> int:
        return len(self.num_vertices)


DEFAULT_SEED = 0x4D45524B + 2


def make_spec(num_graphs: int = 4096, seed: int = DEFAULT_SEED, v_lo: int = 1024,
              v_hi: int = 65536, deg_lo: float = 4.0, deg_hi: float = 32.0,
              upd_lo: float = 0.01, upd_hi: float = 0.10) -> SetSpec:
    """Member sizes log-uniform in [v_lo, v_hi]; average degree from a power
    law with exponent 2 truncated to [deg_lo, deg_hi] (inverse-CDF draw);
    per-step update batch U[upd_lo, upd_hi] of the member's edges, half
    deletes and half inserts; query BFS or WCC by a fair coin."""
    rng = np.random.default_rng(seed)
    G = int(num_graphs)
    nv = np.exp(rng.uniform(np.log(v_lo), np.log(v_hi), G)).astype(np.int64)
    u = rng.random(G)
    deg = 1.0 / (1.0 / deg_lo - u * (1.0 / deg_lo - 1.0 / deg_hi))
    ne = np.maximum(1, np.round(nv * deg)).astype(np.int64)
    frac = rng.uniform(upd_lo, upd_hi, G)
    upd = np.maximum(2, np.round(ne * frac)).astype(np.int64)
    dels = upd // 2
    ins = upd - dels
    query = rng.integers(0, 2, G).astype(np.uint8)
    return SetSpec(nv, ne, dels, ins, query, int(seed))


def _offsets(counts) -> np.ndarray:
    o = np.zeros(len(counts) + 1, dtype=np.int64)
    np.cumsum(np.asarray(counts, dtype=np.int64), out=o[1:])
    return o


def pick_sources(degrees: np.ndarray, offsets: np.ndarray, members: Sequence[int],
                 seed: int) -> np.ndarray:
    """One seeded source per listed member: a random vertex with out-edges
    (the member's first vertex if it has none).  Local ids."""
    rng = np.random.default_rng(seed)
    out = np.zeros(len(members), dtype=np.uint32)
    for i, m in enumerate(members):
        lo, hi = int(offsets[m]), int(offsets[m + 1])
        nz = np.flatnonzero(degrees[lo:hi])
        out[i] = nz[rng.integers(0, len(nz))] if len(nz) else 0
    return out


class BatchedRunner:
    """All members in one GraphSet; one coalesced launch sequence per step
    (the C set runner's, mk_set_runner_step)."""

    def __init__(self, gs: GraphSet, query: np.ndarray, sources_local: np.ndarray):
        self.gs = gs
        self.G = gs.graph
        off = gs.offsets.astype(np.int64)
        self.bfs_members = np.flatnonzero(query == QUERY_BFS)
        self.wcc_members = np.flatnonzero(query == QUERY_WCC)
        glob = (off[self.bfs_members] + sources_local.astype(np.int64)).astype(np.uint32)
        self.sources_global = glob
        src_m = np.zeros(gs.num_graphs, dtype=np.uint32)
        src_m[self.bfs_members] = sources_local
        # the C runner holds the member tables; bfs / wcc are views of its
        # handles
        self.runner = SetRunner(gs, query, src_m)
        self.bfs = self.runner.bfs
        self.wcc = self.runner.wcc
        bsz = off[self.bfs_members + 1] - off[self.bfs_members]
        self._bfs_large = int((bsz > BFS_LOCAL_MAX).sum())
        sizes = off[self.wcc_members + 1] - off[self.wcc_members]
        self._wcc_large = int((sizes > WCC_LOCAL_MAX).sum())
        # every member fits one CTA: the step can also be one launch
        self.single_ok = int((off[1:] - off[:-1]).max()) <= BFS_LOCAL_MAX

    def set_single(self, on: bool) -> None:
        """One cooperative launch per step instead of four (set_single of the
        C runner)."""
        self.runner.set_single(on)

    def update(self, ds, dd, is_, id_, iw, stream=None):
        self.G.DeleteEdges(ds, dd, stream=stream)
        self.G.InsertEdges(is_, id_, vals=iw, stream=stream)

    def query(self, stream=None):
        if self.bfs is not None:
            self.bfs.StaticMembers(stream=stream, timed=False)
        if self.wcc is not None:
            self.wcc.StaticPrepared(stream=stream, timed=False)

    def step(self, batch, stream=None):
        self.runner.step(*batch, stream=stream)

    def launches_per_step(self) -> int:
        if self.runner.single:
            return 1
        # kernels: delete, insert; BFS: 1 shared-memory kernel (plus 2
        # memsets) and the cooperative device-wide kernel when some member is
        # larger than shared memory holds; WCC: 1 shared-memory kernel (plus 1
        # memset), and 5 device-wide kernels for such members
        bfs = (1 + (1 if self._bfs_large else 0)) if self.bfs is not None else 0
        wcc = (1 + (5 if self._wcc_large else 0)) if self.wcc is not None else 0
        return 2 + bfs + wcc

    def member_bfs(self, m_index: int, dist: Optional[np.ndarray] = None) -> np.ndarray:
        """BFS levels of the i-th BFS member (slice of the union result)."""
        d = self.bfs.Distances() if dist is None else dist
        m = self.bfs_members[m_index]
        lo, hi = int(self.gs.offsets[m]), int(self.gs.offsets[m + 1])
        return d[lo:hi]

    def close(self):
        self.runner.close()


class PlainRunner:
    """The per-graph baseline: one DynamicGraph and one BFS or WCC object per
    member, one launch chain per member and step."""

    def __init__(self, graphs: List[DynamicGraph], query: np.ndarray, sources_local: np.ndarray):
        self.graphs = graphs
        self.query_kind = query
        self.algos = []
        it = iter(sources_local.tolist())
        for g, q in zip(graphs, query.tolist()):
            self.algos.append(BFS(g, next(it)) if q == QUERY_BFS else WCC(g))

    def step(self, slices, stream=None):
        """slices[m] = (ds, dd, is_, id_, iw) device views with local ids."""
        for g, a, b in zip(self.graphs, self.algos, slices):
            ds, dd, is_, id_, iw = b
            if ds.numel():
                g.DeleteEdges(ds, dd, stream=stream)
            if is_.numel():
                g.InsertEdges(is_, id_, vals=iw, stream=stream)
            a.Static(stream=stream, timed=False)

    def launches_per_step(self) -> int:
        n = 0
        for q in self.query_kind.tolist():
            n += 2 + (1 if q == QUERY_BFS else 3)
        return n


def pool_slabs_for(num_vertices: int, num_edges: int) -> int:
    """Overflow slabs for a graph built with exact degree hints and then
    updated by batches of a few percent of its edges: about one per vertex
    plus one per ten edges (the automatic size is about twice the bucket
    count, with a 64 Ki-slab floor meant for one large graph)."""
    return int(num_vertices + num_edges // 10 + 1024)
