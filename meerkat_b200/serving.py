"""Serving loop: many resident dynamic graphs answering a stream of update
and query requests, with continuous batching.

All graphs live in one GraphSet (weighted, out-edges), so the requests of
one scheduling round -- at most one per graph, the head of each graph's
queue -- are served by coalesced launches:

  deletes of every graph in the round   one delete launch on the union graph
  inserts                               one insert launch
  BFS / SSSP queries                    one multi-source traversal each
                                        (one source per queried graph)
  WCC queries                           one subset union-find pass

PageRank runs on the member's out-edges directly (push form,
mk_pagerank_range_*).  Triangle counting needs the symmetric graph, so TC
requests run on per-graph views built on first use from a CSR export of the
member and kept current by replaying every later update of that graph on
them.  Views are admitted under a device-memory budget and evicted
least-recently-used.  These heavy requests run after the coalesced fast
work of their round, one segment each, so a triangle count does not hold up
the updates and traversals of other graphs in that round.

Each graph's requests are served in arrival order, so every request sees
exactly the updates of its graph that arrived before it, whether it shares
its round with other graphs' requests ("coalesced") or runs alone ("alone":
one request per round, the plain per-request launch sequence).  The tests
check that every query answer is the same in both modes.

No counterpart in the reference, whose drivers run one graph and one
algorithm per process (src/BFS.cu, src/PageRank.cu, src/TC.cu).
"""
from __future__ import annotations

import collections
import time
from dataclasses import dataclass, field
from typing import Dict, List, Optional

import numpy as np

from . import BFS, SSSP, TC, WCC, DynamicGraph, GraphSet, PageRankRange, gen_rmat_members

INSERT, DELETE, BFS_Q, SSSP_Q, PAGERANK_Q, TC_Q, WCC_Q = range(7)
KIND_NAMES = ["insert", "delete", "bfs", "sssp", "pagerank", "tc", "wcc"]
QUERY_KINDS = (BFS_Q, SSSP_Q, PAGERANK_Q, TC_Q, WCC_Q)


@dataclass
class Request:
    rid: int
    graph: int
    kind: int
    arrival: float          # seconds after the start of the run
    source: int = 0         # local source vertex (BFS / SSSP)
    lo: int = 0             # payload slice [lo, hi) of the update pool
    hi: int = 0
    done: float = -1.0      # completion time (seconds after the start)
    service: float = 0.0    # seconds of the round that served it
    result: object = None   # query answer when results are recorded


@dataclass
class Workload:
    """Graph sizes and a seeded request log with its update payloads (device
    tensors holding global vertex ids)."""
    num_vertices: np.ndarray
    num_edges: np.ndarray
    seed: int
    requests: List[Request] = field(default_factory=list)
    pool_src: object = None
    pool_dst: object = None
    pool_w: object = None


def make_graph_sizes(num_graphs: int, scale_lo: int, scale_hi: int, edge_factor: int, seed: int):
    rng = np.random.default_rng(seed)
    scales = rng.integers(scale_lo, scale_hi + 1, num_graphs)
    nv = (np.int64(1) << scales).astype(np.int64)
    return nv, nv * int(edge_factor)


def build_set(nv, ne, seed: int, device: int = 0, w_lo: int = 1, w_hi: int = 1000,
              pool_fraction: float = 0.0625):
    """The resident graph set (R-MAT members generated on the device) and the
    generated edges (kept for sampling delete payloads)."""
    import torch
    voff = np.zeros(len(nv) + 1, dtype=np.int64)
    np.cumsum(nv, out=voff[1:])
    src, dst, w = gen_rmat_members(voff, ne, seed=seed, w_lo=w_lo, w_hi=w_hi, device=device)
    V = int(voff[-1])
    hints = torch.bincount(src.long(), minlength=V).to(torch.int32).cpu().numpy().view(np.uint32)
    buckets_est = int(V + int(ne.sum()) // 10)
    gs = GraphSet(nv, degree_hints=[hints[voff[m]:voff[m + 1]] for m in range(len(nv))],
                  weighted=True, device=device,
                  pool_slabs=int(buckets_est * pool_fraction) + (1 << 23))
    # load in slices so the per-batch scratch stays small
    step = 1 << 27
    for a in range(0, src.numel(), step):
        gs.graph.InsertEdges(src[a:a + step], dst[a:a + step], vals=w[a:a + step])
    if gs.graph.sync() != 0:
        raise RuntimeError("device error while loading the graph set")
    return gs, (src, dst, w)


def make_requests(wl: Workload, edges, n: int, rate: float, seed: int, device: int = 0,
                  mix=(0.25, 0.25, 0.15, 0.15, 0.10, 0.05, 0.05), upd_lo: int = 1000,
                  upd_hi: int = 1_000_000, w_lo: int = 1, w_hi: int = 1000, t0: float = 0.0):
    """Appends n requests with Poisson arrivals at `rate` per second starting
    at t0.  Kinds drawn from `mix` (insert, delete, bfs, sssp, pagerank, tc,
    wcc); graph uniform; update sizes log-uniform in [upd_lo, upd_hi] (capped
    at the graph's edge count); deletes drawn from the graph's generated
    edges, inserts uniform pairs of distinct vertices; BFS/SSSP sources drawn
    among vertices with out-edges."""
    import torch
    rng = np.random.default_rng(seed)
    dev = f"cuda:{device}"
    src, dst, _ = edges
    nv, ne = wl.num_vertices, wl.num_edges
    G = len(nv)
    voff = np.zeros(G + 1, dtype=np.int64)
    np.cumsum(nv, out=voff[1:])
    eoff = np.zeros(G + 1, dtype=np.int64)
    np.cumsum(ne, out=eoff[1:])
    kinds = rng.choice(len(mix), size=n, p=np.asarray(mix) / np.sum(mix))
    graphs = rng.integers(0, G, n)
    gaps = rng.exponential(1.0 / rate, n)
    arrivals = t0 + np.cumsum(gaps)
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed)
    chunks_s, chunks_d, chunks_w = [], [], []
    pos = 0 if wl.pool_src is None else int(wl.pool_src.numel())
    deg = None
    base = len(wl.requests)
    for i in range(n):
        g, k = int(graphs[i]), int(kinds[i])
        r = Request(rid=base + i, graph=g, kind=k, arrival=float(arrivals[i]))
        if k in (INSERT, DELETE):
            m = int(np.exp(rng.uniform(np.log(upd_lo), np.log(upd_hi))))
            m = max(1, min(m, int(ne[g])))
            if k == DELETE:
                idx = torch.randint(int(eoff[g]), int(eoff[g + 1]), (m,), generator=gen, device=dev)
                chunks_s.append(src[idx])
                chunks_d.append(dst[idx])
                chunks_w.append(torch.zeros(m, dtype=torch.int32, device=dev))
            else:
                n_g = int(nv[g])
                u = torch.randint(0, n_g, (m,), generator=gen, device=dev)
                v = (u + 1 + torch.randint(0, n_g - 1, (m,), generator=gen, device=dev)) % n_g
                chunks_s.append((u + int(voff[g])).int())
                chunks_d.append((v + int(voff[g])).int())
                chunks_w.append(torch.randint(w_lo, w_hi + 1, (m,), generator=gen, device=dev,
                                              dtype=torch.int32))
            r.lo, r.hi = pos, pos + m
            pos += m
        elif k in (BFS_Q, SSSP_Q):
            if deg is None:
                deg = torch.bincount(src.long(), minlength=int(voff[-1]))
            lo = int(voff[g])
            nz = torch.nonzero(deg[lo:lo + int(nv[g])]).flatten()
            r.source = int(nz[int(rng.integers(0, nz.numel()))]) if nz.numel() else 0
        wl.requests.append(r)
    if chunks_s:
        parts = [wl.pool_src] if wl.pool_src is not None else []
        wl.pool_src = torch.cat(parts + chunks_s)
        parts = [wl.pool_dst] if wl.pool_dst is not None else []
        wl.pool_dst = torch.cat(parts + chunks_d)
        parts = [wl.pool_w] if wl.pool_w is not None else []
        wl.pool_w = torch.cat(parts + chunks_w)
    return wl.requests[base:]


HEAVY_KINDS = (PAGERANK_Q, TC_Q)


class _View:
    """The symmetric copy of one member, for triangle counting (the union
    graph holds out-edges only)."""

    def __init__(self, gs: GraphSet, g: int, device: int):
        import torch
        lo, hi = int(gs.offsets[g]), int(gs.offsets[g + 1])
        n = hi - lo
        self.n = n
        rp, col, _ = gs.graph.export_csr_range_device(lo, hi)
        rows = torch.repeat_interleave(torch.arange(n, device=col.device, dtype=torch.int32),
                                       (rp[1:] - rp[:-1]))
        cols = col - lo
        e = int(cols.numel())
        indeg = torch.bincount(cols.long(), minlength=n).to(torch.int32).cpu().numpy().view(np.uint32)
        outdeg = (rp[1:] - rp[:-1]).to(torch.int32).cpu().numpy().view(np.uint32)
        self.graph = DynamicGraph(n, degree_hints=indeg + outdeg, device=device,
                                  pool_slabs=max(4096, (n + e // 10) // 4))
        self.graph.InsertEdges(torch.cat([rows, cols]), torch.cat([cols, rows]))
        del rp, col, rows, cols
        if self.graph.sync() != 0:
            raise RuntimeError("device error while building a view")
        self.tc = TC(self.graph, n)
        # the graph, plus TC's oriented copy of the symmetric edges
        self.bytes = self.graph.info()["device_bytes"] + 8 * n + 4 * e

    def apply(self, kind: int, u, w_, reverse_found):
        """Replays one update of the member (local ids) on the view."""
        import torch
        if kind == INSERT:
            self.graph.InsertEdges(torch.cat([u, w_]), torch.cat([w_, u]))
        else:
            # the undirected edge goes only when neither direction is left
            keep = reverse_found == 0
            uu, ww = u[keep], w_[keep]
            self.graph.DeleteEdges(torch.cat([uu, ww]), torch.cat([ww, uu]))

    def close(self):
        self.tc.close()
        self.graph.close()


class GraphServer:
    """Serves requests on a resident GraphSet within a device-memory budget."""

    def __init__(self, gs: GraphSet, budget_bytes: int, device: int = 0, record: bool = False):
        self.gs = gs
        self.G = gs.graph
        self.device = device
        self.budget = int(budget_bytes)
        self.record = record
        self.off = gs.offsets.astype(np.int64)
        first = [int(self.off[0])]
        self.bfs = BFS(self.G, first)
        self.sssp = SSSP(self.G, first)
        self.wcc = WCC(self.G)
        sizes = np.diff(self.off)
        self.prr = PageRankRange(self.G, int(sizes.max()))
        self.views: "collections.OrderedDict[int, _View]" = collections.OrderedDict()
        V = gs.num_vertices
        info = self.G.info()
        # graph + two traversals (dist, stamp, bitmap, two frontiers, list) + WCC
        # + range PageRank (two FP64 vectors and an FP32 copy of the largest member)
        trav = 8 * V + 4 * V + V // 8 + 2 * 8 * (info["num_buckets"] + 64) + 4 * V
        self.resident = info["device_bytes"] + 2 * trav + 4 * V + V // 4 + 20 * int(sizes.max())
        if self.resident > self.budget:
            raise MemoryError(f"resident set {self.resident} B exceeds the budget {self.budget} B")
        self.view_builds = 0
        self.view_evictions = 0

    def reset_views(self) -> None:
        """Drops every cached view (a run that must start cold)."""
        for v in self.views.values():
            v.close()
        self.views.clear()

    def view_bytes(self) -> int:
        return sum(v.bytes for v in self.views.values())

    def _view(self, g: int) -> _View:
        v = self.views.get(g)
        if v is not None:
            self.views.move_to_end(g)
            return v
        lo, hi = int(self.off[g]), int(self.off[g + 1])
        n, e = hi - lo, int(self.G.count_edges(lo, hi))
        est = 128 * (n + 2 * e // 15) + 8 * n + 4 * e
        while self.views and self.resident + self.view_bytes() + est > self.budget:
            _, old = self.views.popitem(last=False)
            old.close()
            self.view_evictions += 1
        if self.resident + est > self.budget:
            raise MemoryError(f"graph {g}: its symmetric view does not fit the budget")
        v = _View(self.gs, g, self.device)
        self.views[g] = v
        self.view_builds += 1
        # the estimate was short: evict older views until the real size fits
        while len(self.views) > 1 and self.resident + self.view_bytes() > self.budget:
            _, old = self.views.popitem(last=False)
            old.close()
            self.view_evictions += 1
        return v

    # ---- a coalesced round of fast requests: at most one per graph ----
    def serve_fast(self, reqs: List[Request], wl: Workload) -> None:
        import torch
        assert len({r.graph for r in reqs}) == len(reqs), "one request per graph per round"
        assert all(r.kind not in HEAVY_KINDS for r in reqs)
        dels = [r for r in reqs if r.kind == DELETE]
        inss = [r for r in reqs if r.kind == INSERT]
        P_s, P_d, P_w = wl.pool_src, wl.pool_dst, wl.pool_w
        if dels:
            ds = torch.cat([P_s[r.lo:r.hi] for r in dels])
            dd = torch.cat([P_d[r.lo:r.hi] for r in dels])
            self.G.DeleteEdges(ds, dd)
        if inss:
            is_ = torch.cat([P_s[r.lo:r.hi] for r in inss])
            id_ = torch.cat([P_d[r.lo:r.hi] for r in inss])
            iw = torch.cat([P_w[r.lo:r.hi] for r in inss])
            self.G.InsertEdges(is_, id_, vals=iw)
        # keep cached views current (per graph: the same batch, local ids)
        for r in dels + inss:
            v = self.views.get(r.graph)
            if v is None:
                continue
            base = int(self.off[r.graph])
            u, w_ = P_s[r.lo:r.hi] - base, P_d[r.lo:r.hi] - base
            found = None
            if r.kind == DELETE:
                found = torch.zeros(u.numel(), dtype=torch.uint8, device=u.device)
                self.G.SearchEdges(P_d[r.lo:r.hi], P_s[r.lo:r.hi], found)
            v.apply(r.kind, u, w_, found)
        bfs = [r for r in reqs if r.kind == BFS_Q]
        sssp = [r for r in reqs if r.kind == SSSP_Q]
        wccs = [r for r in reqs if r.kind == WCC_Q]
        for trav, rs in ((self.bfs, bfs), (self.sssp, sssp)):
            if rs:
                trav.set_sources([int(self.off[r.graph]) + r.source for r in rs])
                trav.Static(timed=False)
        if wccs:
            self.wcc.StaticRanges([(int(self.off[r.graph]), int(self.off[r.graph + 1]))
                                   for r in wccs], timed=False)
        if self.record:
            self._record(bfs, self.bfs)
            self._record(sssp, self.sssp)
            if wccs:
                lab = self.wcc.Labels().astype(np.int64)
                for r in wccs:
                    lo, hi = int(self.off[r.graph]), int(self.off[r.graph + 1])
                    r.result = (lab[lo:hi] - lo).astype(np.uint32)

    # ---- one PageRank (on the member itself) or triangle-count (on its view) request ----
    def serve_heavy(self, r: Request) -> None:
        if r.kind == PAGERANK_Q:
            # PageRank on the member's out-edges: no view to build
            self.prr.Run(int(self.off[r.graph]), int(self.off[r.graph + 1]), 0.85, 1e-6, 200,
                         timed=False)
            if self.record:
                r.result = self.prr.Values()
        else:
            v = self._view(r.graph)
            v.tc.Static(timed=False)
            r.result = v.tc.GetCount()

    def serve_round(self, reqs: List[Request], wl: Workload) -> None:
        """Fast requests as one coalesced round, then the heavy ones in order."""
        fast = [r for r in reqs if r.kind not in HEAVY_KINDS]
        if fast:
            self.serve_fast(fast, wl)
        for r in reqs:
            if r.kind in HEAVY_KINDS:
                self.serve_heavy(r)

    def _record(self, rs, trav):
        if not rs:
            return
        d = trav.Distances()
        for r in rs:
            lo, hi = int(self.off[r.graph]), int(self.off[r.graph + 1])
            r.result = d[lo:hi].copy()

    def check(self) -> None:
        if self.G.sync() != 0:
            raise RuntimeError("device error in the graph set")

    # ---- open-loop driver ----
    def run(self, reqs: List[Request], wl: Workload, mode: str = "coalesced",
            max_round: int = 0) -> dict:
        """Serves `reqs` (sorted by arrival) against the wall clock: a request
        is admitted once its arrival time has passed.  "coalesced": each round
        takes the head request of every graph with a pending one, runs the fast
        heads (at most max_round if > 0) as coalesced segments by kind (updates,
        then BFS and WCC, then SSSP) and then the
        heavy heads (PageRank / TC) one segment each.  "alone": each
        round runs the single oldest request.  A request completes when the
        GPU has finished its segment.  Returns latency and throughput."""
        import torch
        assert mode in ("coalesced", "alone")
        queues: Dict[int, collections.deque] = collections.defaultdict(collections.deque)
        fifo = collections.deque()
        i, served, rounds, n = 0, 0, 0, len(reqs)
        builds0, evictions0 = self.view_builds, self.view_evictions
        t0 = time.perf_counter() - (reqs[0].arrival if reqs else 0.0)
        while served < n:
            now = time.perf_counter() - t0
            while i < n and reqs[i].arrival <= now:
                queues[reqs[i].graph].append(reqs[i])
                if mode == "alone":
                    fifo.append(reqs[i])
                i += 1
            if served == i:  # idle until the next arrival
                wait = reqs[i].arrival - now
                if wait > 0.0005:
                    time.sleep(wait - 0.0003)
                continue
            segments = []  # (kind of segment, requests)
            if mode == "alone":
                r = fifo.popleft()
                queues[r.graph].popleft()
                segments.append(("heavy" if r.kind in HEAVY_KINDS else "fast", [r]))
            else:
                heads = sorted((q[0] for q in queues.values() if q), key=lambda r: r.arrival)
                fast = [r for r in heads if r.kind not in HEAVY_KINDS]
                heavy = [r for r in heads if r.kind in HEAVY_KINDS]
                if max_round > 0:
                    fast = fast[:max_round]
                # cheap kinds first, each kind group its own segment, so an
                # update does not wait for the round's traversals
                for kinds in ((INSERT, DELETE), (BFS_Q, WCC_Q), (SSSP_Q,)):
                    seg = [r for r in fast if r.kind in kinds]
                    if seg:
                        segments.append(("fast", seg))
                for r in heavy:  # each heavy request its own segment, oldest first
                    segments.append(("heavy", [r]))
                for _, rs in segments:
                    for r in rs:
                        queues[r.graph].popleft()
            for kind, rs in segments:
                start = time.perf_counter() - t0
                if kind == "fast":
                    self.serve_fast(rs, wl)
                else:
                    self.serve_heavy(rs[0])
                torch.cuda.synchronize(self.device)
                done = time.perf_counter() - t0
                for r in rs:
                    r.done = done
                    r.service = done - start
                served += len(rs)
                rounds += 1
        self.check()
        lat = np.array([r.done - r.arrival for r in reqs]) * 1000.0
        span = max(r.done for r in reqs) - min(r.arrival for r in reqs) if reqs else 0.0
        by_kind = {}
        for k in range(len(KIND_NAMES)):
            sel = [r.done - r.arrival for r in reqs if r.kind == k]
            svc = [r.service for r in reqs if r.kind == k]
            if sel:
                by_kind[KIND_NAMES[k]] = {"n": len(sel),
                                          "p50_ms": float(np.percentile(sel, 50) * 1000.0),
                                          "p99_ms": float(np.percentile(sel, 99) * 1000.0),
                                          "service_p50_ms": float(np.percentile(svc, 50) * 1000.0)}
        return {"mode": mode, "requests": n, "rounds": rounds,
                "p50_ms": float(np.percentile(lat, 50)) if n else 0.0,
                "p99_ms": float(np.percentile(lat, 99)) if n else 0.0,
                "mean_ms": float(lat.mean()) if n else 0.0,
                "throughput_rps": n / span if span > 0 else 0.0,
                "by_kind": by_kind, "view_builds": self.view_builds - builds0,
                "view_evictions": self.view_evictions - evictions0}

    def close(self):
        for v in self.views.values():
            v.close()
        self.views.clear()
        for o in (self.bfs, self.sssp, self.wcc, self.prr):
            o.close()
