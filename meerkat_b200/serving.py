"""Serving loop: many resident dynamic graphs answering a stream of update
and query requests, with continuous batching.

All graphs live in one GraphSet (weighted, out-edges).  A graph is a slot: it
holds at most one request on the GPU at a time, so its requests run in
arrival order, and a request that arrives while others are on the GPU is
admitted as soon as its graph's slot and the memory it needs are free.  Each
scheduling round takes the oldest pending request of every free graph:

  deletes of every graph in the round   one delete launch on the union graph
  inserts                               one insert launch
  BFS / SSSP queries                    one multi-source traversal each
                                        (one source per queried graph)
  WCC queries                           one range union-find pass

These fast segments are issued on one CUDA stream without waiting for the
device; a CUDA event after each segment marks its requests complete.
PageRank (push form on the member's out-edges, mk_pagerank_range_*) and
triangle counting (straight from the member's out-edges, mk_tc_range_*) are
heavy: a worker thread runs them one at a time on a second stream, so they
overlap the fast rounds instead of holding them up.

Admission: an insert of m edges needs at most m new slabs, so it waits
while the slabs in use (read back after every insert segment), plus the
inserts still in flight, plus m would pass the slab pool's capacity, and is
rejected when nothing in flight can change that (deletes never free slabs).
Triangle counting's scratch grows to the largest member counted; a member
whose scratch would take the resident set past the memory budget is
rejected.

Each graph's requests are served in arrival order, so every request sees
exactly the updates of its graph that arrived before it, whether it shares
its round with other graphs' requests ("coalesced") or runs alone ("alone":
one request at a time, synchronously: the plain per-request launch
sequence).  The tests check that every query answer is the same in both
modes and equals the oracle's.

No counterpart in the reference, whose drivers run one graph and one
algorithm per process (src/BFS.cu, src/PageRank.cu, src/TC.cu).
"""
from __future__ import annotations

import collections
import queue
import threading
import time
from dataclasses import dataclass, field
from typing import Dict, List

import numpy as np

from . import BFS, SSSP, WCC, GraphSet, PageRankRange, TCRange, gen_rmat_members

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
    service: float = 0.0    # seconds from issue to completion
    result: object = None   # query answer when results are recorded
    status: str = "ok"      # "ok", or why admission refused it


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
FAST_SEGMENTS = ((INSERT, DELETE), (BFS_Q, WCC_Q), (SSSP_Q,))

# triangle-count scratch per member (mk_tc_range): CSR export, row ids,
# reverse flags and the oriented CSR per edge; per-vertex counts and offsets
TC_BYTES_PER_EDGE = 17
TC_BYTES_PER_VERTEX = 64


class GraphServer:
    """Serves requests on a resident GraphSet within a device-memory budget."""

    def __init__(self, gs: GraphSet, budget_bytes: int, device: int = 0, record: bool = False,
                 max_update: int = 1_000_000):
        import torch
        self.gs = gs
        self.G = gs.graph
        self.device = device
        self.dev = torch.device(f"cuda:{device}")
        self.budget = int(budget_bytes)
        self.record = record
        self.off = gs.offsets.astype(np.int64)
        ng = len(self.off) - 1
        sizes = np.diff(self.off)
        first = [int(x) for x in self.off[:-1]]
        ranges = [(int(self.off[g]), int(self.off[g + 1])) for g in range(ng)]
        # the fast stream has the higher priority: its blocks are scheduled
        # ahead of a running PageRank or triangle count's
        self.fast = torch.cuda.Stream(self.dev, priority=-1)
        self.heavy = torch.cuda.Stream(self.dev, priority=0)
        self.bfs = BFS(self.G, first[:1])
        self.sssp = SSSP(self.G, first[:1])
        self.wcc = WCC(self.G)
        self.prr = PageRankRange(self.G, int(sizes.max()))
        self.tcr = TCRange(self.G)
        # size every per-round table for all members once, so rounds never
        # grow a device buffer (growth synchronises the device)
        self.bfs.set_sources(first)
        self.sssp.set_sources(first)
        self.wcc.PrepareRanges(ranges)
        self.G.reserve_batch(ng * int(max_update))
        info = self.G.info()
        V = gs.num_vertices
        # graph + two traversals (dist, stamp, bitmap, two frontiers, list) + WCC
        # + range PageRank (two FP64 vectors and an FP32 copy of the largest member)
        trav = 8 * V + 4 * V + V // 8 + 2 * 8 * (info["num_buckets"] + 64) + 4 * V
        self.resident = info["device_bytes"] + 2 * trav + 4 * V + V // 4 + 20 * int(sizes.max())
        if self.resident > self.budget:
            raise MemoryError(f"resident set {self.resident} B exceeds the budget {self.budget} B")
        self.tc_bytes = 0  # triangle-count scratch held so far
        self.pool_cap = int(info["pool_capacity"])
        self.slabs_used = int(info["slabs_used"])
        self.h_used = torch.zeros(1, dtype=torch.int32).pin_memory()
        self.h_tc = torch.zeros(1, dtype=torch.int64).pin_memory()
        # size the heavy requests' scratch on the member with the most edges
        # (a later growth would synchronise the device mid-run)
        edges = [int(self.G.count_edges(lo, hi)) for lo, hi in ranges]
        big = int(np.argmax(edges))
        warm = Request(rid=-1, graph=big, kind=TC_Q, arrival=0.0)
        self.run_heavy(warm, self.heavy)
        if warm.status != "ok":
            raise MemoryError("triangle-count scratch of the largest member exceeds the budget")
        self.prr.Run(*ranges[big], 0.85, 1e-6, 200, stream=self.heavy, timed=False)
        torch.cuda.synchronize(self.dev)

    def close(self):
        for o in (self.bfs, self.sssp, self.wcc, self.prr, self.tcr):
            o.close()

    # ---- admission ----
    def _tc_need(self, g: int, stream) -> int:
        # (the edge count uses the graph's own accumulator: heavy requests
        # alone call it, one at a time)
        n = int(self.off[g + 1] - self.off[g])
        e = int(self.G.count_edges(int(self.off[g]), int(self.off[g + 1]), stream=stream))
        return TC_BYTES_PER_EDGE * e + TC_BYTES_PER_VERTEX * n

    def _admit(self, r: Request, insert_inflight: int):
        """'go', 'wait' or 'reject' for the head request r (triangle counts
        are admitted against the budget by run_heavy)."""
        if r.kind == INSERT:
            m = r.hi - r.lo
            if self.slabs_used + insert_inflight + m + 1024 <= self.pool_cap:
                return "go"
            return "wait" if insert_inflight else "reject"
        return "go"

    # ---- the work of one fast segment (same-kind requests of distinct graphs) ----
    def issue_fast(self, reqs: List[Request], wl: Workload, stream) -> None:
        import torch
        P_s, P_d, P_w = wl.pool_src, wl.pool_dst, wl.pool_w
        dels = [r for r in reqs if r.kind == DELETE]
        inss = [r for r in reqs if r.kind == INSERT]
        with torch.cuda.stream(stream):
            if dels:
                ds = torch.cat([P_s[r.lo:r.hi] for r in dels])
                dd = torch.cat([P_d[r.lo:r.hi] for r in dels])
                self.G.DeleteEdges(ds, dd, stream=stream)
            if inss:
                is_ = torch.cat([P_s[r.lo:r.hi] for r in inss])
                id_ = torch.cat([P_d[r.lo:r.hi] for r in inss])
                iw = torch.cat([P_w[r.lo:r.hi] for r in inss])
                self.G.InsertEdges(is_, id_, vals=iw, stream=stream)
                self.G.slabs_used_async(self.h_used.data_ptr(), stream=stream)
        bfs = [r for r in reqs if r.kind == BFS_Q]
        sssp = [r for r in reqs if r.kind == SSSP_Q]
        wccs = [r for r in reqs if r.kind == WCC_Q]
        for trav, rs in ((self.bfs, bfs), (self.sssp, sssp)):
            if rs:
                trav.set_sources([int(self.off[r.graph]) + r.source for r in rs], stream=stream)
                trav.Static(stream=stream, timed=False)
        if wccs:
            self.wcc.PrepareRanges([(int(self.off[r.graph]), int(self.off[r.graph + 1]))
                                    for r in wccs], stream=stream)
            self.wcc.StaticPrepared(stream=stream, timed=False)
        if self.record:
            stream.synchronize()
            self._record(bfs, self.bfs)
            self._record(sssp, self.sssp)
            if wccs:
                lab = self.wcc.Labels().astype(np.int64)
                for r in wccs:
                    lo, hi = int(self.off[r.graph]), int(self.off[r.graph + 1])
                    r.result = (lab[lo:hi] - lo).astype(np.uint32)

    # ---- one PageRank or triangle-count request (blocking on `stream`) ----
    def run_heavy(self, r: Request, stream) -> None:
        lo, hi = int(self.off[r.graph]), int(self.off[r.graph + 1])
        if r.kind == PAGERANK_Q:
            self.prr.Run(lo, hi, 0.85, 1e-6, 200, stream=stream, timed=False)
            if self.record:
                r.result = self.prr.Values()
        else:
            need = self._tc_need(r.graph, stream)
            if need > self.tc_bytes and self.resident + need > self.budget:
                r.status = "rejected"
                return
            self.tcr.Run(lo, hi, stream=stream, timed=False)
            self.tc_bytes = max(self.tc_bytes, need)
            self.tcr.count_async(self.h_tc.data_ptr(), stream=stream)
            stream.synchronize()
            r.result = int(self.h_tc[0])

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
        is admitted once its arrival time has passed.  "coalesced": continuous
        batching as described in the module docstring (at most max_round fast
        requests per round if > 0).  "alone": one request at a time, issued
        and waited for (the plain per-request sequence).  A request completes
        when the device has finished its work (CUDA event time).  Returns
        latency and throughput."""
        assert mode in ("coalesced", "alone")
        if mode == "alone":
            return self._run_alone(reqs, wl)
        return self._run_coalesced(reqs, wl, max_round)

    def _summary(self, reqs, mode, rounds, rejected) -> dict:
        self.check()
        done = [r for r in reqs if r.status == "ok"]
        lat = np.array([r.done - r.arrival for r in done]) * 1000.0
        span = (max(r.done for r in reqs) - min(r.arrival for r in reqs)) if reqs else 0.0
        by_kind = {}
        for k in range(len(KIND_NAMES)):
            sel = [r.done - r.arrival for r in done if r.kind == k]
            svc = [r.service for r in done if r.kind == k]
            if sel:
                by_kind[KIND_NAMES[k]] = {"n": len(sel),
                                          "p50_ms": float(np.percentile(sel, 50) * 1000.0),
                                          "p99_ms": float(np.percentile(sel, 99) * 1000.0),
                                          "service_p50_ms": float(np.percentile(svc, 50) * 1000.0),
                                          "service_total_ms": float(np.sum(svc) * 1000.0)}
        n = len(done)
        return {"mode": mode, "requests": len(reqs), "rounds": rounds, "rejected": rejected,
                "p50_ms": float(np.percentile(lat, 50)) if n else 0.0,
                "p99_ms": float(np.percentile(lat, 99)) if n else 0.0,
                "mean_ms": float(lat.mean()) if n else 0.0,
                "throughput_rps": n / span if span > 0 else 0.0,
                "by_kind": by_kind}

    def _run_alone(self, reqs, wl) -> dict:
        s = self.fast
        t0 = time.perf_counter() - (reqs[0].arrival if reqs else 0.0)
        for r in reqs:
            now = time.perf_counter() - t0
            if r.arrival > now:
                time.sleep(r.arrival - now)
            start = time.perf_counter() - t0
            if r.kind in HEAVY_KINDS:
                self.run_heavy(r, s)
            else:
                self.issue_fast([r], wl, s)
            s.synchronize()
            r.done = time.perf_counter() - t0
            r.service = r.done - start
        return self._summary(reqs, "alone", len(reqs), sum(r.status != "ok" for r in reqs))

    def _run_coalesced(self, reqs, wl, max_round) -> dict:
        import torch
        n = len(reqs)
        queues: Dict[int, collections.deque] = collections.defaultdict(collections.deque)
        # a graph's fast requests may queue up behind each other on the fast
        # stream (stream order keeps them in arrival order); a heavy request
        # waits until its graph has nothing in flight, and nothing of its
        # graph is issued while it runs
        fast_pending: Dict[int, int] = collections.defaultdict(int)
        heavy_busy = set()
        inflight = []             # (event, requests, issue time, inserted edges)
        insert_inflight = 0
        heavy_running = 0
        heavy_q: "queue.Queue" = queue.Queue()
        heavy_done: "queue.Queue" = queue.Queue()
        base = torch.cuda.Event(enable_timing=True)
        rounds = rejected = 0
        t0 = time.perf_counter() - (reqs[0].arrival if reqs else 0.0)
        base.record(self.fast)
        base.synchronize()
        t_base = time.perf_counter() - t0

        def worker():
            torch.cuda.set_device(self.dev)
            while True:
                r = heavy_q.get()
                if r is None:
                    return
                start = time.perf_counter() - t0
                self.run_heavy(r, self.heavy)
                ev = torch.cuda.Event(enable_timing=True)
                ev.record(self.heavy)
                ev.synchronize()
                heavy_done.put((r, start, t_base + base.elapsed_time(ev) / 1000.0))

        th = threading.Thread(target=worker, daemon=True)
        th.start()
        i = finished = 0
        try:
            while finished < n:
                progressed = False
                # completions
                still = []
                for ev, rs, start, ins in inflight:
                    if ev.query():
                        done = t_base + base.elapsed_time(ev) / 1000.0
                        for r in rs:
                            r.done, r.service = done, done - start
                            fast_pending[r.graph] -= 1
                        finished += len(rs)
                        if ins:
                            insert_inflight -= ins
                            self.slabs_used = max(self.slabs_used, int(self.h_used[0]) & 0xFFFFFFFF)
                        progressed = True
                    else:
                        still.append((ev, rs, start, ins))
                inflight = still
                while not heavy_done.empty():
                    r, start, done = heavy_done.get()
                    r.done, r.service = done, done - start
                    heavy_busy.discard(r.graph)
                    heavy_running -= 1
                    finished += 1
                    rejected += r.status != "ok"
                    progressed = True
                # arrivals
                now = time.perf_counter() - t0
                while i < n and reqs[i].arrival <= now:
                    queues[reqs[i].graph].append(reqs[i])
                    i += 1
                # one round: the oldest pending request of every free graph
                heads = sorted((q[0] for g, q in queues.items() if q and g not in heavy_busy),
                               key=lambda r: r.arrival)
                fast = []
                for r in heads:
                    heavy = r.kind in HEAVY_KINDS
                    if heavy and fast_pending[r.graph]:
                        continue  # its graph's fast work must finish first
                    if not heavy and max_round > 0 and len(fast) >= max_round:
                        continue
                    verdict = self._admit(r, insert_inflight)
                    if verdict == "wait":
                        continue
                    queues[r.graph].popleft()
                    if verdict == "reject":
                        r.status = "rejected"
                        r.done = r.service = time.perf_counter() - t0
                        finished += 1
                        rejected += 1
                        progressed = True
                        continue
                    if heavy:
                        heavy_busy.add(r.graph)
                        heavy_running += 1
                        heavy_q.put(r)
                    else:
                        fast_pending[r.graph] += 1
                        if r.kind == INSERT:
                            insert_inflight += r.hi - r.lo
                        fast.append(r)
                for kinds in FAST_SEGMENTS:
                    seg = [r for r in fast if r.kind in kinds]
                    if not seg:
                        continue
                    start = time.perf_counter() - t0
                    self.issue_fast(seg, wl, self.fast)
                    ev = torch.cuda.Event(enable_timing=True)
                    ev.record(self.fast)
                    ins = sum(r.hi - r.lo for r in seg if r.kind == INSERT)
                    inflight.append((ev, seg, start, ins))
                    rounds += 1
                    progressed = True
                if not progressed:
                    # nothing to do until an arrival or a completion
                    wait = (reqs[i].arrival - (time.perf_counter() - t0)) if i < n else 1.0
                    if inflight or heavy_running:
                        wait = min(wait, 0.0001)
                    time.sleep(min(max(wait, 0.00002), 0.002))
        finally:
            heavy_q.put(None)
            th.join()
        torch.cuda.synchronize(self.dev)
        return self._summary(reqs, "coalesced", rounds, rejected)
