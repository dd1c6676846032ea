"""Benchmark: batched slab-graph updates on R-MAT scale 22 (the large config).

Workload (`rmat22_mixed_1M`): R-MAT scale 22 (4,194,304 vertices, 67,108,864
distinct directed edges, a/b/c/d = .57/.19/.19/.05, seeded), uint32 weights
uniform in [1, 1000], weighted slab graph with exact degree hints and load
factor 0.7.  One step applies one mixed batch of 1,000,000 edges: a delete
sub-batch of 500,000 present edges, then an insert sub-batch of 500,000
absent edges (uniformly sampled, seeded, generated on the host).

Reported:
  value      edge updates/s over the K timed steps (inputs resident in HBM)
  e2e        the same through the C ABI with pinned host batches: the H2D
             copies of each step's batch and the D2H read of its applied
             counts are inside the timed region (the next step's upload
             overlaps the current step's kernels)
  roofline   algorithmic bytes of the update kernels / their event-timed
             duration vs the measured HBM copy bandwidth
  incremental / decremental BFS and SSSP ms per batch after each sub-batch
  cpu_baseline  the CPU oracle (multithreaded port) applying mixed batches
                on the same graph
  batched    4,096 small graphs (V log-uniform in [1024, 65536]) advanced by
             the batched runner (one graph set, one coalesced launch sequence
             per step, CUDA-graph replay) against the per-graph launch
             sequence on the same members and batches, with every member's
             answer checked equal in both arms
  serving    64 resident R-MAT graphs (scales 18-23) under a 120 GB budget,
             open-loop Poisson requests at two offered rates, served with
             continuous batching and one request at a time (p50 / p99)

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
    python bench.py --workload batched [--graphs G]   # the batched comparison alone
    python bench.py --workload serving [--serving-rates R1,R2,...]   # the serving sweep alone
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

SEED = 0x4D45524B + 1  # large config
METRIC = "edge updates/s"
HALF = 500_000          # sub-batch size (delete, then insert)
SCALE = 22
EDGES = 67_108_864      # 16 * 2^22
W_LO, W_HI = 1, 1000
# algorithmic bytes per applied edge (record + one 128-B slab probe + entry write)
INS_BYTES = 12 + 128 + 8
DEL_BYTES = 8 + 128 + 4


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def measured_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


def profile_traffic():
    """DRAM bytes per update launch from the committed ncu summary, if any."""
    p = ROOT / "profiles" / "k_update_rmat22.md"
    if not p.exists():
        return None
    for line in p.read_text().splitlines():
        if line.startswith("traffic_bytes_per_step:"):
            try:
                return float(line.split(":", 1)[1].strip())
            except ValueError:
                return None
    return None


class Clocks:
    """SM clock and clock-event reasons sampled through NVML by a polling thread
    for the whole timed region (reads only; no GPU setting is changed)."""

    REASONS = {"hw_slowdown": "nvmlClocksEventReasonHwSlowdown",
               "hw_thermal_slowdown": "nvmlClocksEventReasonHwThermalSlowdown",
               "sw_thermal_slowdown": "nvmlClocksEventReasonSwThermalSlowdown",
               "sw_power_cap": "nvmlClocksEventReasonSwPowerCap"}

    def __init__(self, gpu_index: int):
        import threading
        self.samples = []
        self.stop_flag = threading.Event()
        self.t = None
        try:
            import pynvml as N
            N.nvmlInit()
            vis = os.environ.get("CUDA_VISIBLE_DEVICES")
            idx = int(vis.split(",")[gpu_index]) if vis and vis.split(",")[0].isdigit() else gpu_index
            self.N, self.h = N, N.nvmlDeviceGetHandleByIndex(idx)
            self.max_mhz = N.nvmlDeviceGetMaxClockInfo(self.h, N.NVML_CLOCK_SM)
        except Exception as ex:  # no NVML: report nothing rather than guess
            log(f"[bench] NVML unavailable: {ex}")
            self.N = None
            return
        self.t = threading.Thread(target=self._run, daemon=True)
        self.t.start()

    def _sample(self):
        N = self.N
        sm = N.nvmlDeviceGetClockInfo(self.h, N.NVML_CLOCK_SM)
        try:
            r = N.nvmlDeviceGetCurrentClocksEventReasons(self.h)
        except Exception:
            r = N.nvmlDeviceGetCurrentClocksThrottleReasons(self.h)
        self.samples.append((time.perf_counter(), sm, r))

    def _run(self):
        # 2 ms between samples: enough to see the clocks of a sub-second
        # region without holding the GIL against the host-issued arms
        while not self.stop_flag.is_set():
            try:
                self._sample()
            except Exception:
                break
            time.sleep(0.002)

    def stop(self):
        if self.N is None:
            return None
        self.stop_flag.set()
        self.t.join(timeout=5)
        if not self.samples:
            return None
        names = [k for k, attr in self.REASONS.items()
                 if any(r & getattr(self.N, attr, 0) for _, _, r in self.samples)]
        sm = [x for _, x, _ in self.samples]
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(names), "samples": len(sm), "source": "nvml"}


def probe_random_rmw(line_bytes: int, small_words: int, num_ops: int, repeats: int = 5,
                     device: int = 0) -> dict:
    """Operations per second of the update path's memory pattern (random
    128-B line read; + CAS; + a random 4-B read and add) for modes 0, 1, 2,
    best of `repeats` launches each, on a fresh buffer of line_bytes bytes.
    Runs the benchmark-only libmk_bench_probe.so."""
    import ctypes as C

    import torch
    from meerkat_b200.build import build_bench_probe
    L = C.CDLL(str(build_bench_probe()))
    vp = C.c_void_p
    f = L.mkb_probe_random_rmw
    f.restype = C.c_int
    f.argtypes = [vp, C.c_uint64, vp, vp, C.c_uint32, C.c_uint64, C.c_uint32, C.c_uint64, vp, vp,
                  C.POINTER(C.c_float)]
    dev = f"cuda:{device}"
    lines = torch.zeros(line_bytes // 4, dtype=torch.int32, device=dev)
    a = torch.zeros(small_words, dtype=torch.int32, device=dev)
    b = torch.zeros(small_words, dtype=torch.int32, device=dev)
    sink = torch.zeros(1, dtype=torch.int64, device=dev)
    torch.cuda.synchronize(dev)
    out = {}
    for mode in (0, 1, 2, 3, 4):
        best = None
        for r in range(repeats):
            ms = C.c_float(0.0)
            rc = f(lines.data_ptr(), line_bytes // 128, a.data_ptr(), b.data_ptr(), small_words,
                   num_ops, mode, 1000 + r, sink.data_ptr(), None, C.byref(ms))
            if rc != 0:
                raise RuntimeError(f"mkb_probe_random_rmw failed ({rc})")
            best = ms.value if best is None else min(best, ms.value)
        out[mode] = num_ops / (best / 1000.0)
    del lines, a, b, sink
    torch.cuda.empty_cache()
    return {"read_lines_per_s": out[0], "read_cas_per_s": out[1], "update_pattern_per_s": out[2],
            "read_32B_sectors_per_s": out[3], "read_64B_halves_per_s": out[4]}


def make_workload(n_batches: int, source: str = "product"):
    """The R-MAT graph and `n_batches` mixed batches (delete sub-batch of
    present edges, insert sub-batch of absent edges with weights).
    source="oracle" draws the same edges and batches with the oracle's host
    generators, so the reference arm loads no product code."""
    if source == "oracle":
        from oracle import OracleEdgeSet as EdgeSet
        from oracle import gen_rmat
    else:
        from meerkat_b200 import EdgeSet, gen_rmat
    t0 = time.time()
    s, d, w = gen_rmat(SCALE, EDGES, seed=SEED, w_lo=W_LO, w_hi=W_HI)
    log(f"[bench] R-MAT s{SCALE}: {len(s)} edges in {time.time() - t0:.1f}s ({source} generator)")
    t0 = time.time()
    es = EdgeSet(1 << SCALE, s, d)
    batches = []
    rng = np.random.default_rng(SEED)
    for b in range(n_batches):
        ds, dd = es.sample_present(HALF, seed=SEED * 1000 + 2 * b)
        is_, id_ = es.sample_absent(HALF, seed=SEED * 1000 + 2 * b + 1)
        iw = rng.integers(W_LO, W_HI + 1, HALF).astype(np.uint32)
        batches.append((ds, dd, is_, id_, iw))
    log(f"[bench] {n_batches} mixed batches in {time.time() - t0:.1f}s")
    return (s, d, w), batches


def cpu_baseline(graph, batches, max_batches=3, warmup=0):
    """The oracle (C, OpenMP, one thread per host core) applying mixed batches:
    `warmup` untimed batches, then up to `max_batches` timed ones."""
    from oracle import OracleGraph
    s, d, w = graph
    T = os.cpu_count() or 1
    O = OracleGraph(1 << SCALE, threads=T)
    t0 = time.time()
    O.insert(s, d, w)
    log(f"[bench] oracle load {time.time() - t0:.1f}s on {T} threads")
    for (ds, dd, is_, id_, iw) in batches[:warmup]:
        O.delete(ds, dd)
        O.insert(is_, id_, iw)
    times = []
    applied = 0
    for (ds, dd, is_, id_, iw) in batches[warmup:warmup + max_batches]:
        t0 = time.perf_counter()
        n1, _ = O.delete(ds, dd)
        n2, _ = O.insert(is_, id_, iw)
        times.append(time.perf_counter() - t0)
        applied += n1 + n2
    total = sum(times)
    return {"value": applied / total, "unit": METRIC, "cores": T, "kind": "port",
            "sample": f"{len(times)} mixed batches of {2 * HALF} edges on the full R-MAT "
                      f"s{SCALE} graph (hash-set adjacency, one shard per thread)",
            "seconds": total}


def head_slab_share(G, timed_batches):
    """Share of batch edges whose head slab (the bucket slab their probe
    reads first) is also the head slab of another edge of the same
    sub-batch, and distinct head slabs per edge: what sorting a sub-batch by
    slab could save at most (one line read per distinct slab instead of one
    per edge).  Computed on the host from the graph's bucket layout with the
    kernels' bucket hash (mix32, multiply-shift)."""
    boff = G.GetVertexBucketsOffsets().astype(np.uint64)
    nb = G.GetBucketsPerVertex().astype(np.uint64)

    def mix32(x):
        x = x.astype(np.uint64)
        x ^= x >> np.uint64(16)
        x = (x * np.uint64(0x7FEB352D)) & np.uint64(0xFFFFFFFF)
        x ^= x >> np.uint64(15)
        x = (x * np.uint64(0x846CA68B)) & np.uint64(0xFFFFFFFF)
        x ^= x >> np.uint64(16)
        return x

    out = {}
    for name, cols in (("delete", (0, 1)), ("insert", (2, 3))):
        shared = distinct = total = 0
        for b in timed_batches:
            u, v = b[cols[0]].astype(np.int64), b[cols[1]]
            head = boff[u] + ((mix32(v) * nb[u]) >> np.uint64(32))
            _, cnt = np.unique(head, return_counts=True)
            shared += int(cnt[cnt > 1].sum())
            distinct += len(cnt)
            total += len(head)
        out[name + "_edges_sharing_a_head_slab"] = shared / total
        out[name + "_distinct_head_slabs_per_edge"] = distinct / total
    return out


def oracle_large(graph, hist, timed_at, A, gpu, algo):
    """Rank 0, after the GPU work of the updates workload.  The oracle (C,
    OpenMP, every host core) replays every batch the GPU graph received, in
    order, and

    * times three mixed batches (the first three of the K timed ones): the
      CPU baseline of the update half;
    * times the multithreaded CPU implementation of the query half on the
      same graph: static BFS / SSSP from the GPU's source before the A query
      batches, then per batch decremental BFS / SSSP after its deletes and
      incremental after its inserts; static WCC, PageRank (stopped by the
      GPU's rule) and triangle counting on the final graph;
    * checks the GPU's answers at full size: the maintained BFS levels and
      SSSP distances after the A batches bit-exact against the oracle's BFS
      and Dijkstra, with valid parents; after the last batch the degrees,
      the WCC labels and the triangle count exact, and PageRank within L1
      1e-6 of an FP64 solve run to an L1 change of 1e-11 (the pull solver
      the CPU tests pin against the oracle's own iteration).

    Returns (cpu_baseline, cpu_queries, parity)."""
    from oracle import CpuTraversal, OracleGraph, cpu_pagerank, cpu_triangles, cpu_wcc
    s, d, w = graph
    T = os.cpu_count() or 1
    V = 1 << SCALE
    O = OracleGraph(V, threads=T)
    t0 = time.time()
    O.insert(s, d, w)
    log(f"[oracle] s{SCALE} loaded in {time.time() - t0:.1f}s on {T} threads")
    nq = len(hist) - A
    up_times, applied = [], 0
    t0 = time.time()
    for i, (ds, dd, is_, id_, iw) in enumerate(hist[:nq]):
        t1 = time.perf_counter()
        n1, _ = O.delete(ds, dd)
        n2, _ = O.insert(is_, id_, iw)
        if timed_at[0] <= i < timed_at[1]:
            up_times.append(time.perf_counter() - t1)
            applied += n1 + n2
    log(f"[oracle] replayed {nq} mixed batches in {time.time() - t0:.1f}s")
    cb = {"value": applied / sum(up_times), "unit": METRIC, "cores": T, "kind": "port",
          "sample": f"{len(up_times)} mixed batches of {2 * HALF} edges on the full R-MAT "
                    f"s{SCALE} graph (hash-set adjacency, one shard per thread)",
          "seconds": sum(up_times)}

    def ms(fn):
        t1 = time.perf_counter()
        r = fn()
        return 1000.0 * (time.perf_counter() - t1), r

    src = gpu["source"]
    cq = {"cores": T, "kind": "port", "source": src}
    bfs, sssp = CpuTraversal(O, src, False), CpuTraversal(O, src, True)
    cq["bfs_static_ms"], _ = ms(bfs.static)
    cq["sssp_static_ms"], _ = ms(sssp.static)
    rec = {k: [] for k in ("bfs_dec_ms", "sssp_dec_ms", "bfs_inc_ms", "sssp_inc_ms")}
    inv = {"bfs": [], "sssp": []}
    for (ds, dd, is_, id_, iw) in hist[nq:]:
        O.delete(ds, dd)
        rec["bfs_dec_ms"].append(ms(lambda: bfs.decremental(ds, dd))[0])
        rec["sssp_dec_ms"].append(ms(lambda: sssp.decremental(ds, dd))[0])
        inv["bfs"].append(bfs.stats()["invalidated"])
        inv["sssp"].append(sssp.stats()["invalidated"])
        O.insert(is_, id_, iw)
        rec["bfs_inc_ms"].append(ms(lambda: bfs.incremental(is_, id_))[0])
        rec["sssp_inc_ms"].append(ms(lambda: sssp.incremental(is_, id_))[0])
    for k, v in rec.items():
        cq[k + "_p50"] = statistics.median(v)
    cq["invalidated"] = inv
    par = {}
    t0 = time.time()
    want_b, want_s = O.bfs(src), O.sssp(src)
    par["bfs"] = bool(np.array_equal(gpu["bfs"], want_b))
    par["sssp"] = bool(np.array_equal(gpu["sssp"], want_s))
    par["bfs_bad_parents"] = O.check_parents(src, gpu["bfs_packed"], False)
    par["sssp_bad_parents"] = O.check_parents(src, gpu["sssp_packed"], True)
    par["cpu_port_bfs"] = bool(np.array_equal(bfs.distances(), want_b))
    par["cpu_port_sssp"] = bool(np.array_equal(sssp.distances(), want_s))
    del bfs, sssp
    # the 100,000-edge batch of the WCC / PageRank / TC queries: deleted, then
    # inserted again with weight 0
    bs, bd = gpu["batch"]
    O.delete(bs, bd)
    O.insert(bs, bd, np.zeros(len(bs), dtype=np.uint32))
    par["degrees"] = bool(np.array_equal(gpu["degrees"], O.degrees()))
    want_w = O.wcc()
    par["wcc"] = bool(np.array_equal(gpu["wcc"], want_w))
    cq["wcc_static_ms"], lab = ms(lambda: cpu_wcc(O))
    par["cpu_port_wcc"] = bool(np.array_equal(lab, want_w))
    want_t = O.triangles()
    par["triangles"] = int(want_t)
    par["tc"] = int(gpu["triangles"]) == int(want_t)
    cq["tc_static_ms"], n_t = ms(lambda: cpu_triangles(O))
    par["cpu_port_tc"] = int(n_t) == int(want_t)
    # the GPU stops when its L1 change x d / (1 - d) <= tol / 2
    tol = algo.get("pagerank", {}).get("tol", 1e-6)
    cq["pagerank_static_ms"], (_, it) = ms(lambda: cpu_pagerank(O, 0.85, tol * 0.5 * 0.15 / 0.85, 1000))
    cq["pagerank_iterations"] = it
    ref, _ = cpu_pagerank(O, 0.85, 1e-11, 10000)
    par["pagerank_l1"] = float(np.abs(gpu["pagerank"].astype(np.float64) - ref).sum())
    par["pagerank"] = par["pagerank_l1"] <= 1e-6
    par["ok"] = bool(par["bfs"] and par["sssp"] and par["bfs_bad_parents"] == 0 and
                     par["sssp_bad_parents"] == 0 and par["degrees"] and par["wcc"] and
                     par["tc"] and par["pagerank"])
    log(f"[oracle] parity checks in {time.time() - t0:.1f}s: {par}")
    del O
    return cb, cq, par


def verify_replay(G, timed_batches, todev, dev):
    """Checks the graph state after the K captured steps against the batches."""
    import torch
    final = {}
    for ds, dd, is_, id_, _ in timed_batches:
        for a, b in zip(ds.tolist(), dd.tolist()):
            final[(a, b)] = False
        for a, b in zip(is_.tolist(), id_.tolist()):
            final[(a, b)] = True
    keys = np.array(list(final.keys()), dtype=np.uint32).reshape(-1, 2)
    want = np.array(list(final.values()), dtype=np.uint8)
    found = torch.zeros(len(keys), dtype=torch.uint8, device=dev)
    G.SearchEdges(todev(keys[:, 0]), todev(keys[:, 1]), found)
    torch.cuda.synchronize(dev)
    got = found.cpu().numpy()
    bad = int((got != want).sum())
    edges = G.info()["num_edges"]
    return {"ok": bad == 0 and edges == EDGES, "checked": int(len(keys)), "mismatches": bad,
            "num_edges": int(edges)}


def more_queries(mk, G, V, dev, seed):
    """WCC, PageRank and triangle counting on the benchmark graph (static,
    then one decremental and one incremental batch), with the algorithmic
    bytes of each static run: WCC 8 E + 8 V; PageRank 8 E + 16 V per
    iteration; TC 4 x sum over oriented edges of (d+(u) + d+(v)), edges
    oriented from lower to higher (degree, id) on the symmetric graph.

    Returns (timings, finals): finals holds the last answers (WCC labels,
    PageRank values, triangle count) and the host copy of the 100,000-edge
    batch this function deletes from G and inserts again with weight 0, so
    the oracle can replay it and check the answers."""
    import torch
    out = {}
    finals = {}
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    rp, col, _ = G.export_csr_range_device(0, V)
    E = int(col.numel())
    rows = torch.repeat_interleave(torch.arange(V, device=dev, dtype=torch.int32), rp[1:] - rp[:-1])
    pick = torch.randint(0, E, (100_000,), generator=g, device=dev)
    bs, bd = rows[pick].contiguous(), col[pick].contiguous()
    # a reverse copy of the same edges (in-edges): decremental WCC rescans
    # split-off pieces through it; PageRank and pull BFS read it below
    indeg = torch.bincount(col.long(), minlength=V).to(torch.int32).cpu().numpy().view(np.uint32)
    Gr = mk.DynamicGraph(V, degree_hints=indeg, reverse=True, device=dev.index or 0)
    Gr.InsertEdges(rows, col)
    # WCC on the graph itself; the decremental call repairs along the
    # spanning forest with the reverse copy attached (both graphs get the
    # batch first, as a caller keeping them in step would)
    wcc = mk.WCC(G)
    wcc.set_reverse(Gr)
    t = min(wcc.Static() for _ in range(2))
    out["wcc"] = {"static_ms": t, "static_gbs": (8 * E + 8 * V) / (t / 1e3) / 1e9,
                  "static_gbs_note": "8 E + 8 V (one full edge pass) per call; the passes skip "
                                     "the edges inside the largest sampled set, so this is an "
                                     "equivalent rate, not bytes moved"}
    G.DeleteEdges(bs, bd)
    Gr.DeleteEdges(bs, bd)
    out["wcc"]["dec_ms"] = wcc.Decremental(bs, bd)
    dead, rescanned, path = wcc.decremental_stats()
    out["wcc"]["dec_repair"] = {"forest_edges_lost": dead, "vertices_rescanned": rescanned,
                                "path": ["unchanged", "piece rescan", "component rebuild",
                                         "static"][path]}
    G.InsertEdges(bs, bd)  # weight 0 on the re-inserted copies
    Gr.InsertEdges(bs, bd)
    out["wcc"]["inc_ms"] = wcc.Incremental(bs, bd)
    finals["wcc"] = wcc.Labels()
    finals["batch"] = (bs.cpu().numpy().view(np.uint32).copy(), bd.cpu().numpy().view(np.uint32).copy())
    wcc.close()
    # direction-optimizing static BFS: the reverse copy lets large levels pull
    from meerkat_b200.autotune import tune_bfs_pull
    src_bfs = int(torch.argmax(rp[1:] - rp[:-1]))
    bfs_push = mk.BFS(G, src_bfs, V)
    t_push = min(bfs_push.Static() for _ in range(2))
    bfs_pull = mk.BFS(G, src_bfs, V)
    bfs_pull.set_reverse(Gr)
    pull = tune_bfs_pull(G, bfs_pull)
    same = bool(np.array_equal(bfs_push.Distances(), bfs_pull.Distances()))
    out["bfs_pull"] = {"push_only_ms": t_push, "best_ms": min(x["static_ms"] for x in pull["trials"]),
                       "pull_permille": pull["best"], "trials": pull["trials"], "same_levels": same}
    bfs_push.close()
    bfs_pull.close()
    G.set_tuning(pull_permille=0)
    pr = mk.PageRank(Gr, 0.85, 1e-6, V, max_iter=200)
    t_first = pr.Static()  # grows the per-solve CSR and work-item scratch
    t = pr.Static()
    it, _ = pr.stats()
    out["pagerank"] = {"static_ms": t, "first_static_ms": t_first, "iterations": it,
                       "static_gbs": it * (8 * E + 16 * V) / (t / 1e3) / 1e9}
    Gr.DeleteEdges(bs, bd)
    out["pagerank"]["dec_ms"] = pr.Decremental(bs, bd)
    Gr.InsertEdges(bs, bd)
    out["pagerank"]["inc_ms"] = pr.Incremental(bs, bd)
    finals["pagerank"] = pr.Values()
    out["pagerank"]["tol"] = 1e-6
    pr.close()
    Gr.close()
    # triangles on the symmetric graph
    su = torch.cat([rows, col])
    sv = torch.cat([col, rows])
    key = torch.unique(su.long() * V + sv.long())
    su, sv = (key // V).int(), (key % V).int()
    sdeg = torch.bincount(su.long(), minlength=V)
    Gs = mk.DynamicGraph(V, degree_hints=sdeg.to(torch.int32).cpu().numpy().view(np.uint32),
                         device=dev.index or 0)
    Gs.InsertEdges(su, sv)
    fwd = (sdeg[su.long()] < sdeg[sv.long()]) | ((sdeg[su.long()] == sdeg[sv.long()]) & (su < sv))
    ou, ov = su[fwd].long(), sv[fwd].long()
    dplus = torch.bincount(ou, minlength=V)
    tc_bytes = 4 * int((dplus[ou] + dplus[ov]).sum())
    tc = mk.TC(Gs, V)
    t_first = tc.Static()  # sizes the orientation scratch (allocations, first kernel loads)
    t = tc.Static()
    out["tc"] = {"static_ms": t, "first_static_ms": t_first, "triangles": tc.GetCount(),
                 "static_gbs": tc_bytes / (t / 1e3) / 1e9, "sym_edges": int(su.numel())}
    upick = torch.randint(0, int(ou.numel()), (50_000,), generator=g, device=dev)
    uu, uv = ou[upick].int(), ov[upick].int()
    uu, uv = torch.cat([uu, uv]), torch.cat([uv, uu])
    Gs.DeleteEdges(uu, uv)
    out["tc"]["dec_ms"] = tc.Decremental(uu, uv)
    Gs.InsertEdges(uu, uv)
    out["tc"]["inc_ms"] = tc.Incremental(uu, uv)
    finals["triangles"] = tc.GetCount()
    tc.close()
    Gs.close()
    del rp, col, rows, su, sv, key, sdeg, fwd, ou, ov, dplus
    torch.cuda.synchronize(dev)
    torch.cuda.empty_cache()
    peak = measured_peak()[0]
    for k in out:
        if "static_gbs" in out[k]:
            out[k]["static_frac"] = out[k]["static_gbs"] / peak
    return out, finals


def line_summary(line):
    """The headline figures of the updates workload in a few hundred bytes:
    the update rates, the roofline fraction, the query half of the metric
    (GPU and CPU ms per call, p50) and the parity verdict per config."""
    q, cq = line.get("queries", {}), line.get("cpu_queries") or {}
    r3 = lambda x: None if x is None else float(f"{x:.4g}")
    keys = [("bfs_static", "bfs_static_ms", "bfs_static_ms"),
            ("sssp_static", "sssp_static_ms", "sssp_static_ms"),
            ("bfs_inc", "bfs_inc_ms_p50", "bfs_inc_ms_p50"),
            ("bfs_dec", "bfs_dec_ms_p50", "bfs_dec_ms_p50"),
            ("sssp_inc", "sssp_inc_ms_p50", "sssp_inc_ms_p50"),
            ("sssp_dec", "sssp_dec_ms_p50", "sssp_dec_ms_p50")]
    gpu_ms = {k: r3(q.get(a)) for k, a, _ in keys}
    cpu_ms = {k: r3(cq.get(b)) for k, _, b in keys}
    # decremental calls with the reverse graph attached (BFS: level-ordered
    # repair; SSSP: re-seed from in-edges)
    gpu_ms["bfs_dec_rev"] = r3(q.get("bfs_dec_rev_ms_p50"))
    gpu_ms["sssp_dec_rev"] = r3(q.get("sssp_dec_rev_ms_p50"))
    for k in ("wcc", "pagerank", "tc"):
        gpu_ms[k + "_static"] = r3(q.get(k, {}).get("static_ms"))
        cpu_ms[k + "_static"] = r3(cq.get(k + "_static_ms"))
    out = {"updates_per_s": r3(line["value"]), "e2e_updates_per_s": r3(line["e2e"]["value"]),
           "roofline_frac": r3(line["roofline"]["frac"]),
           "cpu_updates_per_s": r3((line.get("cpu_baseline") or {}).get("value")),
           "cpu_cores": cq.get("cores"), "gpu_ms": gpu_ms, "cpu_ms": cpu_ms,
           "parity": line.get("parity")}
    if "batched" in line:
        out["batched_speedup"] = r3(line["batched"]["speedup_vs_plain"])
    if "grid" in line:
        g = line["grid"]
        out["grid_ms_p50"] = {"bfs_dec": r3(g["decremental_p50_ms"]["bfs_ms"]),
                              "sssp_dec": r3(g["decremental_p50_ms"]["sssp_ms"]),
                              "bfs_static": r3(g["static"]["bfs_ms"]),
                              "sssp_static": r3(g["static"]["sssp_ms"])}
    if "serving" in line:
        sv = line["serving"]
        out["serving"] = {"saturation_rps": {m: r3(sv["saturation"][m]["throughput_rps"])
                                             for m in ("coalesced", "alone")},
                          "saturation_ratio": r3(sv["saturation"]["ratio"]),
                          "rates": [{"rps": row["offered_rps"],
                                     **{m: [r3(row[m]["p50_ms"]), r3(row[m]["p99_ms"]),
                                            r3(row[m]["throughput_rps"])]
                                        for m in ("coalesced", "alone")}}
                                    for row in sv["rates"]]}
    return out


def dist_setup(n_gpus):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch.distributed as dist
        import datetime
        backend = "nccl" if os.environ.get("MK_BENCH_BACKEND", "nccl") == "nccl" else "gloo"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return rank, world, local


def max_over_ranks(x: float, world: int, device):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def run_reference(args, rank, world):
    """--impl reference: the reference's CPU path does not exist (the reference is
    GPU-only and does not build here), so the oracle port stands in, timed on
    the host cores on the same config and metric.  Its inputs come from the
    oracle's host generators (the same edges and batches as the GPU arm's), so
    this arm loads only the oracle library."""
    if rank != 0:
        return 0
    K = max(args.steps, 1)
    graph, batches = make_workload(K + args.warmup, source="oracle")
    cb = cpu_baseline(graph, batches, max_batches=K, warmup=args.warmup)
    v = cb["value"]
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": METRIC,
            "n_gpus": args.gpus, "steps": K, "warmup": args.warmup,
            "ms_per_step": 1000.0 * cb["seconds"] / K,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic", "config": config_block(args.gpus),
            "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": v, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def config_block(n):
    name = "rmat22_mixed_1M" if (SCALE, HALF) == (22, 500_000) else f"rmat{SCALE}_mixed_{2 * HALF}"
    return {"workload": name, "graph": f"R-MAT scale {SCALE}, {EDGES} directed edges, "
            "a/b/c/d .57/.19/.19/.05, weights U[1,1000]", "batch": f"{HALF} deletes of present "
            f"edges then {HALF} inserts of absent edges", "load_factor": 0.7,
            "degree_hints": "exact", "l2": "inputs larger than L2 (slab pool ~2.5 GB, random "
            "bucket probes)", "parallelism": f"replicas x{n}" if n > 1 else "single GPU"}


def batched_compare(num_graphs, K, W, rank, world, local):
    """Many small graphs: the batched runner (one GraphSet, one coalesced launch
    sequence per step, CUDA-graph replay) against the plain per-graph launch
    sequence (one DynamicGraph and one BFS/WCC object per member) on the same
    seeded members and batches.  A step = one mixed update batch per member
    (U[1%,10%] of its edges, half deletes of live edges, half inserts of
    random pairs; steps alternate a batch and its inverse, so from the second
    step on the graphs cycle through two states) plus one query per member
    (BFS from a seeded source or the member's components).  The plain arm is
    timed twice: issued from the host, and captured into a CUDA graph.  Every
    member's final BFS levels / component labels must be equal in both arms.
    Returns the summary dict (rank 0 reports it)."""
    import torch

    import meerkat_b200 as mk
    from meerkat_b200 import batched as B
    from meerkat_b200.autotune import VARIANTS, tune_frontier_chunk, tune_updates
    dev = torch.device(f"cuda:{local}")
    stream = torch.cuda.current_stream(dev)
    K = max(2, K + (K % 2))  # even: both arms end in the same state of the cycle
    spec = B.make_spec(num_graphs, seed=B.DEFAULT_SEED + rank)
    Gn = spec.num_graphs
    voff = B._offsets(spec.num_vertices)
    eoff = B._offsets(spec.num_edges)
    V, E = int(voff[-1]), int(eoff[-1])
    t0 = time.time()
    src, dst, w = mk.gen_rmat_members(voff, spec.num_edges, seed=spec.seed, w_lo=1, w_hi=64,
                                      device=local)
    hints_all = torch.bincount(src.long(), minlength=V).to(torch.int32).cpu().numpy().view(np.uint32)
    hints = [hints_all[voff[m]:voff[m + 1]] for m in range(Gn)]
    log(f"[batched] {Gn} graphs, {V} vertices, {E} R-MAT edges in {time.time() - t0:.1f}s")
    t0 = time.time()
    gs = mk.GraphSet(spec.num_vertices, degree_hints=hints, weighted=True, device=local,
                     pool_slabs=B.pool_slabs_for(V, E))
    gs.graph.InsertEdges(src, dst, vals=w)
    assert gs.graph.sync() == 0
    plain = []
    for m in range(Gn):
        lo, hi, base = int(eoff[m]), int(eoff[m + 1]), int(voff[m])
        g = mk.DynamicGraph(int(spec.num_vertices[m]), degree_hints=hints[m], weighted=True,
                            device=local, pool_slabs=B.pool_slabs_for(int(spec.num_vertices[m]),
                                                                      int(spec.num_edges[m])))
        g.InsertEdges(src[lo:hi] - base, dst[lo:hi] - base, vals=w[lo:hi])
        plain.append(g)
    torch.cuda.synchronize(dev)
    assert all(g.sync() == 0 for g in plain)
    # members the oracle checks at the end: the 8 with the most edges and 56
    # more drawn with a seed; their generated edges, in local ids
    sample = np.unique(np.concatenate([
        np.argsort(spec.num_edges)[-8:],
        np.random.default_rng(spec.seed + 9).choice(Gn, size=min(56, Gn), replace=False)]))
    base_edges = {}
    for m in sample.tolist():
        lo, hi, b0 = int(eoff[m]), int(eoff[m + 1]), int(voff[m])
        base_edges[m] = tuple(x[lo:hi].cpu().numpy().view(np.uint32) - (b0 if i < 2 else 0)
                              for i, x in enumerate((src, dst, w)))
    del src, dst, w
    info = gs.graph.info()
    log(f"[batched] union and {Gn} per-graph copies built in {time.time() - t0:.1f}s: {info}")

    deg = gs.graph.degrees()
    bfs_members = np.flatnonzero(spec.query == B.QUERY_BFS)
    srcs = B.pick_sources(deg, voff, bfs_members, seed=spec.seed + 1)
    br = B.BatchedRunner(gs, spec.query, srcs)
    pr = B.PlainRunner(plain, spec.query, srcs)

    # one batch and its inverse, global ids for the set, local ids per member
    fwd = gs.gen_batches(spec.deletes, spec.inserts, seed=spec.seed + 2, w_lo=1, w_hi=64)
    ds, dd, is_, id_, iw = fwd
    gen = torch.Generator(device=dev)
    gen.manual_seed(spec.seed + 3)
    rw = torch.randint(1, 65, (ds.numel(),), generator=gen, device=dev, dtype=torch.int32)
    rev = (is_, id_, ds, dd, rw)
    voff_t = torch.from_numpy(voff).to(dev)

    def local_slices(batch, n_del, n_ins):
        do, io = B._offsets(n_del), B._offsets(n_ins)
        ar = torch.arange(Gn, device=dev)
        od = voff_t[torch.repeat_interleave(ar, torch.from_numpy(n_del).to(dev))]
        oi = voff_t[torch.repeat_interleave(ar, torch.from_numpy(n_ins).to(dev))]
        a, b_, c, d_, e = batch
        a, b_ = (a.long() - od).int(), (b_.long() - od).int()
        c, d_ = (c.long() - oi).int(), (d_.long() - oi).int()
        return [(a[do[m]:do[m + 1]], b_[do[m]:do[m + 1]], c[io[m]:io[m + 1]], d_[io[m]:io[m + 1]],
                 e[io[m]:io[m + 1]]) for m in range(Gn)]

    fwd_local = local_slices(fwd, spec.deletes, spec.inserts)
    rev_local = local_slices(rev, spec.inserts, spec.deletes)
    upd = int(spec.deletes.sum() + spec.inserts.sum())
    both = [fwd, rev]
    both_local = [fwd_local, rev_local]

    # warm-up: one cold step, then 2 rounds of the update tuner (real steps),
    # then the frontier-chunk tuner (static BFS is idempotent)
    nt = 2 * len(VARIANTS)
    Wb = max(W, 1 + nt)
    br.step(both[0])
    tuning = tune_updates(gs.graph, [both[i % 2] for i in range(1, 1 + nt)], stream=stream,
                          rounds=2)
    for i in range(1 + nt, Wb):
        br.step(both[i % 2])
    br.query()
    chunk = tune_frontier_chunk(gs.graph, br.bfs) if br.bfs is not None else None
    for i in range(Wb):
        pr.step(both_local[i % 2])
    torch.cuda.synchronize(dev)
    assert gs.graph.sync() == 0 and all(g.sync() == 0 for g in plain)

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s_ = torch.cuda.current_stream(dev)
        e0.record(s_)
        fn()
        e1.record(s_)
        e1.synchronize()
        return max_over_ranks(e0.elapsed_time(e1), world, dev)

    def capture(fn):
        cs = torch.cuda.Stream(dev)
        cs.wait_stream(stream)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=cs):
            fn(cs)
        torch.cuda.synchronize(dev)
        return g, cs

    clocks = Clocks(local)
    # batched arm: K steps captured into one CUDA graph, replayed once; the
    # four-launch step, then (every member fitting one CTA) the one-launch
    # step over the next K steps (K is even: both end on the same state of
    # the cycle and must give the same answers)
    forms = ["sequence"] + (["single"] if br.single_ok else [])
    form_ms, form_launches, answers = {}, {}, {}
    i0 = Wb
    for form in forms:
        br.set_single(form == "single")
        bg, bs = capture(lambda cs, a0=i0: [br.step(both[i % 2], stream=cs) for i in range(a0, a0 + K)])
        barrier(world)
        with torch.cuda.stream(bs):
            form_ms[form] = timed(bg.replay) / K
        assert gs.graph.sync() == 0
        del bg
        form_launches[form] = br.launches_per_step()
        answers[form] = (br.bfs.Distances() if br.bfs is not None else None,
                         br.wcc.Labels().astype(np.int64) if br.wcc is not None else None)
        i0 += K
    br.set_single(False)
    best = min(forms, key=lambda f: form_ms[f])
    batched_ms = form_ms[best]
    forms_equal = all(all(x is None or np.array_equal(x, y) for x, y in zip(answers[f], answers["sequence"]))
                      for f in forms)
    assert forms_equal, "the one-launch and four-launch steps disagree"
    d_union, l_union = answers["sequence"]
    # plain arm, issued from the host: K steps
    barrier(world)
    plain_ms = timed(lambda: [pr.step(both_local[i % 2]) for i in range(Wb, Wb + K)]) / K
    assert all(g.sync() == 0 for g in plain)
    # plain arm captured: the next two steps of the alternation per graph,
    # replayed K / 2 times, so the plain graphs end on the same state of the
    # two-state cycle as the batched set
    t0 = time.time()
    pg, ps = capture(lambda cs: [pr.step(both_local[(Wb + K + i) % 2], stream=cs)
                                 for i in range(2)])
    cap_s = time.time() - t0
    barrier(world)

    def replays():
        for _ in range(K // 2):
            pg.replay()
    with torch.cuda.stream(ps):
        plain_graph_ms = timed(replays) / K
    clk = clocks.stop()
    assert all(g.sync() == 0 for g in plain)
    del pg

    # every member's answer is the same in both arms
    mism = {"bfs": 0, "wcc": 0}
    for m in range(Gn):
        lo, hi = int(voff[m]), int(voff[m + 1])
        a = pr.algos[m]
        if spec.query[m] == B.QUERY_BFS:
            mism["bfs"] += int(not np.array_equal(a.Distances(), d_union[lo:hi]))
        else:
            mism["wcc"] += int(not np.array_equal(a.Labels().astype(np.int64), l_union[lo:hi] - lo))
    assert mism == {"bfs": 0, "wcc": 0}, mism
    # the oracle replays the sampled members' batches (a batch and its inverse
    # alternate, starting with the batch; every update the set received)
    n_updates = i0 + 2  # warm-up and tuner steps, K timed steps, 2 phase-split steps
    host_local = {m: [tuple(x.cpu().numpy().view(np.uint32) for x in both_local[k][m])
                      for k in (0, 1)] for m in sample.tolist()}
    par = batched_oracle_check(sample, base_edges, host_local, n_updates, spec, srcs, voff,
                               d_union, l_union, gs) if rank == 0 else None
    # phase split of the batched step: two more steps (a batch and its
    # inverse, so the set stays on the same state) with events between phases
    phases = {"update": 0.0, "bfs": 0.0, "wcc": 0.0}
    for i in range(2):
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        ev[0].record(stream)
        br.update(*both[(i0 + i) % 2])
        ev[1].record(stream)
        if br.bfs is not None:
            br.bfs.StaticMembers(timed=False)
        ev[2].record(stream)
        if br.wcc is not None:
            br.wcc.StaticPrepared(timed=False)
        ev[3].record(stream)
        ev[3].synchronize()
        for k, (x, y) in zip(phases, [(0, 1), (1, 2), (2, 3)]):
            phases[k] += ev[x].elapsed_time(ev[y]) / 2
    out = {
        "speedup_vs_plain": plain_ms / batched_ms,
        "speedup_vs_plain_cuda_graph": plain_graph_ms / batched_ms,
        "batched_ms_per_step": batched_ms, "plain_ms_per_step": plain_ms,
        "batched_form": best, "forms_ms_per_step": form_ms,
        "forms_launches_per_step": form_launches, "forms_equal": forms_equal,

        "batched_phases_ms": phases,
        "plain_cuda_graph_ms_per_step": plain_graph_ms, "plain_capture_s": cap_s,
        "steps": K, "warmup": Wb,
        "workload": f"batched_{Gn}_graphs",
        "graphs": f"{Gn} R-MAT members, V log-uniform [1024, 65536], average degree power law "
                  "(exponent 2) on [4, 32], weights U[1,64]",
        "step": "per member: mixed batch of U[1%,10%] of its edges (half deletes of live edges, "
                "half inserts), then one BFS or WCC query (coin flip); a batch and its inverse "
                "alternate",
        "vertices": V, "edges": E, "updates_per_step": upd,
        "batched_updates_per_s": upd / (batched_ms / 1000.0),
        "gpu_launches_per_step": form_launches[best],
        "plain_launches_per_step": pr.launches_per_step(),
        "queries": {"bfs_members": int(len(br.bfs_members)), "wcc_members": int(len(br.wcc_members))},
        "tuning": {"updates": tuning["best"], "frontier_chunk": chunk["best"] if chunk else None},
        "tuning_trials": {"updates": tuning["trials"], "frontier_chunk": chunk["trials"] if chunk else None},
        "equality": {"members_checked": Gn, "bfs_mismatches": mism["bfs"],
                     "wcc_mismatches": mism["wcc"]},
        **({"parity": par} if par is not None else {}),
        "clocks": clk,
        "graph": {"buckets": info["num_buckets"], "slabs_used": info["slabs_used"],
                  "device_bytes": info["device_bytes"]},
    }
    # release the per-graph objects and the runner before the set
    br.close()
    del pr, br
    for g in plain:
        g.close()
    gs.close()
    torch.cuda.synchronize(dev)
    return out


def batched_oracle_check(sample, base_edges, host_local, n_updates, spec, srcs, voff, d_union,
                         l_union, gs):
    """The oracle on a sample of the batched set's members: each member's
    generated edges and its n_updates alternating batches replayed on the CPU,
    then its degrees, BFS levels (BFS members, from the member's source) or
    WCC labels (WCC members) compared bit-exactly with the batched arm's."""
    from meerkat_b200 import batched as B
    from oracle import OracleGraph
    t0 = time.time()
    deg = gs.graph.degrees()
    bfs_index = {int(m): i for i, m in enumerate(np.flatnonzero(spec.query == B.QUERY_BFS))}
    bad = {"degrees": 0, "bfs": 0, "wcc": 0}
    edges_checked = 0
    for m in sample.tolist():
        lo, hi = int(voff[m]), int(voff[m + 1])
        O = OracleGraph(hi - lo)
        bs, bd, bw = base_edges[m]
        O.insert(bs, bd, bw)
        for i in range(n_updates):
            ds, dd, is_, id_, iw = host_local[m][i % 2]
            O.delete(ds, dd)
            O.insert(is_, id_, iw)
        edges_checked += O.num_edges()
        bad["degrees"] += int(not np.array_equal(deg[lo:hi], O.degrees()))
        if spec.query[m] == B.QUERY_BFS:
            bad["bfs"] += int(not np.array_equal(d_union[lo:hi], O.bfs(int(srcs[bfs_index[m]]))))
        else:
            bad["wcc"] += int(not np.array_equal(l_union[lo:hi] - lo, O.wcc().astype(np.int64)))
    out = {"members": int(len(sample)), "largest_included": 8, "edges": int(edges_checked),
           "mismatches": bad, "ok": not any(bad.values())}
    log(f"[batched] oracle check of {len(sample)} members in {time.time() - t0:.1f}s: {out}")
    return out


def serving_compare(num_graphs, scales, rates, N, budget_gb, rank, world, local,
                    rate_fractions=(0.25, 0.5, 0.75)):
    """Open-loop serving: G resident R-MAT graphs (scales uniform in the given
    range, edge factor 16, weights U[1,1000]) in one graph set under a device
    memory budget; mix 50% updates (log-uniform 1K-1M edges, half inserts,
    half deletes), 30% BFS/SSSP, 10% PageRank, 10% TC/WCC.  Two modes serve
    the same request logs: coalesced (continuous batching, heavy requests
    overlapped on a second stream) and alone (one request at a time: the
    plain per-request launch sequence).

    First each mode's saturation throughput: N requests that all arrive at
    once.  Then Poisson arrivals at offered rates below saturation: the given
    `rates`, or, when empty, `rate_fractions` of the alone mode's saturation
    throughput, so both modes run unsaturated.  Returns the summary (rank 0
    reports it)."""
    import torch

    from meerkat_b200 import serving as S
    seed = SEED + 7 + rank
    lo_s, hi_s = scales
    t0 = time.time()
    nv, ne = S.make_graph_sizes(num_graphs, lo_s, hi_s, 16, seed)
    gs, edges = S.build_set(nv, ne, seed, device=local)
    log(f"[serving] {len(nv)} graphs, {int(nv.sum())} vertices, {int(ne.sum())} edges loaded "
        f"in {time.time() - t0:.1f}s: {gs.graph.info()}")
    wl = S.Workload(nv, ne, seed)
    warm = S.make_requests(wl, edges, 64, rate=1e6, seed=seed + 1, device=local)
    sat_reqs = S.make_requests(wl, edges, N, rate=1e9, seed=seed + 2, device=local)
    t_srv = time.time()
    srv = S.GraphServer(gs, budget_bytes=int(budget_gb * 1e9), device=local)
    log(f"[serving] server ready in {time.time() - t_srv:.1f}s (resident {srv.resident / 1e9:.1f} GB)")
    srv.run(warm, wl, mode="coalesced")

    def copy(reqs):
        return [S.Request(r.rid, r.graph, r.kind, r.arrival, r.source, r.lo, r.hi) for r in reqs]

    def slim(out):
        keep = ("p50_ms", "p99_ms", "throughput_rps", "rounds", "rejected")
        return {k: out[k] for k in keep}

    clocks = Clocks(local)
    sat = {}
    for mode in ("coalesced", "alone"):
        t1 = time.time()
        out = srv.run(copy(sat_reqs), wl, mode=mode)
        if mode == "alone":
            sat_alone_kinds = out["by_kind"]
        sat[mode] = slim(out)
        sat[mode]["by_kind_service_p50_ms"] = {k: v["service_p50_ms"] for k, v in out["by_kind"].items()}
        log(f"[serving] saturation {mode}: {out['throughput_rps']:.1f} rps, p50 {out['p50_ms']:.1f} ms,"
            f" {out['rounds']} rounds, {time.time() - t1:.1f}s")
    # what bounds the coalesced mode: heavy requests (PageRank, TC) are not
    # coalesced, so their one-at-a-time GPU time per request (the alone
    # run's service times) caps any schedule's throughput
    heavy_ms = sum(v["service_total_ms"] for k, v in sat_alone_kinds.items()
                   if k in ("pagerank", "tc")) / N
    fast_ms = sum(v["service_total_ms"] for k, v in sat_alone_kinds.items()
                  if k not in ("pagerank", "tc")) / N
    sat["heavy_bound"] = {"heavy_ms_per_request": heavy_ms, "fast_ms_per_request": fast_ms,
                          "max_rps_if_fast_work_were_free": 1000.0 / heavy_ms if heavy_ms else None}
    if not rates:
        rates = [round(f * sat["alone"]["throughput_rps"], 1) for f in rate_fractions]
    table = []
    for j, rate in enumerate(rates):
        reqs = S.make_requests(wl, edges, N, rate=rate, seed=seed + 100 + j, device=local)
        row = {"offered_rps": rate}
        for mode in (("coalesced", "alone") if j % 2 == 0 else ("alone", "coalesced")):
            t1 = time.time()
            out = srv.run(copy(reqs), wl, mode=mode)
            log(f"[serving] {rate:.1f} rps {mode}: p50 {out['p50_ms']:.2f} ms p99 "
                f"{out['p99_ms']:.2f} ms, {out['throughput_rps']:.1f} rps, {out['rounds']} rounds, "
                f"{time.time() - t1:.1f}s")
            row[mode] = slim(out)
        table.append(row)
    clk = clocks.stop()
    del edges
    out = {
        "workload": f"serving_{len(nv)}_graphs",
        "graphs": f"{len(nv)} R-MAT graphs, scales U{{{lo_s}..{hi_s}}}, edge factor 16, "
                  "weights U[1,1000]",
        "vertices": int(nv.sum()), "edges": int(ne.sum()),
        "mix": "25% insert, 25% delete (1K-1M edges, log-uniform), 15% BFS, 15% SSSP, "
               "10% PageRank, 5% TC, 5% WCC; graph uniform",
        "arrivals": "open-loop Poisson", "requests_per_rate": N, "budget_gb": budget_gb,
        "saturation": {**sat, "ratio": sat["coalesced"]["throughput_rps"] /
                       max(sat["alone"]["throughput_rps"], 1e-9),
                       "what": f"{N} requests arriving at once"},
        "rates": table, "clocks": clk, "warmup_requests": len(warm),
        "resident_bytes": srv.resident, "tc_scratch_bytes": srv.tc_bytes,
    }
    srv.close()
    gs.close()
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    return out


def run_serving(args, rank, world, local):
    import torch

    from meerkat_b200.build import build
    if rank == 0:
        build()
    barrier(world)
    torch.cuda.set_device(local)
    scales = tuple(int(x) for x in args.serving_scales.split(","))
    rates = [float(x) for x in args.serving_rates.split(",") if x.strip() not in ("", "auto")]
    r = serving_compare(args.serving_graphs, scales, rates, args.serving_requests,
                        args.serving_budget_gb, rank, world, local)
    top = r["saturation"]["coalesced"]
    if rank == 0:
        line = {
            "metric": "serving saturation throughput (coalesced)",
            "value": top["throughput_rps"], "unit": "requests/s", "n_gpus": world,
            "steps": len(r["rates"]), "warmup": r["warmup_requests"],
            "ms_per_step": top["p50_ms"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic",
            "config": {k: r[k] for k in ("workload", "graphs", "vertices", "edges", "mix",
                                         "arrivals", "requests_per_rate", "budget_gb")},
            "p50_ms": top["p50_ms"], "p99_ms": top["p99_ms"],
            "rates": r["rates"], "saturation": r["saturation"], "clocks": r["clocks"],
            "resident_bytes": r["resident_bytes"], "tc_scratch_bytes": r["tc_scratch_bytes"],
        }
        print(json.dumps(line), flush=True)
    barrier(world)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def grid_stress(side, nbatch, batch, rank, world, local):
    """High-diameter decremental stress: side x side 4-neighbour grid, both
    directions, plus 1% random long-range shortcut edges, weights U[1,1000].
    nbatch delete-only batches of `batch` edges, 80% drawn from the current
    SSSP tree and 20% from the generated edges, then nbatch insert batches of
    `batch` random local edges (Chebyshev radius <= 2).  After each batch:
    decremental / incremental BFS, SSSP (from the centre) and WCC, ms each.
    At the end the maintained BFS levels, SSSP distances and WCC labels must
    equal a fresh static recompute on the final graph."""
    import torch

    import meerkat_b200 as mk
    dev = torch.device(f"cuda:{local}")
    V = side * side
    grid_edges = 4 * side * (side - 1)
    t0 = time.time()
    s, d, w = mk.gen_grid(side, grid_edges // 100, seed=SEED + 21 + rank, w_lo=1, w_hi=1000)
    E = len(s)

    def todev(a):
        return torch.from_numpy(np.ascontiguousarray(a, dtype=np.uint32).view(np.int32)).to(dev)

    G = mk.DynamicGraph(V, degree_hints=np.bincount(s, minlength=V).astype(np.uint32),
                        weighted=True, device=local)
    G.InsertEdges(todev(s), todev(d), vals=todev(w))
    assert G.sync() == 0
    log(f"[grid] {side}x{side}: {V} vertices, {E} edges in {time.time() - t0:.1f}s")
    src = (side // 2) * side + side // 2
    bfs, sssp, wcc = mk.BFS(G, src, V), mk.SSSP(G, src, V), mk.WCC(G)
    # a reverse copy (in-edges) kept in step outside the timed calls lets
    # decremental WCC rescan only the pieces a batch split off
    Gr = mk.DynamicGraph(V, degree_hints=np.bincount(d, minlength=V).astype(np.uint32),
                         reverse=True, device=local)
    Gr.InsertEdges(todev(s), todev(d))
    Gr.reserve_batch(batch)
    wcc.set_reverse(Gr)
    from meerkat_b200.autotune import tune_sssp_delta
    nf = tune_sssp_delta(G, sssp, deltas=(0, 4096, 16384, 65536))
    # deletes aimed at the SSSP tree cut off large subtrees: recompute from the
    # centre once 0.5% of the vertices are invalidated instead of repairing
    G.set_tuning(recompute_permille=5)
    static = {"bfs_ms": min(bfs.Static() for _ in range(2)),
              "sssp_ms": min(sssp.Static() for _ in range(2)),
              "wcc_ms": min(wcc.Static() for _ in range(2))}
    static["bfs_levels"], _ = bfs.stats()
    static["sssp_levels"], _ = sssp.stats()
    rng = np.random.default_rng(SEED + 22 + rank)
    rec = {k: [] for k in ("update_ms", "bfs_ms", "sssp_ms", "wcc_ms")}
    dec, inc = {k: [] for k in rec}, {k: [] for k in rec}
    repair = {"bfs": [], "sssp": [], "wcc": []}
    history = []  # host copies of every batch, for the oracle replay
    INFINF = np.uint64(2**64 - 1)
    for b in range(nbatch):
        packed = sssp.packed()
        par = (packed & np.uint64(0xFFFFFFFF)).astype(np.int64)
        tree = np.flatnonzero((packed != INFINF) & (par != np.arange(V)))
        nt = min(len(tree), int(0.8 * batch))
        pick = rng.choice(tree, size=nt, replace=False)
        ridx = rng.integers(0, E, batch - nt)
        ds = np.concatenate([par[pick], s[ridx]]).astype(np.uint32)
        dd = np.concatenate([pick, d[ridx]]).astype(np.uint32)
        tds, tdd = todev(ds), todev(dd)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        G.DeleteEdges(tds, tdd)
        e1.record()
        e1.synchronize()
        dec["update_ms"].append(e0.elapsed_time(e1))
        Gr.DeleteEdges(tds, tdd)
        dec["bfs_ms"].append(bfs.Decremental(tds, tdd))
        dec["sssp_ms"].append(sssp.Decremental(tds, tdd))
        dec["wcc_ms"].append(wcc.Decremental(tds, tdd))
        repair["bfs"].append(bfs.decremental_stats())
        repair["sssp"].append(sssp.decremental_stats())
        repair["wcc"].append(wcc.decremental_stats())
        history.append(("del", ds, dd, None))
    for b in range(nbatch):
        u = rng.integers(0, V, batch)
        dx = rng.integers(-2, 3, batch)
        dy = rng.integers(-2, 3, batch)
        r, c = u // side + dy, u % side + dx
        ok = (r >= 0) & (r < side) & (c >= 0) & (c < side) & ((dx != 0) | (dy != 0))
        r, c, u = np.where(ok, r, u // side), np.where(ok, c, u % side), u
        v = (r * side + c).astype(np.uint32)
        uw = rng.integers(1, 1001, batch).astype(np.uint32)
        tis, tid, tiw = todev(u), todev(v), todev(uw)
        history.append(("ins", u.astype(np.uint32), v, uw))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        G.InsertEdges(tis, tid, vals=tiw)
        e1.record()
        e1.synchronize()
        inc["update_ms"].append(e0.elapsed_time(e1))
        Gr.InsertEdges(tis, tid)
        inc["bfs_ms"].append(bfs.Incremental(tis, tid))
        inc["sssp_ms"].append(sssp.Incremental(tis, tid, wgt=tiw))
        inc["wcc_ms"].append(wcc.Incremental(tis, tid))
    assert G.sync() == 0
    # full-size check: the maintained answers equal a fresh recompute
    got = (bfs.Distances(), sssp.Distances(), wcc.Labels())
    fb, fs, fw = mk.BFS(G, src, V), mk.SSSP(G, src, V), mk.WCC(G)
    fb.Static(), fs.Static(), fw.Static()
    same = {"bfs": bool(np.array_equal(got[0], fb.Distances())),
            "sssp": bool(np.array_equal(got[1], fs.Distances())),
            "wcc": bool(np.array_equal(got[2], fw.Labels()))}
    comps = int(len(np.unique(got[2])))
    gpu_deg = G.degrees()
    for o in (fb, fs, fw, bfs, sssp, wcc):
        o.close()
    Gr.close()
    G.close()
    torch.cuda.synchronize(dev)
    torch.cuda.empty_cache()
    assert all(same.values()), same
    # the oracle replays the same batches: the maintained answers bit-exact
    par = None
    if rank == 0:
        from oracle import OracleGraph
        t0 = time.time()
        O = OracleGraph(V, threads=os.cpu_count() or 1)
        O.insert(s, d, w)
        for op, a, b, c in history:
            O.delete(a, b) if op == "del" else O.insert(a, b, c)
        par = {"degrees": bool(np.array_equal(gpu_deg, O.degrees())),
               "bfs": bool(np.array_equal(got[0], O.bfs(src))),
               "sssp": bool(np.array_equal(got[1], O.sssp(src))),
               "wcc": bool(np.array_equal(got[2], O.wcc()))}
        par["ok"] = all(par.values())
        del O
        log(f"[grid] oracle replay and checks in {time.time() - t0:.1f}s: {par}")
    p50 = lambda xs: statistics.median(xs) if xs else None
    out = {"workload": f"grid{side}_decremental_stress", "vertices": V, "edges": E,
           "tuning": {"sssp_delta": nf["best"], "recompute_permille": 5},
           "batches": nbatch, "batch": batch, "source": src, "static": static,
           "decremental_p50_ms": {k: p50(v) for k, v in dec.items()},
           "incremental_p50_ms": {k: p50(v) for k, v in inc.items()},
           "decremental_repair": {
               **{k: {"invalidated": [int(x) for x, _ in repair[k]],
                      "recomputed": [bool(r) for _, r in repair[k]],
                      "ms": [round(x, 3) for x in dec[k + "_ms"]]} for k in ("bfs", "sssp")},
               "wcc": {"forest_edges_lost": [int(x) for x, _, _ in repair["wcc"]],
                       "path": [["unchanged", "piece rescan", "component rebuild", "static"][p]
                                for _, _, p in repair["wcc"]],
                       "ms": [round(x, 3) for x in dec["wcc_ms"]]}},
           "recompute_rule": "a decremental call recomputes from the source once its "
                             "invalidation walk passes recompute_permille of the vertices",
           "components_after": comps, "matches_static_recompute": same}
    if par is not None:
        out["parity"] = par
    return out


def run_batched(args, rank, world, local):
    import torch
    from meerkat_b200.build import build
    if rank == 0:
        build()
    barrier(world)
    torch.cuda.set_device(local)
    r = batched_compare(args.graphs, args.steps, args.warmup, rank, world, local)
    if rank == 0:
        line = {
            "metric": "batched step speedup (per-graph launches / batched runner)",
            "value": r["speedup_vs_plain"], "unit": "x", "n_gpus": world, "steps": r["steps"],
            "warmup": r["warmup"], "ms_per_step": r["batched_ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic",
            "config": {"workload": r["workload"], "graphs": r["graphs"], "step": r["step"],
                       "l2": "inputs larger than L2 (union slab pool and per-graph pools)"},
            "gpu_launches": r["steps"] * r["gpu_launches_per_step"], "clocks": r["clocks"],
            "batched": r,
        }
        print(json.dumps(line), flush=True)
    barrier(world)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--algo-batches", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--scale", type=int, default=22,
                    help="R-MAT scale (22 = the benchmark config; smaller only for profiling)")
    ap.add_argument("--batch", type=int, default=500_000, help="edges per sub-batch")
    ap.add_argument("--update-kernel", default="auto", choices=["auto", "0", "1", "2"],
                    help="auto = autotune on the first batches; 0/1 pins a variant")
    ap.add_argument("--workload", default="updates", choices=["updates", "batched", "serving"],
                    help="updates = the headline mixed-batch benchmark; batched = many small "
                         "graphs, batched runner against per-graph launches")
    ap.add_argument("--graphs", type=int, default=4096, help="member graphs (batched workload)")
    ap.add_argument("--batched-graphs", type=int, default=4096,
                    help="updates workload: also run the batched many-graph comparison on this "
                         "many graphs and attach it to the line (0 = skip)")
    ap.add_argument("--batched-steps", type=int, default=6)
    ap.add_argument("--serving-graphs", type=int, default=64)
    ap.add_argument("--serving-scales", default="18,23", help="R-MAT scale range lo,hi")
    ap.add_argument("--serving-rates", default="auto",
                    help="offered req/s, comma separated; auto = 25/50/75%% of the alone mode's "
                         "saturation throughput")
    ap.add_argument("--serving-requests", type=int, default=300, help="requests per rate")
    ap.add_argument("--serving-budget-gb", type=float, default=120.0)
    ap.add_argument("--serving-in-line", default="auto",
                    help="updates workload: offered rates of the serving comparison attached to "
                         "the line (auto = 25/50/75%% of the alone mode's saturation; '' = skip)")
    ap.add_argument("--serving-in-line-requests", type=int, default=150)
    ap.add_argument("--grid-side", type=int, default=4096,
                    help="updates workload: side of the grid decremental stress run attached to "
                         "the line (0 = skip)")
    args = ap.parse_args()
    if args.workload == "serving":
        rank, world, local = dist_setup(args.gpus)
        if args.impl == "reference":
            if rank == 0:
                print(json.dumps({"impl": "reference", "workload": "serving",
                                  "unavailable": "the reference has no serving loop and no "
                                  "CPU path; the oracle port is timed by the updates workload"}))
            return 0
        return run_serving(args, rank, world, local)
    if args.workload == "batched":
        rank, world, local = dist_setup(args.gpus)
        if args.impl == "reference":
            if rank == 0:
                print(json.dumps({"impl": "reference", "workload": "batched",
                                  "unavailable": "the reference has no many-graph runner and no "
                                  "CPU path; the oracle port is timed by the updates workload"}))
            return 0
        return run_batched(args, rank, world, local)
    global SCALE, EDGES, HALF
    SCALE, EDGES, HALF = args.scale, 16 << args.scale, args.batch
    rank, world, local = dist_setup(args.gpus)
    if args.impl == "reference":
        return run_reference(args, rank, world)

    import torch

    import meerkat_b200 as mk
    from meerkat_b200.build import build
    if rank == 0:
        build()
    barrier(world)
    torch.cuda.set_device(local)
    dev = torch.device(f"cuda:{local}")
    W, K, A = args.warmup, args.steps, args.algo_batches
    from meerkat_b200.autotune import VARIANTS, tune_updates
    T = 2 * len(VARIANTS)  # two tuning rounds
    graph, batches = make_workload(T + W + 2 * K + W + A + 2)
    allb = batches  # every batch G receives, in order (the oracle replays them)
    s, d, w = graph
    V = 1 << SCALE

    def todev(a):
        return torch.from_numpy(np.ascontiguousarray(a, dtype=np.uint32).view(np.int32)).to(dev)

    hints = np.bincount(s, minlength=V).astype(np.uint32)
    G = mk.DynamicGraph(V, load_factor=0.7, degree_hints=hints, weighted=True, device=local)
    G.reserve_batch(HALF)
    t0 = time.time()
    G.InsertEdges(todev(s), todev(d), vals=todev(w))
    assert G.sync() == 0
    info = G.info()
    log(f"[bench] graph built in {time.time() - t0:.1f}s: {info}")

    stream = torch.cuda.current_stream(dev)
    # autotune the update kernel on the first T batches (they are real updates)
    variants = VARIANTS if args.update_kernel == "auto" else [(int(args.update_kernel), 0)] * 4
    tuning = tune_updates(G, [tuple(todev(x) for x in b) for b in batches[:T]], variants=variants,
                          stream=stream, rounds=2)
    log(f"[bench] tuning: {tuning}")
    batches = batches[T:]
    dbatches = [tuple(todev(x) for x in b) for b in batches[:W + K]]

    def step(b, ev=None):
        ds, dd, is_, id_, iw = b
        if ev is not None:
            ev[0].record(stream)
        G.DeleteEdges(ds, dd)
        if ev is not None:
            ev[1].record(stream)
        G.InsertEdges(is_, id_, vals=iw)
        if ev is not None:
            ev[2].record(stream)

    for i in range(W):
        step(dbatches[i])
    torch.cuda.synchronize(dev)
    assert G.sync() == 0
    # The K timed steps are captured into one CUDA graph and replayed once, so
    # the timed region holds exactly K steps of device work with no host
    # submission gaps (the host-driven path is measured by e2e below).  Every
    # step consumes its own batch, so the graph is replayed exactly once.
    cap_stream = torch.cuda.Stream(dev)
    cap_stream.wait_stream(stream)
    cgraph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(cgraph, stream=cap_stream):
        for i in range(K):
            ds, dd, is_, id_, iw = dbatches[W + i]
            G.DeleteEdges(ds, dd, stream=cap_stream)
            G.InsertEdges(is_, id_, vals=iw, stream=cap_stream)
    torch.cuda.synchronize(dev)
    barrier(world)
    clocks = Clocks(local)
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(dev)
    with torch.cuda.stream(cap_stream):  # replay() launches on the current stream
        t_host0 = time.perf_counter()
        start.record(cap_stream)
        cgraph.replay()
        stop.record(cap_stream)
        stop.synchronize()
        host_ms = (time.perf_counter() - t_host0) * 1000.0
    torch.cuda.synchronize(dev)
    clk = clocks.stop()
    barrier(world)
    ms = start.elapsed_time(stop)
    ms_max = max_over_ranks(ms, world, dev)
    assert G.sync() == 0
    del cgraph
    # the replay really applied the K batches: every inserted edge of every
    # timed batch is present unless a later batch deleted it, every deleted
    # edge absent unless a later batch re-inserted it, and the edge count is
    # unchanged (each step deletes and inserts HALF edges)
    verify = verify_replay(G, batches[W:W + K], todev, dev)
    assert verify["ok"], verify
    upd_per_step = 2 * HALF
    value = world * K * upd_per_step / (ms_max / 1000.0)
    # per-call split (host-driven, events around each call) for reference
    split_b = batches[W + K:W + K + 2]
    del_ms, ins_ms = [], []
    for b in split_b:
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        step(tuple(todev(x) for x in b), ev)
        torch.cuda.synchronize(dev)
        del_ms.append(ev[0].elapsed_time(ev[1]))
        ins_ms.append(ev[1].elapsed_time(ev[2]))
    assert G.sync() == 0

    # ---- e2e through the C ABI with pinned host batches ----
    # Step i+1's batch is uploaded from pinned host memory on a copy stream
    # while step i's kernels run (two device buffer sets), and every step's
    # two applied counts come back to pinned host memory with stream-ordered
    # copies.  W untimed steps run the same pipeline first (fresh batches, in
    # sequence); the timed region runs from the first upload of the K timed
    # steps to their last count.  Every pinned batch buffer is DMA'd once
    # before any of this: the first transfer out of a freshly pinned
    # allocation costs about a third more than later ones (measured 3.1-3.3
    # against 4.7 G/s for the whole pipeline), and a streaming producer
    # recycles its pinned staging buffers, paying that once.  A step's five
    # arrays sit back to back in one pinned buffer and go up in one copy into
    # one device buffer (its five views are the arguments of the calls): five
    # separate copies per step cost about 9 % of the link in per-copy
    # overhead.
    pinned = []
    for b in batches[W + K + 2:W + 2 * K + 2 + W]:
        pinned.append(torch.from_numpy(np.ascontiguousarray(np.concatenate(
            [np.asarray(x, dtype=np.uint32) for x in b])).view(np.int32)).pin_memory())
    dev_bufs = [torch.empty(5 * HALF, dtype=torch.int32, device=dev) for _ in range(2)]
    sets = [[buf.narrow(0, j * HALF, HALF) for j in range(5)] for buf in dev_bufs]
    counts = torch.zeros(2 * (W + K), dtype=torch.int64).pin_memory()
    copy_s, comp_s = torch.cuda.Stream(dev), torch.cuda.Stream(dev)
    copied = [torch.cuda.Event() for _ in range(2)]
    used = [torch.cuda.Event() for _ in range(2)]

    def upload(i):
        k = i % 2
        with torch.cuda.stream(copy_s):
            if i >= 2:
                copy_s.wait_event(used[k])
            dev_bufs[k].copy_(pinned[i], non_blocking=True)
            copied[k].record(copy_s)

    with torch.cuda.stream(copy_s):
        for i, pb in enumerate(pinned):
            dev_bufs[i % 2].copy_(pb, non_blocking=True)
    torch.cuda.synchronize(dev)

    def pipeline(i0, n):
        """Steps i0 .. i0+n-1 of the pinned batches; returns CUDA-event ms."""
        if n == 0:
            return 0.0
        torch.cuda.synchronize(dev)
        barrier(world)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(copy_s)
        upload(i0)
        for i in range(i0, i0 + n):
            if i + 1 < i0 + n:
                upload(i + 1)
            k = i % 2
            comp_s.wait_event(copied[k])
            b = sets[k]
            G.DeleteEdges(b[0], b[1], stream=comp_s)
            G.last_applied_async(counts.data_ptr() + 16 * i, stream=comp_s)  # 8-byte D2H
            G.InsertEdges(b[2], b[3], vals=b[4], stream=comp_s)
            G.last_applied_async(counts.data_ptr() + 16 * i + 8, stream=comp_s)
            used[k].record(comp_s)
        e1.record(comp_s)
        e1.synchronize()
        torch.cuda.synchronize(dev)
        return e0.elapsed_time(e1)

    pipeline(0, W)
    e2e_ms = max_over_ranks(pipeline(W, K), world, dev)
    assert G.sync() == 0
    e2e_value = world * K * upd_per_step / (e2e_ms / 1000.0)
    applied_e2e = int(counts.sum())
    assert applied_e2e == (W + K) * upd_per_step, applied_e2e
    # the host link alone: the same pinned copy per step, no kernels
    lk0, lk1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(copy_s):
        for i in range(3):
            dev_bufs[i % 2].copy_(pinned[i], non_blocking=True)
        lk0.record(copy_s)
        for i in range(K):
            dev_bufs[i % 2].copy_(pinned[W + i], non_blocking=True)
        lk1.record(copy_s)
    lk1.synchronize()
    link_gbs = K * HALF * 4 * 5 / (lk0.elapsed_time(lk1) / 1e3) / 1e9
    h2d = HALF * 4 * 5
    d2h = 16

    # ---- incremental / decremental BFS and SSSP on the same graph ----
    algo = {}
    bfs = sssp = None
    if A > 0:
        src_v = int(np.argmax(hints))
        bfs, sssp = mk.BFS(G, src_v, V), mk.SSSP(G, src_v, V)
        algo["bfs_static_ms"] = min(bfs.Static() for _ in range(2))
        # the project tuner picks the static near-far step on this graph
        # (static calls are idempotent); the dynamic calls below keep it
        from meerkat_b200.autotune import tune_sssp_delta
        nf = tune_sssp_delta(G, sssp, deltas=(0, 1000, 4000, 16000))
        algo["sssp_static_ms"] = min(t["static_ms"] for t in nf["trials"])
        algo["sssp_delta"] = nf["best"]
        algo["sssp_static_ms_plain"] = next(t["static_ms"] for t in nf["trials"] if t["sssp_delta"] == 0)
        # a weighted reverse copy of the same edges, kept in step with G, lets a
        # second pair of traversals re-seed decremental calls from in-edges
        rp_, col_, w_ = G.export_csr_range_device(0, V, weights=True)
        rows_ = torch.repeat_interleave(torch.arange(V, device=dev, dtype=torch.int32),
                                        rp_[1:] - rp_[:-1])
        indeg_ = torch.bincount(col_.long(), minlength=V).to(torch.int32).cpu().numpy().view(np.uint32)
        Gr = mk.DynamicGraph(V, degree_hints=indeg_, weighted=True, reverse=True, device=local)
        Gr.InsertEdges(rows_, col_, vals=w_)
        assert Gr.sync() == 0
        del rp_, col_, w_, rows_
        bfs_r, sssp_r = mk.BFS(G, src_v, V), mk.SSSP(G, src_v, V)
        bfs_r.set_reverse(Gr)
        sssp_r.set_reverse(Gr)
        bfs_r.Static()
        sssp_r.Static()
        rec = {k: [] for k in ("bfs_dec_ms", "sssp_dec_ms", "bfs_inc_ms", "sssp_inc_ms",
                               "bfs_dec_rev_ms", "sssp_dec_rev_ms")}
        gbs = {k: [] for k in rec}
        repair = {"bfs": [], "sssp": []}  # (invalidated, recomputed) per decremental call

        def timed_dynamic(key, trav, s_bytes, call):
            # algorithmic bytes: sum over vertices whose distance changed of
            # 8 + (s + 8) x out-degree (a lower bound: vertices invalidated
            # and restored to the same distance are not counted)
            before = trav.Distances()
            ms = call()
            changed = np.flatnonzero(trav.Distances() != before)
            deg = G.degrees().astype(np.int64)
            nbytes = int(8 * len(changed) + (s_bytes + 8) * deg[changed].sum())
            rec[key].append(ms)
            gbs[key].append(nbytes / (ms / 1e3) / 1e9)

        for b in batches[W + 2 * K + 2 + W:W + 2 * K + 2 + W + A]:
            ds, dd, is_, id_, iw = (todev(x) for x in b)
            G.DeleteEdges(ds, dd)
            Gr.DeleteEdges(ds, dd)
            timed_dynamic("bfs_dec_ms", bfs, 4, lambda: bfs.Decremental(ds, dd))
            timed_dynamic("sssp_dec_ms", sssp, 8, lambda: sssp.Decremental(ds, dd))
            repair["bfs"].append(bfs.decremental_stats())
            repair["sssp"].append(sssp.decremental_stats())
            timed_dynamic("bfs_dec_rev_ms", bfs_r, 4, lambda: bfs_r.Decremental(ds, dd))
            timed_dynamic("sssp_dec_rev_ms", sssp_r, 8, lambda: sssp_r.Decremental(ds, dd))
            G.InsertEdges(is_, id_, vals=iw)
            Gr.InsertEdges(is_, id_, vals=iw)
            timed_dynamic("bfs_inc_ms", bfs, 4, lambda: bfs.Incremental(is_, id_))
            timed_dynamic("sssp_inc_ms", sssp, 8, lambda: sssp.Incremental(is_, id_, wgt=iw))
            bfs_r.Incremental(is_, id_, timed=False)
            sssp_r.Incremental(is_, id_, wgt=iw, timed=False)
        assert np.array_equal(bfs.Distances(), bfs_r.Distances())
        assert np.array_equal(sssp.Distances(), sssp_r.Distances())
        for o in (bfs_r, sssp_r, Gr):
            o.close()
        assert G.sync() == 0
        peak_q = measured_peak()[0]
        for k, v in rec.items():
            algo[k + "_p50"] = statistics.median(v)
            g = statistics.median(gbs[k])
            algo[k.replace("_ms", "_gbs") + "_p50"] = g
            algo[k.replace("_ms", "_frac") + "_p50"] = g / peak_q
        algo["source"] = src_v
        algo["decremental_repair"] = {
            k: {"invalidated": [int(x) for x, _ in v], "recomputed": [bool(r) for _, r in v],
                "invalidated_share_p50": statistics.median(x for x, _ in v) / V}
            for k, v in repair.items()}
        # the maintained answers after the A batches, for the oracle check
        gpu_final = {"source": src_v, "bfs": bfs.Distances(), "sssp": sssp.Distances(),
                     "bfs_packed": bfs.packed(), "sssp_packed": sssp.packed()}
        bfs.close()
        sssp.close()
        bfs = sssp = None
        mq, mq_finals = more_queries(mk, G, V, dev, SEED + 11)
        algo.update(mq)
        gpu_final.update(mq_finals)
        gpu_final["degrees"] = G.degrees()

    peak, peak_kind = measured_peak()
    upd_bytes = HALF * DEL_BYTES + HALF * INS_BYTES
    upd_ms = ms / K  # device time of one delete + insert pair (graph replay)
    achieved = upd_bytes / (upd_ms / 1000.0) / 1e9
    traffic = profile_traffic()
    share = head_slab_share(G, batches[W:W + min(K, 4)])
    # the same random-line pattern without decision logic, on a buffer the
    # size of the slab pool: what the memory system gives this access pattern
    ceiling = probe_random_rmw(int(info["pool_capacity"]) * 128, V, 2 * HALF, device=local)
    cb = cpu_q = parity_large = None
    if rank == 0 and not args.no_cpu_baseline:
        if A > 0:
            hist = allb[:T + W + 2 * K + 2 + W + A]
            timed_at = (T + W, T + W + 3)  # the CPU times the first 3 of the K timed batches
            cb, cpu_q, parity_large = oracle_large(graph, hist, timed_at, A, gpu_final, algo)
            del gpu_final
        else:
            cb = cpu_baseline(graph, batches[W:W + K], max_batches=3)
    batched = None
    if args.batched_graphs > 0:
        del bfs, sssp
        G.close()
        torch.cuda.synchronize(dev)
        r = batched_compare(args.batched_graphs, args.batched_steps, W, rank, world, local)
        batched = {k: r[k] for k in (
            "workload", "speedup_vs_plain", "speedup_vs_plain_cuda_graph", "batched_ms_per_step",
            "plain_ms_per_step", "plain_cuda_graph_ms_per_step", "batched_updates_per_s",
            "updates_per_step", "vertices", "edges", "gpu_launches_per_step",
            "batched_form", "forms_ms_per_step", "forms_launches_per_step", "forms_equal",
            "plain_launches_per_step", "queries", "tuning", "equality", "clocks", "steps")
            if k in r}
        if "parity" in r:
            batched["parity"] = r["parity"]
    grid = None
    if args.grid_side > 0:
        grid = grid_stress(args.grid_side, 10, 500_000, rank, world, local)
    serving = None
    if args.serving_in_line:
        rates = [float(x) for x in args.serving_in_line.split(",") if x.strip() not in ("", "auto")]
        scales = tuple(int(x) for x in args.serving_scales.split(","))
        r = serving_compare(args.serving_graphs, scales, rates, args.serving_in_line_requests,
                            args.serving_budget_gb, rank, world, local)
        serving = {k: r[k] for k in ("workload", "vertices", "edges", "requests_per_rate",
                                     "budget_gb", "clocks", "saturation", "rates")}
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": K,
            "warmup": W, "ms_per_step": ms_max / K, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u32", "data": "synthetic",
            "config": config_block(world),
            "e2e": {"value": e2e_value, "unit": METRIC, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h,
                    "upload_gbs": K * h2d / (e2e_ms / 1e3) / 1e9,
                    "h2d_link_gbs": link_gbs,
                    "link_note": "h2d_link_gbs: the same pinned copies with no kernels; "
                                 "upload_gbs / h2d_link_gbs is how close e2e is to the host link",
                    "pinned_note": "each step's batch sits in its own pinned buffer, DMA'd once "
                                   "before the timed region (a first transfer from a freshly "
                                   "pinned buffer is about a third slower); every timed step "
                                   "uploads its 10 MB (its five arrays back to back, one copy)"},
            "gpu_launches": 2 * K,  # one delete and one insert kernel per step
            "roofline": {"bound": "hbm", "kernel": "k_update delete + insert (one mixed batch, graph replay)",
                         "achieved": achieved, "peak": peak, "peak_kind": peak_kind,
                         "unit": "GB/s", "frac": achieved / peak,
                         "algorithmic_bytes_per_step": upd_bytes,
                         "traffic": traffic,
                         "head_slab_sharing": share,
                         "pattern_ceiling": {
                             "what": "benchmark probe: random 128-B line read + CAS + random "
                                     "4-B read and add per operation, no decision logic, "
                                     f"{2 * HALF} operations on a {int(info['pool_capacity']) * 128 >> 20} MiB buffer",
                             **ceiling,
                             "frac": (upd_per_step / (ms / K / 1000.0)) / ceiling["update_pattern_per_s"]}},
            "host_driven_delete_ms": statistics.mean(del_ms),
            "host_driven_insert_ms": statistics.mean(ins_ms),
            "tuning": tuning["best"],
            "replay_check": verify,
            "replay_host_ms": host_ms,
            "clocks": clk,
            "queries": algo,
            "graph": {"slabs_used": info["slabs_used"], "buckets": info["num_buckets"],
                      "device_bytes": info["device_bytes"]},
        }
        if "bfs_pull" in algo:
            algo["bfs_pull"].pop("trials", None)
        if cb is not None:
            line["cpu_baseline"] = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}
        if cpu_q is not None:
            line["cpu_queries"] = cpu_q
        parity = {}
        if parity_large is not None:
            line["parity_large"] = parity_large
            parity["large"] = "ok" if parity_large["ok"] else "MISMATCH"
        if batched is not None:
            line["batched"] = batched
            if "parity" in batched:
                parity["batched"] = "ok" if batched["parity"]["ok"] else "MISMATCH"
        if serving is not None:
            line["serving"] = serving
        if grid is not None:
            line["grid"] = grid
            if "parity" in grid:
                parity["grid"] = "ok" if grid["parity"]["ok"] else "MISMATCH"
        line["parity"] = parity
        # a compact digest last, so a reader of the line's tail sees it
        line["summary"] = line_summary(line)
        print(json.dumps(line), flush=True)
    barrier(world)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
