"""Autotuner for the update path.

Measures every update-kernel variant (mk_tuning.update_kernel and
update_blocks_per_sm) on live update batches of the caller's graph and keeps
the fastest.  Each trial applies a real mixed batch (deletes of present
edges, then inserts of absent edges), so tuning consumes batches exactly like
the timed run and leaves the graph in a valid state.  Results can be cached
in a JSON file keyed by GPU name and graph shape.

There is no counterpart in the reference (it has one insert and one delete
kernel with fixed 128-thread blocks, include/Graph/SlabGraphImpl.cuh:6-62).
"""
from __future__ import annotations

import json
import os
from pathlib import Path
from typing import Iterable, List, Optional, Sequence, Tuple

# (update_kernel, update_blocks_per_sm): warp-staged TMA kernel, lane-per-edge
# kernel, warp-cooperative kernel at full and at half residency (an even
# count, so the rotating rounds give every variant both batch kinds)
VARIANTS: Tuple[Tuple[int, int], ...] = ((0, 0), (1, 6), (2, 0), (2, 4))


def _key(G, device_name: str) -> str:
    info = G.info()
    return (f"{device_name}|V={info['num_vertices']}|E~{info['num_edges'] >> 20}M|"
            f"w={info['weighted']}|r={info['reverse']}")


def cache_path() -> Path:
    return Path(os.environ.get("MK_TUNING_CACHE",
                               Path.home() / ".cache" / "meerkat_b200" / "tuning.json"))


def load_cached(G, device_name: str) -> Optional[dict]:
    p = cache_path()
    if not p.exists():
        return None
    try:
        return json.loads(p.read_text()).get(_key(G, device_name))
    except (OSError, ValueError):
        return None


def store_cached(G, device_name: str, best: dict) -> None:
    p = cache_path()
    try:
        p.parent.mkdir(parents=True, exist_ok=True)
        data = json.loads(p.read_text()) if p.exists() else {}
        data[_key(G, device_name)] = best
        p.write_text(json.dumps(data, indent=1, sort_keys=True))
    except (OSError, ValueError):
        pass


def tune_updates(G, batches: Iterable[Sequence], variants: Sequence[Tuple[int, int]] = VARIANTS,
                 stream=None, rounds: int = 1) -> dict:
    """Times one mixed batch per variant and round (batches: (del_src, del_dst,
    ins_src, ins_dst, ins_w) device tensors, valid in sequence; rounds x
    len(variants) of them are consumed) and selects the variant with the
    smallest step time, taking each variant's best round (a variant's first
    launch also loads its kernel, so one round alone can mislead).  Round r
    visits the variants rotated by r, so with an even variant count and
    batches of two alternating kinds every variant meets both kinds.
    Returns {"best": {...}, "trials": [...]}."""
    import torch
    it = iter(batches)
    trials: List[dict] = []
    s = stream if stream is not None else torch.cuda.current_stream()
    n = len(variants)
    for r in range(max(1, rounds)):
        for j in range(n):
            kern, bps = variants[(j + r) % n]
            b = next(it)
            G.set_tuning(update_kernel=kern, update_blocks_per_sm=bps)
            e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
            e0.record(s)
            G.DeleteEdges(b[0], b[1], stream=s)
            e1.record(s)
            G.InsertEdges(b[2], b[3], vals=b[4], stream=s)
            e2.record(s)
            e2.synchronize()
            if G.sync() != 0:
                raise RuntimeError("device error during tuning")
            trials.append({"update_kernel": kern, "update_blocks_per_sm": bps,
                           "delete_ms": e0.elapsed_time(e1), "insert_ms": e1.elapsed_time(e2)})

    def best_ms(v):
        return min(t["delete_ms"] + t["insert_ms"] for t in trials
                   if (t["update_kernel"], t["update_blocks_per_sm"]) == v)

    best = min(variants, key=best_ms)
    G.set_tuning(update_kernel=best[0], update_blocks_per_sm=best[1])
    return {"best": {"update_kernel": best[0], "update_blocks_per_sm": best[1]},
            "trials": trials}


# buckets per BFS/SSSP frontier work item
CHUNKS: Tuple[int, ...] = (1, 2, 4, 8, 16, 32)


def tune_frontier_chunk(G, traversal, chunks: Sequence[int] = CHUNKS, repeats: int = 2) -> dict:
    """Times traversal.Static() (idempotent: it recomputes from the sources)
    once per frontier chunk size, keeps the fastest on G.  Returns
    {"best": chunk, "trials": [{"frontier_chunk": c, "static_ms": t}, ...]}."""
    trials: List[dict] = []
    for c in chunks:
        G.set_tuning(frontier_chunk=c)
        t = min(traversal.Static() for _ in range(max(1, repeats)))
        trials.append({"frontier_chunk": int(c), "static_ms": t})
    best = min(trials, key=lambda t: t["static_ms"])
    G.set_tuning(frontier_chunk=best["frontier_chunk"])
    return {"best": best["frontier_chunk"], "trials": trials}


# static SSSP near-far steps (0 = plain level-synchronous)
SSSP_DELTAS: Tuple[int, ...] = (0, 128, 512, 2048, 8192)


def tune_sssp_delta(G, sssp, deltas: Sequence[int] = SSSP_DELTAS, repeats: int = 2) -> dict:
    """Times sssp.Static() (idempotent) once per near-far step, keeps the
    fastest on G.  Returns {"best": delta, "trials": [...]}."""
    trials: List[dict] = []
    for dl in deltas:
        G.set_tuning(sssp_delta=dl)
        t = min(sssp.Static() for _ in range(max(1, repeats)))
        trials.append({"sssp_delta": int(dl), "static_ms": t})
    best = min(trials, key=lambda t: t["static_ms"])
    G.set_tuning(sssp_delta=best["sssp_delta"])
    return {"best": best["sssp_delta"], "trials": trials}


# static BFS pull thresholds, per mille of the vertices (0 = never pull)
PULL_PERMILLE: Tuple[int, ...] = (0, 5, 20, 50, 150)


def tune_bfs_pull(G, bfs, perms: Sequence[int] = PULL_PERMILLE, repeats: int = 2) -> dict:
    """Times bfs.Static() (a BFS with a reverse graph attached) once per pull
    threshold, keeps the fastest on G.  Returns {"best": ..., "trials": [...]}."""
    trials: List[dict] = []
    for pm in perms:
        G.set_tuning(pull_permille=pm)
        t = min(bfs.Static() for _ in range(max(1, repeats)))
        trials.append({"pull_permille": int(pm), "static_ms": t})
    best = min(trials, key=lambda t: t["static_ms"])
    G.set_tuning(pull_permille=best["pull_permille"])
    return {"best": best["pull_permille"], "trials": trials}
