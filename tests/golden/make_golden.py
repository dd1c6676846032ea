"""Generates tests/golden/rmat10.npz: a small seeded R-MAT graph, one insert and
one delete batch, and the expected BFS / SSSP / WCC / PageRank / triangle
results after each step, computed with scipy.sparse.csgraph and networkx
(independent of both the CUDA library and the oracle).

The reference (meerkat-pkd/Meerkat) ships no golden vectors and cannot be
built here, so these vectors pin the oracle against independent
implementations of the same definitions:
  BFS levels / SSSP uint32 distances from the source, 0xFFFFFFFF unreachable;
  WCC label = minimum vertex id of the weakly connected component;
  PageRank with teleport (1-d)/N and dangling mass spread uniformly, d = 0.85;
  triangle count of the symmetrised simple graph.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import networkx as nx
import numpy as np
import scipy.sparse as sp
from scipy.sparse import csgraph

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from meerkat_b200 import EdgeSet, gen_rmat  # noqa: E402  (host-only generator)

INF = 0xFFFFFFFF
SCALE, EDGES, SEED, SRC = 10, 8192, 0x4D45524B, 0
V = 1 << SCALE


def expected(src, dst, w):
    A = sp.csr_matrix((w.astype(np.float64), (src, dst)), shape=(V, V))
    B = sp.csr_matrix((np.ones(len(src)), (src, dst)), shape=(V, V))
    bfs = csgraph.shortest_path(B, method="D", directed=True, unweighted=True, indices=SRC)
    sssp = csgraph.dijkstra(A, directed=True, indices=SRC)
    to_u32 = lambda d: np.where(np.isinf(d), INF, d).astype(np.uint64).astype(np.uint32)
    ncomp, lab = csgraph.connected_components(B, directed=True, connection="weak")
    mins = np.full(ncomp, V, dtype=np.int64)
    np.minimum.at(mins, lab, np.arange(V))
    wcc = mins[lab].astype(np.uint32)
    G = nx.DiGraph()
    G.add_nodes_from(range(V))
    G.add_edges_from(zip(src.tolist(), dst.tolist()))
    pr = nx.pagerank(G, alpha=0.85, tol=1e-15, max_iter=100000)
    pr = np.array([pr[i] for i in range(V)], dtype=np.float64)
    U = nx.Graph()
    U.add_nodes_from(range(V))
    U.add_edges_from(zip(src.tolist(), dst.tolist()))
    tri = sum(nx.triangles(U).values()) // 3
    return dict(bfs=to_u32(bfs), sssp=to_u32(sssp), wcc=wcc, pr=pr, tc=np.uint64(tri))


def main():
    s, d, w = gen_rmat(SCALE, EDGES, seed=SEED, w_lo=1, w_hi=64)
    es = EdgeSet(V, s, d)
    ins_s, ins_d = es.sample_absent(200, seed=SEED + 1)
    ins_w = (np.arange(200, dtype=np.uint32) % 64) + 1
    del_s, del_d = es.sample_present(200, seed=SEED + 2)

    out = dict(src=s, dst=d, w=w, ins_src=ins_s, ins_dst=ins_d, ins_w=ins_w, del_src=del_s,
               del_dst=del_d)
    for k, v in expected(s, d, w).items():
        out["base_" + k] = v
    # after the insert batch
    s1 = np.concatenate([s, ins_s])
    d1 = np.concatenate([d, ins_d])
    w1 = np.concatenate([w, ins_w])
    for k, v in expected(s1, d1, w1).items():
        out["ins_" + k] = v
    # after the delete batch
    gone = set(zip(del_s.tolist(), del_d.tolist()))
    keep = np.array([(a, b) not in gone for a, b in zip(s1.tolist(), d1.tolist())])
    for k, v in expected(s1[keep], d1[keep], w1[keep]).items():
        out["del_" + k] = v
    path = Path(__file__).resolve().parent / "rmat10.npz"
    np.savez_compressed(path, **out)
    print(f"wrote {path} ({path.stat().st_size} bytes)")


if __name__ == "__main__":
    main()
