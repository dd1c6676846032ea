"""CPU: the oracle against independent implementations on many small seeded
graphs (sizes 1..300, sparse to dense, self loops, duplicate and absent
batch entries).  The batch semantics are modelled here with a dict (self
loops skipped, a duplicate or re-inserted edge keeps the minimum weight, a
delete of an absent edge is a no-op); BFS / SSSP / WCC come from
scipy.sparse.csgraph, triangles from networkx, PageRank from an FP64 power
iteration of the same formula."""
import networkx as nx
import numpy as np
import pytest
import scipy.sparse as sp
from scipy.sparse import csgraph

from oracle import OracleGraph

INF = 0xFFFFFFFF


def model_insert(edges, s, d, w):
    for a, b, c in zip(s.tolist(), d.tolist(), w.tolist()):
        if a == b:
            continue
        edges[(a, b)] = min(c, edges.get((a, b), c))


def model_delete(edges, s, d):
    for a, b in zip(s.tolist(), d.tolist()):
        edges.pop((a, b), None)


def expected(V, edges, src):
    if edges:
        keys = np.array(list(edges.keys()), dtype=np.int64)
        wts = np.array(list(edges.values()), dtype=np.float64)
    else:
        keys = np.zeros((0, 2), np.int64)
        wts = np.zeros(0)
    A = sp.csr_matrix((wts, (keys[:, 0], keys[:, 1])), shape=(V, V))
    B = sp.csr_matrix((np.ones(len(keys)), (keys[:, 0], keys[:, 1])), shape=(V, V))
    bfs = csgraph.shortest_path(B, method="D", directed=True, unweighted=True, indices=src)
    sssp = csgraph.dijkstra(A, directed=True, indices=src)
    to_u32 = lambda x: np.where(np.isinf(x), INF, x).astype(np.uint32)
    _, comp = csgraph.connected_components(B, directed=True, connection="weak")
    first = np.full(comp.max() + 1, V, dtype=np.int64)
    np.minimum.at(first, comp, np.arange(V))
    wcc = first[comp].astype(np.uint32)
    U = nx.Graph()
    U.add_nodes_from(range(V))
    U.add_edges_from((a, b) for a, b in edges if a != b)
    tri = sum(nx.triangles(U).values()) // 3
    outdeg = np.bincount(keys[:, 0], minlength=V).astype(np.float64)
    pr = np.full(V, 1.0 / V)
    for _ in range(10000):
        contrib = np.where(outdeg > 0, pr / np.maximum(outdeg, 1), 0.0)
        nxt = np.full(V, (1 - 0.85) / V + 0.85 * pr[outdeg == 0].sum() / V)
        np.add.at(nxt, keys[:, 1], 0.85 * contrib[keys[:, 0]])
        delta = np.abs(nxt - pr).sum()
        pr = nxt
        if delta < 1e-15:
            break
    return to_u32(bfs), to_u32(sssp), wcc, tri, pr


def check(g, V, edges, src):
    bfs, sssp, wcc, tri, pr = expected(V, edges, src)
    np.testing.assert_array_equal(g.bfs(src), bfs)
    np.testing.assert_array_equal(g.sssp(src), sssp)
    np.testing.assert_array_equal(g.wcc(), wcc)
    assert g.triangles() == tri
    got, _ = g.pagerank(d=0.85, tol=1e-14)
    assert np.abs(got - pr).sum() < 1e-9
    assert g.num_edges() == len(edges)
    deg = np.zeros(V, np.int64)
    for a, _ in edges:
        deg[a] += 1
    np.testing.assert_array_equal(g.degrees(), deg)


@pytest.mark.parametrize("case", range(24))
def test_oracle_matches_independent_implementations(case):
    rng = np.random.default_rng(1000 + case)
    V = int(rng.choice([1, 2, 3, 7, 31, 64, 150, 300]))
    dense = case % 3 == 0
    E = int(rng.integers(0, (V * V if dense else 4 * V) + 1))
    s = rng.integers(0, V, E)
    d = rng.integers(0, V, E) if not dense else (s + rng.integers(0, 3, E)) % V
    w = rng.integers(1, 1001, E)
    g = OracleGraph(V, threads=1 + case % 3)
    edges = {}
    g.insert(s, d, w)
    model_insert(edges, s, d, w)
    src = int(rng.integers(0, V))
    check(g, V, edges, src)
    # insert batch: new pairs, duplicates of live edges with random weights
    n2 = int(rng.integers(0, 2 * V + 1))
    s2 = np.concatenate([rng.integers(0, V, n2), s[: n2 // 2]])
    d2 = np.concatenate([rng.integers(0, V, n2), d[: n2 // 2]])
    w2 = rng.integers(1, 1001, len(s2))
    g.insert(s2, d2, w2)
    model_insert(edges, s2, d2, w2)
    check(g, V, edges, src)
    # delete batch: half live edges, half random (mostly absent) pairs
    live = list(edges.keys())
    k = len(live) // 2
    pick = rng.permutation(len(live))[:k] if k else np.zeros(0, np.int64)
    s3 = np.array([live[i][0] for i in pick] + rng.integers(0, V, k).tolist(), dtype=np.int64)
    d3 = np.array([live[i][1] for i in pick] + rng.integers(0, V, k).tolist(), dtype=np.int64)
    g.delete(s3, d3)
    model_delete(edges, s3, d3)
    check(g, V, edges, src)
