"""GPU: bounded device-side waits run out and are reported, without a fault.

The persistent BFS/SSSP and PageRank kernels separate their levels and
passes with grid barriers whose waits are bounded by the graph's
`wait_limit_us` (4 s by default); the reference spins without a bound
(include/Util/Lock.cuh:43-56, include/Util/UnionFind.cuh:197-213).  Here the
limit is set to 1 microsecond on a graph whose traversal needs over a
hundred levels, so blocks that reach a barrier before the others give up:
the call must return MK_ERR_TIMEOUT with every block gone (the device stays
usable), and once the default is restored the next calls on the same
handles must match the oracle again."""
import numpy as np
import pytest

import meerkat_b200 as mk
from helpers import degree_hints, to_dev
from oracle import OracleGraph

pytestmark = pytest.mark.gpu

PR_L1_TOL = 1e-6


def _grid(side):
    s, d, w = mk.gen_grid(side, 0, seed=3, w_lo=1, w_hi=9)
    return side * side, s, d, w


def test_traversal_barrier_limit_expires_and_recovers():
    V, s, d, w = _grid(64)  # 126 BFS levels from a corner
    G = mk.DynamicGraph(V, degree_hints=degree_hints(s, V), weighted=True)
    G.InsertEdges(to_dev(s), to_dev(d), vals=to_dev(w))
    assert G.sync() == 0
    O = OracleGraph(V)
    O.insert(s, d, w)
    bfs, sssp = mk.BFS(G, 0, V), mk.SSSP(G, 0, V)
    G.set_tuning(wait_limit_us=1)
    for t in (bfs, sssp):
        with pytest.raises(mk.MeerkatError, match="MK_ERR_TIMEOUT"):
            t.Static()
        with pytest.raises(mk.MeerkatError, match="MK_ERR_TIMEOUT"):
            t.Distances()
    # untimed: reported by the next read of the results
    bfs.Static(timed=False)
    with pytest.raises(mk.MeerkatError, match="MK_ERR_TIMEOUT"):
        bfs.Distances()
    assert G.sync() == 0  # the graph itself is untouched
    G.set_tuning(wait_limit_us=0)
    bfs.Static()
    sssp.Static()
    np.testing.assert_array_equal(bfs.Distances(), O.bfs(0))
    np.testing.assert_array_equal(sssp.Distances(), O.sssp(0))
    # and the dynamic calls work on the recovered state
    ds, dd = s[:200], d[:200]
    G.DeleteEdges(to_dev(ds), to_dev(dd))
    O.delete(ds, dd)
    bfs.Decremental(to_dev(ds), to_dev(dd))
    sssp.Decremental(to_dev(ds), to_dev(dd))
    np.testing.assert_array_equal(bfs.Distances(), O.bfs(0))
    np.testing.assert_array_equal(sssp.Distances(), O.sssp(0))
    for o in (bfs, sssp, G):
        o.close()


def test_pagerank_barrier_limit_expires_and_recovers():
    V, s, d, w = _grid(256)
    Gr = mk.DynamicGraph(V, degree_hints=degree_hints(d, V), reverse=True)
    Gr.InsertEdges(to_dev(s), to_dev(d))
    assert Gr.sync() == 0
    O = OracleGraph(V)
    O.insert(s, d)
    pr = mk.PageRank(Gr, 0.85, 1e-6, V)
    Gr.set_tuning(wait_limit_us=1)
    with pytest.raises(mk.MeerkatError, match="MK_ERR_TIMEOUT"):
        pr.Static()
    Gr.set_tuning(wait_limit_us=0)
    pr.Static()
    want, _ = O.pagerank(0.85, 1e-13)
    assert np.abs(pr.Values().astype(np.float64) - want).sum() <= PR_L1_TOL
    pr.close()
    Gr.close()
