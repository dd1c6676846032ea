"""GPU: triangle counting of graph-set members straight from their out-edges
(mk_tc_range_*), against the oracle's count on each member's symmetrised
simple graph.  Members mix one-way and reciprocal edges, a hub whose
oriented degree exceeds the one-warp limit, an empty member, and updates
between runs."""
import numpy as np
import pytest

import meerkat_b200 as mk
from helpers import to_dev
from oracle import OracleGraph

pytestmark = pytest.mark.gpu


def _member_edges(n, m, seed, hub=False, recip=0.3):
    rng = np.random.default_rng(seed)
    s, d, _ = mk.gen_rmat(int(np.log2(n)), m, seed=seed, w_lo=1, w_hi=9)
    k = int(len(s) * recip)  # reverse copies of some edges
    s = np.concatenate([s, d[:k]])
    d = np.concatenate([d, s[:k]])
    if hub:  # vertex 1 linked both ways to 3,000 others (oriented degree > 1,024)
        o = rng.choice(np.arange(2, n), size=3000, replace=False).astype(np.uint32)
        s = np.concatenate([s, np.full(3000, 1, np.uint32), o[:1500]])
        d = np.concatenate([d, o, np.full(1500, 1, np.uint32)])
    return s.astype(np.uint32), d.astype(np.uint32)


@pytest.mark.parametrize("weighted", [False, True])
def test_tc_range_matches_oracle(weighted):
    sizes = [4096, 8192, 2048, 16]
    S = mk.GraphSet(sizes, weighted=weighted)
    off = S.offsets.astype(np.int64)
    oracles, gs, gd = [], [], []
    for m, n in enumerate(sizes):
        if n == 16:
            s = d = np.zeros(0, np.uint32)
        else:
            s, d = _member_edges(n, 12 * n, 50 + m, hub=(m == 1))
        O = OracleGraph(n)
        O.insert(s, d)
        oracles.append(O)
        gs.append(s + off[m])
        gd.append(d + off[m])
    src, dst = np.concatenate(gs), np.concatenate(gd)
    S.graph.InsertEdges(to_dev(src), to_dev(dst),
                        vals=to_dev(np.ones(len(src), np.uint32)) if weighted else None)
    assert S.graph.sync() == 0
    t = mk.TCRange(S.graph)
    for rnd in range(2):
        for m in range(len(sizes)):
            t.Run(int(off[m]), int(off[m + 1]))
            assert t.GetCount() == oracles[m].triangles(), (rnd, m)
        # delete a slice of member 1's edges (including reciprocal ones) and rerun
        ds, dd = gs[1][::7], gd[1][::7]
        S.graph.DeleteEdges(to_dev(ds), to_dev(dd))
        oracles[1].delete(ds - off[1], dd - off[1])
        assert S.graph.sync() == 0
    t.close()
    S.close()


def test_tc_range_on_a_whole_graph_equals_symmetric_tc():
    V = 1 << 12
    s, d, _ = mk.gen_rmat(12, 60000, seed=8)
    G = mk.DynamicGraph(V, degree_hints=np.bincount(s, minlength=V).astype(np.uint32))
    G.InsertEdges(to_dev(s), to_dev(d))
    O = OracleGraph(V)
    O.insert(s, d)
    t = mk.TCRange(G)
    ms = t.Run(0, V)
    assert ms >= 0 and t.GetCount() == O.triangles()
    t.close()
    G.close()


def test_tc_range_flags_an_edge_leaving_the_range():
    S = mk.GraphSet([64, 64])
    S.graph.InsertEdges(to_dev(np.array([1, 2, 3], np.uint32)), to_dev(np.array([2, 3, 70], np.uint32)))
    assert S.graph.sync() == 0
    t = mk.TCRange(S.graph)
    t.Run(0, 64)
    assert t.GetCount() == 0
    with pytest.raises(mk.MeerkatError, match="MK_ERR_INVALID"):
        S.graph.sync()
    t.close()
    S.close()
