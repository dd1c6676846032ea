"""Edge cases of the update path and the algorithms: empty and degenerate
batches, tiny graphs, and a size-independent round trip at a larger size."""
import numpy as np
import pytest

import meerkat_b200 as mk

from helpers import assert_same_graph, make_pair, symmetrise, to_dev

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("variant", [0, 1, 2])
def test_empty_and_degenerate_batches(variant):
    import torch
    V = 512
    s, d, w = mk.gen_rmat(9, 3000, seed=3, w_lo=1, w_hi=9)
    G, O = make_pair(V, s, d, w, weighted=True, variant=variant)
    empty = torch.empty(0, dtype=torch.int32, device="cuda:0")
    G.InsertEdges(empty, empty, vals=empty)
    assert G.sync() == 0 and G.last_applied() == 0
    G.DeleteEdges(empty, empty)
    assert G.sync() == 0 and G.last_applied() == 0
    # a batch of self-loops only: nothing applied, nothing changes
    loops = to_dev(np.arange(100, dtype=np.uint32))
    G.InsertEdges(loops, loops, vals=loops)
    assert G.sync() == 0 and G.last_applied() == 0
    G.DeleteEdges(loops, loops)
    assert G.sync() == 0 and G.last_applied() == 0
    assert_same_graph(G, O, weighted=True)
    # the algorithms accept empty batches and keep their answers
    bfs, sssp, wcc = mk.BFS(G, 0, V), mk.SSSP(G, 0, V), mk.WCC(G)
    bfs.Static(), sssp.Static(), wcc.Static()
    bfs.Incremental(empty, empty, n=0)
    bfs.Decremental(empty, empty, n=0)
    sssp.Incremental(empty, empty, n=0, wgt=empty)
    wcc.Incremental(empty, empty, n=0)
    np.testing.assert_array_equal(bfs.Distances(), O.bfs(0))
    np.testing.assert_array_equal(sssp.Distances(), O.sssp(0))
    np.testing.assert_array_equal(wcc.Labels(), O.wcc())


def test_single_vertex_graph():
    import torch
    G = mk.DynamicGraph(1)
    z = torch.zeros(4, dtype=torch.int32, device="cuda:0")
    G.InsertEdges(z, z)
    assert G.sync() == 0 and G.last_applied() == 0
    assert G.degrees().tolist() == [0]
    bfs = mk.BFS(G, 0, 1)
    bfs.Static()
    assert bfs.Distances().tolist() == [0]
    wcc = mk.WCC(G)
    wcc.Static()
    assert wcc.Labels().tolist() == [0]
    rp, col, _ = G.export_csr()
    assert rp.tolist() == [0, 0] and len(col) == 0


def test_tc_and_pagerank_accept_empty_batches():
    import torch
    V = 1 << 10
    s, d, _ = mk.gen_rmat(10, 6000, seed=5)
    ss, sd = symmetrise(s, d)
    Gs, Os = make_pair(V, ss, sd)
    tc = mk.TC(Gs, V)
    tc.Static()
    empty = torch.empty(0, dtype=torch.int32, device="cuda:0")
    tc.Incremental(empty, empty, n=0)
    tc.Decremental(empty, empty, n=0)
    assert tc.GetCount() == Os.triangles()
    Gr, _ = make_pair(V, s, d, reverse=True)
    pr = mk.PageRank(Gr, 0.85, 1e-6, V, max_iter=500)
    pr.Static()
    before = pr.Values()
    pr.Incremental(empty, empty, n=0)
    assert np.abs(pr.Values() - before).sum() <= 1e-6


def test_insert_delete_round_trip_at_scale_20():
    """A million absent edges inserted and deleted again leave exactly the
    original adjacency (compared as sorted CSR) and one tombstone each."""
    import torch
    V = 1 << 20
    s, d, w = mk.gen_rmat(20, 8 << 20, seed=99, w_lo=1, w_hi=1000)
    hints = np.bincount(s, minlength=V).astype(np.uint32)
    G = mk.DynamicGraph(V, degree_hints=hints, weighted=True)
    G.InsertEdges(to_dev(s), to_dev(d), vals=to_dev(w))
    assert G.sync() == 0
    rp0, col0, w0 = G.export_csr(sort_rows=True)
    es = mk.EdgeSet(V, s, d)
    is_, id_ = es.sample_absent(1 << 20, seed=100)
    ti, td = to_dev(is_), to_dev(id_)
    G.InsertEdges(ti, td, vals=to_dev(np.full(1 << 20, 7, np.uint32)))
    assert G.sync() == 0 and G.last_applied() == 1 << 20
    G.DeleteEdges(ti, td)
    assert G.sync() == 0 and G.last_applied() == 1 << 20
    rp1, col1, w1 = G.export_csr(sort_rows=True)
    np.testing.assert_array_equal(rp0, rp1)
    np.testing.assert_array_equal(col0, col1)
    np.testing.assert_array_equal(w0, w1)
    tomb = G.tombstones().astype(np.int64)
    np.testing.assert_array_equal(tomb, np.bincount(is_, minlength=V))
