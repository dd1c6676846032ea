"""GPU parity of BFS, SSSP, PageRank, TC and WCC (static, incremental,
decremental) against the golden vectors and the oracle.

Integer results are bit-exact; BFS/SSSP parents must be valid shortest-path
parents; PageRank must be within L1 <= 1e-6 of the FP64 oracle."""
from pathlib import Path

import numpy as np
import pytest

import meerkat_b200 as mk
from helpers import degree_hints, make_pair, symmetrise, to_dev
from oracle import OracleGraph

pytestmark = pytest.mark.gpu

GOLD = Path(__file__).resolve().parent / "golden" / "rmat10.npz"
PR_L1_TOL = 1e-6  # north-star tolerance for FP32 PageRank vs the FP64 oracle


@pytest.fixture(scope="module")
def gold():
    return dict(np.load(GOLD))


def test_golden_fixture_through_the_abi(gold):
    V = 1024
    s, d, w = gold["src"], gold["dst"], gold["w"]
    G = mk.DynamicGraph(V, degree_hints=degree_hints(s, V), weighted=True)
    Gr = mk.DynamicGraph(V, degree_hints=degree_hints(d, V), reverse=True)
    ss, sd = symmetrise(s, d)
    Gs = mk.DynamicGraph(V, degree_hints=degree_hints(ss, V))
    ts, td, tw = to_dev(s), to_dev(d), to_dev(w)
    G.InsertEdges(ts, td, vals=tw)
    Gr.InsertEdges(ts, td)
    Gs.InsertEdges(to_dev(ss), to_dev(sd))
    for g in (G, Gr, Gs):
        assert g.sync() == 0
    bfs, sssp = mk.BFS(G, 0, V), mk.SSSP(G, 0, V)
    pr = mk.PageRank(Gr, 0.85, 1e-6, V, max_iter=500)
    tc, wcc = mk.TC(Gs, V), mk.WCC(G)
    bfs.Static(len(s))
    sssp.Static(len(s))
    pr.Static()
    tc.Static(len(ss))
    wcc.Static()

    def check(prefix):
        np.testing.assert_array_equal(bfs.Distances(), gold[prefix + "bfs"])
        np.testing.assert_array_equal(sssp.Distances(), gold[prefix + "sssp"])
        np.testing.assert_array_equal(wcc.Labels(), gold[prefix + "wcc"])
        assert np.abs(pr.Values().astype(np.float64) - gold[prefix + "pr"]).sum() <= PR_L1_TOL
        assert tc.GetCount() == int(gold[prefix + "tc"])

    check("base_")
    # insert batch: graph first, then the algorithms with the same batch
    i_s, i_d, i_w = to_dev(gold["ins_src"]), to_dev(gold["ins_dst"]), to_dev(gold["ins_w"])
    G.InsertEdges(i_s, i_d, vals=i_w)
    Gr.InsertEdges(i_s, i_d)
    sym_s = to_dev(np.concatenate([gold["ins_src"], gold["ins_dst"]]))
    sym_d = to_dev(np.concatenate([gold["ins_dst"], gold["ins_src"]]))
    Gs.InsertEdges(sym_s, sym_d)
    bfs.Incremental(i_s, i_d)
    sssp.Incremental(i_s, i_d, wgt=i_w)
    wcc.Incremental(i_s, i_d)
    pr.Incremental(i_s, i_d)
    tc.Incremental(sym_s, sym_d)
    check("ins_")
    # delete batch
    d_s, d_d = to_dev(gold["del_src"]), to_dev(gold["del_dst"])
    G.DeleteEdges(d_s, d_d)
    Gr.DeleteEdges(d_s, d_d)
    # an undirected edge leaves the symmetric graph only if neither direction
    # survives in the directed graph
    alive = set(zip(np.concatenate([s, gold["ins_src"]]).tolist(),
                    np.concatenate([d, gold["ins_dst"]]).tolist()))
    alive -= set(zip(gold["del_src"].tolist(), gold["del_dst"].tolist()))
    gone = np.array([(a, b) not in alive and (b, a) not in alive
                     for a, b in zip(gold["del_src"].tolist(), gold["del_dst"].tolist())])
    us, ud = gold["del_src"][gone], gold["del_dst"][gone]
    sym_s = to_dev(np.concatenate([us, ud]))
    sym_d = to_dev(np.concatenate([ud, us]))
    Gs.DeleteEdges(sym_s, sym_d)
    bfs.Decremental(d_s, d_d)
    sssp.Decremental(d_s, d_d)
    wcc.Decremental(d_s, d_d)
    pr.Decremental(d_s, d_d)
    tc.Decremental(sym_s, sym_d)
    check("del_")


def _traversal_rounds(V, s, d, w, rounds, batch, seed, hints="exact", tuning=None):
    G, O = make_pair(V, s, d, w, weighted=True, hints=hints)
    if tuning:
        G.set_tuning(**tuning)
    es = mk.EdgeSet(V, s, d)
    src = int(np.argmax(np.bincount(s, minlength=V)))
    bfs, sssp = mk.BFS(G, src, V), mk.SSSP(G, src, V)
    bfs.Static()
    sssp.Static()
    rng = np.random.default_rng(seed)

    def check():
        np.testing.assert_array_equal(bfs.Distances(), O.bfs(src))
        np.testing.assert_array_equal(sssp.Distances(), O.sssp(src))
        assert O.check_parents(src, bfs.packed(), weighted=False) == 0
        assert O.check_parents(src, sssp.packed(), weighted=True) == 0

    check()
    for r in range(rounds):
        ds, dd = es.sample_present(batch, seed=seed * 100 + 2 * r)
        # also delete some current shortest-path tree edges (subtree invalidation)
        packed = sssp.packed()
        par = (packed & 0xFFFFFFFF).astype(np.uint32)
        tree_v = np.nonzero((packed != np.uint64(2**64 - 1)) & (par != np.arange(V)))[0]
        pick = rng.choice(tree_v, size=min(batch // 2, len(tree_v)), replace=False)
        ts, td = par[pick], pick.astype(np.uint32)
        ds = np.concatenate([ds, ts]).astype(np.uint32)
        dd = np.concatenate([dd, td]).astype(np.uint32)
        tds, tdd = to_dev(ds), to_dev(dd)
        G.DeleteEdges(tds, tdd)
        assert G.sync() == 0
        O.delete(ds, dd)
        bfs.Decremental(tds, tdd)
        sssp.Decremental(tds, tdd)
        check()
        ins_s, ins_d = es.sample_absent(batch, seed=seed * 100 + 2 * r + 1)
        ins_w = rng.integers(1, 65, batch).astype(np.uint32)
        tis, tid, tiw = to_dev(ins_s), to_dev(ins_d), to_dev(ins_w)
        G.InsertEdges(tis, tid, vals=tiw)
        assert G.sync() == 0
        O.insert(ins_s, ins_d, ins_w)
        bfs.Incremental(tis, tid)
        sssp.Incremental(tis, tid, wgt=tiw)
        check()


def test_traversals_rmat_rounds():
    V = 1 << 13
    s, d, w = mk.gen_rmat(13, 80000, seed=21, w_lo=1, w_hi=64)
    _traversal_rounds(V, s, d, w, rounds=3, batch=2000, seed=5)


def test_traversals_rmat_hints_one():
    V = 1 << 12
    s, d, w = mk.gen_rmat(12, 40000, seed=22, w_lo=1, w_hi=1000)
    _traversal_rounds(V, s, d, w, rounds=2, batch=1000, seed=6, hints="ones")


def test_traversals_grid_high_diameter():
    side = 64
    s, d, w = mk.gen_grid(side, 80, seed=7, w_lo=1, w_hi=1000)
    _traversal_rounds(side * side, s, d, w, rounds=3, batch=600, seed=7)


def test_incremental_with_stale_batch_entries():
    """Incremental SSSP seeds from the stored edges, not from the batch: an
    entry for a live edge with a larger weight changes nothing, one with a
    smaller weight lowers the edge (upsert-min), self loops are ignored."""
    V = 6
    G, O = make_pair(V, np.array([0, 1, 2], np.uint32), np.array([1, 2, 3], np.uint32),
                     np.array([10, 10, 10], np.uint32), weighted=True)
    sssp = mk.SSSP(G, 0, V)
    sssp.Static()
    bs = np.array([0, 0, 4, 3, 1], np.uint32)
    bd = np.array([2, 1, 4, 5, 2], np.uint32)
    bw = np.array([3, 1, 1, 1, 50], np.uint32)  # (0,1) live with weight 10, (1,2) too
    tbs, tbd, tbw = to_dev(bs), to_dev(bd), to_dev(bw)
    G.InsertEdges(tbs, tbd, vals=tbw)
    assert G.sync() == 0
    O.insert(bs, bd, bw)
    sssp.Incremental(tbs, tbd, wgt=tbw)
    np.testing.assert_array_equal(sssp.Distances(), O.sssp(0))


def test_pagerank_static_and_dynamic():
    V = 1 << 13
    s, d, _ = mk.gen_rmat(13, 80000, seed=31)
    G, O = make_pair(V, s, d, reverse=True)
    Of = OracleGraph(V)
    Of.insert(s, d)
    pr = mk.PageRank(G, 0.85, 1e-6, V, out_degree=np.bincount(s, minlength=V), max_iter=1000)
    pr.Static()
    ref, _ = Of.pagerank(0.85, 1e-14)
    assert np.abs(pr.Values().astype(np.float64) - ref).sum() <= PR_L1_TOL
    es = mk.EdgeSet(V, s, d)
    for r in range(2):
        ds, dd = es.sample_present(3000, seed=40 + r)
        tds, tdd = to_dev(ds), to_dev(dd)
        G.DeleteEdges(tds, tdd)
        Of.delete(ds, dd)
        pr.Decremental(tds, tdd)
        ref, _ = Of.pagerank(0.85, 1e-14)
        assert np.abs(pr.Values().astype(np.float64) - ref).sum() <= PR_L1_TOL
        is_, id_ = es.sample_absent(3000, seed=50 + r)
        tis, tid = to_dev(is_), to_dev(id_)
        G.InsertEdges(tis, tid)
        Of.insert(is_, id_)
        pr.Incremental(tis, tid)
        ref, _ = Of.pagerank(0.85, 1e-14)
        assert np.abs(pr.Values().astype(np.float64) - ref).sum() <= PR_L1_TOL
    # out-degrees counted from the graph when none are given
    pr2 = mk.PageRank(G, 0.85, 1e-6, V, max_iter=1000)
    pr2.Static()
    assert np.abs(pr2.Values().astype(np.float64) - ref).sum() <= PR_L1_TOL


def _sym_batch(s, d):
    return (np.concatenate([s, d]).astype(np.uint32), np.concatenate([d, s]).astype(np.uint32))


@pytest.mark.parametrize("scale,edges", [(11, 30000), (13, 120000)])
def test_triangles_static_and_dynamic(scale, edges):
    V = 1 << scale
    s, d, _ = mk.gen_rmat(scale, edges, seed=61)
    ss, sd = symmetrise(s, d)
    G, O = make_pair(V, ss, sd)
    tc = mk.TC(G, V)
    tc.Static()
    assert tc.GetCount() == O.triangles()
    es = mk.EdgeSet(V, ss, sd)
    rng = np.random.default_rng(62)
    for r in range(3):
        # delete undirected edges (both directions)
        ds, dd = es.sample_present(1500, seed=70 + r)
        keep = ds < dd
        us, ud = ds[keep], dd[keep]
        bs, bd = _sym_batch(us, ud)
        tbs, tbd = to_dev(bs), to_dev(bd)
        G.DeleteEdges(tbs, tbd)
        O.delete(bs, bd)
        tc.Decremental(tbs, tbd)
        assert tc.GetCount() == O.triangles()
        # insert undirected edges, some closing triangles around hubs
        hs = rng.integers(0, 64, 800).astype(np.uint32)
        hd = rng.integers(0, V, 800).astype(np.uint32)
        bs, bd = _sym_batch(hs, hd)
        tbs, tbd = to_dev(bs), to_dev(bd)
        G.InsertEdges(tbs, tbd)
        O.insert(bs, bd)
        tc.Incremental(tbs, tbd)
        assert tc.GetCount() == O.triangles()


def test_wcc_static_and_dynamic():
    V = 1 << 12
    s, d, _ = mk.gen_rmat(12, 6000, seed=81)  # sparse: many components
    G, O = make_pair(V, s, d)
    wcc = mk.WCC(G)
    wcc.Static()
    np.testing.assert_array_equal(wcc.Labels(), O.wcc())
    es = mk.EdgeSet(V, s, d)
    for r in range(3):
        ds, dd = es.sample_present(1500, seed=90 + r)
        tds, tdd = to_dev(ds), to_dev(dd)
        G.DeleteEdges(tds, tdd)
        O.delete(ds, dd)
        wcc.Decremental(tds, tdd)
        np.testing.assert_array_equal(wcc.Labels(), O.wcc())
        is_, id_ = es.sample_absent(800, seed=95 + r)
        tis, tid = to_dev(is_), to_dev(id_)
        G.InsertEdges(tis, tid)
        O.insert(is_, id_)
        wcc.Incremental(tis, tid)
        np.testing.assert_array_equal(wcc.Labels(), O.wcc())


@pytest.mark.parametrize("with_rev,weighted", [(True, False), (True, True), (False, False)])
def test_wcc_decremental_over_the_spanning_forest(with_rev, weighted):
    """Decremental WCC repairs along its spanning forest: with a reverse
    graph it may rescan only the pieces a lost forest edge split off (path
    1), without one it rebuilds the affected components (path 2, or the
    static passes when they hold most vertices: path 3); a batch that
    removes no forest edge changes nothing (path 0).  Labels equal the
    oracle's after every batch."""
    V = 1 << 12
    s, d, w = mk.gen_rmat(12, 9000, seed=83, w_lo=1, w_hi=50)  # sparse: many components
    G = mk.DynamicGraph(V, degree_hints=degree_hints(s, V), weighted=weighted)
    G.InsertEdges(to_dev(s), to_dev(d), vals=to_dev(w) if weighted else None)
    O = OracleGraph(V)
    O.insert(s, d, w if weighted else None)
    Gr = None
    if with_rev:
        Gr = mk.DynamicGraph(V, degree_hints=degree_hints(d, V), reverse=True)
        Gr.InsertEdges(to_dev(s), to_dev(d))
    wcc = mk.WCC(G)
    if Gr is not None:
        wcc.set_reverse(Gr)
    wcc.Static()
    np.testing.assert_array_equal(wcc.Labels(), O.wcc())
    es = mk.EdgeSet(V, s, d)
    paths = []
    for r in range(6):
        ds, dd = es.sample_present(400 if r % 2 else 2500, seed=120 + r)
        tds, tdd = to_dev(ds), to_dev(dd)
        G.DeleteEdges(tds, tdd)
        if Gr is not None:
            Gr.DeleteEdges(tds, tdd)
        O.delete(ds, dd)
        wcc.Decremental(tds, tdd)
        np.testing.assert_array_equal(wcc.Labels(), O.wcc())
        dead, rescanned, path = wcc.decremental_stats()
        assert (path == 0) <= (dead == 0) and (path in (1, 2)) <= (dead > 0)
        paths.append(path)
        is_, id_ = es.sample_absent(700, seed=130 + r)
        tis, tid = to_dev(is_), to_dev(id_)
        G.InsertEdges(tis, tid)
        if Gr is not None:
            Gr.InsertEdges(tis, tid)
        O.insert(is_, id_)
        wcc.Incremental(tis, tid)
        np.testing.assert_array_equal(wcc.Labels(), O.wcc())
    # which path a batch takes depends on the forest the concurrent unions
    # happened to record; the labels above are checked on every path
    if not with_rev:
        assert 1 not in paths and (2 in paths or 3 in paths)


def _core_and_leaves(rng):
    """A core of 1,000 vertices (ring plus 8 random core edges each), 1,500
    leaves joined by leaf -> core edges, 1,500 leaves reached only by core ->
    leaf edges (out-degree 0: linked by no sample, only by their in-edges),
    50 separate pairs and 252 isolated vertices (4,352 in all); no
    duplicate edges."""
    core = np.arange(1000, dtype=np.uint32)
    s = [core, np.repeat(core, 8)]
    d = [np.roll(core, -1), rng.integers(0, 1000, 8000).astype(np.uint32)]
    out_leaves = np.arange(1000, 2500, dtype=np.uint32)
    in_leaves = np.arange(2500, 4000, dtype=np.uint32)
    s += [out_leaves, rng.integers(0, 1000, 1500).astype(np.uint32)]
    d += [rng.integers(0, 1000, 1500).astype(np.uint32), in_leaves]
    s.append(np.arange(4000, 4100, 2, dtype=np.uint32))
    d.append(np.arange(4001, 4100, 2, dtype=np.uint32))
    s, d = np.concatenate(s), np.concatenate(d)
    keep = s != d
    s, d = s[keep], d[keep]
    _, first = np.unique(s.astype(np.uint64) << np.uint64(32) | d, return_index=True)
    first.sort()
    return 4352, s[first], d[first]


def _rings(rng):
    """512 separate rings of 8 vertices: no sampled set holds more than a
    few samples."""
    V = 4096
    x = np.arange(V, dtype=np.uint32)
    return V, x, (x & ~np.uint32(7)) | ((x + 1) & np.uint32(7))


def _hubs_outside(rng):
    """A core of 6,000 vertices (ring plus 4 random core edges each) holds
    most samples; outside it a source hub with 700 out-edges to its own
    leaves and a sink hub with 700 in-edges from its own leaves: both hubs
    span many buckets, so their edges are listed as several scan items."""
    core = np.arange(6000, dtype=np.uint32)
    s = [core, np.repeat(core, 4), np.full(700, 6000, np.uint32), np.arange(6801, 7501, dtype=np.uint32)]
    d = [np.roll(core, -1), rng.integers(0, 6000, 24000).astype(np.uint32),
         np.arange(6001, 6701, dtype=np.uint32), np.full(700, 6800, np.uint32)]
    s, d = np.concatenate(s), np.concatenate(d)
    keep = s != d
    s, d = s[keep], d[keep]
    _, first = np.unique(s.astype(np.uint64) << np.uint64(32) | d, return_index=True)
    first.sort()
    return 8192, s[first], d[first]


@pytest.mark.parametrize("weighted", [False, True])
@pytest.mark.parametrize("shape", ["core_and_leaves", "rings", "hubs_outside"])
def test_wcc_static_with_reverse_graph(shape, weighted):
    """Static WCC with a reverse graph attached: when one sampled set holds
    most samples (core_and_leaves) only the vertices outside it have their
    out- and in-edges scanned, and leaves reached only by in-edges must be
    joined through the reverse graph; with no such set (rings) every
    out-edge is scanned once; hubs outside the set (hubs_outside) are split
    into several scan items.  Labels equal the oracle's, repeated calls
    included, and after a deletion batch that falls back to them."""
    rng = np.random.default_rng(71)
    V, s, d = {"core_and_leaves": _core_and_leaves, "rings": _rings,
               "hubs_outside": _hubs_outside}[shape](rng)
    w = (np.arange(len(s)) % 40 + 1).astype(np.uint32)
    G, O = make_pair(V, s, d, w=w if weighted else None, weighted=weighted)
    Gr = mk.DynamicGraph(V, degree_hints=degree_hints(d, V), reverse=True)
    Gr.InsertEdges(to_dev(s), to_dev(d))
    wcc = mk.WCC(G)
    wcc.set_reverse(Gr)
    for _ in range(3):
        wcc.Static()
        np.testing.assert_array_equal(wcc.Labels(), O.wcc())
    # the core's ring and random edges go: most of the graph is affected
    ds, dd = s[:9000], d[:9000]
    tds, tdd = to_dev(ds), to_dev(dd)
    G.DeleteEdges(tds, tdd)
    Gr.DeleteEdges(tds, tdd)
    O.delete(ds, dd)
    wcc.Decremental(tds, tdd)
    np.testing.assert_array_equal(wcc.Labels(), O.wcc())
    wcc.Static()
    np.testing.assert_array_equal(wcc.Labels(), O.wcc())


@pytest.mark.parametrize("weighted", [False, True])
def test_wcc_decremental_rescans_only_split_off_pieces(weighted):
    """A hub with 2,047 leaves (leaf -> hub) and 1,500 leaf -> leaf edges:
    deleting leaf -> hub edges cuts single leaves (or small groups) off the
    hub's piece; with the reverse graph attached only those pieces are
    rescanned (path 1), and leaves that still reach the hub through another
    leaf keep the hub's label."""
    V = 2048
    rng = np.random.default_rng(29)
    leaves = np.arange(1, V, dtype=np.uint32)
    ls = rng.integers(1, V, 1500).astype(np.uint32)
    ld = rng.integers(1, V, 1500).astype(np.uint32)
    keep = ls != ld
    s = np.concatenate([leaves, ls[keep]])
    d = np.concatenate([np.zeros(V - 1, np.uint32), ld[keep]])
    w = (np.arange(len(s)) % 50 + 1).astype(np.uint32)
    G, O = make_pair(V, s, d, w=w if weighted else None, weighted=weighted)
    Gr, _ = make_pair(V, s, d, reverse=True)
    wcc = mk.WCC(G)
    wcc.set_reverse(Gr)
    wcc.Static()
    np.testing.assert_array_equal(wcc.Labels(), O.wcc())
    for r in range(3):
        cut = rng.choice(leaves, 100, replace=False).astype(np.uint32)
        zero = np.zeros(len(cut), np.uint32)
        tds, tdd = to_dev(cut), to_dev(zero)
        G.DeleteEdges(tds, tdd)
        Gr.DeleteEdges(tds, tdd)
        O.delete(cut, zero)
        wcc.Decremental(tds, tdd)
        np.testing.assert_array_equal(wcc.Labels(), O.wcc())
        dead, rescanned, path = wcc.decremental_stats()
        assert dead > 0 and path == 1 and 0 < rescanned < V // 4
        G.InsertEdges(tds, tdd, vals=to_dev(np.full(len(cut), 7, np.uint32)) if weighted else None)
        Gr.InsertEdges(tds, tdd)
        O.insert(cut, zero, np.full(len(cut), 7, np.uint32) if weighted else None)
        wcc.Incremental(tds, tdd)
        np.testing.assert_array_equal(wcc.Labels(), O.wcc())


def test_wcc_forest_edge_with_a_surviving_reverse_edge_changes_nothing():
    """On a symmetric graph a batch that deletes one direction of each pair
    removes no connection: the forest keeps the reverse edges and the call
    takes path 0."""
    V = 1 << 11
    s0, d0, _ = mk.gen_rmat(11, 5000, seed=85)
    s, d = symmetrise(s0, d0)
    G, O = make_pair(V, s, d)
    wcc = mk.WCC(G)
    wcc.Static()
    want = O.wcc()
    keep = s < d
    for r in range(2):
        pick = np.random.default_rng(140 + r).choice(np.flatnonzero(keep), 1500, replace=False)
        ds, dd = (s[pick], d[pick]) if r == 0 else (d[pick], s[pick])
        tds, tdd = to_dev(ds), to_dev(dd)
        G.DeleteEdges(tds, tdd)
        O.delete(ds, dd)
        wcc.Decremental(tds, tdd)
        assert wcc.decremental_stats()[2] == 0
        np.testing.assert_array_equal(wcc.Labels(), want)
        np.testing.assert_array_equal(O.wcc(), want)
        tis, tid = to_dev(ds), to_dev(dd)
        G.InsertEdges(tis, tid)
        O.insert(ds, dd)
        wcc.Incremental(tis, tid)
        np.testing.assert_array_equal(wcc.Labels(), want)


def test_wcc_decremental_splits_paths_along_the_forest():
    """Directed paths (deep forest): deleting path edges splits components
    into pieces that must get their own min-id labels; with the reverse graph
    attached the pieces are rescanned or the components rebuilt."""
    V = 1 << 14
    rng = np.random.default_rng(19)
    perm = rng.permutation(V).astype(np.uint32)
    paths = perm.reshape(64, -1)
    s = paths[:, :-1].ravel()
    d = paths[:, 1:].ravel()
    G, O = make_pair(V, s, d)
    Gr, _ = make_pair(V, s, d, reverse=True)
    wcc = mk.WCC(G)
    wcc.set_reverse(Gr)
    wcc.Static()
    for r in range(3):
        pick = rng.choice(len(s), 40, replace=False)
        ds, dd = s[pick], d[pick]
        tds, tdd = to_dev(ds), to_dev(dd)
        G.DeleteEdges(tds, tdd)
        Gr.DeleteEdges(tds, tdd)
        O.delete(ds, dd)
        wcc.Decremental(tds, tdd)
        assert wcc.decremental_stats()[2] in (1, 2, 3)
        np.testing.assert_array_equal(wcc.Labels(), O.wcc())


def test_algorithms_with_a_foreign_batch_fall_back_to_recompute():
    """Dynamic calls whose batch is not the graph's last update recompute."""
    V = 1 << 10
    s, d, _ = mk.gen_rmat(10, 6000, seed=3)
    G, O = make_pair(V, s, d)
    wcc = mk.WCC(G)
    wcc.Static()
    es = mk.EdgeSet(V, s, d)
    ds, dd = es.sample_present(500, seed=4)
    G.DeleteEdges(to_dev(ds), to_dev(dd))
    O.delete(ds, dd)
    wcc.Decremental(to_dev(ds), to_dev(dd))  # fresh tensors: different pointers
    np.testing.assert_array_equal(wcc.Labels(), O.wcc())


def test_wcc_labels_are_roots_on_deep_trees():
    """Long random paths give deep union-find trees; every label must be the
    component minimum on every run (the compress pass walks to the root
    without path-halving stores, which could otherwise overwrite a finished
    label with a non-root ancestor)."""
    V = 1 << 20
    rng = np.random.default_rng(17)
    perm = rng.permutation(V).astype(np.uint32)
    # 16 paths of V/16 vertices each, vertex ids shuffled
    paths = perm.reshape(16, -1)
    s = paths[:, :-1].ravel()
    d = paths[:, 1:].ravel()
    G, _ = make_pair(V, s, d, hints="ones")
    want = np.empty(V, np.uint32)
    for row in paths:
        want[row] = row.min()
    wcc = mk.WCC(G)
    for _ in range(8):
        wcc.Static()
        np.testing.assert_array_equal(wcc.Labels(), want)


@pytest.mark.parametrize("delta", [1, 50, 700, 100000])
def test_sssp_near_far_static_matches_oracle(delta):
    """Static SSSP with the near-far split (sssp_delta) on a skewed graph and
    a high-diameter grid: same distances as the oracle, valid parents, and
    the dynamic calls that follow still agree."""
    for V, (s, d, w) in ((1 << 13, mk.gen_rmat(13, 90000, seed=23, w_lo=1, w_hi=1000)),
                         (64 * 64, mk.gen_grid(64, 100, seed=8, w_lo=1, w_hi=1000))):
        G, O = make_pair(V, s, d, w, weighted=True)
        G.set_tuning(sssp_delta=delta)
        src = int(np.argmax(np.bincount(s, minlength=V)))
        sssp = mk.SSSP(G, src, V)
        sssp.Static()
        np.testing.assert_array_equal(sssp.Distances(), O.sssp(src))
        assert O.check_parents(src, sssp.packed(), weighted=True) == 0
        es = mk.EdgeSet(V, s, d)
        ds, dd = es.sample_present(len(s) // 10, seed=delta % 97)
        tds, tdd = to_dev(ds), to_dev(dd)
        G.DeleteEdges(tds, tdd)
        O.delete(ds, dd)
        sssp.Decremental(tds, tdd)
        np.testing.assert_array_equal(sssp.Distances(), O.sssp(src))
        sssp.Static()  # near-far again on the changed graph
        np.testing.assert_array_equal(sssp.Distances(), O.sssp(src))
        assert O.check_parents(src, sssp.packed(), weighted=True) == 0


@pytest.mark.parametrize("tuning", [{"recompute_permille": 0},
                                    {"recompute_permille": 1},
                                    {"recompute_permille": 1, "sssp_delta": 300}])
def test_decremental_recompute_fallback(tuning):
    """Decremental BFS/SSSP either repair the invalidated subtrees or, past the
    recompute threshold, recompute from the source (with or without the
    near-far split): the answers are the oracle's either way."""
    side = 48
    s, d, w = mk.gen_grid(side, 60, seed=12, w_lo=1, w_hi=1000)
    _traversal_rounds(side * side, s, d, w, rounds=3, batch=500, seed=13, tuning=tuning)
    V = 1 << 12
    s, d, w = mk.gen_rmat(12, 40000, seed=14, w_lo=1, w_hi=1000)
    _traversal_rounds(V, s, d, w, rounds=2, batch=1500, seed=15, tuning=tuning)


@pytest.mark.parametrize("pull", [1, 50])
def test_bfs_pull_levels_match_oracle(pull):
    """Static BFS with a reverse graph attached pulls its large levels
    bottom-up: same levels as the oracle, valid parents, before and after an
    update applied to both graphs."""
    for V, (s, d, w) in ((1 << 13, mk.gen_rmat(13, 100000, seed=31, w_lo=1, w_hi=9)),
                         (64 * 64, mk.gen_grid(64, 100, seed=9, w_lo=1, w_hi=9))):
        G, O = make_pair(V, s, d, w, weighted=True)
        Gr, _ = make_pair(V, s, d, reverse=True)
        G.set_tuning(pull_permille=pull)
        src = int(np.argmax(np.bincount(s, minlength=V)))
        bfs = mk.BFS(G, src, V)
        bfs.set_reverse(Gr)
        bfs.Static()
        np.testing.assert_array_equal(bfs.Distances(), O.bfs(src))
        assert O.check_parents(src, bfs.packed(), weighted=False) == 0
        es = mk.EdgeSet(V, s, d)
        ds, dd = es.sample_present(len(s) // 5, seed=pull)
        for g in (G, Gr):
            g.DeleteEdges(to_dev(ds), to_dev(dd))
        O.delete(ds, dd)
        bfs.Static()
        np.testing.assert_array_equal(bfs.Distances(), O.bfs(src))
        assert O.check_parents(src, bfs.packed(), weighted=False) == 0
        with pytest.raises(mk.MeerkatError):
            mk.SSSP(G, src, V).set_reverse(Gr)  # SSSP needs a weighted reverse graph


def test_decremental_reseed_from_reverse_graph():
    """Decremental BFS/SSSP with a reverse graph attached re-seed invalidated
    vertices from their own in-edges (weighted reverse copy for SSSP): the
    oracle's answers after every delete and insert batch, including deletes
    of shortest-path-tree edges."""
    for V, (s, d, w) in ((1 << 12, mk.gen_rmat(12, 50000, seed=41, w_lo=1, w_hi=1000)),
                         (48 * 48, mk.gen_grid(48, 60, seed=42, w_lo=1, w_hi=1000))):
        G, O = make_pair(V, s, d, w, weighted=True)
        Gr, _ = make_pair(V, s, d, w, weighted=True, reverse=True)
        G.set_tuning(recompute_permille=0)  # always repair, never recompute
        src = int(np.argmax(np.bincount(s, minlength=V)))
        bfs, sssp = mk.BFS(G, src, V), mk.SSSP(G, src, V)
        bfs.set_reverse(Gr)
        sssp.set_reverse(Gr)
        bfs.Static()
        sssp.Static()
        es = mk.EdgeSet(V, s, d)
        rng = np.random.default_rng(43)
        for r in range(3):
            ds, dd = es.sample_present(len(s) // 20, seed=50 + r)
            par = (sssp.packed() & np.uint64(0xFFFFFFFF)).astype(np.int64)
            dist = sssp.Distances()
            tree = np.flatnonzero((dist != mk.MK_INF) & (par != np.arange(V)))
            pick = rng.choice(tree, size=min(len(tree), 200), replace=False)
            # and BFS tree edges: the BFS repair re-parents or invalidates their heads
            bpar = (bfs.packed() & np.uint64(0xFFFFFFFF)).astype(np.int64)
            btree = np.flatnonzero((bfs.Distances() != mk.MK_INF) & (bpar != np.arange(V)))
            bpick = rng.choice(btree, size=min(len(btree), 200), replace=False)
            ds = np.concatenate([ds, par[pick], bpar[bpick]]).astype(np.uint32)
            dd = np.concatenate([dd, pick, bpick]).astype(np.uint32)
            for g in (G, Gr):
                g.DeleteEdges(to_dev(ds), to_dev(dd))
            O.delete(ds, dd)
            bfs.Decremental(to_dev(ds), to_dev(dd))
            sssp.Decremental(to_dev(ds), to_dev(dd))
            np.testing.assert_array_equal(bfs.Distances(), O.bfs(src))
            np.testing.assert_array_equal(sssp.Distances(), O.sssp(src))
            assert O.check_parents(src, bfs.packed(), weighted=False) == 0
            assert O.check_parents(src, sssp.packed(), weighted=True) == 0
            is_, id_ = es.sample_absent(len(s) // 20, seed=60 + r)
            iw = rng.integers(1, 1001, len(is_)).astype(np.uint32)
            for g in (G, Gr):
                g.InsertEdges(to_dev(is_), to_dev(id_), vals=to_dev(iw))
            O.insert(is_, id_, iw)
            bfs.Incremental(to_dev(is_), to_dev(id_))
            sssp.Incremental(to_dev(is_), to_dev(id_), wgt=to_dev(iw))
            np.testing.assert_array_equal(bfs.Distances(), O.bfs(src))
            np.testing.assert_array_equal(sssp.Distances(), O.sssp(src))
        with pytest.raises(mk.MeerkatError):
            Gu, _ = make_pair(V, s, d, reverse=True)  # unweighted reverse
            mk.SSSP(G, src, V).set_reverse(Gu)


def test_bfs_repair_invalidates_only_vertices_whose_level_rises():
    """With the reverse graph, decremental BFS invalidates only the vertices
    whose level really rises (the others take a parent one level up), so it
    invalidates no more than the whole-subtree walk without the reverse
    graph, and exactly the oracle's count of vertices whose level changed or
    that became unreachable; both give the oracle's levels."""
    V = 1 << 13
    s, d, w = mk.gen_rmat(13, 120000, seed=61, w_lo=1, w_hi=9)
    G, O = make_pair(V, s, d, w, weighted=True)
    Gr, _ = make_pair(V, s, d, w, weighted=True, reverse=True)
    G.set_tuning(recompute_permille=0)
    src = int(np.argmax(np.bincount(s, minlength=V)))
    plain, rep = mk.BFS(G, src, V), mk.BFS(G, src, V)
    rep.set_reverse(Gr)
    plain.Static()
    rep.Static()
    rng = np.random.default_rng(62)
    for r in range(3):
        before = O.bfs(src)
        par = (rep.packed() & np.uint64(0xFFFFFFFF)).astype(np.int64)
        tree = np.flatnonzero((before != mk.MK_INF) & (par != np.arange(V)))
        pick = rng.choice(tree, size=min(len(tree), 400), replace=False)
        ds, dd = par[pick].astype(np.uint32), pick.astype(np.uint32)
        for g in (G, Gr):
            g.DeleteEdges(to_dev(ds), to_dev(dd))
        O.delete(ds, dd)
        plain.Decremental(to_dev(ds), to_dev(dd))
        rep.Decremental(to_dev(ds), to_dev(dd))
        after = O.bfs(src)
        np.testing.assert_array_equal(rep.Distances(), after)
        np.testing.assert_array_equal(plain.Distances(), after)
        assert O.check_parents(src, rep.packed(), weighted=False) == 0
        inv_rep, rec_rep = rep.decremental_stats()
        inv_plain, _ = plain.decremental_stats()
        assert not rec_rep
        assert inv_rep == int((after != before).sum())
        assert inv_rep <= inv_plain
    for o in (plain, rep, G, Gr):
        o.close()
