"""GPU parity of the slab graph against the oracle.  Mirrors the reference's
structural tests (test/GraphTest.cu): DegreeCountTest (:647-681),
ElementTest (:716-871), PartialDelete (:873-956), FullDelete (:958-1007) and
the weighted WGraphTest (:1009-1215), with seeded inputs instead of the
missing `simple` fixture."""
import numpy as np
import pytest

import meerkat_b200 as mk
from helpers import assert_same_graph, degree_hints, make_pair, to_dev
from oracle import OracleGraph

pytestmark = pytest.mark.gpu

V12 = 1 << 12


@pytest.fixture(scope="module")
def rmat12():
    return mk.gen_rmat(12, 60000, seed=11, w_lo=1, w_hi=64)


VARIANTS = [0, 1, 2]  # update kernels: warp-staged TMA, lane per edge, warp-cooperative


@pytest.mark.parametrize("variant", VARIANTS)
@pytest.mark.parametrize("weighted", [False, True])
@pytest.mark.parametrize("hints", ["exact", "ones"])
def test_degree_and_element(rmat12, weighted, hints, variant):
    s, d, w = rmat12
    G, O = make_pair(V12, s, d, w, weighted=weighted, hints=hints, variant=variant)
    assert G.last_applied() == len(s)
    assert_same_graph(G, O, weighted)
    info = G.info()
    assert info["num_edges"] == len(s)
    assert info["keys_per_slab"] == (15 if weighted else 31)


@pytest.mark.parametrize("variant", VARIANTS)
@pytest.mark.parametrize("weighted", [False, True])
def test_partial_delete(rmat12, weighted, variant):
    s, d, w = rmat12
    G, O = make_pair(V12, s, d, w, weighted=weighted, variant=variant)
    rng = np.random.default_rng(45)
    sel = rng.random(len(s)) < 0.45
    ds, dd = to_dev(s[sel]), to_dev(d[sel])
    G.DeleteEdges(ds, dd)
    assert G.sync() == 0
    assert G.last_applied() == int(sel.sum())
    O.delete(s[sel], d[sel])
    assert_same_graph(G, O, weighted)


@pytest.mark.parametrize("variant", VARIANTS)
def test_full_delete_leaves_tombstones(rmat12, variant):
    s, d, _ = rmat12
    G, O = make_pair(V12, s, d, variant=variant)
    deg0 = G.degrees().copy()
    G.DeleteEdges(to_dev(s), to_dev(d))
    assert G.sync() == 0
    assert (G.degrees() == 0).all()
    np.testing.assert_array_equal(G.tombstones(), deg0)


@pytest.mark.parametrize("variant", VARIANTS)
def test_batch_semantics_weighted(variant):
    V = 16
    G, O = make_pair(V, np.array([], np.uint32), np.array([], np.uint32), weighted=True,
                     variant=variant)
    src = np.array([1, 2, 2, 3, 1, 4, 4, 4], np.uint32)
    dst = np.array([1, 3, 3, 4, 2, 5, 5, 6], np.uint32)
    w = np.array([5, 7, 8, 9, 2, 11, 12, 13], np.uint32)
    ts, td, tw = to_dev(src), to_dev(dst), to_dev(w)
    G.InsertEdges(ts, td, vals=tw)
    assert G.sync() == 0
    n, ap = O.insert(src, dst, w)
    assert G.last_applied() == n == 5
    assert_same_graph(G, O, weighted=True)
    # re-insert of live edges with larger weights: nothing changes
    G.InsertEdges(to_dev([2, 4]), to_dev([3, 5]), vals=to_dev([100, 100]))
    assert G.sync() == 0 and G.last_applied() == 0
    assert_same_graph(G, O, weighted=True)
    # with smaller weights (several copies in one batch): the minimum is kept
    G.InsertEdges(to_dev([4, 2, 4, 4]), to_dev([5, 3, 5, 6]), vals=to_dev([9, 3, 4, 20]))
    assert G.sync() == 0 and G.last_applied() == 0
    O.insert([4, 2, 4, 4], [5, 3, 5, 6], [9, 3, 4, 20])
    assert_same_graph(G, O, weighted=True)
    # delete absent, self loop, duplicate
    dsrc = np.array([2, 2, 7, 1], np.uint32)
    ddst = np.array([3, 3, 8, 1], np.uint32)
    G.DeleteEdges(to_dev(dsrc), to_dev(ddst))
    assert G.sync() == 0
    n, _ = O.delete(dsrc, ddst)
    assert G.last_applied() == n == 1
    assert_same_graph(G, O, weighted=True)
    # insert after delete reuses nothing but is live again
    G.InsertEdges(to_dev([2]), to_dev([3]), vals=to_dev([42]))
    O.insert([2], [3], [42])
    assert G.sync() == 0
    assert_same_graph(G, O, weighted=True)


def test_search_edges(rmat12):
    import torch
    s, d, w = rmat12
    G, O = make_pair(V12, s, d, w, weighted=True)
    rng = np.random.default_rng(3)
    qs = np.concatenate([s[:500], rng.integers(0, V12, 500).astype(np.uint32)])
    qd = np.concatenate([d[:500], rng.integers(0, V12, 500).astype(np.uint32)])
    found = torch.zeros(len(qs), dtype=torch.uint8, device="cuda:0")
    wout = torch.zeros(len(qs), dtype=torch.int32, device="cuda:0")
    G.SearchEdges(to_dev(qs), to_dev(qd), found, wout)
    f = found.cpu().numpy()
    wo = wout.cpu().numpy().view(np.uint32)
    for i in range(len(qs)):
        import ctypes
        ow = ctypes.c_uint32(0)
        from oracle.oracle import _L
        has = _L().og_has_edge(O._h, int(qs[i]), int(qd[i]), ctypes.byref(ow))
        assert bool(f[i]) == bool(has)
        if has:
            assert wo[i] == ow.value


def test_reverse_graph_is_transpose(rmat12):
    s, d, _ = rmat12
    G, O = make_pair(V12, s, d, reverse=True)
    assert_same_graph(G, O)


def test_out_of_range_ids_report_invalid():
    G, O = make_pair(8, np.array([], np.uint32), np.array([], np.uint32))
    G.InsertEdges(to_dev([1, 9, 2]), to_dev([2, 1, 3]))
    with pytest.raises(mk.MeerkatError) as e:
        G.sync()
    assert e.value.status == 1
    O.insert([1, 2], [2, 3])
    assert_same_graph(G, O)


@pytest.mark.parametrize("variant", VARIANTS)
def test_pool_exhaustion_reports_oom_and_stays_consistent(variant):
    V = 64
    rng = np.random.default_rng(5)
    s = rng.integers(0, V, 4000).astype(np.uint32)
    d = rng.integers(0, V, 4000).astype(np.uint32)
    G = mk.DynamicGraph(V, degree_hints=None, pool_slabs=16)
    G.set_tuning(update_kernel=variant)
    G.InsertEdges(to_dev(s), to_dev(d))
    with pytest.raises(mk.MeerkatError) as e:
        G.sync()
    assert e.value.status == 2
    # whatever was stored is a consistent set: export == degrees, no duplicates
    rp, col, _ = G.export_csr()
    deg = G.degrees()
    assert (np.diff(rp) == deg).all()
    for u in range(V):
        row = col[rp[u]:rp[u + 1]]
        assert len(np.unique(row)) == len(row)
        assert u not in row


@pytest.mark.parametrize("variant", VARIANTS)
def test_small_config_insert_delete(variant):
    """Small config: R-MAT s16, 1,048,576 edges, +10k absent, -10k present."""
    V = 1 << 16
    s, d, w = mk.gen_rmat(16, 1 << 20, seed=0x4D45524B, w_lo=1, w_hi=64)
    G, O = make_pair(V, s, d, w, weighted=True, hints="ones", variant=variant)
    es = mk.EdgeSet(V, s, d)
    ins_s, ins_d = es.sample_absent(10000, seed=1)
    ins_w = (np.arange(10000, dtype=np.uint32) % 64) + 1
    G.InsertEdges(to_dev(ins_s), to_dev(ins_d), vals=to_dev(ins_w))
    assert G.sync() == 0 and G.last_applied() == 10000
    O.insert(ins_s, ins_d, ins_w)
    del_s, del_d = es.sample_present(10000, seed=2)
    G.DeleteEdges(to_dev(del_s), to_dev(del_d))
    assert G.sync() == 0 and G.last_applied() == 10000
    O.delete(del_s, del_d)
    assert_same_graph(G, O, weighted=True)


def test_tuning_round_trip_and_validation():
    G, _ = make_pair(64, np.array([1], np.uint32), np.array([2], np.uint32))
    assert G.get_tuning() == {"update_kernel": 0, "update_blocks_per_sm": 0, "frontier_chunk": 0,
                              "sssp_delta": 0, "recompute_permille": 100,
                              "pull_permille": 0, "wait_limit_us": 0}
    G.set_tuning(update_kernel=1, update_blocks_per_sm=3)
    G.set_tuning(frontier_chunk=16)  # keeps the other knobs
    assert G.get_tuning() == {"update_kernel": 1, "update_blocks_per_sm": 3, "frontier_chunk": 16,
                              "sssp_delta": 0, "recompute_permille": 100,
                              "pull_permille": 0, "wait_limit_us": 0}
    with pytest.raises(mk.MeerkatError):
        G.set_tuning(update_kernel=7)
    with pytest.raises(mk.MeerkatError):
        G.set_tuning(frontier_chunk=4096)
