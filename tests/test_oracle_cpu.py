"""CPU: the multithreaded CPU baseline (oracle/mk_cpu.c) against the oracle's
sequential definitions, on seeded R-MAT graphs through insert and delete
batches: BFS levels and SSSP distances bit-exact after static, incremental
and decremental calls (parents checked for validity), PageRank within 1e-12
L1 of the sequential FP64 iteration, triangle counts and WCC labels exact."""
import numpy as np
import pytest

import meerkat_b200 as mk
from oracle import (CpuTraversal, OracleEdgeSet, OracleGraph, cpu_pagerank, cpu_triangles,
                    cpu_wcc, cpu_wcc_incremental)


def _graph(scale, edges, seed, threads):
    V = 1 << scale
    s, d, w = mk.gen_rmat(scale, edges, seed=seed, w_lo=1, w_hi=64)
    O = OracleGraph(V, threads=threads)
    O.insert(s, d, w)
    return V, s, d, O


@pytest.mark.parametrize("scale,edges,threads,tree_bias", [(8, 1500, 1, False), (11, 20000, 4, True),
                                                           (13, 120000, 8, False)])
def test_traversals_through_batches(scale, edges, threads, tree_bias):
    V, s, d, O = _graph(scale, edges, 17 + scale, threads)
    es = OracleEdgeSet(V, s, d)
    rng = np.random.default_rng(scale)
    src = int(np.argmax(O.degrees()))
    bfs, sssp = CpuTraversal(O, src, False), CpuTraversal(O, src, True)
    bfs.static()
    sssp.static()
    np.testing.assert_array_equal(bfs.distances(), O.bfs(src))
    np.testing.assert_array_equal(sssp.distances(), O.sssp(src))
    n = max(edges // 20, 10)
    for r in range(4):
        if tree_bias:  # delete tree edges of the SSSP: whole subtrees go invalid
            p = sssp.packed()
            kids = np.flatnonzero((p != np.uint64(2**64 - 1)) & (np.arange(V) != src))
            pick = rng.choice(kids, size=min(n, len(kids)), replace=False)
            ds = (p[pick] & np.uint64(0xFFFFFFFF)).astype(np.uint32)
            dd = pick.astype(np.uint32)
        else:
            ds, dd = es.sample_present(n, seed=1000 + r)
        O.delete(ds, dd)
        bfs.decremental(ds, dd)
        sssp.decremental(ds, dd)
        np.testing.assert_array_equal(bfs.distances(), O.bfs(src))
        np.testing.assert_array_equal(sssp.distances(), O.sssp(src))
        assert O.check_parents(src, bfs.packed(), False) == 0
        assert O.check_parents(src, sssp.packed(), True) == 0
        is_, id_ = es.sample_absent(n, seed=2000 + r)
        iw = rng.integers(1, 65, n).astype(np.uint32)
        O.insert(is_, id_, iw)
        bfs.incremental(is_, id_)
        sssp.incremental(is_, id_)
        np.testing.assert_array_equal(bfs.distances(), O.bfs(src))
        np.testing.assert_array_equal(sssp.distances(), O.sssp(src))
        assert O.check_parents(src, sssp.packed(), True) == 0


def test_decremental_recompute_rule():
    V, s, d, O = _graph(10, 6000, 5, 4)
    src = int(np.argmax(O.degrees()))
    t = CpuTraversal(O, src, False)
    t.static()
    # delete every out-edge of the source: the whole tree goes invalid
    rp, col, _ = O.csr()
    ds = np.full(int(rp[src + 1] - rp[src]), src, dtype=np.uint32)
    dd = col[rp[src]:rp[src + 1]].astype(np.uint32)
    O.delete(ds, dd)
    t.decremental(ds, dd)
    st = t.stats()
    assert st["recomputed"] and st["invalidated"] * 10 > V
    np.testing.assert_array_equal(t.distances(), O.bfs(src))


@pytest.mark.parametrize("threads", [1, 8])
def test_pagerank_triangles_wcc(threads):
    V, s, d, O = _graph(12, 40000, 9, threads)
    want, _ = O.pagerank(0.85, 1e-14)
    got, it = cpu_pagerank(O, 0.85, 1e-14)
    assert np.abs(got - want).sum() <= 1e-12
    warm, it2 = cpu_pagerank(O, 0.85, 1e-14, warm=got)
    assert it2 < it and np.abs(warm - want).sum() <= 1e-12
    assert cpu_triangles(O) == O.triangles()
    np.testing.assert_array_equal(cpu_wcc(O), O.wcc())
    # incremental WCC: unions of a batch that joins components
    V2 = 4096
    O2 = OracleGraph(V2, threads=threads)
    rng = np.random.default_rng(3)
    a = rng.integers(0, V2, 1500).astype(np.uint32)
    b = rng.integers(0, V2, 1500).astype(np.uint32)
    O2.insert(a, b)
    lab = cpu_wcc(O2)
    x = rng.integers(0, V2, 800).astype(np.uint32)
    y = rng.integers(0, V2, 800).astype(np.uint32)
    O2.insert(x, y)
    np.testing.assert_array_equal(cpu_wcc_incremental(lab, x, y), O2.wcc())
