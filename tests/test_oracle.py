"""CPU tests: the oracle against the golden vectors (scipy / networkx) and
hand-checked known answers for the reference's batch semantics."""
from pathlib import Path

import numpy as np
import pytest

from oracle import OracleGraph

GOLD = Path(__file__).resolve().parent / "golden" / "rmat10.npz"
INF = 0xFFFFFFFF


@pytest.fixture(scope="module")
def gold():
    return dict(np.load(GOLD))


def _check_state(g: OracleGraph, gold, prefix):
    np.testing.assert_array_equal(g.bfs(0), gold[prefix + "bfs"])
    np.testing.assert_array_equal(g.sssp(0), gold[prefix + "sssp"])
    np.testing.assert_array_equal(g.wcc(), gold[prefix + "wcc"])
    pr, _ = g.pagerank(d=0.85, tol=1e-14)
    assert np.abs(pr - gold[prefix + "pr"]).sum() < 1e-9
    assert g.triangles() == int(gold[prefix + "tc"])


@pytest.mark.parametrize("threads", [1, 3])
def test_oracle_matches_golden(gold, threads):
    g = OracleGraph(1024, threads=threads)
    n, applied = g.insert(gold["src"], gold["dst"], gold["w"])
    assert n == len(gold["src"]) and applied.all()
    _check_state(g, gold, "base_")
    n, applied = g.insert(gold["ins_src"], gold["ins_dst"], gold["ins_w"])
    assert n == len(gold["ins_src"])
    _check_state(g, gold, "ins_")
    n, applied = g.delete(gold["del_src"], gold["del_dst"])
    assert n == len(gold["del_src"])
    _check_state(g, gold, "del_")


def test_insert_semantics_known_answers():
    g = OracleGraph(8)
    # self loop skipped, duplicate in batch: one edge with the smaller weight,
    # out-of-range skipped
    n, ap = g.insert([1, 2, 2, 3, 9, 1], [1, 3, 3, 4, 0, 2], [5, 7, 8, 9, 1, 2])
    assert n == 3
    assert ap.tolist() == [0, 1, 0, 1, 0, 1]
    rp, col, w = g.csr(weights=True)
    assert col.tolist() == [2, 3, 4] and w.tolist() == [2, 7, 9]
    # re-insert of a live edge adds nothing; a larger weight changes nothing
    n, ap = g.insert([2], [3], [100])
    assert n == 0 and ap.tolist() == [0]
    _, _, w = g.csr(weights=True)
    assert w.tolist() == [2, 7, 9]
    # ... and a smaller one lowers it (upsert-min)
    n, ap = g.insert([3, 3], [4, 4], [6, 5])
    assert n == 0 and ap.tolist() == [0, 0]
    _, _, w = g.csr(weights=True)
    assert w.tolist() == [2, 7, 5]
    assert g.degrees().tolist() == [0, 1, 1, 1, 0, 0, 0, 0]


def test_delete_semantics_known_answers():
    g = OracleGraph(6)
    g.insert([0, 0, 1, 2], [1, 2, 2, 3])
    n, ap = g.delete([0, 0, 5, 2, 2], [1, 1, 4, 2, 3])
    assert n == 2 and ap.tolist() == [1, 0, 0, 0, 1]
    assert g.num_edges() == 2
    assert g.degrees().tolist() == [1, 1, 0, 0, 0, 0]
    # delete then re-insert
    n, _ = g.insert([0], [1], [4])
    assert n == 1 and g.num_edges() == 3


def test_traversal_known_answers():
    # 0 -> 1 (w 5), 0 -> 2 (w 1), 2 -> 1 (w 1), 1 -> 3 (w 2), 4 isolated
    g = OracleGraph(5)
    g.insert([0, 0, 2, 1], [1, 2, 1, 3], [5, 1, 1, 2])
    assert g.bfs(0).tolist() == [0, 1, 1, 2, INF]
    assert g.sssp(0).tolist() == [0, 2, 1, 4, INF]
    packed = np.array([(0 << 32) | 0, (2 << 32) | 2, (1 << 32) | 0, (4 << 32) | 1, 2**64 - 1],
                      dtype=np.uint64)
    assert g.check_parents(0, packed, weighted=True) == 0
    packed[1] = (2 << 32) | 0  # wrong parent (edge 0->1 weighs 5)
    assert g.check_parents(0, packed, weighted=True) == 1
    assert g.wcc().tolist() == [0, 0, 0, 0, 4]


def test_triangles_symmetrised():
    g = OracleGraph(5)
    # one directed triangle 0->1->2->0 plus a chord making a second: {0,2,3}
    g.insert([0, 1, 2, 2, 3], [1, 2, 0, 3, 0])
    assert g.triangles() == 2


def test_pagerank_dangling_and_sum():
    g = OracleGraph(4)
    g.insert([0, 1, 2], [1, 2, 0])  # vertex 3 dangling and isolated
    pr, it = g.pagerank(d=0.85, tol=1e-15)
    assert abs(pr.sum() - 1.0) < 1e-12
    assert pr[0] == pytest.approx(pr[1]) == pytest.approx(pr[2])
    assert pr[3] < pr[0]
