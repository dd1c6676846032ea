"""CPU: the oracle's host generators (oracle/mk_gen.c), which the benchmark's
reference arm uses so that it loads no product code, draw exactly the edges
and update batches of the product's generators (meerkat_b200/csrc/gen.cpp)."""
import numpy as np
import pytest

import meerkat_b200 as mk
from oracle import OracleEdgeSet, gen_rmat


@pytest.mark.parametrize("scale,edges,seed", [(4, 40, 1), (10, 8192, 7), (14, 262144, 0x4D45524B + 1)])
def test_rmat_same_edges(scale, edges, seed):
    s, d, w = mk.gen_rmat(scale, edges, seed=seed, w_lo=1, w_hi=1000)
    os_, od, ow = gen_rmat(scale, edges, seed=seed, w_lo=1, w_hi=1000)
    np.testing.assert_array_equal(s, os_)
    np.testing.assert_array_equal(d, od)
    np.testing.assert_array_equal(w, ow)


def test_rmat_rejects_too_dense():
    with pytest.raises(ValueError):
        gen_rmat(3, 40, seed=1)


def test_edgeset_same_batches():
    V = 1 << 12
    s, d, _ = mk.gen_rmat(12, 40000, seed=3)
    a, b = mk.EdgeSet(V, s, d), OracleEdgeSet(V, s, d)
    assert len(a) == len(b) == 40000
    for k in range(6):
        for name in ("sample_present", "sample_absent"):
            x = getattr(a, name)(5000, seed=100 + k)
            y = getattr(b, name)(5000, seed=100 + k)
            np.testing.assert_array_equal(x[0], y[0])
            np.testing.assert_array_equal(x[1], y[1])
        assert len(a) == len(b)
    with pytest.raises(ValueError):
        b.sample_present(len(b) + 1, seed=1)


def test_edgeset_skips_invalid_and_duplicates():
    V = 16
    s = np.array([1, 1, 2, 3, 3, 20], dtype=np.uint32)
    d = np.array([2, 2, 2, 4, 5, 1], dtype=np.uint32)
    a, b = mk.EdgeSet(V, s, d), OracleEdgeSet(V, s, d)
    assert len(a) == len(b) == 3
    np.testing.assert_array_equal(a.sample_present(3, seed=5)[0], b.sample_present(3, seed=5)[0])
