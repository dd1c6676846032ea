"""Host logic of the batched many-graph workload (no GPU): the seeded member
spec and the source picker."""
import numpy as np

from meerkat_b200 import batched as B


def test_spec_shapes_ranges_and_determinism():
    a = B.make_spec(4096)
    b = B.make_spec(4096)
    for x, y in zip((a.num_vertices, a.num_edges, a.deletes, a.inserts, a.query),
                    (b.num_vertices, b.num_edges, b.deletes, b.inserts, b.query)):
        assert np.array_equal(x, y)
    assert a.num_graphs == 4096
    assert a.num_vertices.min() >= 1024 and a.num_vertices.max() < 65536
    deg = a.num_edges / a.num_vertices
    assert deg.min() >= 4.0 - 1e-3 and deg.max() <= 32.0 + 1e-3
    # power law with exponent 2 on [4, 32]: the median degree sits near 6.4
    assert 5.5 < np.median(deg) < 7.5
    upd = a.deletes + a.inserts
    frac = upd / a.num_edges
    assert frac.min() >= 0.01 - 2 / a.num_edges.min() and frac.max() <= 0.10 + 1e-6
    assert (np.abs(a.deletes - a.inserts) <= 1).all()
    assert set(np.unique(a.query)) <= {B.QUERY_BFS, B.QUERY_WCC}
    assert 0.45 < (a.query == B.QUERY_WCC).mean() < 0.55
    c = B.make_spec(4096, seed=B.DEFAULT_SEED + 1)
    assert not np.array_equal(a.num_vertices, c.num_vertices)


def test_sources_have_out_edges():
    sizes = np.array([5, 8, 3, 6])
    off = B._offsets(sizes)
    deg = np.zeros(int(off[-1]), np.uint32)
    deg[off[0] + 2] = 1           # member 0: only vertex 2 has out-edges
    deg[off[1]:off[2]] = 3        # member 1: every vertex
    # member 2: none -> its first vertex
    deg[off[3] + 5] = 7           # member 3: only vertex 5
    src = B.pick_sources(deg, off, [0, 1, 2, 3], seed=11)
    assert src[0] == 2 and src[2] == 0 and src[3] == 5
    assert 0 <= src[1] < 8
    assert np.array_equal(src, B.pick_sources(deg, off, [0, 1, 2, 3], seed=11))


def test_pool_sizing_covers_the_load():
    # heads one per vertex at least, plus room for growth
    for v, e in ((1024, 4096), (65536, 2_000_000), (3, 0)):
        assert B.pool_slabs_for(v, e) >= v
