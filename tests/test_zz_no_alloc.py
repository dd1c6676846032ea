"""mk_graph_export_csr_noalloc against mk_graph_export_csr, through the C ABI.

The no-allocation export keeps its scratch in a fixed device array inside the
library.  Its output must equal the plain export's bit for bit (integer data:
the tolerance is zero) on consecutive calls that share that array, and a call
after the first must not change the device's free memory."""
import numpy as np
import pytest

import meerkat_b200 as mk
from meerkat_b200._lib import MK_ERR_INVALID, lib

from helpers import degree_hints, to_dev

pytestmark = pytest.mark.gpu

MAX_BUCKETS = 1 << 18


def buffers(G):
    import torch
    E = G.info()["num_edges"]
    rp = torch.full((G.num_vertices + 1,), -1, dtype=torch.int64, device="cuda:0")
    col = torch.full((max(E, 1),), -1, dtype=torch.int32, device="cuda:0")
    w = torch.full((max(E, 1),), -1, dtype=torch.int32, device="cuda:0") if G.weighted else None
    return E, rp, col, w


def call(G, fn_name, rp, col, w):
    st = getattr(lib(), fn_name)(G.handle, rp.data_ptr(), col.data_ptr(),
                                 w.data_ptr() if w is not None else None, None)
    assert st == 0, lib().mk_last_error_string().decode()


def export(G, fn_name):
    import torch
    E, rp, col, w = buffers(G)
    call(G, fn_name, rp, col, w)
    torch.cuda.synchronize()
    return (rp.cpu().numpy(), col.cpu().numpy()[:E],
            w.cpu().numpy()[:E] if w is not None else None)


def assert_same(a, b):
    for x, y in zip(a, b):
        if x is None:
            assert y is None
        else:
            np.testing.assert_array_equal(x, y)


@pytest.mark.parametrize("weighted", [True, False])
def test_noalloc_export_matches_plain_export_on_consecutive_calls(weighted):
    import torch
    V = 1 << 14
    s, d, w = mk.gen_rmat(14, 150000, seed=77, w_lo=1, w_hi=500)
    G = mk.DynamicGraph(V, degree_hints=degree_hints(s, V), weighted=weighted)
    G.InsertEdges(to_dev(s), to_dev(d), vals=to_dev(w) if weighted else None)
    assert G.sync() == 0
    assert G.info()["num_buckets"] <= MAX_BUCKETS

    first = export(G, "mk_graph_export_csr_noalloc")  # sets up the scratch
    second = export(G, "mk_graph_export_csr_noalloc")
    plain = export(G, "mk_graph_export_csr")
    assert_same(first, plain)
    assert_same(second, plain)
    assert first[0][-1] == len(s)

    # change the graph, then the next two calls again share the scratch
    es = mk.EdgeSet(V, s, d)
    ds, dd = es.sample_present(20000, seed=5)
    G.DeleteEdges(to_dev(ds), to_dev(dd))
    is_, id_ = es.sample_absent(7000, seed=6)
    G.InsertEdges(to_dev(is_), to_dev(id_), vals=to_dev(np.full(7000, 3, np.uint32)))
    assert G.sync() == 0
    third = export(G, "mk_graph_export_csr_noalloc")
    fourth = export(G, "mk_graph_export_csr_noalloc")
    plain = export(G, "mk_graph_export_csr")
    assert_same(third, plain)
    assert_same(fourth, plain)
    assert third[0][-1] == len(s) - 20000 + 7000

    # no allocation: with the output buffers in place, two more calls leave
    # the device's free memory and the graph's own byte count unchanged
    E, rp, col, wb = buffers(G)
    bytes_before = G.info()["device_bytes"]
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    call(G, "mk_graph_export_csr_noalloc", rp, col, wb)
    call(G, "mk_graph_export_csr_noalloc", rp, col, wb)
    torch.cuda.synchronize()
    free_after = torch.cuda.mem_get_info()[0]
    assert free_after == free_before
    assert G.info()["device_bytes"] == bytes_before
    np.testing.assert_array_equal(rp.cpu().numpy(), plain[0])
    np.testing.assert_array_equal(col.cpu().numpy()[:E], plain[1])
    G.close()


def test_noalloc_export_at_its_bucket_limit():
    """A graph of exactly 262,144 buckets: the last tile of the scan and the
    final row offset sit at the end of the fixed scratch."""
    V = MAX_BUCKETS  # no hints: one bucket per vertex
    rng = np.random.default_rng(11)
    s = rng.integers(0, V, 5000).astype(np.uint32)
    d = rng.integers(0, V, 5000).astype(np.uint32)
    s[:3] = V - 1  # rows at the very end of the range
    d[:3] = np.array([0, 1, 2], np.uint32)
    G = mk.DynamicGraph(V, weighted=True)
    G.InsertEdges(to_dev(s), to_dev(d), vals=to_dev(np.arange(5000, dtype=np.uint32) % 97 + 1))
    assert G.sync() == 0
    assert G.info()["num_buckets"] == MAX_BUCKETS
    E = G.info()["num_edges"]
    for _ in range(2):
        got = export(G, "mk_graph_export_csr_noalloc")
        plain = export(G, "mk_graph_export_csr")
        assert_same(got, plain)
        assert got[0][-1] == E
    G.close()


def test_noalloc_export_rejects_graphs_beyond_its_scratch():
    G = mk.DynamicGraph(MAX_BUCKETS + 1000)  # one bucket per vertex
    assert G.info()["num_buckets"] > MAX_BUCKETS
    import torch
    rp = torch.empty(G.num_vertices + 1, dtype=torch.int64, device="cuda:0")
    col = torch.empty(1, dtype=torch.int32, device="cuda:0")
    st = lib().mk_graph_export_csr_noalloc(G.handle, rp.data_ptr(), col.data_ptr(), None, None)
    assert st == MK_ERR_INVALID
    assert "262144" in lib().mk_last_error_string().decode()
    G.close()
