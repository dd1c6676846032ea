"""Batched runner against the per-graph launch sequence and the oracle: every
member's answer after each step is that of the member alone."""
import numpy as np
import pytest

import meerkat_b200 as mk
from meerkat_b200 import batched as B
from oracle import OracleGraph


def build(spec, dev, weighted=True):
    import torch
    voff = B._offsets(spec.num_vertices)
    eoff = B._offsets(spec.num_edges)
    src, dst, w = mk.gen_rmat_members(voff, spec.num_edges, seed=spec.seed, w_lo=1, w_hi=64)
    V = int(voff[-1])
    hints = torch.bincount(src.long(), minlength=V).to(torch.int32).cpu().numpy().view(np.uint32)
    gs = mk.GraphSet(spec.num_vertices, degree_hints=[hints[voff[m]:voff[m + 1]]
                                                      for m in range(spec.num_graphs)],
                     weighted=weighted)
    gs.graph.InsertEdges(src, dst, vals=w if weighted else None)
    assert gs.graph.sync() == 0
    s_h = src.cpu().numpy().view(np.uint32).astype(np.int64)
    d_h = dst.cpu().numpy().view(np.uint32).astype(np.int64)
    w_h = w.cpu().numpy().view(np.uint32)
    plain, oracles = [], []
    for m in range(spec.num_graphs):
        lo, hi, base = int(eoff[m]), int(eoff[m + 1]), int(voff[m])
        g = mk.DynamicGraph(int(spec.num_vertices[m]), weighted=True)
        g.InsertEdges(src[lo:hi] - base, dst[lo:hi] - base, vals=w[lo:hi])
        assert g.sync() == 0
        plain.append(g)
        O = OracleGraph(int(spec.num_vertices[m]))
        O.insert((s_h[lo:hi] - base).astype(np.uint32), (d_h[lo:hi] - base).astype(np.uint32),
                 w_h[lo:hi])
        oracles.append(O)
    return gs, plain, oracles, voff


@pytest.mark.gpu
@pytest.mark.parametrize("capture", [False, True])
def test_batched_runner_matches_plain_and_oracle(capture):
    import torch
    spec = B.make_spec(48, seed=11, v_lo=32, v_hi=700, deg_lo=2, deg_hi=12, upd_lo=0.05,
                       upd_hi=0.3)
    gs, plain, oracles, voff = build(spec, "cuda:0")
    Gn = spec.num_graphs
    bfs_members = np.flatnonzero(spec.query == B.QUERY_BFS)
    srcs = B.pick_sources(gs.graph.degrees(), voff, bfs_members, seed=3)
    br = B.BatchedRunner(gs, spec.query, srcs)
    pr = B.PlainRunner(plain, spec.query, srcs)
    src_of = dict(zip(bfs_members.tolist(), srcs.tolist()))
    for step in range(3):
        ds, dd, is_, id_, iw = gs.gen_batches(spec.deletes, spec.inserts, seed=100 + step)
        batch = (ds, dd, is_, id_, iw)
        if capture:
            s = torch.cuda.Stream()
            s.wait_stream(torch.cuda.current_stream())
            br.update(*batch, stream=s)  # warm the launch path outside the capture
            torch.cuda.synchronize()
            # undo is not needed: capture only the queries, replay twice
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, stream=s):
                br.query(stream=s)
            with torch.cuda.stream(s):
                g.replay()
                g.replay()
            torch.cuda.synchronize()
            del g
        else:
            br.step(batch)
        check_step(spec, batch, voff, oracles, gs, br, src_of, pr, plain)


def check_step(spec, batch, voff, oracles, gs, br, src_of, pr=None, plain=()):
    """Applies one set batch to the oracles (and, when given, the plain
    per-graph runner with local ids), then compares every member's answer,
    and the set's degrees, with the oracle's."""
    import torch
    Gn = spec.num_graphs
    h = [x.cpu().numpy().view(np.uint32).astype(np.int64) for x in batch[:4]]
    h.append(batch[4].cpu().numpy().view(np.uint32).astype(np.int64) if batch[4] is not None
             else np.ones(len(h[2]), dtype=np.int64))
    do, io = B._offsets(spec.deletes), B._offsets(spec.inserts)
    slices = []
    for m in range(Gn):
        base = int(voff[m])
        a = slice(do[m], do[m + 1])
        b = slice(io[m], io[m + 1])
        loc = [(h[0][a] - base), (h[1][a] - base), (h[2][b] - base), (h[3][b] - base)]
        loc = [x.astype(np.uint32) for x in loc] + [h[4][b].astype(np.uint32)]
        oracles[m].delete(loc[0], loc[1])
        oracles[m].insert(loc[2], loc[3], loc[4])
        slices.append(tuple(torch.from_numpy(x.view(np.int32)).cuda() for x in loc))
    if pr is not None:
        pr.step(slices)
    torch.cuda.synchronize()
    assert gs.graph.sync() == 0 and all(g.sync() == 0 for g in plain)
    d_union = br.bfs.Distances()
    l_union = br.wcc.Labels().astype(np.int64)
    deg = gs.graph.degrees()
    for m in range(Gn):
        lo, hi = int(voff[m]), int(voff[m + 1])
        np.testing.assert_array_equal(deg[lo:hi], oracles[m].degrees())
        if spec.query[m] == B.QUERY_BFS:
            want = oracles[m].bfs(src_of[m])
            np.testing.assert_array_equal(d_union[lo:hi], want)
            if pr is not None:
                np.testing.assert_array_equal(pr.algos[m].Distances(), want)
        else:
            want = oracles[m].wcc()
            np.testing.assert_array_equal(l_union[lo:hi] - lo, want)
            if pr is not None:
                np.testing.assert_array_equal(pr.algos[m].Labels(), want)


@pytest.mark.gpu
@pytest.mark.parametrize("capture,weighted,single", [
    (False, False, False), (True, True, False), (True, False, False),
    (False, True, True), (True, True, True), (False, False, True)])
def test_runner_step_matches_oracle(capture, weighted, single):
    """The whole batched step through the C set runner (mk_set_runner_step:
    both update kernels and both member queries, or the one cooperative
    launch), issued directly or captured into a CUDA graph and replayed:
    every member's answer and the set's degrees equal the oracle's after
    each step, on weighted and unweighted sets, and the applied-insert count
    is published as after the four launches."""
    import torch
    spec = B.make_spec(48, seed=12, v_lo=32, v_hi=700, deg_lo=2, deg_hi=12, upd_lo=0.05,
                       upd_hi=0.3)
    gs, _, oracles, voff = build(spec, "cuda:0", weighted=weighted)
    bfs_members = np.flatnonzero(spec.query == B.QUERY_BFS)
    srcs = B.pick_sources(gs.graph.degrees(), voff, bfs_members, seed=4)
    br = B.BatchedRunner(gs, spec.query, srcs)
    if single:
        assert br.single_ok
        br.set_single(True)
    assert br.launches_per_step() == br.runner.launches_per_step() == (1 if single else 4)
    gs.graph.reserve_batch(int(max(spec.inserts.sum(), spec.deletes.sum())))
    src_of = dict(zip(bfs_members.tolist(), srcs.tolist()))
    for step in range(3):
        batch = gs.gen_batches(spec.deletes, spec.inserts, seed=200 + step, weights=weighted)
        if capture:
            s = torch.cuda.Stream()
            s.wait_stream(torch.cuda.current_stream())
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, stream=s):
                br.step(batch, stream=s)
            with torch.cuda.stream(s):
                g.replay()
            torch.cuda.synchronize()
            del g
        else:
            br.step(batch)
        edges_before = sum(O.num_edges() for O in oracles)
        check_step(spec, batch, voff, oracles, gs, br, src_of)
        # inserts applied = the edge count's growth + the deletes applied
        grown = sum(O.num_edges() for O in oracles) - edges_before
        assert grown <= gs.graph.last_applied() <= int(spec.inserts.sum())
    br.close()
    gs.close()


def test_spec_is_seeded_and_in_range():
    a = B.make_spec(500, seed=5)
    b = B.make_spec(500, seed=5)
    assert (a.num_vertices == b.num_vertices).all() and (a.query == b.query).all()
    assert a.num_vertices.min() >= 1024 and a.num_vertices.max() <= 65536
    deg = a.num_edges / a.num_vertices
    assert deg.min() >= 3.9 and deg.max() <= 32.1
    frac = (a.deletes + a.inserts) / a.num_edges
    assert frac.min() >= 0.009 and frac.max() <= 0.101
    assert 150 < int((a.query == B.QUERY_BFS).sum()) < 350
