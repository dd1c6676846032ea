"""Graph sets: many small graphs in one union graph.  Every member's result
must equal the oracle's result for that member alone."""
import numpy as np
import pytest

import meerkat_b200 as mk
from oracle import OracleGraph

from helpers import degree_hints, to_dev

pytestmark = pytest.mark.gpu

INFINF = np.uint64(2**64 - 1)


def members(n=12, seed=40):
    """n seeded R-MAT graphs of scale 7..10 (local ids)."""
    out = []
    for m in range(n):
        scale = 7 + m % 4
        V = 1 << scale
        s, d, w = mk.gen_rmat(scale, V * (2 + m % 3), seed=seed + m, w_lo=1, w_hi=64)
        out.append((V, s, d, w))
    return out


def build_set(mem, chunk=None):
    nv = [V for V, *_ in mem]
    hints = [degree_hints(s, V) for V, s, _, _ in mem]
    S = mk.GraphSet(nv, degree_hints=hints, weighted=True)
    if chunk is not None:
        S.graph.set_tuning(frontier_chunk=chunk)
    off = S.offsets.astype(np.int64)
    s = np.concatenate([s + off[m] for m, (_, s, _, _) in enumerate(mem)]).astype(np.uint32)
    d = np.concatenate([d + off[m] for m, (_, _, d, _) in enumerate(mem)]).astype(np.uint32)
    w = np.concatenate([w for *_, w in mem]).astype(np.uint32)
    S.graph.InsertEdges(to_dev(s), to_dev(d), vals=to_dev(w))
    assert S.graph.sync() == 0
    oracles = []
    for V, ms, md, mw in mem:
        O = OracleGraph(V)
        O.insert(ms, md, mw)
        oracles.append(O)
    return S, oracles


def local_packed(packed, lo, hi):
    """Member slice of a packed dist<<32|parent array with local parent ids."""
    p = packed[lo:hi].copy()
    live = p != INFINF
    p[live] = (p[live] & np.uint64(0xFFFFFFFF00000000)) | ((p[live] & np.uint64(0xFFFFFFFF)) - np.uint64(lo))
    return p


@pytest.mark.parametrize("chunk", [None, 1, 64])
def test_multi_source_traversals_and_subset_wcc_match_members(chunk):
    mem = members()
    S, oracles = build_set(mem, chunk)
    off = S.offsets.astype(np.int64)
    G = S.graph
    # one source (the member's hub) for every even member; odd members stay unreached
    src_local = {m: int(np.argmax(np.bincount(s, minlength=V)))
                 for m, (V, s, _, _) in enumerate(mem) if m % 2 == 0}
    sources = [off[m] + v for m, v in src_local.items()]
    bfs, sssp = mk.BFS(G, sources), mk.SSSP(G, sources)
    wcc = mk.WCC(G)
    bfs.Static()
    sssp.Static()
    wcc.Static()

    def check(labels_expected=None):
        bd, sd = bfs.Distances(), sssp.Distances()
        bp, sp = bfs.packed(), sssp.packed()
        lab = wcc.Labels()
        for m, O in enumerate(oracles):
            lo, hi = off[m], off[m + 1]
            if m in src_local:
                v = src_local[m]
                np.testing.assert_array_equal(bd[lo:hi], O.bfs(v))
                np.testing.assert_array_equal(sd[lo:hi], O.sssp(v))
                assert O.check_parents(v, local_packed(bp, lo, hi), weighted=False) == 0
                assert O.check_parents(v, local_packed(sp, lo, hi), weighted=True) == 0
            else:
                assert (bd[lo:hi] == mk.MK_INF).all() and (sd[lo:hi] == mk.MK_INF).all()
            if labels_expected is None:
                np.testing.assert_array_equal(lab[lo:hi].astype(np.int64) - lo, O.wcc())
            else:
                np.testing.assert_array_equal(lab[lo:hi], labels_expected[lo:hi])

    check()
    labels_before = wcc.Labels()
    # one mixed batch over all members: deletes (incl. tree edges) then inserts
    rng = np.random.default_rng(9)
    packed = sssp.packed()
    del_s, del_d, ins_s, ins_d, ins_w = [], [], [], [], []
    for m, (V, s, d, _) in enumerate(mem):
        es = mk.EdgeSet(V, s, d)
        ds, dd = es.sample_present(len(s) // 8, seed=100 + m)
        if m in src_local:
            lp = local_packed(packed, off[m], off[m + 1])
            par = (lp & np.uint64(0xFFFFFFFF)).astype(np.int64)
            tree = np.nonzero((lp != INFINF) & (par != np.arange(V)))[0]
            pick = rng.choice(tree, size=min(8, len(tree)), replace=False)
            ds = np.concatenate([ds, par[pick]]).astype(np.uint32)
            dd = np.concatenate([dd, pick]).astype(np.uint32)
        is_, id_ = es.sample_absent(len(s) // 10, seed=200 + m)
        iw = rng.integers(1, 65, len(is_)).astype(np.uint32)
        oracles[m].delete(ds, dd)
        oracles[m].insert(is_, id_, iw)
        del_s.append(ds + off[m]), del_d.append(dd + off[m])
        ins_s.append(is_ + off[m]), ins_d.append(id_ + off[m]), ins_w.append(iw)
    cat = lambda xs: to_dev(np.concatenate(xs).astype(np.uint32))
    tds, tdd = cat(del_s), cat(del_d)
    G.DeleteEdges(tds, tdd)
    assert G.sync() == 0
    bfs.Decremental(tds, tdd)
    sssp.Decremental(tds, tdd)
    tis, tid, tiw = cat(ins_s), cat(ins_d), cat(ins_w)
    G.InsertEdges(tis, tid, vals=tiw)
    assert G.sync() == 0
    bfs.Incremental(tis, tid)
    sssp.Incremental(tis, tid, wgt=tiw)
    # recompute components of the odd members only: even members keep their
    # (now stale) labels
    flags = np.array([m % 2 for m in range(len(mem))], np.uint8)
    wcc.StaticSubset(S.select_bits(flags))
    expect = labels_before.copy()
    for m, O in enumerate(oracles):
        if m % 2:
            expect[off[m]:off[m + 1]] = O.wcc() + off[m]
    check(expect)


def test_select_bits_layout():
    S = mk.GraphSet([5, 40, 1, 30])
    bits = S.select_bits(np.array([1, 0, 1, 1], np.uint8)).cpu().numpy().view(np.uint32)
    V = S.num_vertices
    got = np.array([(bits[v >> 5] >> (v & 31)) & 1 for v in range(V)])
    owner = np.searchsorted(S.offsets, np.arange(V), side="right") - 1
    np.testing.assert_array_equal(got, np.array([1, 0, 1, 1])[owner])
    assert (bits[-1] >> (V & 31)) == 0  # padding bits stay clear


def test_device_generators_stay_inside_members():
    import torch
    nv = [300, 1024, 77, 5000, 2048, 1]
    S = mk.GraphSet(nv, weighted=True)
    off = S.offsets.astype(np.int64)
    epg = [2000, 8000, 300, 40000, 0, 5]
    src, dst, w = S.gen_rmat(epg, seed=3, w_lo=2, w_hi=9)
    s = src.cpu().numpy().view(np.uint32).astype(np.int64)
    d = dst.cpu().numpy().view(np.uint32).astype(np.int64)
    ww = w.cpu().numpy().view(np.uint32)
    assert len(s) == sum(epg)
    owner = np.repeat(np.arange(len(nv)), epg)
    assert ((s >= off[owner]) & (s < off[owner + 1])).all()
    assert ((d >= off[owner]) & (d < off[owner + 1])).all()
    single = owner == 5
    assert (s[~single] != d[~single]).all() and (s[single] == d[single]).all()
    assert ww.min() >= 2 and ww.max() <= 9
    # same seed, same edges
    src2, dst2, _ = S.gen_rmat(epg, seed=3, w_lo=2, w_hi=9)
    assert torch.equal(src, src2) and torch.equal(dst, dst2)
    # R-MAT skew inside member 3: its low ids are the heavy ones
    deg = np.bincount(s[owner == 3] - off[3], minlength=nv[3])
    assert deg[:64].sum() > deg[-64:].sum()
    S.graph.InsertEdges(src, dst, vals=w)
    assert S.graph.sync() == 0
    dpg = [100, 200, 50, 500, 10, 3]  # member 4 has no edge, member 5 only loops
    ipg = [30, 60, 10, 100, 10, 2]
    ds, dd, is_, id_, iw = S.gen_batches(dpg, ipg, seed=5, w_lo=2, w_hi=9)
    dsh = ds.cpu().numpy().view(np.uint32).astype(np.int64)
    ddh = dd.cpu().numpy().view(np.uint32).astype(np.int64)
    own_d = np.repeat(np.arange(len(nv)), dpg)
    live = (own_d != 4) & (own_d != 5)
    found = torch.zeros(len(dsh), dtype=torch.uint8, device="cuda:0")
    S.graph.SearchEdges(ds, dd, found)
    torch.cuda.synchronize()
    assert found.cpu().numpy()[live].all()
    assert ((dsh >= off[own_d]) & (dsh < off[own_d + 1])).all()
    assert (dsh[~live] == ddh[~live]).all()  # no live edge: a self-loop no-op
    ish = is_.cpu().numpy().view(np.uint32).astype(np.int64)
    idh = id_.cpu().numpy().view(np.uint32).astype(np.int64)
    own_i = np.repeat(np.arange(len(nv)), ipg)
    assert ((ish >= off[own_i]) & (ish < off[own_i + 1])).all()
    assert ((idh >= off[own_i]) & (idh < off[own_i + 1])).all()
    assert (ish[own_i != 5] != idh[own_i != 5]).all()
    iwh = iw.cpu().numpy().view(np.uint32)
    assert iwh.min() >= 2 and iwh.max() <= 9


def test_multi_source_rejects_bad_sources():
    S = mk.GraphSet([10, 10], weighted=True)
    with pytest.raises(mk.MeerkatError):
        mk.BFS(S.graph, [1, 1])
    with pytest.raises(mk.MeerkatError):
        mk.SSSP(S.graph, [3, 20])


def test_wcc_ranges_touch_only_their_members():
    mem = members(n=8, seed=60)
    S, oracles = build_set(mem)
    off = S.offsets.astype(np.int64)
    wcc = mk.WCC(S.graph)
    wcc.Static()
    before = wcc.Labels()
    # delete a third of member 1's and member 5's edges, recompute only those
    for m in (1, 5):
        V, s, d, _ = mem[m]
        es = mk.EdgeSet(V, s, d)
        ds, dd = es.sample_present(len(s) // 3, seed=7 + m)
        S.graph.DeleteEdges(to_dev(ds + off[m]), to_dev(dd + off[m]))
        oracles[m].delete(ds, dd)
    assert S.graph.sync() == 0
    wcc.StaticRanges([(off[1], off[2]), (off[5], off[6])])
    lab = wcc.Labels()
    for m, O in enumerate(oracles):
        lo, hi = off[m], off[m + 1]
        if m in (1, 5):
            np.testing.assert_array_equal(lab[lo:hi].astype(np.int64) - lo, O.wcc())
        else:
            np.testing.assert_array_equal(lab[lo:hi], before[lo:hi])


def test_range_pagerank_matches_each_member():
    mem = members(n=6, seed=70)
    S, oracles = build_set(mem)
    off = S.offsets.astype(np.int64)
    prr = mk.PageRankRange(S.graph, int(np.diff(off).max()))
    for m, O in enumerate(oracles):
        prr.Run(off[m], off[m + 1], 0.85, 1e-6, 500)
        want, _ = O.pagerank(0.85, 1e-14)
        got = prr.Values().astype(np.float64)
        assert len(got) == off[m + 1] - off[m]
        assert np.abs(got - want).sum() <= 1e-6, m
    # after an update of one member, its ranks follow (live out-degrees)
    V, s, d, _ = mem[2]
    es = mk.EdgeSet(V, s, d)
    ds, dd = es.sample_present(len(s) // 4, seed=3)
    S.graph.DeleteEdges(to_dev(ds + off[2]), to_dev(dd + off[2]))
    assert S.graph.sync() == 0
    oracles[2].delete(ds, dd)
    prr.Run(off[2], off[3], 0.85, 1e-6, 500)
    want, _ = oracles[2].pagerank(0.85, 1e-14)
    assert np.abs(prr.Values().astype(np.float64) - want).sum() <= 1e-6
    with pytest.raises(mk.MeerkatError):
        prr.Run(0, off[-1])  # larger than max_vertices


def _random_member(V, E, rng):
    s = rng.integers(0, V, E).astype(np.uint32)
    d = rng.integers(0, V, E).astype(np.uint32)
    keep = s != d
    return s[keep], d[keep], rng.integers(1, 65, keep.sum()).astype(np.uint32)


def test_wcc_prepared_ranges_shared_memory_and_device_wide_members():
    """Members up to 65,536 vertices run in shared memory, larger ones through
    the device-wide pass; both must give each member's own labels, also when
    the prepared call is captured into a CUDA graph and replayed after an
    update."""
    import torch
    rng = np.random.default_rng(91)
    sizes = [65536, 70000, 3, 1, 20000, 1024, 4096]
    mem = []
    for m, V in enumerate(sizes):
        if m == 5:  # no edges at all
            s = d = w = np.zeros(0, np.uint32)
        elif m == 6:  # one long path in a shuffled order: deep union trees
            perm = rng.permutation(V).astype(np.uint32)
            s, d = perm[:-1], perm[1:]
            w = np.ones(V - 1, np.uint32)
        else:  # sparse: many components
            s, d, w = _random_member(V, max(1, int(V * 0.6)), rng)
        mem.append((V, s, d, w))
    S, oracles = build_set(mem)
    off = S.offsets.astype(np.int64)
    wcc = mk.WCC(S.graph)
    ranges = [(off[m], off[m + 1]) for m in range(len(sizes))]
    wcc.PrepareRanges(ranges)
    wcc.StaticPrepared()
    assert S.graph.sync() == 0

    def check():
        lab = wcc.Labels().astype(np.int64)
        for m, O in enumerate(oracles):
            np.testing.assert_array_equal(lab[off[m]:off[m + 1]] - off[m], O.wcc(), err_msg=str(m))
    check()
    # capture, update two members (one per path), replay
    cs = torch.cuda.Stream()
    cs.wait_stream(torch.cuda.current_stream())
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=cs):
        wcc.StaticPrepared(stream=cs, timed=False)
    torch.cuda.synchronize()
    for m in (1, 6):
        V, s, d, _ = mem[m]
        pick = rng.choice(len(s), size=len(s) // 5, replace=False)
        S.graph.DeleteEdges(to_dev(s[pick] + off[m]), to_dev(d[pick] + off[m]))
        oracles[m].delete(s[pick], d[pick])
    assert S.graph.sync() == 0
    torch.cuda.synchronize()
    g.replay()
    torch.cuda.synchronize()
    assert S.graph.sync() == 0
    check()
    del g


def test_wcc_range_not_closed_under_edges_is_reported():
    S = mk.GraphSet([100, 100])
    # an edge from member 0 into member 1 breaks the closure of member 0
    S.graph.InsertEdges(to_dev(np.array([5, 7], np.uint32)), to_dev(np.array([150, 8], np.uint32)))
    assert S.graph.sync() == 0
    wcc = mk.WCC(S.graph)
    wcc.StaticRanges([(0, 100)])
    with pytest.raises(mk.MeerkatError, match="vertex range"):
        S.graph.sync()


def test_bfs_static_members_equals_device_wide_static():
    """The shared-memory member BFS gives the distances of the device-wide
    static BFS and a valid BFS tree (parents are not unique: the reference's
    relaxation keeps the first of equal-distance parents, BFSImpl.cuh:311-314),
    for members at the shared-memory limit, above it (device-wide path), tiny,
    edgeless and deep; the dynamic calls that follow it stay exact; a captured
    replay after an update matches a fresh static run."""
    import torch
    rng = np.random.default_rng(92)
    sizes = [65535, 70000, 3, 1, 20000, 1024, 4096, 300]
    mem = []
    for m, V in enumerate(sizes):
        if m == 5:
            s = d = w = np.zeros(0, np.uint32)
        elif m == 6:  # a shuffled path: 4095 levels
            perm = rng.permutation(V).astype(np.uint32)
            s, d = perm[:-1], perm[1:]
            w = np.ones(V - 1, np.uint32)
        else:
            s, d, w = _random_member(V, max(1, int(V * 3)), rng)
        mem.append((V, s, d, w))
    S, oracles = build_set(mem)
    off = S.offsets.astype(np.int64)
    src_local = []
    for m, (V, s, d, _) in enumerate(mem):
        if m == 6:
            src_local.append(int(s[0]))  # the head of the path
        else:
            src_local.append(int(np.argmax(np.bincount(s, minlength=V))) if len(s) else 0)
    sources = [int(off[m] + v) for m, v in enumerate(src_local)]
    ranges = [(off[m], off[m + 1]) for m in range(len(sizes))]
    bfs = mk.BFS(S.graph, sources)
    bfs.Static()
    want = bfs.Distances()
    bfs.PrepareMembers(ranges)
    bfs.StaticMembers()
    assert S.graph.sync() == 0
    dist = bfs.Distances()
    np.testing.assert_array_equal(dist, want)
    packed = bfs.packed()
    for m, O in enumerate(oracles):
        np.testing.assert_array_equal(dist[off[m]:off[m + 1]], O.bfs(src_local[m]), err_msg=str(m))
        assert O.check_parents(src_local[m], local_packed(packed, off[m], off[m + 1]),
                               weighted=False) == 0, m
    # a decremental call after the member static: tree edges of two members
    del_s, del_d = [], []
    for m in (0, 6):
        V, s, d, _ = mem[m]
        lp = local_packed(packed, off[m], off[m + 1])
        par = (lp & np.uint64(0xFFFFFFFF)).astype(np.int64)
        tree = np.nonzero((lp != INFINF) & (par != np.arange(V)))[0]
        pick = rng.choice(tree, size=min(16, len(tree)), replace=False)
        oracles[m].delete(par[pick].astype(np.uint32), pick.astype(np.uint32))
        del_s.append(par[pick] + off[m])
        del_d.append(pick + off[m])
    tds = to_dev(np.concatenate(del_s).astype(np.uint32))
    tdd = to_dev(np.concatenate(del_d).astype(np.uint32))
    S.graph.DeleteEdges(tds, tdd)
    assert S.graph.sync() == 0
    bfs.Decremental(tds, tdd)
    dist = bfs.Distances()
    for m in (0, 6):
        np.testing.assert_array_equal(dist[off[m]:off[m + 1]], oracles[m].bfs(src_local[m]))
    # captured member static, replayed after an insert batch
    cs = torch.cuda.Stream()
    cs.wait_stream(torch.cuda.current_stream())
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=cs):
        bfs.StaticMembers(stream=cs, timed=False)
    torch.cuda.synchronize()
    V, s, d, _ = mem[4]
    es = mk.EdgeSet(V, s, d)
    is_, id_ = es.sample_absent(2000, seed=5)
    S.graph.InsertEdges(to_dev(is_ + off[4]), to_dev(id_ + off[4]),
                        vals=to_dev(np.ones(len(is_), np.uint32)))
    assert S.graph.sync() == 0
    oracles[4].insert(is_, id_, np.ones(len(is_), np.uint32))
    torch.cuda.synchronize()
    g.replay()
    torch.cuda.synchronize()
    got = bfs.Distances()
    del g
    np.testing.assert_array_equal(got[off[4]:off[5]], oracles[4].bfs(src_local[4]))
    bfs.Static()
    np.testing.assert_array_equal(got, bfs.Distances())


def test_bfs_prepare_members_rejects_bad_tables():
    S = mk.GraphSet([10, 10, 10], weighted=True)
    bfs = mk.BFS(S.graph, [1, 12])
    with pytest.raises(mk.MeerkatError):
        bfs.PrepareMembers([(0, 10)])                 # one range per source
    with pytest.raises(mk.MeerkatError):
        bfs.PrepareMembers([(0, 10), (20, 30)])       # source 12 outside (20, 30)
    with pytest.raises(mk.MeerkatError):
        bfs.PrepareMembers([(0, 15), (10, 20)])       # overlapping
    with pytest.raises(mk.MeerkatError):
        bfs.StaticMembers()                           # nothing prepared
    sssp = mk.SSSP(S.graph, [1])
    with pytest.raises((mk.MeerkatError, AttributeError)):
        sssp.PrepareMembers([(0, 10)])
