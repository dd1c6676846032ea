"""GPU parity on the small benchmark configuration at its stated size.

R-MAT scale 16 (65,536 vertices, 1,048,576 distinct directed edges,
a/b/c/d = .57/.19/.19/.05, seed 0x4D45524B), uint32 weights uniform in
[1, 64].  One insert batch of 10,000 uniformly random absent edges, then one
delete batch of 10,000 uniformly chosen present edges.  Before the batches
and after each one: BFS and SSSP from vertex 0 (static, then incremental /
decremental with the batch, the reference drivers' protocol of
src/BFS.cu:111-121 and src/SSSP.cu:144-155), PageRank (damping 0.85, tol
1e-6, FP32 values; PageRank.cuh:32-46 on the reverse graph), triangle
counting on the symmetrised graph (TC.cuh:28-40) and union-find WCC.  Every
result is compared with the CPU oracle: levels, distances, triangle counts
and WCC labels bit-exact, BFS/SSSP parents valid, PageRank L1 <= 1e-6 of
the FP64 oracle."""
import numpy as np
import pytest

import meerkat_b200 as mk
from helpers import assert_same_graph, degree_hints, to_dev
from oracle import OracleGraph

pytestmark = pytest.mark.gpu

SCALE, EDGES, SEED = 16, 1_048_576, 0x4D45524B
BATCH = 10_000
PR_L1_TOL = 1e-6  # FP32 PageRank against the FP64 oracle


def test_small_config_sequence():
    V = 1 << SCALE
    s, d, w = mk.gen_rmat(SCALE, EDGES, seed=SEED, w_lo=1, w_hi=64)
    es = mk.EdgeSet(V, s, d)
    ins_s, ins_d = es.sample_absent(BATCH, seed=SEED + 1)
    ins_w = np.random.default_rng(SEED).integers(1, 65, BATCH).astype(np.uint32)
    del_s, del_d = es.sample_present(BATCH, seed=SEED + 2)

    O = OracleGraph(V, threads=8)
    O.insert(s, d, w)
    G = mk.DynamicGraph(V, load_factor=0.7, degree_hints=degree_hints(s, V), weighted=True)
    Gr = mk.DynamicGraph(V, load_factor=0.7, degree_hints=degree_hints(d, V), reverse=True)
    G.InsertEdges(to_dev(s), to_dev(d), vals=to_dev(w))
    Gr.InsertEdges(to_dev(s), to_dev(d))
    # symmetric copy for triangle counting, maintained with the same batches
    sym = {}
    for a, b in zip(s.tolist(), d.tolist()):
        sym[(min(a, b), max(a, b))] = sym.get((min(a, b), max(a, b)), 0) + 1
    und = np.array(list(sym.keys()), dtype=np.uint32).reshape(-1, 2)
    ss = np.concatenate([und[:, 0], und[:, 1]])
    sd = np.concatenate([und[:, 1], und[:, 0]])
    Gs = mk.DynamicGraph(V, load_factor=0.7, degree_hints=degree_hints(ss, V))
    Gs.InsertEdges(to_dev(ss), to_dev(sd))
    for g in (G, Gr, Gs):
        assert g.sync() == 0
    assert_same_graph(G, O, weighted=True)

    bfs, sssp = mk.BFS(G, 0, V), mk.SSSP(G, 0, V)
    pr = mk.PageRank(Gr, 0.85, 1e-6, V)
    tc, wcc = mk.TC(Gs, V), mk.WCC(G)
    bfs.Static(EDGES)
    sssp.Static(EDGES)
    pr.Static()
    tc.Static(len(ss))
    wcc.Static()

    def check(stage):
        assert G.sync() == 0, stage
        np.testing.assert_array_equal(bfs.Distances(), O.bfs(0), err_msg=stage)
        np.testing.assert_array_equal(sssp.Distances(), O.sssp(0), err_msg=stage)
        assert O.check_parents(0, bfs.packed(), weighted=False) == 0, stage
        assert O.check_parents(0, sssp.packed(), weighted=True) == 0, stage
        np.testing.assert_array_equal(wcc.Labels(), O.wcc(), err_msg=stage)
        assert tc.GetCount() == O.triangles(), stage
        want, _ = O.pagerank(0.85, 1e-13)
        l1 = float(np.abs(pr.Values().astype(np.float64) - want).sum())
        assert l1 <= PR_L1_TOL, (stage, l1)

    check("static")

    # insert batch: the graphs first, then the algorithms with the same batch
    n_ins, applied = O.insert(ins_s, ins_d, ins_w)
    assert n_ins == BATCH
    t_s, t_d, t_w = to_dev(ins_s), to_dev(ins_d), to_dev(ins_w)
    G.InsertEdges(t_s, t_d, vals=t_w)
    Gr.InsertEdges(t_s, t_d)
    new_und = []
    for a, b in zip(ins_s.tolist(), ins_d.tolist()):
        k = (min(a, b), max(a, b))
        if k not in sym:
            new_und.append(k)
        sym[k] = sym.get(k, 0) + 1
    nu = np.array(new_und, dtype=np.uint32).reshape(-1, 2)
    sy_s, sy_d = to_dev(np.concatenate([nu[:, 0], nu[:, 1]])), to_dev(np.concatenate([nu[:, 1], nu[:, 0]]))
    Gs.InsertEdges(sy_s, sy_d)
    assert G.last_applied() == BATCH
    bfs.Incremental(t_s, t_d)
    sssp.Incremental(t_s, t_d, wgt=t_w)
    pr.Incremental(t_s, t_d)
    tc.Incremental(sy_s, sy_d)
    wcc.Incremental(t_s, t_d)
    assert_same_graph(G, O, weighted=True)
    check("insert 10k")

    # delete batch
    n_del, _ = O.delete(del_s, del_d)
    assert n_del == BATCH
    t_s, t_d = to_dev(del_s), to_dev(del_d)
    G.DeleteEdges(t_s, t_d)
    Gr.DeleteEdges(t_s, t_d)
    gone = []
    for a, b in zip(del_s.tolist(), del_d.tolist()):
        k = (min(a, b), max(a, b))
        sym[k] -= 1
        if sym[k] == 0:
            del sym[k]
            gone.append(k)
    gu = np.array(gone, dtype=np.uint32).reshape(-1, 2)
    sy_s, sy_d = to_dev(np.concatenate([gu[:, 0], gu[:, 1]])), to_dev(np.concatenate([gu[:, 1], gu[:, 0]]))
    Gs.DeleteEdges(sy_s, sy_d)
    assert G.last_applied() == BATCH
    bfs.Decremental(t_s, t_d)
    sssp.Decremental(t_s, t_d)
    pr.Decremental(t_s, t_d)
    tc.Decremental(sy_s, sy_d)
    wcc.Decremental(t_s, t_d)
    assert_same_graph(G, O, weighted=True)
    check("delete 10k")
    for o in (bfs, sssp, pr, tc, wcc, G, Gr, Gs):
        o.close()
