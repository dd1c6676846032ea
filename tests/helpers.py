"""Shared helpers of the GPU parity tests."""
from __future__ import annotations

import numpy as np

import meerkat_b200 as mk
from oracle import OracleGraph


def to_dev(a, device="cuda:0"):
    """numpy uint32 array -> int32 CUDA tensor with the same bits."""
    import torch
    a = np.ascontiguousarray(a, dtype=np.uint32)
    return torch.from_numpy(a.view(np.int32)).to(device)


def degree_hints(src, V):
    return np.bincount(np.asarray(src, dtype=np.int64), minlength=V).astype(np.uint32)


def make_pair(V, src, dst, w=None, weighted=False, reverse=False, hints="exact",
              load_factor=0.7, pool_slabs=0, variant=None):
    """Builds the GPU graph and the oracle graph from the same edge list."""
    if hints == "exact":
        h = degree_hints(dst if reverse else src, V)
    elif hints == "ones":
        h = None
    else:
        h = hints
    G = mk.DynamicGraph(V, load_factor=load_factor, degree_hints=h, weighted=weighted,
                        reverse=reverse, pool_slabs=pool_slabs)
    if variant is not None:
        G.set_tuning(update_kernel=variant)
    O = OracleGraph(V)
    if len(src):
        s, d = to_dev(src), to_dev(dst)
        ww = to_dev(w) if (weighted and w is not None) else None
        G.InsertEdges(s, d, vals=ww)
        assert G.sync() == 0
        if reverse:
            O.insert(dst, src, w if weighted else None)
        else:
            O.insert(src, dst, w if weighted else None)
    return G, O


def assert_same_graph(G: mk.DynamicGraph, O: OracleGraph, weighted=False):
    np.testing.assert_array_equal(G.degrees(), O.degrees())
    rp, col, w = G.export_csr(sort_rows=True)
    orp, ocol, ow = O.csr(weights=weighted)
    np.testing.assert_array_equal(rp, orp)
    np.testing.assert_array_equal(col, ocol)
    if weighted:
        np.testing.assert_array_equal(w, ow)


def symmetrise(src, dst):
    s = np.concatenate([src, dst]).astype(np.uint32)
    d = np.concatenate([dst, src]).astype(np.uint32)
    keys = np.unique(s.astype(np.uint64) << 32 | d.astype(np.uint64))
    return (keys >> 32).astype(np.uint32), (keys & 0xFFFFFFFF).astype(np.uint32)
