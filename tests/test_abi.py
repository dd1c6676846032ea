"""CPU tests of the C ABI: the library loads and exports every declared
symbol, host-only generators are deterministic and valid."""
import ctypes
import re
import subprocess
from pathlib import Path

import numpy as np

import meerkat_b200 as mk
from meerkat_b200._lib import LIB_PATH, SIGNATURES

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "meerkat_b200.h"


def declared_symbols():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(mk_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    syms = declared_symbols()
    assert len(syms) > 40
    lib = ctypes.CDLL(str(LIB_PATH))
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing
    # nm agrees (C linkage, no mangling)
    out = subprocess.run(["nm", "-D", "--defined-only", str(LIB_PATH)], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r"\bT (mk_[a-z0-9_]+)$", out, flags=re.M))
    assert set(syms) <= exported


def test_python_bindings_cover_the_header():
    bound = {name for name, _, _ in SIGNATURES}
    assert set(declared_symbols()) <= bound


def test_python_bindings_match_the_header_arity():
    """Every ctypes prototype takes as many arguments as the C declaration."""
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    protos = {}
    for m in re.finditer(r"\b(mk_[a-z0-9_]+)\s*\(([^;{]*?)\)\s*;", text, flags=re.S):
        params = m.group(2).strip()
        protos[m.group(1)] = 0 if params in ("", "void") else len(params.split(","))
    assert len(protos) > 40
    bad = [(name, protos[name], len(args)) for name, _, args in SIGNATURES
           if name in protos and protos[name] != len(args)]
    assert not bad, bad


def test_version_string():
    assert "sm_100a" in mk.version()


def test_rmat_is_deterministic_distinct_and_loop_free():
    s1, d1, w1 = mk.gen_rmat(12, 30000, seed=7, w_lo=1, w_hi=64)
    s2, d2, w2 = mk.gen_rmat(12, 30000, seed=7, w_lo=1, w_hi=64)
    assert (s1 == s2).all() and (d1 == d2).all() and (w1 == w2).all()
    keys = s1.astype(np.uint64) << 32 | d1.astype(np.uint64)
    assert len(np.unique(keys)) == 30000
    assert (s1 != d1).all() and s1.max() < 4096 and d1.max() < 4096
    assert w1.min() >= 1 and w1.max() <= 64
    # skew: vertex 0 quadrant is the heaviest (a = 0.57)
    deg = np.bincount(s1, minlength=4096)
    assert deg[:64].sum() > deg[-64:].sum()
    s3, _, _ = mk.gen_rmat(12, 30000, seed=8)
    assert not (s1 == s3).all()


def test_grid_generator_shape():
    side = 16
    s, d, w = mk.gen_grid(side, 10, seed=3, w_lo=1, w_hi=1000)
    assert len(s) == 4 * side * (side - 1) + 10
    keys = s.astype(np.uint64) << 32 | d.astype(np.uint64)
    assert len(np.unique(keys)) == len(keys)
    g = s[: 4 * side * (side - 1)]
    h = d[: 4 * side * (side - 1)]
    dr = np.abs(g.astype(np.int64) // side - h.astype(np.int64) // side)
    dc = np.abs(g.astype(np.int64) % side - h.astype(np.int64) % side)
    assert ((dr + dc) == 1).all()
    # both directions present
    fw = set(zip(g.tolist(), h.tolist()))
    assert all((b, a) in fw for a, b in fw)


def test_edgeset_sampling_is_valid():
    s, d, _ = mk.gen_rmat(10, 5000, seed=1)
    es = mk.EdgeSet(1024, s, d)
    assert len(es) == 5000
    present = set(zip(s.tolist(), d.tolist()))
    ds, dd = es.sample_present(1000, seed=2)
    dele = list(zip(ds.tolist(), dd.tolist()))
    assert len(set(dele)) == 1000 and all(e in present for e in dele)
    present -= set(dele)
    ins, ind = es.sample_absent(1000, seed=3)
    ins_l = list(zip(ins.tolist(), ind.tolist()))
    assert len(set(ins_l)) == 1000
    assert all(e not in present and e[0] != e[1] for e in ins_l)
    assert len(es) == 5000
    # a deleted edge may come back only through sample_absent
    ds2, dd2 = es.sample_present(len(es), seed=4)
    assert len(set(zip(ds2.tolist(), dd2.tolist()))) == 5000


def test_graph_create_rejects_bad_arguments_without_gpu():
    import pytest
    with pytest.raises(mk.MeerkatError):
        mk.DynamicGraph(0)
    with pytest.raises(mk.MeerkatError):
        mk.DynamicGraph(16, load_factor=0.0)
