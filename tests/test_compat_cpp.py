"""The C++ drop-in shim (include/meerkat_compat.hpp) compiles and links
against libmeerkat_b200.so without a GPU, and on a GPU a reference-style
driver using it (tests/cpp/drop_in_driver.cpp) matches the oracle."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

import meerkat_b200 as mk
from meerkat_b200._lib import LIB_PATH
from oracle import OracleGraph

ROOT = Path(__file__).resolve().parent.parent
SRC = ROOT / "tests" / "cpp" / "drop_in_driver.cpp"
FILE_DRIVER = ROOT / "tests" / "cpp" / "bfs_file_driver.cpp"
SET_DRIVER = ROOT / "tests" / "cpp" / "set_runner_driver.cpp"


def build_driver(tmp_path, src=SRC) -> Path:
    exe = tmp_path / src.stem
    cmd = ["/usr/bin/g++" if Path("/usr/bin/g++").exists() else "g++", "-std=c++17", "-O2",
           f"-I{ROOT / 'include'}", "-I/usr/local/cuda/include", str(src), "-o", str(exe),
           f"-L{LIB_PATH.parent}", "-lmeerkat_b200", f"-Wl,-rpath,{LIB_PATH.parent}",
           "-L/usr/local/cuda/lib64", "-lcudart", "-Wl,-rpath,/usr/local/cuda/lib64"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_shim_compiles_and_links(tmp_path):
    exe = build_driver(tmp_path)
    assert exe.exists()
    assert build_driver(tmp_path, FILE_DRIVER).exists()
    assert build_driver(tmp_path, SET_DRIVER).exists()


@pytest.mark.gpu
@pytest.mark.parametrize("op", ["0", "1"])
def test_reference_file_workflow_matches_oracle(tmp_path, op):
    """The reference's BFS driver workflow: graph file + <prefix>.batch.<i>
    files in its text formats, update then Incremental/Decremental."""
    exe = build_driver(tmp_path, FILE_DRIVER)
    V = 1 << 11
    s, d, _ = mk.gen_rmat(11, 12000, seed=9)
    mk.write_edge_list(tmp_path / "g.txt", V, s, d)
    es = mk.EdgeSet(V, s, d)
    O = OracleGraph(V)
    O.insert(s, d)
    for i in range(3):
        if op == "0":
            bs, bd = es.sample_absent(700, seed=20 + i)
            O.insert(bs, bd)
        else:
            bs, bd = es.sample_present(700, seed=20 + i)
            O.delete(bs, bd)
        mk.write_batch(tmp_path / f"upd.batch.{i}", bs, bd)
    r = subprocess.run([str(exe), str(tmp_path / "g.txt"), op, str(tmp_path / "upd"), "3"],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    lines = r.stdout.strip().splitlines()
    assert lines[0].startswith(str(tmp_path / "g.txt")) and lines[0].count(",") == 4
    got = np.array(list(map(int, lines[1:])), dtype=np.uint32)
    np.testing.assert_array_equal(got, O.bfs(0))


@pytest.mark.gpu
@pytest.mark.parametrize("rev", ["", "rev"])
def test_reference_style_driver_matches_oracle(tmp_path, rev):
    """The reference's driver sequence on the shim; with rev the algorithms
    also get reverse graphs (SetReverse) kept in step with every batch."""
    exe = build_driver(tmp_path)
    r = subprocess.run([str(exe), "12"] + ([rev] if rev else []), capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    lines = r.stdout.strip().splitlines()
    got = np.array([list(map(int, ln.split())) for ln in lines[1:]], dtype=np.uint64)
    scale, V = 12, 1 << 12
    E = 8 << scale
    s, d, w = mk.gen_rmat(scale, E, seed=7, w_lo=1, w_hi=64)
    O = OracleGraph(V)
    O.insert(s, d, w)
    nb = E // 8
    O.delete(s[:nb], d[:nb])
    O.insert(s[:nb // 2], d[:nb // 2], w[:nb // 2])
    np.testing.assert_array_equal(got[:, 0], O.bfs(0))
    np.testing.assert_array_equal(got[:, 1], O.sssp(0))
    np.testing.assert_array_equal(got[:, 2], O.wcc())


@pytest.mark.gpu
@pytest.mark.parametrize("capture", ["0", "1"])
@pytest.mark.parametrize("single", ["0", "1"])
def test_cpp_batched_step_matches_oracle(tmp_path, capture, single):
    """The batched many-graph step through the C++ shim (GraphSet +
    GraphSetRunner over mk_set_runner_*), four launches or one cooperative
    launch per step, issued step by step and captured into a CUDA graph:
    every member's BFS levels or WCC labels equal the oracle's on that
    member alone after the same update steps."""
    exe = build_driver(tmp_path, SET_DRIVER)
    G, K = 6, 5
    r = subprocess.run([str(exe), str(G), str(K), capture, single], capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    lines = r.stdout.strip().splitlines()
    assert len(lines) == G
    for m, ln in enumerate(lines):
        f = list(map(int, ln.split()))
        assert f[0] == m
        kind, src, got = f[1], f[2], np.array(f[3:], dtype=np.uint32)
        n = 256 << (m % 4)
        scale = n.bit_length() - 1
        E = 6 * n
        s, d, w = mk.gen_rmat(scale, E, seed=100 + m, w_lo=1, w_hi=64)
        O = OracleGraph(n)
        O.insert(s, d, w)
        us, ud = s[:E // 10], d[:E // 10]
        for k in range(K):
            if k % 2 == 0:
                O.delete(us, ud)
            else:
                O.insert(us, ud, np.full(len(us), 7, np.uint32))
        assert len(got) == n
        if kind == 0:
            np.testing.assert_array_equal(got, O.bfs(src))
        else:
            np.testing.assert_array_equal(got, O.wcc())
