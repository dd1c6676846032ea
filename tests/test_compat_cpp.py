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


def build_driver(tmp_path) -> Path:
    exe = tmp_path / "drop_in_driver"
    cmd = ["/usr/bin/g++" if Path("/usr/bin/g++").exists() else "g++", "-std=c++17", "-O2",
           f"-I{ROOT / 'include'}", "-I/usr/local/cuda/include", str(SRC), "-o", str(exe),
           f"-L{LIB_PATH.parent}", "-lmeerkat_b200", f"-Wl,-rpath,{LIB_PATH.parent}",
           "-L/usr/local/cuda/lib64", "-lcudart", "-Wl,-rpath,/usr/local/cuda/lib64"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_shim_compiles_and_links(tmp_path):
    exe = build_driver(tmp_path)
    assert exe.exists()


@pytest.mark.gpu
def test_reference_style_driver_matches_oracle(tmp_path):
    exe = build_driver(tmp_path)
    r = subprocess.run([str(exe), "12"], capture_output=True, text=True, timeout=300)
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
