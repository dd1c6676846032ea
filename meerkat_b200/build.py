"""Builds libmeerkat_b200.so in-tree with nvcc for sm_100a.

    python -m meerkat_b200.build          # incremental build
    python -m meerkat_b200.build --clean  # rebuild everything

Objects go to meerkat_b200/_build/, the shared library to
meerkat_b200/libmeerkat_b200.so (both git-ignored; the .so travels with the
repository snapshot to the GPU machine).
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libmeerkat_b200.so"
# benchmark-only probe library (not part of the product library or header)
BENCH_SRC = PKG / "bench_native" / "probe.cu"
BENCH_LIB = PKG / "libmk_bench_probe.so"
INCLUDE = PKG.parent / "include"

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
# the system g++ ships libgomp (an environment CXX may not)
HOSTCXX = ["-ccbin", "/usr/bin/g++"] if Path("/usr/bin/g++").exists() else []
ARCH = HOSTCXX + ["-gencode", "arch=compute_100a,code=sm_100a"]
CUFLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "--extended-lambda",
    "-Xcompiler", "-fPIC,-fopenmp,-O3", f"-I{INCLUDE}",
]


def _sources():
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))


def _headers():
    return sorted(list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list(INCLUDE.glob("*.h")))


def _needs(obj: Path, src: Path, headers) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return src.stat().st_mtime > t or any(h.stat().st_mtime > t for h in headers)


def _compile(src: Path, extra) -> Path:
    obj = BUILD / (src.name + ".o")
    cmd = [NVCC, *CUFLAGS, *extra, "-c", str(src), "-o", str(obj)]
    if src.suffix == ".cpp":
        cmd = [NVCC, *HOSTCXX, "-x", "c++", "-std=c++17", "-O3", "-Xcompiler", "-fPIC,-fopenmp,-O3",
               f"-I{INCLUDE}", "-c", str(src), "-o", str(obj)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return obj


def build(clean: bool = False, verbose: bool = False, ptxas_v: bool = False) -> Path:
    if clean and BUILD.exists():
        shutil.rmtree(BUILD)
    BUILD.mkdir(exist_ok=True)
    headers = _headers()
    srcs = _sources()
    extra = ["-Xptxas", "-v"] if ptxas_v else []
    todo = [s for s in srcs if ptxas_v or _needs(BUILD / (s.name + ".o"), s, headers)]
    if todo:
        with cf.ThreadPoolExecutor(max_workers=min(8, len(todo))) as ex:
            list(ex.map(lambda s: _compile(s, extra), todo))
    objs = [BUILD / (s.name + ".o") for s in srcs]
    if todo or not LIB.exists() or any(o.stat().st_mtime > LIB.stat().st_mtime for o in objs):
        cmd = [NVCC, *ARCH, "-shared", "-o", str(LIB), *map(str, objs),
               "-Xcompiler", "-fopenmp", "-lgomp", "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        if verbose:
            print(f"built {LIB}")
    return LIB


def build_bench_probe() -> Path:
    """Builds libmk_bench_probe.so (bench.py's memory-pattern probe)."""
    if BENCH_LIB.exists() and BENCH_LIB.stat().st_mtime >= BENCH_SRC.stat().st_mtime:
        return BENCH_LIB
    cmd = [NVCC, *CUFLAGS, "-shared", "-o", str(BENCH_LIB), str(BENCH_SRC), "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {BENCH_SRC.name}:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return BENCH_LIB


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--clean", action="store_true")
    ap.add_argument("--ptxas-v", action="store_true", help="print register / smem usage")
    a = ap.parse_args(argv)
    build(clean=a.clean, verbose=True, ptxas_v=a.ptxas_v)
    build_bench_probe()


if __name__ == "__main__":
    sys.exit(main())
