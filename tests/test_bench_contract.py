"""The benchmark's reference arm (CPU oracle, no GPU needed) prints one JSON
line with the contract's keys, on a small graph."""
import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def test_reference_arm_line():
    cmd = [sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--scale", "14",
           "--batch", "2000", "--steps", "2", "--warmup", "1"]
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["metric"] == line["unit"] == "edge updates/s"
    assert line["value"] > 0 and line["higher_is_better"] is True
    assert line["steps"] == 2 and line["warmup"] == 1 and line["n_gpus"] == 1
    assert line["config"]["workload"] == "rmat14_mixed_4000"
    cb = line["cpu_baseline"]
    assert {"value", "unit", "cores", "kind", "sample"} <= set(cb)
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == line["value"]
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"],
                           "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_loads_no_product_code():
    """The reference arm draws its inputs with the oracle's generators: the
    product library never enters the process."""
    code = (
        "import sys; sys.argv = ['bench.py', '--impl', 'reference', '--scale', '12', '--batch', "
        "'1000', '--steps', '1', '--warmup', '1']\n"
        "import bench\n"
        "assert bench.main() == 0\n"
        "maps = open('/proc/self/maps').read()\n"
        "assert 'libmeerkat_b200' not in maps, 'product library loaded'\n"
        "assert 'libmk_oracle' in maps\n"
        "assert 'meerkat_b200' not in sys.modules\n")
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True,
                         timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]


def _oracle_answers(scale, hist, A):
    """What a correct GPU run would report, computed with the oracle."""
    import numpy as np

    import bench
    from oracle import OracleGraph, cpu_pagerank
    (s, d, w), _ = bench.make_workload(0, source="oracle")
    O = OracleGraph(1 << scale, threads=4)
    O.insert(s, d, w)
    for ds, dd, is_, id_, iw in hist:
        O.delete(ds, dd)
        O.insert(is_, id_, iw)
    src = int(np.argmax(O.degrees()))
    gpu = {"source": src, "bfs": O.bfs(src), "sssp": O.sssp(src)}
    # parents: the oracle's own valid tree from the CPU port
    from oracle import CpuTraversal
    tb, ts = CpuTraversal(O, src, False), CpuTraversal(O, src, True)
    tb.static()
    ts.static()
    gpu["bfs_packed"], gpu["sssp_packed"] = tb.packed(), ts.packed()
    bs, bd = s[:500].copy(), d[:500].copy()
    O.delete(bs, bd)
    O.insert(bs, bd, np.zeros(500, dtype=np.uint32))
    gpu["batch"] = (bs, bd)
    gpu["degrees"] = O.degrees()
    gpu["wcc"] = O.wcc()
    gpu["triangles"] = O.triangles()
    gpu["pagerank"] = cpu_pagerank(O, 0.85, 1e-12)[0].astype(np.float32)
    return gpu


def test_oracle_large_parity_and_cpu_queries():
    """bench.oracle_large on a scale-12 run: the oracle's own answers pass,
    a planted wrong distance fails."""
    import bench
    saved = bench.SCALE, bench.EDGES, bench.HALF
    bench.SCALE, bench.EDGES, bench.HALF = 12, 16 << 12, 1000
    try:
        _check_oracle_large(bench)
    finally:
        bench.SCALE, bench.EDGES, bench.HALF = saved


def _check_oracle_large(bench):
    graph, batches = bench.make_workload(6, source="oracle")
    A = 2
    gpu = _oracle_answers(12, batches, A)
    cb, cq, par = bench.oracle_large(graph, batches, (0, 3), A, gpu, {})
    assert par["ok"], par
    assert cb["value"] > 0 and cb["kind"] == "port"
    for k in ("bfs_static_ms", "sssp_static_ms", "bfs_dec_ms_p50", "sssp_inc_ms_p50",
              "wcc_static_ms", "tc_static_ms", "pagerank_static_ms"):
        assert cq[k] >= 0
    assert par["cpu_port_bfs"] and par["cpu_port_sssp"] and par["cpu_port_tc"]
    gpu["sssp"] = gpu["sssp"].copy()
    v = int(next(i for i in range(len(gpu["sssp"])) if gpu["sssp"][i] not in (0, 0xFFFFFFFF)))
    gpu["sssp"][v] += 1
    _, _, par = bench.oracle_large(graph, batches, (0, 3), A, gpu, {})
    assert not par["ok"] and not par["sssp"]


def test_line_summary_is_compact():
    import bench
    line = {"value": 1e9, "e2e": {"value": 5e8}, "roofline": {"frac": 0.2},
            "cpu_baseline": {"value": 2e7},
            "queries": {"bfs_static_ms": 2.0, "bfs_inc_ms_p50": 0.1, "wcc": {"static_ms": 2.0}},
            "cpu_queries": {"cores": 16, "bfs_static_ms": 50.0},
            "parity": {"large": "ok"}}
    out = bench.line_summary(line)
    assert out["gpu_ms"]["bfs_static"] == 2.0 and out["cpu_ms"]["bfs_static"] == 50.0
    assert out["parity"] == {"large": "ok"}
    assert len(__import__("json").dumps(out)) < 2000
