"""CPU oracle of the dynamic-graph semantics (test infrastructure only).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
package, as the checker.  See mk_oracle.c for the restated semantics and the
reference lines they follow.
"""
from .oracle import (CpuTraversal, OracleEdgeSet, OracleGraph, build_oracle,  # noqa: F401
                     cpu_pagerank, cpu_triangles, cpu_wcc, cpu_wcc_incremental, gen_rmat)
