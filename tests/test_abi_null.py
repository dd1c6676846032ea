"""CPU: every C-ABI entry point called with null handles and pointers (and
zero sizes) returns an error status instead of crashing; destroy functions
accept NULL like free().  Runs in a child process so a crash fails the test
instead of the session."""
import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent

PROBE = r"""
import ctypes as C, json, sys
sys.path.insert(0, sys.argv[1])
from meerkat_b200._lib import lib, SIGNATURES
L = lib()
out = {}
ints = (C.c_uint32, C.c_int32, C.c_uint64, C.c_int64, C.c_int, C.c_uint8, C.c_size_t)
for name, restype, argtypes in SIGNATURES:
    if name in ("mk_version", "mk_last_error_string"):
        continue
    args = []
    for a in argtypes:
        if a in (C.c_float, C.c_double):
            args.append(0.0)
        elif isinstance(a, type) and issubclass(a, ints):
            args.append(0)
        else:
            args.append(None)
    out[name] = int(getattr(L, name)(*args))
print(json.dumps(out))
"""


def test_null_arguments_return_errors():
    r = subprocess.run([sys.executable, "-c", PROBE, str(ROOT)], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    status = json.loads(r.stdout.strip().splitlines()[-1])
    assert len(status) > 60
    for name, st in status.items():
        if name.endswith("_destroy") or name == "mk_edgeset_size":
            assert st == 0, name
        else:
            assert st != 0, name
