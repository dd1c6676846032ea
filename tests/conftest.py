import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def _has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _has_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA device on this machine")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Builds the CUDA library (cross-compiles without a GPU) and the oracle."""
    from meerkat_b200.build import build
    from oracle import build_oracle
    if not os.environ.get("MK_SKIP_BUILD"):
        build()
    build_oracle()
    yield


@pytest.fixture
def dev():
    import torch
    return torch.device("cuda:0")


def to_dev(a, device="cuda:0"):
    """numpy uint32 array -> int32 CUDA tensor with the same bits."""
    import numpy as np
    import torch
    a = np.ascontiguousarray(a, dtype=np.uint32)
    return torch.from_numpy(a.view(np.int32)).to(device)
