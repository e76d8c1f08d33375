import json
import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = Path(__file__).with_name("golden") / "golden.json"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: long-running case")


def _cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _cuda_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def golden():
    return json.loads(GOLDEN.read_text())


@pytest.fixture(scope="session", autouse=True)
def built_library():
    """Builds the native library and the CPU checker once per session."""
    import __graft_entry__ as ge
    ge.build()


def host_csr(d):
    import cgp_b200 as cgp
    w = None
    if "weights" in d:
        w = np.asarray(d["weights"], np.float32)
    return cgp.HostCsr(np.asarray(d["row_offsets"], np.int64),
                       np.asarray(d["col_indices"], np.int32), w)


def as_expected(vec, dtype):
    out = []
    for x in vec:
        out.append(np.inf if x == "inf" else x)
    return np.asarray(out, dtype)
