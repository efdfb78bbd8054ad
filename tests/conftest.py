import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(ROOT, "geraf-sens_b200")
for p in (ROOT, PKG_DIR):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN_DIR = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")


def rel_l2(a, b):
    import numpy as np

    a = np.asarray(a, dtype=np.complex128) if np.iscomplexobj(a) else np.asarray(a, np.float64)
    b = np.asarray(b, dtype=np.complex128) if np.iscomplexobj(b) else np.asarray(b, np.float64)
    den = np.linalg.norm(b.ravel())
    return float(np.linalg.norm((a - b).ravel()) / (den if den > 0 else 1.0))


_PARITY = []


@pytest.fixture
def parity_log():
    """Records measured parity figures; written to $GERAF_PARITY_OUT at session end."""
    def log(test, **figures):
        _PARITY.append({"test": test, **{k: (float(v) if not isinstance(v, str) else v)
                                         for k, v in figures.items()}})
    return log


def pytest_sessionfinish(session, exitstatus):
    path = os.environ.get("GERAF_PARITY_OUT")
    if path and _PARITY:
        import json

        with open(path, "w") as f:
            json.dump(_PARITY, f, indent=1)
