import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def load_golden(name):
    return dict(np.load(os.path.join(GOLDEN, name)))


def fields(d, prefix):
    return [d[f"{prefix}_{n}"] for n in ("rho", "mx", "my", "E", "bxf", "byf")]


@pytest.fixture(scope="session")
def oracle_built():
    from oracle import oracle

    oracle.oracle_lib()
    return oracle


def gpu_available():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False
