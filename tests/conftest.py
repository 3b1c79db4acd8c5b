import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, os.path.join(ROOT, "ray-tracing_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def golden(name):
    return np.load(os.path.join(GOLDEN, name), allow_pickle=False)


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:  # pragma: no cover
        return False


@pytest.fixture(scope="session")
def ctx():
    """One liblrt context on cuda:0 for the GPU tests (the library must be built; no fallback)."""
    if not gpu_available():
        pytest.skip("no CUDA device")
    import lrt
    c = lrt.Context(0)
    yield c
    c.close()


def rel_close(a, b, rtol=1e-5, atol=1e-7):
    """|a - b| <= rtol * max(|a|, |b|) + atol, elementwise (NaNs equal)"""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    both_nan = np.isnan(a) & np.isnan(b)
    same_inf = np.isinf(a) & np.isinf(b) & (np.sign(a) == np.sign(b))
    ok = np.abs(a - b) <= rtol * np.maximum(np.abs(a), np.abs(b)) + atol
    return ok | both_nan | same_inf
