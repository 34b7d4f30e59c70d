import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the perix_b200 kernels")


def load_golden(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def port():
    from oracle import PortOracle, port_available
    if not port_available():
        import subprocess
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "port"], check=True, capture_output=True)
    return PortOracle()


@pytest.fixture(scope="session")
def ctx():
    """One perix_b200 context for the GPU tests (the library is built in-tree first)."""
    from perix_b200.build import build
    build()
    import perix_b200 as px
    c = px.Context(0)
    yield c
    c.close()


def scaled_err(a, b, off):
    """max over nodes/ops of |a-b| / max_t |b| over the node's family, per operator slot (family-scaled)."""
    a = np.asarray(a).reshape(b.shape)
    n = off.size - 1
    worst = 0.0
    lens = np.diff(off)
    node_of = np.repeat(np.arange(n), lens)
    scale = np.zeros((n, b.shape[1]))
    np.maximum.at(scale, node_of, np.abs(b))
    denom = scale[node_of]
    d = np.abs(a - b)
    mask = denom > 0
    if mask.any():
        worst = float((d[mask] / denom[mask]).max())
    if (~mask).any():
        worst = max(worst, float(d[~mask].max()))
    return worst
