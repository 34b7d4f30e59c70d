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


def graded_cloud(dim, n=(24, 16, 8), h0=1e-3, grade=0.6, jitter=0.1, seed=4):
    """A point cloud whose spacing grows by `grade` across x (cell-centred columns of width h0 (1 + grade x/Lx)),
    uniform h0 in y (and z), jittered by U(+-jitter h) per coordinate; volumes are the local cell sizes.  Its
    volumes vary smoothly, so a variable horizon (delta_i ~ V_i^(1/dim)) differs from node to node."""
    rng = np.random.default_rng(seed)
    nx = n[0]
    w = h0 * (1.0 + grade * (np.arange(nx) + 0.5) / nx)
    xc = np.cumsum(w) - 0.5 * w
    axes = [np.arange(k) for k in n[1:dim]]
    grid = np.meshgrid(np.arange(nx), *axes, indexing="ij")
    idx = np.stack([g.reshape(-1) for g in grid], -1)
    xyz = np.zeros((idx.shape[0], 3))
    xyz[:, 0] = xc[idx[:, 0]]
    for a in range(1, dim):
        xyz[:, a] = (idx[:, a] + 0.5) * h0
    hx = w[idx[:, 0]]
    xyz[:, 0] += rng.uniform(-jitter, jitter, idx.shape[0]) * hx
    for a in range(1, dim):
        xyz[:, a] += rng.uniform(-jitter, jitter, idx.shape[0]) * h0
    vols = hx * h0 ** (dim - 1)
    return xyz, vols
