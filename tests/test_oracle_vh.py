"""Variable horizon on the host, against the reference (oracle/_ref/libperix_ref.so): the per-node horizon and rim
spacing from the node volumes (PDMesh::computeVariableHorizon, CreatePDMesh.cpp:828-905) and the dual families
(createNeighborNodes with NodeHorizon, CreatePDMesh.cpp:932-938, 1043-1057), bit for bit on graded 2D and 3D
clouds."""
import numpy as np
import pytest

from conftest import graded_cloud
from oracle import ref_available

pytestmark = pytest.mark.skipif(not ref_available(), reason="reference harness not built")


@pytest.mark.parametrize("dim", [2, 3])
def test_variable_horizon_and_families_match_reference(dim):
    import perix_b200 as px
    from oracle import RefMesh
    h0 = 1e-3
    xyz, vols = graded_cloud(dim, n=(24, 16, 8) if dim == 2 else (14, 9, 8))
    m = RefMesh.cloud_vh(dim, xyz, vols, h0, h0, h0 if dim == 3 else 0.0, 3.015 * h0)
    assert np.ptp(m.node_delta) > 0.1 * m.node_delta.max()  # the horizons do vary
    d, sp = px.variable_horizon(dim, vols, m.delta, h0)
    assert np.array_equal(d, m.node_delta)
    assert np.array_equal(sp, m.node_spacing)
    off, ids = px.families_vh(xyz, d, dim == 3)
    assert np.array_equal(off, m.off)
    assert np.array_equal(ids, m.ids)
    # dual families: some members lie beyond the node's own horizon
    x = xyz[:, :dim]
    node = np.repeat(np.arange(off.size - 1), np.diff(off))
    r = np.linalg.norm(x[ids - 1] - x[node], axis=1)
    assert (r > d[node]).any()
