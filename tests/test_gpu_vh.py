"""Variable horizon on the device, against the reference (oracle/_ref): graded 2D and 3D clouds whose node horizons
follow their volumes (PDMesh::computeVariableHorizon) and whose families are the dual families.

* g-build: node i's moment system over the bonds within its own delta_i, its own rim spacing, zero operators beyond
  delta_i (CalcPDOperators.cpp:113-147, 307-354): FP64 within 1e-12 on both schedules' build (the warp-per-node
  kernel reads the horizons), mixed within 1e-6.
* explicit fracture: each bond breaks at s_c(0.5 (delta_i + delta_j)) (ExplicitPDDOFracElement.cpp:254-261): a rate
  call on every step schedule and ten steps, health identical, acceleration within 1e-12, u within 1e-10.
* the drop-in: the reference element with UseCuda on the same mesh hands nodeHorizon / nodeSpacing to the shim."""
import math

import numpy as np
import pytest

from conftest import graded_cloud, scaled_err
from oracle import dropin_available, ref_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not ref_available(), reason="reference harness not built")]

H0 = 1e-3


def _mesh(dim, dropin=False):
    from oracle import RefMesh
    xyz, vols = graded_cloud(dim, n=(24, 16, 8) if dim == 2 else (14, 9, 8))
    return RefMesh.cloud_vh(dim, xyz, vols, H0, H0, H0 if dim == 3 else 0.0, 3.015 * H0, dropin=dropin)


def _geometry(ctx, m):
    ctx.set_geometry(m.coords, m.vols, m.off, m.ids, m.delta, m.dx_char, m.dim)
    ctx.set_node_horizons(m.node_delta, m.node_spacing)


@pytest.mark.parametrize("dim", [2, 3])
def test_vh_gbuild_matches_reference(ctx, dim):
    m = _mesh(dim)
    g_ref, deg = m.gbuild()
    assert deg.sum() == 0
    _geometry(ctx, m)
    nd, _ = ctx.gbuild(2, 0)
    assert nd == 0
    g = ctx.get_ops()
    assert scaled_err(g, g_ref, m.off) <= 1e-12
    # bonds beyond the node's own horizon carry zero operators, as in the reference
    x = m.coords.reshape(-1, 3)[:, :dim]
    node = np.repeat(np.arange(m.n), np.diff(m.off))
    far = np.linalg.norm(x[m.ids - 1] - x[node], axis=1) > m.node_delta[node]
    assert far.any() and np.all(g[far] == 0.0) and np.all(g_ref[far] == 0.0)
    ctx.gbuild(2, 1)
    assert scaled_err(ctx.get_ops(), g_ref, m.off) <= 1e-6


def _epf_ref(m, dim):
    from oracle import RefEpf
    E, nu, rho = (190e9, 0.3, 8000.0) if dim == 2 else (72e9, 0.22, 2440.0)
    G0 = (0.01 ** 2 * 12 * E * 3.015 * H0 / (5 * math.pi)) if dim == 2 else (0.004 ** 2 * 6 * E * 3.015 * H0 / 5)
    el = RefEpf(m, E, nu, rho, G0)
    el.rate(np.zeros(dim * m.n))
    return el, el.constants(), E, rho, G0


def _epf_device(ctx, m, k, E, rho, G0, variant):
    import perix_b200 as px
    _geometry(ctx, m)
    ctx.epf_setup(k["C11"], k["C12"], k["C66"], rho, (0.0,) * m.dim, k["sc"], True)
    ctx.epf_set_variable_horizon_stretch(G0, E, False)
    try:
        ctx.epf_set_variant(variant)
    except px.PxbError as e:
        assert e.status == 7
        pytest.skip("variant %d does not fit these families" % variant)


@pytest.mark.parametrize("variant", list(range(21)))
@pytest.mark.parametrize("dim", [2, 3])
def test_vh_explicit_rate_and_steps_match_reference(ctx, dim, variant):
    m = _mesh(dim)
    el, k, E, rho, G0 = _epf_ref(m, dim)
    rng = np.random.default_rng(20 + dim)
    # amplitudes at which the reference breaks ~1.5 % (2D, s_c = 0.01) and ~3.5 % (3D, s_c = 0.004) of the bonds
    u = rng.standard_normal(dim * m.n) * (5e-6 if dim == 2 else 3e-6)
    a_ref, h_ref, _ = el.rate(u)
    assert (h_ref == 0).any()
    _epf_device(ctx, m, k, E, rho, G0, variant)
    a, nbk = ctx.epf_rate(u)
    h = ctx.epf_state()[2]
    assert 0 < nbk and np.array_equal(h, (h_ref > 0).astype(np.uint8))
    assert np.abs(a - a_ref).max() <= 1e-12 * np.abs(a_ref).max()
    # ten steps from the same field (a fresh reference element, no BCs on the free cloud)
    el2, _, _, _, _ = _epf_ref(m, dim)
    dt = 0.8 * H0 / math.sqrt(k["C11"] / rho)
    u_r, uo_r, hh_r, _ = el2.run(u * 0.5, None, dt, 10, [])
    _epf_device(ctx, m, k, E, rho, G0, variant)
    ctx.epf_start(u * 0.5, None, dt)
    ctx.epf_advance(10, chunk=5)
    u_d, uo_d, h_d, _ = ctx.epf_state()
    assert np.array_equal(h_d, (hh_r > 0).astype(np.uint8))
    assert np.abs(u_d - u_r).max() <= 1e-10 * np.abs(u_r).max()
    assert np.abs(uo_d - uo_r).max() <= 1e-10 * np.abs(u_r).max()


@pytest.mark.skipif(not dropin_available(), reason="drop-in harness not built")
@pytest.mark.parametrize("dim", [2, 3])
def test_vh_dropin_element_through_shim(dim):
    """ExplicitPDDOFracElement with UseCuda on the variable-horizon mesh: the element passes nodeHorizon and
    nodeSpacing to perix_cuda::assembleExplicitPDDOFracAccel; health and acceleration equal its CPU loop's."""
    import perix_b200 as px
    px.lib().pxb_cuda_shutdown()
    m = _mesh(dim, dropin=True)
    gpu, _, _, _, _ = _epf_ref(m, dim)
    cpu, _, _, _, _ = _epf_ref(m, dim)
    gpu.use_cuda(True)
    rng = np.random.default_rng(30 + dim)
    base = rng.standard_normal(dim * m.n) * (1.5e-6 if dim == 2 else 3e-6)
    for scale in (0.5, 1.0, 1.5):
        a_c, h_c, _ = cpu.rate(base * scale)
        a_g, h_g, _ = gpu.rate(base * scale)
        assert np.array_equal(h_g, h_c)
        assert np.abs(a_g - a_c).max() <= 1e-12 * np.abs(a_c).max()
    assert (h_c == 0).sum() > 0
    px.lib().pxb_cuda_shutdown()
