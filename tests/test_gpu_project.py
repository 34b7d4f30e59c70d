"""Output projections of the explicit fracture state (pxb_epf_project) against the reference element's own
ExplicitPDDOFracElement::computeNodalProjection (through oracle/_ref): damage, von Mises, stress and strain on
lattices with mirror ghosts, after one rate evaluation at a random field that breaks part of the bonds (the same
bonds in both, as the step parity tests establish).  Damage is a count ratio and must be identical; the tensors
within 1e-12 of the largest value of the field (the gradient sums cancel per node)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dim", [2, 3])
def test_projections_match_reference_element(ctx, dim):
    from oracle import RefEpf, RefMesh, ref_available
    if not ref_available():
        pytest.skip("the reference harness is not built")
    if dim == 2:
        m = RefMesh.structured(2, 24, 16, 0, [0, 0.024, 0, 0.016], 3.015, 2)
    else:
        m = RefMesh.structured(3, 6, 6, 5, [0, 0.006, 0, 0.006, 0, 0.005], 3.015, 2)
    E, nu, rho, G0 = 190e9, 0.3, 8000.0, 2e3
    el = RefEpf(m, E, nu, rho, G0)
    rng = np.random.default_rng(9 + dim)
    u = rng.standard_normal(m.n * dim) * 2e-6
    _, h_ref, _ = el.rate(u)
    k = el.constants()  # the element derives s_c in its first preprocess
    assert k["sc"] > 0
    assert 0 < (h_ref == 0).sum() < h_ref.size
    ctx.set_geometry(m.coords, m.vols, m.off, m.ids, m.delta, m.dx_char, dim, mirror=m.mirror)
    ctx.epf_setup(k["C11"], k["C12"], k["C66"], rho, (0.0,) * dim, k["sc"], True)
    ctx.epf_rate(u)
    _, _, h, _ = ctx.epf_state()
    assert np.array_equal(h, (h_ref > 0).astype(np.uint8))
    got = ctx.epf_project(u, plane_strain=True)
    assert np.array_equal(got["damage"], el.project("damage", u))
    for name in ("vonMises", "stress", "strain"):
        ref = el.project(name, u)
        assert np.abs(got[name] - ref).max() <= 1e-12 * np.abs(ref).max(), name
