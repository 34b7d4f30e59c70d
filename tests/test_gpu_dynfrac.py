"""Implicit PDDO dynamic-fracture assembly (pxb_assemble_cached; boundary of the reference's
perix_cuda::assembleCached) against the reference's PDDODynamicFracElement (golden fixtures dynfrac2d/3d from
tests/golden/make_golden.py): the element is initialised, commits one step (velocity history, bond failure by
stretch: 22 % / 28 % of the bonds break) and is assembled at a perturbed state; perix_b200 gets the element's
committed velocity (in a 3-slot node cache, the reference layout) and bond health.  Every K entry within 1e-12
of the largest neighbour-block entry of its row, every rhs entry within 1e-12 of the largest bond term of its
row or of the entry itself (the nodal inertia dominates)."""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dim", [2, 3])
def test_dynfrac_matches_reference_element(ctx, dim):
    d = load_golden("dynfrac%dd" % dim)
    s = d["scalars"]
    ctx.set_geometry(d["coords"], d["vols"], d["off"], d["ids"], s[0], s[4], dim, mirror=d["mirror"])
    nd, _ = ctx.gbuild(2, 0)
    assert nd == 0
    ctx.csr_set_pattern(d["rowptr"], d["cols"], dim)
    E, nu, rho, G0, dt, bx, by, bz = (float(x) for x in d["params"])
    C11, C12, C66 = (float(x) for x in d["consts"])
    n = d["vols"].size
    nodecache = np.zeros((n, 3))
    nodecache[:, :dim] = d["vel"].reshape(n, dim)
    prm = dict(C11=C11, C12=C12, C66=C66, rho=rho, dt=dt, b=(bx, by, bz))
    kv, rhs = ctx.assemble_cached(prm, d["u"], d["uold"], nodecache=nodecache.reshape(-1), ncache=3,
                                  bondcache=d["health"], nbcache=1)
    kref, rref = d["kvals"], d["rhs"]
    rp, cols = d["rowptr"], d["cols"]
    rows = np.repeat(np.arange(rp.size - 1), np.diff(rp))
    nbr = (cols // dim) != (rows // dim)
    ks = np.zeros(rp.size - 1)
    np.maximum.at(ks, rows[nbr], np.abs(kref[nbr]))
    assert (np.abs(kv - kref) <= 1e-12 * np.maximum(ks[rows], np.abs(kref))).all()
    u = d["u"]
    du = u[cols] - u[(rows // dim) * dim + (cols % dim)]
    rs = np.zeros(rp.size - 1)
    np.maximum.at(rs, rows[nbr], np.abs(kref[nbr] * du[nbr]))
    assert (np.abs(rhs - rref) <= 1e-12 * np.maximum(rs, np.abs(rref))).all()
