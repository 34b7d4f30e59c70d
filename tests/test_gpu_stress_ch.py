"""Stress-coupled Cahn-Hilliard assembly (pxb_assemble_stress_ch; boundary of the reference's
perix_cuda::assembleStressCahnHilliard).  Rows per node: c, mu, u (ndof = dim + 2).

* Against the reference's CPU element (StressCahnHilliardElement preprocess + nodal/bond callbacks, accumulated
  as formResidualAndJacobianParallel does; golden fixtures stressch2d/3d from tests/golden/make_golden.py):
  every K entry within 1e-12 of the largest neighbour-block entry of its row, every rhs entry within 1e-12 of
  the largest bond term of its row (the bond sums cancel to far below their terms).
* With frozen bond health (kres on broken bonds) and backward-Euler inertia, against the reference's own GPU
  assembler (its CUDA translation unit built for sm_100a, oracle/ref_cuda_harness.cu), same tolerances."""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


def _setup(ctx, d, dim):
    s = d["scalars"]
    ctx.set_geometry(d["coords"], d["vols"], d["off"], d["ids"], s[0], s[4], dim, mirror=d["mirror"])
    nd, _ = ctx.gbuild(2, 0)
    assert nd == 0
    ctx.ch_set_geometry(d["rev"], d["lapbond"], d["isghost"])
    ctx.csr_set_pattern(d["rowptr"], d["cols"], dim + 2)
    E, nu, Omega, cref, D, chi, kappa, dt = (float(x) for x in d["params"])
    C11, C12, C66, A, Kh, Ch = (float(x) for x in d["consts"])
    return dict(C11=C11, C12=C12, C66=C66, A=A, Kh=Kh, Ch=Ch, Omega=Omega, cref=cref, chi=chi, kappa=kappa, dt=dt,
                kres=1e-8, rho=0.0)


def _row_scales(d, dim, kref):
    """Per row: the largest |K| entry outside the row's own node block, and the largest bond term
    |K_IJ (u_j - u_i)| entering the row's residual."""
    nd = dim + 2
    rp, cols = d["rowptr"], d["cols"]
    rows = np.repeat(np.arange(rp.size - 1), np.diff(rp))
    nbr = (cols // nd) != (rows // nd)
    ks = np.zeros(rp.size - 1)
    np.maximum.at(ks, rows[nbr], np.abs(kref[nbr]))
    u = d["u"]
    du = u[cols] - u[(rows // nd) * nd + (cols % nd)]
    rs = np.zeros(rp.size - 1)
    np.maximum.at(rs, rows[nbr], np.abs(kref[nbr] * du[nbr]))
    return rows, ks, rs


@pytest.mark.parametrize("dim", [2, 3])
def test_stress_ch_matches_reference_element(ctx, dim):
    d = load_golden("stressch%dd" % dim)
    p = _setup(ctx, d, dim)
    kv, rhs = ctx.assemble_stress_ch(p, d["mnode"], d["u"], d["uold"])
    rows, ks, rs = _row_scales(d, dim, d["kvals"])
    assert (np.abs(kv - d["kvals"]) <= 1e-12 * ks[rows]).all()
    nd = dim + 2
    # nodal parts of the rhs (c, mu rows) are O(1) next to the bond sums: scale by both
    scale = np.maximum(rs, np.abs(d["rhs"]))
    assert (np.abs(rhs - d["rhs"]) <= 1e-12 * scale).all()
    assert rhs.size == d["u"].size and kv.size == d["kvals"].size and nd == d["u"].size // d["vols"].size


def _p13(p):
    return np.array([p[k] for k in ("C11", "C12", "C66", "A", "Kh", "Ch", "Omega", "cref", "chi", "kappa", "dt",
                                    "kres", "rho")])


def _fracture_inertia(d, dim, p):
    rng = np.random.default_rng(5 + dim)
    n, nb = d["vols"].size, d["ids"].size
    health = (rng.uniform(size=nb) > 0.1).astype(np.float64)
    vel = rng.standard_normal(n * dim) * 1e-3
    return health, vel, dict(p, rho=2.0e3, kres=1e-3)


def _check(d, dim, kv, rhs, kr, rr):
    rows, ks, rs = _row_scales(d, dim, kr)
    assert (np.abs(kv - kr) <= 1e-12 * np.maximum(ks[rows], np.abs(kr))).all()
    assert (np.abs(rhs - rr) <= 1e-12 * np.maximum(rs, np.abs(rr))).all()


@pytest.mark.parametrize("dim", [2, 3])
def test_stress_ch_fracture_and_inertia_vs_restatement(ctx, port, dim):
    """Broken bonds (kres) and backward-Euler inertia against the numpy restatement (oracle/stress_ch.py, pinned
    to the reference element by tests/test_oracle.py) on perix_b200's FP64 operators."""
    from oracle.stress_ch import stress_ch_assemble
    d = load_golden("stressch%dd" % dim)
    p = _setup(ctx, d, dim)
    health, vel, q = _fracture_inertia(d, dim, p)
    kv, rhs = ctx.assemble_stress_ch(q, d["mnode"], d["u"], d["uold"], health=health, vel=vel)
    pqr = port.qindices(dim, 2)[0].reshape(-1, 3)
    kr, rr = stress_ch_assemble(dim, d["off"], d["ids"], ctx.get_ops(), pqr, d["vols"], d["rev"], d["lapbond"],
                                d["isghost"], d["mnode"], d["u"], d["uold"], d["rowptr"], d["cols"], q,
                                health=health, vel=vel)
    _check(d, dim, kv, rhs, kr, rr)


def test_stress_ch_2d_matches_reference_gpu(ctx):
    """The reference's own GPU assembler (its CUDA translation unit for sm_100a), plain and with broken bonds and
    inertia (2D; on the 3D fixture the reference's GPU path disagrees with its own CPU element, which perix_b200
    follows)."""
    from oracle import ref_cuda_available, ref_cuda_stress_ch
    if not ref_cuda_available():
        pytest.skip("the reference's CUDA assembler is not built (make -C oracle refcuda)")
    d = load_golden("stressch2d")
    p = _setup(ctx, d, 2)
    s = d["scalars"]
    geo = (d["rev"], d["lapbond"], d["isghost"], d["mnode"], d["u"], d["uold"])
    kv, rhs = ctx.assemble_stress_ch(p, d["mnode"], d["u"], d["uold"])
    kr, rr = ref_cuda_stress_ch(2, d["coords"], d["vols"], d["off"], d["ids"], s[0], s[4], d["rowptr"], d["cols"],
                                _p13(p), *geo)
    _check(d, 2, kv, rhs, kr, rr)
    health, vel, q = _fracture_inertia(d, 2, p)
    kv, rhs = ctx.assemble_stress_ch(q, d["mnode"], d["u"], d["uold"], health=health, vel=vel)
    kr, rr = ref_cuda_stress_ch(2, d["coords"], d["vols"], d["off"], d["ids"], s[0], s[4], d["rowptr"], d["cols"],
                                _p13(q), *geo, health=health, vel=vel)
    _check(d, 2, kv, rhs, kr, rr)
