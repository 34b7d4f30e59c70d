"""The oracle (plain-C restatement, oracle/pddo_oracle.c) pinned against the reference: golden fixtures made by
the reference's own code (tests/golden/make_golden.py), the reference's known-answer tests, and - where the
reference-sourced harness oracle/_ref/libperix_ref.so is built - the reference itself at full config sizes."""
import math

import numpy as np
import pytest

from conftest import load_golden, scaled_err

FIXTURES = [("poisson16", 2), ("lattice3d", 3), ("cloud2d", 2), ("cloud3d", 3), ("epf2d", 2), ("epf3d", 3)]


def crack_args(d):
    cracks = d["cracks"] if "cracks" in d else None
    planes = d["plane"].reshape(1, -1) if "plane" in d else None
    return cracks, planes, ("cracks" in d or "plane" in d)


@pytest.mark.parametrize("name,dim", FIXTURES)
def test_families_bit_exact(port, name, dim):
    d = load_golden(name)
    cracks, planes, fo = crack_args(d)
    mirror = d["mirror"] if d["mirror"].any() else None
    off, ids = port.families(d["coords"], d["scalars"][0], dim == 3, cracks=cracks, planes=planes, mirror=mirror,
                             force_only=fo)
    assert np.array_equal(off, d["off"])
    assert np.array_equal(ids, d["ids"])


@pytest.mark.parametrize("name", ["poisson16", "lattice3d"])
def test_csr_pattern_bit_exact(port, name):
    d = load_golden(name)
    rp, cols = port.csr_pattern(d["off"], d["ids"], d["mirror"], 1)
    assert np.array_equal(rp, d["rowptr1"]) and np.array_equal(cols, d["cols1"])
    if "rowptr2" in d:
        rp, cols = port.csr_pattern(d["off"], d["ids"], d["mirror"], 2)
        assert np.array_equal(rp, d["rowptr2"]) and np.array_equal(cols, d["cols2"])


@pytest.mark.parametrize("name,dim", FIXTURES[:4])
def test_gbuild_within_1e12(port, name, dim):
    d = load_golden(name)
    s = d["scalars"]
    ops, deg = port.gbuild(dim, 2, d["coords"], d["vols"], d["off"], d["ids"], s[0], s[4])
    assert np.array_equal(deg, d["degenerate"])
    assert scaled_err(ops, d["ops"], d["off"]) <= 1e-12


@pytest.mark.parametrize("name,dim", FIXTURES[:4])
def test_apply_within_1e12(port, name, dim):
    d = load_golden(name)
    out = port.apply(d["off"], d["ids"], d["ops"], d["u"])
    assert np.abs(out - d["apply"]).max() <= 1e-12 * np.abs(d["apply"]).max()


def test_poisson_assembly(port):
    d = load_golden("poisson16")
    kv, rhs = port.poisson_assemble(2, d["off"], d["ids"], d["ops"], [2, 4], 1.0, d["f"], d["u"], d["rowptr1"],
                                    d["cols1"])
    assert np.abs(kv - d["kvals"]).max() <= 1e-13 * np.abs(d["kvals"]).max()
    assert np.abs(rhs - d["rhs"]).max() <= 1e-13 * np.abs(d["rhs"]).max()


def navier(d, dim, port):
    if dim == 2:
        return d["opcache"][:, [2, 3, 4]]
    s = d["scalars"]
    ops, _ = port.gbuild(3, 2, d["coords"], d["vols"], d["off"], d["ids"], s[0], s[4])
    return ops[:, [3, 6, 8, 4, 5, 7]]


@pytest.mark.parametrize("name,dim", [("epf2d", 2), ("epf3d", 3)])
def test_crack_seed_matches_reference(port, name, dim):
    d = load_golden(name)
    cracks, planes, _ = crack_args(d)
    n = d["coords"].size // 3
    node = np.repeat(np.arange(n), np.diff(d["off"])) + 1
    cut = np.array([port.crack_cuts(d["coords"], d["mirror"], cracks, planes, i, j) for i, j in zip(node, d["ids"])])
    assert np.array_equal(~cut, d["health0"].astype(bool))


@pytest.mark.parametrize("name,dim", [("epf2d", 2), ("epf3d", 3)])
def test_epf_rate(port, name, dim):
    d = load_golden(name)
    sc, C11, C12, C66 = d["consts"][:4]
    a, h = port.epf_rate(dim, d["coords"], d["off"], d["ids"], navier(d, dim, port), (C11, C12, C66),
                         float(d["rho"]), np.zeros(dim), sc, d["u_rand"], d["health0"].astype(float))
    assert np.array_equal((h > 0).astype(np.uint8), d["health_rand"])
    assert np.abs(a - d["a_rand"]).max() <= 1e-13 * np.abs(d["a_rand"]).max()


def golden_bcs(d, dim):
    if dim == 2:
        y1, y2 = d["y_band"]
        bcs = [dict(kind="neumann", comps=[0, 1], nodes=d[g + "_ghosts"]) for g in ("left", "right", "bottom", "top")]
        bcs.append(dict(kind="dirichlet", comps=[0], nodes=d["left_ghosts"], value=[0, 0], velocity=[16.5, 0],
                        direct=True, box=[-1, 1, y1, y2, -1, 1]))
        return bcs
    Ly, h = float(d["Ly"]), float(d["h"])
    mir = d["mirror"]
    xyz = d["coords"].reshape(-1, 3)
    lo, hi = xyz[mir == 0].min(axis=0), xyz[mir == 0].max(axis=0)
    bcs = []
    for axis in range(3):
        for side, bound in ((0, lo[axis]), (1, hi[axis])):
            sel = (mir > 0) & ((xyz[:, axis] < bound) if side == 0 else (xyz[:, axis] > bound))
            bcs.append(dict(kind="neumann", comps=[0, 1, 2], nodes=np.nonzero(sel)[0] + 1))
    alld = np.arange(1, xyz.shape[0] + 1)
    bcs.append(dict(kind="dirichlet", comps=[1], nodes=alld, value=[0, 0, 0], velocity=[0, 2.0, 0], direct=True,
                    box=[-1, 1, Ly - 3 * h, 1, -1, 1]))
    bcs.append(dict(kind="dirichlet", comps=[1], nodes=alld, value=[0, 0, 0], velocity=[0, -2.0, 0], direct=True,
                    box=[-1, 1, -1, 3 * h, -1, 1]))
    return bcs


@pytest.mark.parametrize("name,dim", [("epf2d", 2), ("epf3d", 3)])
def test_epf_trajectory(port, name, dim):
    d = load_golden(name)
    sc, C11, C12, C66 = d["consts"][:4]
    n = d["coords"].size // 3
    u, uo, h = port.epf_run(dim, d["coords"], d["mirror"], d["off"], d["ids"], navier(d, dim, port), (C11, C12, C66),
                            float(d["rho"]), np.zeros(dim), sc, np.zeros(n * dim), None, float(d["dt"]),
                            int(d["nsteps"]), golden_bcs(d, dim), d["health0"].astype(float))
    assert np.array_equal((h > 0).astype(np.uint8), d["health"])
    assert np.abs(u - d["u"]).max() <= 1e-12 * np.abs(d["u"]).max()
    assert np.abs(uo - d["uold"]).max() <= 1e-12 * np.abs(d["u"]).max()


# ---- the reference's own known-answer tests (tests/ExplicitPDDOFracElementTests.cpp:96-154,
#      tests/InitialVelocityTests.cpp:78-90) -------------------------------------------------------------------
def nine_point():
    coords = np.array([[i, j, 0.0] for j in (-1, 0, 1) for i in (-1, 0, 1)], float)
    off = np.arange(0, 73, 8, dtype=np.int32)
    ids = np.array([j for i in range(1, 10) for j in range(1, 10) if j != i], np.int32)
    return coords, off, ids


def test_known_answers_explicit_element(port):
    coords, off, ids = nine_point()
    E, nu, rho = 100.0, 0.25, 4.0
    ops, deg = port.gbuild(2, 2, coords, np.ones(9), off, ids, 4.0, 0.0, volume_correction=False)
    assert deg.sum() == 0
    nav = ops[:, [2, 4, 3]]
    Cv = port.elastic_constants(2, True, E, nu)
    a, _ = port.epf_rate(2, coords, off, ids, nav, Cv, rho, np.array([8.0, -12.0]), 0.0, np.zeros(18), np.ones(72),
                         damage_on=False)
    assert abs(a[8] - 2.0) < 1e-11 and abs(a[9] + 3.0) < 1e-11
    c11 = E / (1 - nu * nu)
    assert abs(1.0 / math.sqrt(c11 / rho) - 1.0 / math.sqrt(Cv[0] / rho)) < 1e-15
    sc = port.critical_stretch(2, True, 1e-5, E, 4.0)
    u = 0.02 * coords[:, :2].ravel()
    a, h = port.epf_rate(2, coords, off, ids, nav, Cv, rho, np.zeros(2), sc, u, np.ones(72))
    assert 1.0 - h[off[4]:off[5]].mean() == 1.0
    a, h2 = port.epf_rate(2, coords, off, ids, nav, Cv, rho, np.zeros(2), sc, np.zeros(18), h)
    assert 1.0 - h2[off[4]:off[5]].mean() == 1.0 and abs(a[8]) == 0.0 and abs(a[9]) == 0.0


def test_known_answer_central_difference_start(port):
    coords, off, ids = nine_point()
    nav = np.zeros((72, 3))
    u, uo, h = port.epf_run(2, coords, None, off, ids, nav, (0.0, 0.0, 0.0), 1.0, np.zeros(2), 0.0, np.zeros(18),
                            np.full(18, 2.0), 0.1, 1, [], np.ones(72))
    assert np.abs(u - 0.2).max() < 1e-14


# ---- against the reference itself at config sizes (where the reference harness is built) -------------------
def _ref():
    from oracle import ref_available
    if not ref_available():
        pytest.skip("reference harness oracle/_ref/libperix_ref.so not built here")
    from oracle import RefMesh
    return RefMesh


def test_vs_reference_poisson64_full(port):
    RefMesh = _ref()
    m = RefMesh.structured(2, 64, 64, 0, [0, 1, 0, 1], 3.015, 2)
    assert m.n == 4352 and m.nb == 117172
    off, ids = port.families(m.coords, m.delta, False, mirror=m.mirror)
    assert np.array_equal(off, m.off) and np.array_equal(ids, m.ids)
    rp, cols = port.csr_pattern(off, ids, m.mirror, 1)
    rr, rc = m.csr_pattern(1)
    assert rp[-1] == 121524 and np.array_equal(rp, rr) and np.array_equal(cols, rc)
    g_ref, _ = m.gbuild()
    g, _ = port.gbuild(2, 2, m.coords, m.vols, off, ids, m.delta, m.dx_char)
    assert scaled_err(g, g_ref, off) <= 1e-12


def test_vs_reference_plate_families(port):
    RefMesh = _ref()
    h = 5e-4
    cracks = [[0.0, 0.05 - 25 * h, 50 * h, 0.05 - 25 * h], [0.0, 0.05 + 25 * h, 50 * h, 0.05 + 25 * h]]
    m = RefMesh.structured(2, 400, 200, 0, [0, 0.2, 0, 0.1], 3.015, 2, cracks=cracks, force_only=True)
    assert m.n == 81200 and m.nb == 2251924
    off, ids = port.families(m.coords, m.delta, False, cracks=cracks, mirror=m.mirror, force_only=True)
    assert np.array_equal(off, m.off) and np.array_equal(ids, m.ids)


def test_vs_reference_3d_slab_gbuild(port):
    RefMesh = _ref()
    m = RefMesh.structured(3, 16, 16, 6, [0, 0.016, 0, 0.016, 0, 0.006], 3.015, 2)
    off, ids = port.families(m.coords, m.delta, True, mirror=m.mirror)
    assert np.array_equal(off, m.off) and np.array_equal(ids, m.ids)
    g_ref, _ = m.gbuild()
    g, _ = port.gbuild(3, 2, m.coords, m.vols, off, ids, m.delta, m.dx_char)
    assert scaled_err(g, g_ref, off) <= 1e-12


@pytest.mark.skipif(not __import__("oracle").ref_available(), reason="reference harness not built here")
def test_poisson64_solve_with_reference_assembly():
    """The 64x64 Poisson workload with the reference's own Poisson assembly: the relative L2 error of the solved field against
    sin(pi x) sin(pi y) over the bulk nodes (the value the GPU path is held to)."""
    import math
    import perix_b200 as px
    from bench import poisson_solve
    from oracle import RefMesh
    m = RefMesh.structured(2, 64, 64, 0, [0, 1, 0, 1], 3.015, 2)
    m.gbuild()
    x, y = m.coords[0::3], m.coords[1::3]
    f = 2 * math.pi ** 2 * np.sin(math.pi * x) * np.sin(math.pi * y)
    kv, rhs, _ = m.poisson_assemble(1.0, f, np.zeros(m.n))
    rp, cols = m.csr_pattern(1)
    L = px.lattice(2, 64, 64, 0, [0.0, 1.0, 0.0, 1.0])
    _, err = poisson_solve(px, kv, rhs, L, rp, cols)
    assert abs(err - 1.4357e-3) <= 1e-6


@pytest.mark.parametrize("dim", [2, 3])
def test_stress_ch_restatement_vs_reference_element(dim):
    """The numpy restatement of the stress-coupled CH assembly (oracle/stress_ch.py) against the reference's
    StressCahnHilliardElement on its own operators, and against the committed fixture of the same mesh."""
    RefMesh = _ref()
    from conftest import load_golden
    from oracle.stress_ch import stress_ch_assemble
    d = load_golden("stressch%dd" % dim)
    if dim == 2:
        m = RefMesh.structured(2, 24, 24, 0, [0, 1, 0, 1], 3.015, 2)
    else:
        m = RefMesh.structured(3, 5, 5, 4, [0, 0.5, 0, 0.5, 0, 0.4], 3.015, 2)
    assert np.array_equal(m.off, d["off"]) and np.array_equal(m.ids, d["ids"])
    ops, _ = m.gbuild()
    E, nu, Omega, cref, D, chi, kappa, dt = (float(x) for x in d["params"])
    kv, rhs, geo, _ = m.stress_ch_assemble(E, nu, False, Omega, cref, D, chi, kappa, dt, d["u"], d["uold"])
    assert np.array_equal(kv, d["kvals"]) and np.array_equal(rhs, d["rhs"])
    C11, C12, C66, A, Kh, Ch = (float(x) for x in geo["consts"])
    prm = dict(C11=C11, C12=C12, C66=C66, A=A, Kh=Kh, Ch=Ch, Omega=Omega, cref=cref, chi=chi, kappa=kappa, dt=dt,
               kres=1e-8, rho=0.0)
    pqr = m.qindices()[0]
    ko, ro = stress_ch_assemble(dim, m.off, m.ids, ops, pqr, m.vols, geo["rev"], geo["lapbond"], geo["isghost"],
                                geo["mnode"], d["u"], d["uold"], d["rowptr"], d["cols"], prm)
    rp, cols = d["rowptr"], d["cols"]
    nd = dim + 2
    rows = np.repeat(np.arange(rp.size - 1), np.diff(rp))
    nbr = (cols // nd) != (rows // nd)
    ks = np.zeros(rp.size - 1)
    np.maximum.at(ks, rows[nbr], np.abs(kv[nbr]))
    assert (np.abs(ko - kv) <= 1e-12 * np.maximum(ks[rows], np.abs(kv))).all()
    du = d["u"][cols] - d["u"][(rows // nd) * nd + (cols % nd)]
    rs = np.zeros(rp.size - 1)
    np.maximum.at(rs, rows[nbr], np.abs(kv[nbr] * du[nbr]))
    assert (np.abs(ro - rhs) <= 1e-12 * np.maximum(rs, np.abs(rhs))).all()
