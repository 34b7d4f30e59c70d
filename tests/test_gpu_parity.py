"""GPU parity: perix_b200 kernels (through the C-ABI) against the golden fixtures made by the reference's own
code and against the C restatement (oracle) at sizes it finishes in seconds.

Tolerances: g-functions and operator applies within 1e-12 relative in FP64 (relative to the
operator's own magnitude over the family); mixed precision within 1e-6; families/CSR bit-exact; damage sets
identical except bonds whose stretch lies within 1e-9 of critical; explicit trajectories within 1e-10 relative
(60 central-difference steps accumulate round-off from the reordered family sums)."""
import math

import numpy as np
import pytest

from conftest import load_golden, scaled_err

pytestmark = pytest.mark.gpu

G_TOL64 = 1e-12
G_TOLMIX = 1e-6


def geometry(ctx, d, dim):
    s = d["scalars"]
    ctx.set_geometry(d["coords"], d["vols"], d["off"], d["ids"], s[0], s[4], dim, mirror=d["mirror"])


@pytest.mark.parametrize("name,dim", [("poisson16", 2), ("lattice3d", 3), ("cloud2d", 2), ("cloud3d", 3)])
def test_gbuild_fp64_matches_reference(ctx, name, dim):
    d = load_golden(name)
    geometry(ctx, d, dim)
    nd, first = ctx.gbuild(2, 0)
    assert nd == 0
    g = ctx.get_ops()
    assert g.shape == d["ops"].shape
    assert scaled_err(g, d["ops"], d["off"]) <= G_TOL64


@pytest.mark.parametrize("name,dim", [("poisson16", 2), ("lattice3d", 3), ("cloud2d", 2), ("cloud3d", 3)])
def test_gbuild_mixed_within_1e6(ctx, name, dim):
    d = load_golden(name)
    geometry(ctx, d, dim)
    ctx.gbuild(2, 1)
    g = ctx.get_ops()
    assert scaled_err(g, d["ops"], d["off"]) <= G_TOLMIX


def test_gbuild_poisson64_full_size_vs_oracle(ctx, port):
    import perix_b200 as px
    L = px.lattice(2, 64, 64, 0, [0, 1, 0, 1])
    delta = 3.015 * L.dxyz[0] * (1 + 1e-6)
    off, ids = px.families(L.coords, delta, False, mirror=L.mirror)
    ctx.set_geometry(L.coords, L.vols, off, ids, delta, L.dxyz[0], 2, mirror=L.mirror)
    ctx.gbuild(2, 0)
    g = ctx.get_ops()
    ref, deg = port.gbuild(2, 2, L.coords, L.vols, off, ids, delta, L.dxyz[0])
    assert deg.sum() == 0
    assert scaled_err(g, ref, off) <= G_TOL64


@pytest.mark.parametrize("name,dim", [("poisson16", 2), ("lattice3d", 3), ("cloud2d", 2), ("cloud3d", 3)])
def test_apply_and_adjoint(ctx, port, name, dim):
    d = load_golden(name)
    geometry(ctx, d, dim)
    ctx.gbuild(2, 0)
    nop = d["ops"].shape[1]
    slots = np.arange(nop, dtype=np.int32)
    out = ctx.apply(d["u"], slots)
    # per-node scale: sum_t |g| |u_j - u_i|
    du = np.abs(d["u"][d["ids"] - 1] - np.repeat(d["u"], np.diff(d["off"])))
    scale = np.zeros((d["off"].size - 1, nop))
    np.add.at(scale, np.repeat(np.arange(d["off"].size - 1), np.diff(d["off"])), np.abs(d["ops"]) * du[:, None])
    err = np.abs(out - d["apply"]) / np.maximum(scale, 1e-300)
    assert err.max() <= G_TOL64
    # adjoint: <A u, y> == <u, A^T y>
    rng = np.random.default_rng(5)
    y = rng.standard_normal(out.shape)
    ubar = ctx.apply_adjoint(y, slots)
    lhs = float((out * y).sum())
    rhs = float((d["u"] * ubar).sum())
    assert abs(lhs - rhs) <= 1e-11 * (abs(lhs) + np.abs(out * y).sum())


@pytest.mark.parametrize("name,dim", [("cloud2d", 2), ("cloud3d", 3), ("lattice3d", 3)])
def test_apply_mixed_error_stated(ctx, name, dim):
    """Mixed apply (FP32-stored g widened to FP64 for the products, second derivatives corrected by the
    first-moment defect of their stored operators) against the FP64 reference, slot by slot relative to the
    slot's largest value: first and second derivatives within 1e-6."""
    d = load_golden(name)
    geometry(ctx, d, dim)
    ctx.gbuild(2, 1)
    nop = d["ops"].shape[1]
    out = ctx.apply(d["u"], np.arange(nop, dtype=np.int32))
    rel = np.abs(out - d["apply"]).max(axis=0) / np.abs(d["apply"]).max(axis=0)
    assert rel.max() <= G_TOLMIX


@pytest.mark.parametrize("slots", [[0, 1, 2, 3, 4], [3], [1, 4, 2]])
def test_apply_mixed_adjoint_is_transpose(ctx, slots):
    """With the defect correction the mixed forward is G u - C (G1 u); its adjoint must be the exact transpose,
    also when the first-derivative slots are not among the requested ones."""
    d = load_golden("cloud2d")
    geometry(ctx, d, 2)
    ctx.gbuild(2, 1)
    s = np.asarray(slots, np.int32)
    out = ctx.apply(d["u"], s)
    y = np.random.default_rng(8).standard_normal(out.shape)
    ubar = ctx.apply_adjoint(y, s)
    lhs, rhs = float((out * y).sum()), float((d["u"] * ubar).sum())
    assert abs(lhs - rhs) <= 1e-11 * np.abs(out * y).sum()


def test_ch_assembly_matches_reference(ctx):
    """Conservative Cahn-Hilliard (2 dof) K and rhs against the reference element (CahnHilliardElement
    preprocess + callbacks in the formResidualAndJacobianParallel accumulation), on the element's own geometry
    (lambda-corrected Laplacian, reverse bonds, ghost flags) and Picard mobility.  K entries within 1e-12 of the
    row's largest neighbour-block entry (the 1/dt diagonal would otherwise hide the bond terms), rhs within
    1e-12 of its largest entry."""
    d = load_golden("ch32")
    geometry(ctx, d, 2)
    ctx.csr_set_pattern(d["rowptr2"], d["cols2"], 2)
    ctx.ch_set_geometry(d["rev"], d["lapbond"], d["isghost"])
    chi, kappa, M0, dt = (float(x) for x in d["params"])
    kv, rhs = ctx.assemble_ch(kappa, chi, dt, d["mnode"], d["u"], d["uold"])
    rp, cols, ref = d["rowptr2"], d["cols2"], d["kvals"]
    rows = np.repeat(np.arange(rp.size - 1), np.diff(rp))
    nbr_block = (cols // 2) != (rows // 2)
    scale = np.zeros(rp.size - 1)
    np.maximum.at(scale, rows[nbr_block], np.abs(ref[nbr_block]))
    assert (np.abs(kv - ref) <= 1e-12 * scale[rows]).all()
    assert np.abs(rhs - d["rhs"]).max() <= 1e-12 * np.abs(d["rhs"]).max()


def test_ch_device_geometry_and_mobility(ctx):
    """The CH geometry and mobility built on the device (pxb_ch_build_geometry, pxb_ch_mobility_d) against the
    reference element's own arrays, then the whole assembly from them against the reference K and rhs."""
    import torch
    d = load_golden("ch32")
    geometry(ctx, d, 2)
    ctx.gbuild(2, 0)
    ctx.ch_build_geometry()
    rev, lap, ghost = ctx.ch_get_geometry()
    assert np.array_equal(rev, d["rev"]) and np.array_equal(ghost, d["isghost"])
    assert scaled_err(lap.reshape(-1, 1), d["lapbond"].reshape(-1, 1), d["off"]) <= 1e-12
    chi, kappa, M0, dt = (float(x) for x in d["params"])
    dev = torch.device("cuda", 0)
    ctx.set_stream(torch.cuda.current_stream(dev).cuda_stream)
    u = torch.from_numpy(d["u"]).to(dev)
    uo = torch.from_numpy(d["uold"]).to(dev)
    mn = torch.empty(ctx.n, dtype=torch.float64, device=dev)
    ctx.ch_mobility_d(M0, u.data_ptr(), mn.data_ptr())
    assert np.abs(mn.cpu().numpy() - d["mnode"]).max() <= 1e-15
    ctx.csr_set_pattern(d["rowptr2"], d["cols2"], 2)
    kv = torch.empty(d["kvals"].size, dtype=torch.float64, device=dev)
    rhs = torch.empty(2 * ctx.n, dtype=torch.float64, device=dev)
    ctx.assemble_ch_d(kappa, chi, dt, mn.data_ptr(), u.data_ptr(), uo.data_ptr(), kv.data_ptr(), rhs.data_ptr())
    torch.cuda.synchronize(dev)
    rp, cols, ref = d["rowptr2"], d["cols2"], d["kvals"]
    rows = np.repeat(np.arange(rp.size - 1), np.diff(rp))
    nbr_block = (cols // 2) != (rows // 2)
    scale = np.zeros(rp.size - 1)
    np.maximum.at(scale, rows[nbr_block], np.abs(ref[nbr_block]))
    assert (np.abs(kv.cpu().numpy() - ref) <= 1e-12 * scale[rows]).all()
    assert np.abs(rhs.cpu().numpy() - d["rhs"]).max() <= 1e-12 * np.abs(d["rhs"]).max()


def test_poisson64_solve_l2_error(ctx, port):
    """The 64x64 Poisson problem end to end: 64x64 lattice, order 2, FP64 g-build and Poisson assembly on the GPU, the
    reference's Dirichlet row replacement on the ghost layer, one solve.  The solution matches the solve of the
    C restatement's assembly of the same system (1e-9) and the relative L2 error against sin(pi x) sin(pi y) is
    the reference's (1.44e-3 with the reference's own assembly, tests/test_oracle.py)."""
    import perix_b200 as px
    from bench import poisson_solve
    L = px.lattice(2, 64, 64, 0, [0.0, 1.0, 0.0, 1.0])
    delta = 3.015 * L.dxyz[0] * (1 + 1e-6)
    off, ids = px.families(L.coords, delta, False, mirror=L.mirror)
    rowptr, cols = px.csr_pattern(off, ids, L.mirror, 1)
    ctx.set_geometry(L.coords, L.vols, off, ids, delta, L.dxyz[0], 2, mirror=L.mirror)
    ctx.gbuild(2, 0)
    ctx.csr_set_pattern(rowptr, cols, 1)
    x, y = L.coords[0::3], L.coords[1::3]
    f = 2 * math.pi ** 2 * np.sin(math.pi * x) * np.sin(math.pi * y)
    kv, rhs = ctx.assemble_scalar(0, 1.0, np.zeros(L.n), f_node=f)
    U, err = poisson_solve(px, kv, rhs, L, rowptr, cols)
    g, _ = port.gbuild(2, 2, L.coords, L.vols, off, ids, delta, L.dxyz[0])
    kv_o, rhs_o = port.poisson_assemble(2, off, ids, g, [2, 4], 1.0, f, np.zeros(L.n), rowptr, cols)
    U_o, err_o = poisson_solve(px, kv_o, rhs_o, L, rowptr, cols)
    assert np.abs(U - U_o).max() <= 1e-9
    assert abs(err - 1.4357e-3) <= 1e-6 and abs(err - err_o) <= 1e-9


def test_poisson_assembly_matches_reference(ctx):
    d = load_golden("poisson16")
    geometry(ctx, d, 2)
    ctx.gbuild(2, 0)
    ctx.csr_set_pattern(d["rowptr1"], d["cols1"], 1)
    kv, rhs = ctx.assemble_scalar(0, 1.0, d["u"], f_node=d["f"])
    assert np.abs(kv - d["kvals"]).max() <= 1e-12 * np.abs(d["kvals"]).max()
    assert np.abs(rhs - d["rhs"]).max() <= 1e-12 * np.abs(d["rhs"]).max()


# ---------------------------------------------------------------------------------------- explicit fracture
def epf_context(ctx, d, dim, precision=0):
    geometry(ctx, d, dim)
    sc, C11, C12, C66 = d["consts"][:4]
    ctx.epf_setup(C11, C12, C66, float(d["rho"]), (0, 0, 0), sc, True, health0=d["health0"], precision=precision)
    return sc


def plate_bcs(d, px):
    y1, y2 = d["y_band"]
    bcs = [px.BC("neumann", [0, 1], d[g + "_ghosts"]) for g in ("left", "right", "bottom", "top")]
    bcs.append(px.BC("dirichlet", [0], d["left_ghosts"], value=[0, 0], velocity=[16.5, 0], direct=True,
                     box=[-1, 1, y1, y2, -1, 1]))
    return bcs


def slab_bcs(d, px, mesh_n):
    Ly, h = float(d["Ly"]), float(d["h"])
    import perix_b200.api as api  # noqa: F401
    mir = d["mirror"]
    # ghost groups from the mirror map + coordinates (ghosts sit outside the box faces)
    xyz = d["coords"].reshape(-1, 3)
    lo = xyz[mir == 0].min(axis=0)
    hi = xyz[mir == 0].max(axis=0)
    bcs = []
    for axis in range(3):
        for side, bound in ((0, lo[axis]), (1, hi[axis])):
            sel = (mir > 0) & ((xyz[:, axis] < bound) if side == 0 else (xyz[:, axis] > bound))
            bcs.append(px.BC("neumann", [0, 1, 2], np.nonzero(sel)[0] + 1))
    alld = np.arange(1, mesh_n + 1)
    bcs.append(px.BC("dirichlet", [1], alld, value=[0, 0, 0], velocity=[0, 2.0, 0], direct=True,
                     box=[-1, 1, Ly - 3 * h, 1, -1, 1]))
    bcs.append(px.BC("dirichlet", [1], alld, value=[0, 0, 0], velocity=[0, -2.0, 0], direct=True,
                     box=[-1, 1, -1, 3 * h, -1, 1]))
    return bcs


@pytest.mark.parametrize("variant", list(range(21)))
@pytest.mark.parametrize("name,dim", [("epf2d", 2), ("epf3d", 3)])
def test_epf_rate_matches_reference(ctx, name, dim, variant):
    """The per-step drop-in call on every schedule variant (the staged ones run their RATE epilogue)."""
    import perix_b200 as px
    d = load_golden(name)
    epf_context(ctx, d, dim)
    try:
        ctx.epf_set_variant(variant)
    except px.PxbError as e:
        assert e.status == 7  # families too large for this tile size
        pytest.skip("variant %d does not fit these families" % variant)
    a, nbk = ctx.epf_rate(d["u_rand"])
    _, _, h, _ = ctx.epf_state()
    assert np.array_equal(h, d["health_rand"])
    assert nbk == int((d["health0"] == 1).sum() - (d["health_rand"] == 1).sum())
    assert np.abs(a - d["a_rand"]).max() <= 1e-12 * np.abs(d["a_rand"]).max()


@pytest.mark.parametrize("variant", list(range(21)))
@pytest.mark.parametrize("name,dim", [("epf2d", 2), ("epf3d", 3)])
def test_epf_trajectory_matches_reference(ctx, name, dim, variant):
    """Every schedule variant of the step kernel (lane groups, CSR-stream tiles, TMA-staged tiles)."""
    import perix_b200 as px
    d = load_golden(name)
    epf_context(ctx, d, dim)
    try:
        ctx.epf_set_variant(variant)
    except px.PxbError as e:
        assert e.status == 7  # families too large for this tile size
        pytest.skip("variant %d does not fit these families" % variant)
    n = d["coords"].size // 3
    bcs = plate_bcs(d, px) if dim == 2 else slab_bcs(d, px, n)
    ctx.epf_set_bcs(bcs)
    ctx.epf_start(np.zeros(n * dim), None, float(d["dt"]))
    ctx.epf_advance(int(d["nsteps"]), chunk=16)
    u, uo, h, t = ctx.epf_state()
    assert np.array_equal(h, d["health"])
    scale = np.abs(d["u"]).max()
    assert np.abs(u - d["u"]).max() <= 1e-10 * scale
    assert np.abs(uo - d["uold"]).max() <= 1e-10 * scale


def test_epf_mixed_close_to_fp64(ctx):
    import perix_b200 as px
    d = load_golden("epf2d")
    n = d["coords"].size // 3
    res = {}
    for prec in (0, 1):
        epf_context(ctx, d, 2, precision=prec)
        ctx.epf_set_bcs(plate_bcs(d, px))
        ctx.epf_start(np.zeros(n * 2), None, float(d["dt"]))
        ctx.epf_advance(int(d["nsteps"]))
        res[prec] = ctx.epf_state()
    u64, u32 = res[0][0], res[1][0]
    assert np.abs(u32 - u64).max() <= 1e-6 * np.abs(u64).max()


def test_known_answers_nine_point(ctx):
    """Reference tests/ExplicitPDDOFracElementTests.cpp:96-154 on the nine-point all-to-all mesh."""
    import perix_b200 as px
    coords = np.array([[i, j, 0.0] for j in (-1, 0, 1) for i in (-1, 0, 1)], float)
    off = np.arange(0, 73, 8, dtype=np.int32)
    ids = np.array([j for i in range(1, 10) for j in range(1, 10) if j != i], np.int32)
    ctx.set_geometry(coords, np.ones(9), off, ids, 4.0, 0.0, 2)
    E, nu, rho = 100.0, 0.25, 4.0
    C11, C12, C66 = px.elastic_constants(2, True, E, nu)
    ctx.epf_setup(C11, C12, C66, rho, (8.0, -12.0, 0.0), 0.0, True)
    a, _ = ctx.epf_rate(np.zeros(18))
    assert abs(a[8] - 2.0) < 1e-12 and abs(a[9] + 3.0) < 1e-12
    sc = px.critical_stretch(2, True, 1e-5, E, 4.0)
    ctx.epf_setup(C11, C12, C66, rho, (0, 0, 0), sc, True)
    a, nbk = ctx.epf_rate(0.02 * coords[:, :2].ravel())
    _, _, h, _ = ctx.epf_state()
    assert h[off[4]:off[5]].sum() == 0                      # damage 1.0 at the centre node
    a, _ = ctx.epf_rate(np.zeros(18))                       # irreversible
    _, _, h2, _ = ctx.epf_state()
    assert h2[off[4]:off[5]].sum() == 0
    assert abs(a[8]) < 1e-300 and abs(a[9]) < 1e-300


def test_central_difference_start(ctx):
    """Reference tests/InitialVelocityTests.cpp:78-90: v0=2, dt=0.1, zero acceleration -> u=0.2 after a step."""
    coords = np.array([[i, j, 0.0] for j in (-1, 0, 1) for i in (-1, 0, 1)], float)
    off = np.arange(0, 73, 8, dtype=np.int32)
    ids = np.array([j for i in range(1, 10) for j in range(1, 10) if j != i], np.int32)
    ctx.set_geometry(coords, np.ones(9), off, ids, 4.0, 0.0, 2)
    ctx.epf_setup(0.0, 0.0, 0.0, 1.0, (0, 0, 0), 0.0, True)   # zero stiffness: a = 0
    ctx.epf_start(np.zeros(18), np.full(18, 2.0), 0.1)
    ctx.epf_advance(1)
    u, _, _, t = ctx.epf_state()
    assert np.allclose(u, 0.2, atol=1e-14, rtol=0)
    assert abs(t - 0.1) < 1e-15


def _device_families_case(name):
    import perix_b200 as px
    from bench import clouds_generate
    if name == "plate2d":
        from bench import plate_setup
        w = plate_setup(px)
        return w["L"].coords, w["L"].vols, w["delta"], 2, w["L"].mirror
    if name == "slab3d":
        from bench import slab_setup
        w = slab_setup(px, nx=30, ny=30, nz=10)
        return w["L"].coords, w["L"].vols, w["delta"], 3, w["L"].mirror
    if name == "poisson64":
        L = px.lattice(2, 64, 64, 0, [0.0, 1.0, 0.0, 1.0])
        return L.coords, L.vols, 3.015 * L.dxyz[0] * (1 + 1e-6), 2, L.mirror
    cl = clouds_generate(px, nclouds=2, nmin=3000, nmax=6000, seed=3)[0 if name == "cloud2d" else 1]
    return cl["coords3"], cl["vols"], cl["delta"], cl["dim"], None


@pytest.mark.parametrize("name", ["plate2d", "slab3d", "poisson64", "cloud2d", "cloud3d"])
def test_device_families_equal_host(ctx, name):
    """Families built on the device (pxb_set_geometry_points) equal the host build (pxb_families, itself bit-equal
    to the reference's createNeighborNodes): same offsets, same ids in the same order."""
    import perix_b200 as px
    coords, vols, delta, dim, mirror = _device_families_case(name)
    off_h, ids_h = px.families(coords, delta, dim == 3, mirror=mirror)
    ctx.set_geometry_points(coords, vols, delta, delta, delta / 3.015, dim, mirror=mirror)
    off_d, ids_d = ctx.get_families()
    assert np.array_equal(off_d, off_h)
    assert np.array_equal(ids_d, ids_h)
