"""Generate the golden fixtures under tests/golden/ from the REFERENCE's own code.

Requires oracle/_ref/libperix_ref.so (built by `make -C oracle ref` from the reference sources), so it runs
where the reference tree is present; its outputs (*.npz) are committed and used by the tests everywhere.

    PYTHONPATH=. python tests/golden/make_golden.py

Every array saved here comes out of reference code: mesh generators + createPDMesh + createNeighborNodes,
PDOperators::calcAMatrix/calcOperators, SparseMatrix::initFromPDMesh, the PoissonElement bond callback in the
formResidualAndJacobianParallel loop, and ExplicitPDDOFracElement::preprocessIteration (with the
central-difference + BC restatement of ref_harness.cpp for trajectories).
"""
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import RefEpf, RefMesh  # noqa: E402


def save(name, **arrays):
    path = os.path.join(HERE, name + ".npz")
    np.savez_compressed(path, **arrays)
    print("wrote", path, "%.1f KB" % (os.path.getsize(path) / 1024))


def mesh_arrays(m):
    return dict(coords=m.coords, vols=m.vols, mirror=m.mirror, off=m.off, ids=m.ids,
                scalars=np.array([m.delta, m.dx, m.dy, m.dz, m.dx_char, m.nop]))


def poisson_fixture():
    """The Poisson workload at 16x16: sigma=1, f=2 pi^2 sin(pi x) sin(pi y), a random u."""
    m = RefMesh.structured(2, 16, 16, 0, [0, 1, 0, 1], 3.015, 2)
    ops, deg = m.gbuild()
    rp1, cols1 = m.csr_pattern(1)
    rp2, cols2 = m.csr_pattern(2)
    x = m.coords[0::3]
    y = m.coords[1::3]
    f = 2 * math.pi ** 2 * np.sin(math.pi * x) * np.sin(math.pi * y)
    rng = np.random.default_rng(11)
    u = rng.standard_normal(m.n)
    kv, rhs, _ = m.poisson_assemble(1.0, f, u)
    apply_u = m.apply(u)
    save("poisson16", **mesh_arrays(m), ops=ops, degenerate=deg, rowptr1=rp1, cols1=cols1, rowptr2=rp2,
         cols2=cols2, f=f, u=u, kvals=kv, rhs=rhs, apply=apply_u,
         groups=np.concatenate([m.group(g + "nodes_ghost") for g in ("left", "right", "bottom", "top")]))


def ch_fixture():
    """The Cahn-Hilliard workload scaled to a 32x32 lattice, h = 1/32, delta = 3.015h, c0 = 0.5 + U(-0.01, 0.01) (seeded), chi = 2.5,
    M0 = 1, kappa = 1e-4, dt = 1e-6; u = (c, mu) interleaved with mu = f'(c) plus noise; uold = u with c moved."""
    m = RefMesh.structured(2, 32, 32, 0, [0, 1, 0, 1], 3.015, 2)
    rp2, cols2 = m.csr_pattern(2)
    rng = np.random.default_rng(21)
    chi, kappa, M0, dt = 2.5, 1e-4, 1.0, 1e-6
    c = 0.5 + rng.uniform(-0.01, 0.01, m.n)
    mu = np.log(c / (1 - c)) + chi * (1 - 2 * c) + rng.standard_normal(m.n) * 1e-3
    u = np.stack([c, mu], 1).reshape(-1)
    uold = u.copy()
    uold[0::2] -= rng.uniform(-1e-4, 1e-4, m.n)
    kv, rhs, geo, _ = m.ch_assemble(chi, kappa, M0, dt, u, uold)
    save("ch32", **mesh_arrays(m), rowptr2=rp2, cols2=cols2, u=u, uold=uold,
         params=np.array([chi, kappa, M0, dt]), kvals=kv, rhs=rhs, **geo)


def stress_ch_fixture(dim):
    """Stress-coupled Cahn-Hilliard (ndof = dim + 2: c, mu, u) through the reference's StressCahnHilliardElement:
    2D 24x24 lattice on the unit square, 3D 5x5x4 on [0,0.5]x[0,0.5]x[0,0.4], delta = 3.015h, plane strain,
    E = 1e3, nu = 0.3, Omega = 0.05, cref = 0.5, D = 1, chi = 2.5, kappa = 1e-4, dt = 1e-6; c = 0.5 + U(+-0.05),
    mu = f'(c) plus noise, displacements N(0, (1e-3 h)^2) (seeded); uold = u with c moved."""
    if dim == 2:
        m = RefMesh.structured(2, 24, 24, 0, [0, 1, 0, 1], 3.015, 2)
        h = 1.0 / 24
    else:
        m = RefMesh.structured(3, 5, 5, 4, [0, 0.5, 0, 0.5, 0, 0.4], 3.015, 2)
        h = 0.1
    nd = dim + 2
    rp, cols = m.csr_pattern(nd)
    rng = np.random.default_rng(31 + dim)
    E, nu, Omega, cref, D, chi, kappa, dt = 1e3, 0.3, 0.05, 0.5, 1.0, 2.5, 1e-4, 1e-6
    c = 0.5 + rng.uniform(-0.05, 0.05, m.n)
    mu = np.log(c / (1 - c)) + chi * (1 - 2 * c) + rng.standard_normal(m.n) * 1e-3
    u = np.zeros((m.n, nd))
    u[:, 0] = c
    u[:, 1] = mu
    u[:, 2:] = rng.standard_normal((m.n, dim)) * 1e-3 * h
    u = u.reshape(-1)
    uold = u.copy()
    uold[0::nd] -= rng.uniform(-1e-4, 1e-4, m.n)
    kv, rhs, geo, _ = m.stress_ch_assemble(E, nu, False, Omega, cref, D, chi, kappa, dt, u, uold)
    save("stressch%dd" % dim, **mesh_arrays(m), rowptr=rp, cols=cols, u=u, uold=uold,
         params=np.array([E, nu, Omega, cref, D, chi, kappa, dt]), kvals=kv, rhs=rhs, **geo)


def dynfrac_fixture(dim):
    """Implicit PDDO dynamic fracture (ndof = dim) through the reference's PDDODynamicFracElement: 2D 20x20 on
    [0,0.2]^2, 3D 5x5x4 on [0,0.5]x[0,0.5]x[0,0.4], delta = 3.015h, plane strain, E = 190e9, nu = 0.3,
    rho = 8000, G0 = 2e4, dt = 1e-7, body force (1e3, -2e3, 5e2); uprev = 0, uold = a smooth stretch plus
    noise (amplitude 1.5e-3 in 2D, 5e-4 in 3D; noise 5e-5 h) that breaks part of the bonds at the commit,
    u = uold plus noise (seeded)."""
    if dim == 2:
        m = RefMesh.structured(2, 20, 20, 0, [0, 0.2, 0, 0.2], 3.015, 2)
        h = 0.01
    else:
        m = RefMesh.structured(3, 5, 5, 4, [0, 0.5, 0, 0.5, 0, 0.4], 3.015, 2)
        h = 0.1
    rp, cols = m.csr_pattern(dim)
    rng = np.random.default_rng(41 + dim)
    E, nu, rho, G0, dt = 190e9, 0.3, 8000.0, 2e4, 1e-7
    b = (1e3, -2e3, 5e2)
    x = m.coords.reshape(-1, 3)[:, :dim]
    uprev = np.zeros(m.n * dim)
    amp = 1.5e-3 if dim == 2 else 5e-4
    uold = (amp * x * x / x.max() + rng.standard_normal(x.shape) * 5e-5 * h).reshape(-1)
    u = uold + rng.standard_normal(m.n * dim) * 1e-4 * h
    kv, rhs, vel, health, consts = m.dynfrac_assemble(E, nu, rho, G0, dt, uprev, uold, u, b=b)
    save("dynfrac%dd" % dim, **mesh_arrays(m), rowptr=rp, cols=cols, uprev=uprev, uold=uold, u=u,
         params=np.array([E, nu, rho, G0, dt] + list(b)), kvals=kv, rhs=rhs, vel=vel, health=health, consts=consts)


def lattice3d_fixture():
    m = RefMesh.structured(3, 5, 5, 4, [0, 0.5, 0, 0.5, 0, 0.4], 3.015, 2)
    ops, deg = m.gbuild()
    rp1, cols1 = m.csr_pattern(1)
    rng = np.random.default_rng(12)
    u = rng.standard_normal(m.n)
    save("lattice3d", **mesh_arrays(m), ops=ops, degenerate=deg, rowptr1=rp1, cols1=cols1, u=u, apply=m.apply(u))


def cloud_fixture(dim, n_side, seed):
    """Jittered lattice cloud (no ghosts), uniform jitter +-0.2h, horizon 3.015h: boundary-truncated families."""
    rng = np.random.default_rng(seed)
    h = 1.0 / n_side
    g = (np.arange(n_side) + 0.5) * h
    if dim == 2:
        X, Y = np.meshgrid(g, g, indexing="xy")
        pts = np.stack([X.ravel(), Y.ravel(), np.zeros(X.size)], 1)
    else:
        X, Y, Z = np.meshgrid(g, g, g[: max(3, n_side // 2)], indexing="ij")
        pts = np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1)
    pts[:, :dim] += rng.uniform(-0.2 * h, 0.2 * h, size=(pts.shape[0], dim))
    vols = np.full(pts.shape[0], h ** dim)
    m = RefMesh.cloud(dim, pts.ravel(), vols, h, h, h if dim == 3 else 0.0, 3.015 * h, 2)
    ops, deg = m.gbuild()
    coef = rng.standard_normal(20)
    x, y, z = m.coords[0::3], m.coords[1::3], m.coords[2::3]
    u = cubic(coef, x, y, z, dim)
    save("cloud%dd" % dim, **mesh_arrays(m), ops=ops, degenerate=deg, u=u, coef=coef, apply=m.apply(u))


def cubic(c, x, y, z, dim):
    """Random cubic polynomial with coefficients c (N(0,1))."""
    if dim == 2:
        mons = [np.ones_like(x), x, y, x * x, x * y, y * y, x ** 3, x * x * y, x * y * y, y ** 3]
    else:
        mons = [np.ones_like(x), x, y, z, x * x, x * y, x * z, y * y, y * z, z * z, x ** 3, y ** 3, z ** 3,
                x * x * y, x * x * z, y * y * x, y * y * z, z * z * x, z * z * y, x * y * z]
    return sum(ci * mi for ci, mi in zip(c, mons))


def plate_bcs(m, dim, y_lo, y_hi, vx):
    """The notched-plate BCs, in list order: zero Neumann on every ghost wall, then a prescribed x-velocity (direct
    pin) on the left ghosts between the slits (it overrides the Neumann copy there)."""
    bcs = [dict(kind="neumann", comps=list(range(dim)), nodes=m.group(g + "nodes_ghost"))
           for g in ("left", "right", "bottom", "top")]
    bcs.append(dict(kind="dirichlet", comps=[0], nodes=m.group("leftnodes_ghost"), value=[0.0] * dim,
                    velocity=[vx] + [0.0] * (dim - 1), direct=True, box=[-1, 1, y_lo, y_hi, -1, 1]))
    return bcs


def epf2d_fixture():
    """The notched plate scaled to 40x20 nodes, h=0.5 mm, two force-only slits of 5h at y = Ly/2 +- 2.5h, 16.5 m/s pull."""
    nx, ny, h = 40, 20, 5e-4
    Lx, Ly = nx * h, ny * h
    y1, y2 = Ly / 2 - 2.5 * h, Ly / 2 + 2.5 * h
    cracks = [[0.0, y1, 5 * h, y1], [0.0, y2, 5 * h, y2]]
    m = RefMesh.structured(2, nx, ny, 0, [0, Lx, 0, Ly], 3.015, 2, cracks=cracks, force_only=True)
    E, nu, rho, sc = 190e9, 0.3, 8000.0, 0.01
    G0 = sc * sc * 12 * E * m.delta / (5 * math.pi)
    el = RefEpf(m, E, nu, rho, G0, plane_stress=False)
    bcs = plate_bcs(m, 2, y1, y2, 16.5)
    u0 = np.zeros(2 * m.n)
    a0, h0, _ = el.rate(u0)                       # seeds force-only notch health, a at rest
    consts = el.constants()
    dt = 0.8 * h / math.sqrt(consts["C11"] / rho)
    opc = el.opcache()
    # a rate at a random displacement field (same seeded health)
    rng = np.random.default_rng(21)
    ur = rng.standard_normal(2 * m.n) * 1e-6
    el2 = RefEpf(m, E, nu, rho, G0, plane_stress=False)
    ar, hr, _ = el2.rate(ur)
    # trajectory
    el3 = RefEpf(m, E, nu, rho, G0, plane_stress=False)
    nsteps = 60
    u, uo, hh, _ = el3.run(u0, None, dt, nsteps, bcs)
    save("epf2d", **mesh_arrays(m), cracks=np.array(cracks), E=E, nu=nu, rho=rho, G0=G0,
         consts=np.array([consts["sc"], consts["C11"], consts["C12"], consts["C66"], consts["stable_dt"]]), dt=dt,
         y_band=np.array([y1, y2]), health0=(h0 > 0).astype(np.uint8), a0=a0, opcache=opc, u_rand=ur, a_rand=ar,
         health_rand=(hr > 0).astype(np.uint8), nsteps=nsteps, u=u, uold=uo, health=(hh > 0).astype(np.uint8),
         left_ghosts=m.group("leftnodes_ghost"), right_ghosts=m.group("rightnodes_ghost"),
         bottom_ghosts=m.group("bottomnodes_ghost"), top_ghosts=m.group("topnodes_ghost"))


def slab_bcs(m, Ly, h):
    """The notched-slab BCs, in list order: zero Neumann on every ghost wall, then +-2 m/s y-velocity pins (direct) on
    every node (bulk and ghost) of the top and bottom three-layer strips."""
    bcs = [dict(kind="neumann", comps=[0, 1, 2], nodes=m.group(g + "nodes_ghost"))
           for g in ("left", "right", "bottom", "top", "back", "front")]
    bcs.append(dict(kind="dirichlet", comps=[1], nodes=m.group("alldomain"), value=[0, 0, 0], velocity=[0, 2.0, 0],
                    direct=True, box=[-1, 1, Ly - 3 * h, 1, -1, 1]))
    bcs.append(dict(kind="dirichlet", comps=[1], nodes=m.group("alldomain"), value=[0, 0, 0], velocity=[0, -2.0, 0],
                    direct=True, box=[-1, 1, -1, 3 * h, -1, 1]))
    return bcs


def epf3d_fixture():
    """The notched slab scaled to 10x10x4 nodes, h=1 mm, central edge notch plane (force-only), +-2 m/s on top/bottom layers."""
    nx, ny, nz, h = 10, 10, 4, 1e-3
    Lx, Ly, Lz = nx * h, ny * h, nz * h
    plane = [0.0, Ly / 2, -1.0, 3 * h, Ly / 2, -1.0, 3 * h, Ly / 2, 1.0, 0.0, Ly / 2, 1.0]
    m = RefMesh.structured(3, nx, ny, nz, [0, Lx, 0, Ly, 0, Lz], 3.015, 2, planes=[plane], force_only=True)
    E, nu, rho, sc = 72e9, 0.22, 2440.0, 0.004
    G0 = sc * sc * 6 * E * m.delta / 5
    el = RefEpf(m, E, nu, rho, G0)
    bcs = slab_bcs(m, Ly, h)
    u0 = np.zeros(3 * m.n)
    a0, h0, _ = el.rate(u0)
    consts = el.constants()
    dt = 0.8 * h / math.sqrt(consts["C11"] / rho)
    rng = np.random.default_rng(31)
    ur = rng.standard_normal(3 * m.n) * 2e-6
    el2 = RefEpf(m, E, nu, rho, G0)
    ar, hr, _ = el2.rate(ur)
    el3 = RefEpf(m, E, nu, rho, G0)
    nsteps = 40
    u, uo, hh, _ = el3.run(u0, None, dt, nsteps, bcs)
    save("epf3d", **mesh_arrays(m), plane=np.array(plane), E=E, nu=nu, rho=rho, G0=G0,
         consts=np.array([consts["sc"], consts["C11"], consts["C12"], consts["C66"], consts["stable_dt"]]), dt=dt,
         health0=(h0 > 0).astype(np.uint8), a0=a0, u_rand=ur, a_rand=ar, health_rand=(hr > 0).astype(np.uint8),
         nsteps=nsteps, u=u, uold=uo, health=(hh > 0).astype(np.uint8), Ly=Ly, h=h)


if __name__ == "__main__":
    poisson_fixture()
    lattice3d_fixture()
    cloud_fixture(2, 24, 7)
    cloud_fixture(3, 8, 8)
    epf2d_fixture()
    epf3d_fixture()
    ch_fixture()
    stress_ch_fixture(2)
    stress_ch_fixture(3)
    dynfrac_fixture(2)
    dynfrac_fixture(3)
