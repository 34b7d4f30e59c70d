"""Test infrastructure only (the oracle): a numpy restatement of the stress-coupled Cahn-Hilliard assembly.

It follows the reference's StressCahnHilliardElement (src/ElmtSystem/StressCahnHilliardElement.cpp:282-466, bond
and nodal callbacks) together with the fracture gate and inertia of its device assembler
(src/PDSystem/CudaAssembleKernels.cu:685-874: mechanical operators scaled by 1 or kres per bond,
-rho (u - u_old - v dt)/dt^2 on the displacement rows).  Bonds are row-owned and accumulated in family order,
as PDSystem::formResidualAndJacobianParallel does (FormResidualAndJacobianParallel.cpp:114-171); the bond block
K_IJ is stored per bond and K_II = -K_IJ summed into the diagonal block with the nodal Jacobian.
Sign convention K = -dF/dU, rhs = +F.  Only tests import it.
"""
import numpy as np


def _slot(pqr, p, q, r):
    for k, t in enumerate(pqr):
        if tuple(t) == (p, q, r):
            return k
    raise KeyError((p, q, r))


def stress_ch_assemble(dim, off, ids, ops, pqr, vols, rev, lapbond, isghost, mnode, u, uold, rowptr, cols, prm,
                       health=None, vel=None):
    """off/ids: family CSR (ids 1-based); ops[nb, nop] FP64 g-functions with multi-indices pqr; prm: dict with
    C11 C12 C66 A Kh Ch Omega cref chi kappa dt kres rho.  Returns (kvals, rhs)."""
    nd = dim + 2
    off = np.asarray(off, np.int64)
    n = off.size - 1
    nb = int(off[-1])
    i = np.repeat(np.arange(n), np.diff(off))
    j = np.asarray(ids, np.int64)[:nb] - 1
    ops = np.asarray(ops, np.float64).reshape(nb, -1)
    u = np.asarray(u, np.float64).reshape(n, nd)
    uold = np.zeros_like(u) if uold is None else np.asarray(uold, np.float64).reshape(n, nd)
    g = np.ones(nb) if health is None else np.where(np.asarray(health) > 0.0, 1.0, prm["kres"])
    G = lambda p, q, r: g * ops[:, _slot(pqr, p, q, r)]
    G1 = [G(1, 0, 0), G(0, 1, 0)] + ([G(0, 0, 1)] if dim == 3 else [])
    Gxx, Gxy, Gyy = G(2, 0, 0), G(1, 1, 0), G(0, 2, 0)
    vols = np.asarray(vols, np.float64)
    mnode = np.asarray(mnode, np.float64)
    lap = np.asarray(lapbond, np.float64)
    rev = np.asarray(rev, np.int64)
    ghostJ = np.asarray(isghost)[j] != 0
    Vi, Vj, Mi, Mj = vols[i], vols[j], mnode[i], mnode[j]
    paired = (rev >= 0) & (Vi > 0.0)
    lap_rev = lap[np.where(rev >= 0, rev, 0)]
    with np.errstate(divide="ignore", invalid="ignore"):
        w = np.where(paired, 0.5 * (Mi * lap + (Vj / np.where(Vi > 0, Vi, 1.0)) * Mj * lap_rev), Mi * lap)
    coeff_c = np.where(ghostJ, 0.0, -w)
    kappa_lap = np.where(ghostJ, 0.0, prm["kappa"] * lap)
    K = np.zeros((nb, nd, nd))
    K[:, 0, 1] = coeff_c
    K[:, 1, 0] = kappa_lap
    for d in range(dim):
        K[:, 1, 2 + d] = prm["Omega"] * prm["Kh"] * G1[d]
        K[:, 2 + d, 0] = -prm["A"] * G1[d]
    C11, C12, C66 = prm["C11"], prm["C12"], prm["C66"]
    if dim == 2:
        K[:, 2, 2] = C11 * Gxx + C66 * Gyy
        K[:, 3, 3] = C66 * Gxx + C11 * Gyy
        K[:, 2, 3] = K[:, 3, 2] = (C12 + C66) * Gxy
    else:
        Gzz, Gxz, Gyz = G(0, 0, 2), G(1, 0, 1), G(0, 1, 1)
        a = C12 + C66
        K[:, 2, 2] = C11 * Gxx + C66 * (Gyy + Gzz)
        K[:, 3, 3] = C11 * Gyy + C66 * (Gxx + Gzz)
        K[:, 4, 4] = C11 * Gzz + C66 * (Gxx + Gyy)
        K[:, 2, 3] = K[:, 3, 2] = a * Gxy
        K[:, 2, 4] = K[:, 4, 2] = a * Gxz
        K[:, 3, 4] = K[:, 4, 3] = a * Gyz
    du = u[j] - u[i]
    R = np.einsum("tab,tb->ta", K, du)
    # nodal terms (regular-solution free energy with swelling; optional inertia)
    c, mu, cold = u[:, 0], u[:, 1], uold[:, 0]
    cc = np.clip(c, 1e-8, 1 - 1e-8)
    fp = np.log(cc / (1 - cc)) + prm["chi"] * (1 - 2 * cc)
    fpp = 1 / (cc * (1 - cc)) - 2 * prm["chi"]
    dt = prm["dt"]
    rl = np.zeros((n, nd))
    kii = np.zeros((n, nd, nd))
    rl[:, 0] = (c - cold) / dt
    rl[:, 1] = mu - fp + prm["Omega"] * prm["Ch"] * (c - prm["cref"])
    kii[:, 0, 0] = -(1.0 / dt)
    kii[:, 1, 0] = -(-fpp + prm["Omega"] * prm["Ch"])
    kii[:, 1, 1] = -1.0
    if prm.get("rho", 0.0) > 0.0 and vel is not None:
        c0 = prm["rho"] / (dt * dt)
        v = np.asarray(vel, np.float64).reshape(n, dim)
        for d in range(dim):
            rl[:, 2 + d] += -c0 * (u[:, 2 + d] - uold[:, 2 + d] - v[:, d] * dt)
            kii[:, 2 + d, 2 + d] += c0
    np.add.at(rl, i, R)
    np.add.at(kii, i, K)
    # scatter into the CSR: bond blocks -K_IJ, diagonal blocks kii
    rowptr = np.asarray(rowptr, np.int64)
    cols = np.asarray(cols, np.int64)
    ncol = n * nd
    keys = np.repeat(np.arange(rowptr.size - 1), np.diff(rowptr)) * ncol + cols
    kv = np.zeros(cols.size)
    a_idx, b_idx = np.meshgrid(np.arange(nd), np.arange(nd), indexing="ij")
    rk = (i[:, None, None] * nd + a_idx[None]) * ncol + (j[:, None, None] * nd + b_idx[None])
    kv[np.searchsorted(keys, rk.reshape(-1))] = -K.reshape(-1)
    nodes = np.arange(n)
    dk = (nodes[:, None, None] * nd + a_idx[None]) * ncol + (nodes[:, None, None] * nd + b_idx[None])
    kv[np.searchsorted(keys, dk.reshape(-1))] = kii.reshape(-1)
    return kv, rl.reshape(-1)
