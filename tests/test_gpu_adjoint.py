"""Adjoint kernels through torch.autograd (perix_b200.autograd): gradient checks.

References: (1) a plain-torch FP64 restatement of the same operators built from the oracle's g-functions,
differentiated by torch's own autograd; (2) central finite differences of the forward path, taken through
the device's fused explicit loop (pxb_epf_start / pxb_epf_advance with damage off), which is independent of
the torch loop being differentiated.  Tolerance: 1e-6 relative for finite differences; 1e-10 against the FP64
torch restatement; mixed precision within 1e-5 of the FP64 gradient (see the test for why)."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NX, NY, H = 60, 30, 5e-4
NSTEPS = 60
E0, NU, RHO = 190e9, 0.3, 8000.0


def _torch():
    import torch
    return torch, torch.device("cuda", 0)


@pytest.fixture(scope="module")
def plate(port):
    import perix_b200 as px
    L = px.lattice(2, NX, NY, 0, [0.0, NX * H, 0.0, NY * H])
    delta = 3.015 * L.dxyz[0] * (1.0 + 1e-6)
    y1, y2 = (NY / 2 - 5) * H, (NY / 2 + 5) * H
    cracks = [[0.0, y1, 10 * H, y1], [0.0, y2, 10 * H, y2]]
    off, ids = px.families(L.coords, delta, False, cracks=cracks, mirror=L.mirror, force_only=True)
    health0 = (1 - px.crack_cut_mask(L.coords, L.mirror, off, ids, cracks=cracks)).astype(np.uint8)
    bcs = [px.BC("neumann", [0, 1], L.group(w + "nodes_ghost")) for w in ("left", "right", "bottom", "top")]
    bcs.append(px.BC("dirichlet", [0], L.group("leftnodes_ghost"), value=[0, 0], velocity=[16.5, 0], direct=True,
                     box=[-1, 1, y1, y2, -1, 1]))
    g, deg = port.gbuild(2, 2, L.coords, L.vols, off, ids, delta, L.dxyz[0])
    assert deg.sum() == 0
    C11, _, _ = px.elastic_constants(2, False, E0, NU)
    dt = 0.8 * H / math.sqrt(C11 / RHO)
    return dict(L=L, delta=delta, off=off, ids=ids, health0=health0, bcs=bcs, g=g, dt=dt)


def _ctx(ctx, w, E, precision=0):
    import perix_b200 as px
    L = w["L"]
    ctx.set_geometry(L.coords, L.vols, w["off"], w["ids"], w["delta"], L.dxyz[0], 2, mirror=L.mirror)
    C11, C12, C66 = px.elastic_constants(2, False, E, NU)
    ctx.epf_setup(C11, C12, C66, RHO, (0.0, 0.0), 0.0, True, health0=w["health0"], precision=precision)
    return ctx


def _torch_force(w, u, C):
    """FP64 restatement: a_i = sum_t h_t P_t (u_j - u_i) / rho with P from (Gxx, Gyy, Gxy) and C."""
    torch, dev = _torch()
    off, ids, g = w["off"], w["ids"], w["g"]
    n = off.size - 1
    src = torch.from_numpy(np.repeat(np.arange(n), np.diff(off))).to(dev)
    nbr = torch.from_numpy((ids - 1).astype(np.int64)).to(dev)
    h = torch.from_numpy(w["health0"].astype(np.float64)).to(dev)
    G = torch.from_numpy(np.ascontiguousarray(g[:, [2, 4, 3]])).to(dev)
    U = u.view(n, 2)
    e = U[nbr] - U[src]
    p11 = C[0] * G[:, 0] + C[2] * G[:, 1]
    p22 = C[2] * G[:, 0] + C[0] * G[:, 1]
    pxy = (C[1] + C[2]) * G[:, 2]
    f = torch.stack([h * (p11 * e[:, 0] + pxy * e[:, 1]), h * (pxy * e[:, 0] + p22 * e[:, 1])], dim=1)
    Lsum = torch.zeros(n, 2, dtype=torch.float64, device=dev).index_add(0, src, f)
    return (Lsum / RHO).reshape(-1)


def test_apply_adjoint_through_autograd(ctx, plate):
    """Dot-product identity and autograd against the torch restatement D^k u = sum_t g^k_t (u_j - u_i)."""
    torch, dev = _torch()
    from perix_b200.autograd import pddo_apply
    w = plate
    L = w["L"]
    ctx.set_geometry(L.coords, L.vols, w["off"], w["ids"], w["delta"], L.dxyz[0], 2, mirror=L.mirror)
    ctx.gbuild(2, 0)
    n = L.n
    slots = [0, 1, 2, 3, 4]
    rng = np.random.default_rng(3)
    u = torch.tensor(rng.standard_normal(n), device=dev, requires_grad=True)
    y = torch.tensor(rng.standard_normal((n, 5)), device=dev)
    D = pddo_apply(ctx, u, slots)
    (D * y).sum().backward()
    # restatement
    off, ids, g = w["off"], w["ids"], w["g"]
    src = torch.from_numpy(np.repeat(np.arange(n), np.diff(off))).to(dev)
    nbr = torch.from_numpy((ids - 1).astype(np.int64)).to(dev)
    u2 = u.detach().clone().requires_grad_(True)
    Gt = torch.from_numpy(g).to(dev)
    Dref = torch.zeros(n, 5, dtype=torch.float64, device=dev).index_add(0, src, Gt * (u2[nbr] - u2[src])[:, None])
    (Dref * y).sum().backward()
    assert (D.detach() - Dref.detach()).abs().max() <= 1e-12 * Dref.abs().max()
    assert (u.grad - u2.grad).abs().max() <= 1e-12 * u2.grad.abs().max()
    # <D u, y> = <u, D^T y>
    lhs = float((D.detach() * y).sum())
    rhs = float((u.detach() * u.grad).sum())
    assert abs(lhs - rhs) <= 1e-12 * (D.detach().abs() * y.abs()).sum().item()


def test_frozen_force_gradients(ctx, plate):
    torch, dev = _torch()
    import perix_b200 as px
    from perix_b200.autograd import frozen_force
    w = plate
    _ctx(ctx, w, E0)
    n = w["L"].n
    rng = np.random.default_rng(4)
    u = torch.tensor(rng.standard_normal(2 * n) * 1e-6, device=dev, requires_grad=True)
    C = torch.tensor(px.elastic_constants(2, False, E0, NU), dtype=torch.float64, device=dev, requires_grad=True)
    abar = torch.tensor(rng.standard_normal(2 * n), device=dev)
    a = frozen_force(ctx, u, C)
    (a * abar).sum().backward()
    u2 = u.detach().clone().requires_grad_(True)
    C_ref = C.detach().clone().requires_grad_(True)
    aref = _torch_force(w, u2, C_ref)
    (aref * abar).sum().backward()
    assert (a.detach() - aref.detach()).abs().max() <= 1e-12 * aref.abs().max()
    assert (u.grad - u2.grad).abs().max() <= 1e-10 * u2.grad.abs().max()
    assert (C.grad - C_ref.grad).abs().max() <= 1e-10 * C_ref.grad.abs().max()


def _device_final(ctx, w, E, u0):
    """u^N from the fused device loop (damage off: frozen mask)."""
    _ctx(ctx, w, E)
    ctx.epf_set_bcs(w["bcs"])
    ctx.epf_start(u0, None, w["dt"])
    ctx.epf_advance(NSTEPS, chunk=20)
    return ctx.epf_state()[0]


def _loop_grad(ctx, w, u_obs, u0, precision=0, checkpoint_every=10, reference_force=False):
    torch, dev = _torch()
    from perix_b200.autograd import BcPlan, elastic_constants_t, explicit_loop, set_constants
    _ctx(ctx, w, E0, precision)
    L = w["L"]
    plan = BcPlan(w["bcs"], L.coords, L.mirror, 2, dev)
    E = torch.tensor(E0, dtype=torch.float64, device=dev, requires_grad=True)
    u0t = torch.tensor(u0, device=dev, requires_grad=True)
    C = elastic_constants_t(2, False, E, NU)
    set_constants(ctx, C, RHO)
    force = (lambda pctx, u, Cv: _torch_force(w, u, Cv)) if reference_force else None
    uN, _ = explicit_loop(ctx, u0t, None, w["dt"], NSTEPS, C, plan, checkpoint_every=checkpoint_every, force=force)
    J = 0.5 * ((uN - torch.tensor(u_obs, device=dev)) ** 2).sum()
    J.backward()
    return float(J), float(E.grad), u0t.grad.cpu().numpy(), uN.detach().cpu().numpy()


@pytest.fixture(scope="module")
def loop_case(ctx, plate):
    w = plate
    n = w["L"].n
    rng = np.random.default_rng(5)
    u0 = rng.standard_normal(2 * n) * 1e-7
    u_obs = _device_final(ctx, w, 1.02 * E0, u0)
    return w, u0, u_obs


def _J(ctx, w, E, u0, u_obs):
    uN = _device_final(ctx, w, E, u0)
    return 0.5 * float(((uN - u_obs) ** 2).sum())


def _J_torch_loop(ctx, w, E, u0, u_obs, precision):
    """J through the torch loop's own forward (the function the adjoint differentiates), no tape."""
    torch, dev = _torch()
    from perix_b200.autograd import BcPlan, elastic_constants_t, explicit_loop, set_constants
    _ctx(ctx, w, E0, precision)
    L = w["L"]
    plan = BcPlan(w["bcs"], L.coords, L.mirror, 2, dev)
    with torch.no_grad():
        C = elastic_constants_t(2, False, torch.tensor(E, dtype=torch.float64, device=dev), NU)
        set_constants(ctx, C, RHO)
        uN, _ = explicit_loop(ctx, torch.tensor(u0, device=dev), None, w["dt"], NSTEPS, C, plan)
        return 0.5 * float(((uN - torch.tensor(u_obs, device=dev)) ** 2).sum())


def test_explicit_loop_forward_matches_device_loop(ctx, loop_case):
    w, u0, u_obs = loop_case
    _, _, _, uN = _loop_grad(ctx, w, u_obs, u0)
    ref = _device_final(ctx, w, E0, u0)
    assert np.abs(uN - ref).max() <= 1e-10 * np.abs(ref).max()


def test_dJ_dE_against_finite_differences(ctx, loop_case):
    w, u0, u_obs = loop_case
    J, dE, _, _ = _loop_grad(ctx, w, u_obs, u0)
    h = 1e-5 * E0
    fd = (_J(ctx, w, E0 + h, u0, u_obs) - _J(ctx, w, E0 - h, u0, u_obs)) / (2 * h)
    assert abs(dE - fd) <= 1e-6 * abs(fd)


def test_dJ_du0_against_finite_differences(ctx, loop_case):
    w, u0, u_obs = loop_case
    _, _, du0, _ = _loop_grad(ctx, w, u_obs, u0)
    rng = np.random.default_rng(6)
    d = rng.standard_normal(u0.size)
    eps = 1e-3 * np.abs(u0).max()
    fd = (_J(ctx, w, E0, u0 + eps * d, u_obs) - _J(ctx, w, E0, u0 - eps * d, u_obs)) / (2 * eps)
    ad = float(du0 @ d)
    assert abs(ad - fd) <= 1e-6 * abs(fd)


def test_checkpointed_equals_stored_and_fp64_reference(ctx, loop_case):
    w, u0, u_obs = loop_case
    _, dE_ck, du_ck, _ = _loop_grad(ctx, w, u_obs, u0, checkpoint_every=10)
    _, dE_st, du_st, _ = _loop_grad(ctx, w, u_obs, u0, checkpoint_every=0)
    assert abs(dE_ck - dE_st) <= 1e-12 * abs(dE_st)
    assert np.abs(du_ck - du_st).max() <= 1e-12 * np.abs(du_st).max()
    _, dE_ref, du_ref, _ = _loop_grad(ctx, w, u_obs, u0, reference_force=True)
    assert abs(dE_ck - dE_ref) <= 1e-10 * abs(dE_ref)
    assert np.abs(du_ck - du_ref).max() <= 1e-10 * np.abs(du_ref).max()


def test_mixed_adjoint_against_its_forward(ctx, loop_case):
    """Mixed precision (FP32 operator storage): the adjoint is the exact derivative of the mixed forward (finite
    differences of that forward within 1e-6), and stays within 1e-5 of the FP64 gradient.  The second bound is
    looser than the forward's 1e-6 because the misfit against a 2 % different modulus is a difference of
    nearly equal fields: the FP32 rounding of the operators (~1e-7 of u) is amplified ~50x in dJ/dE."""
    w, u0, u_obs = loop_case
    _, dE64, du64, _ = _loop_grad(ctx, w, u_obs, u0, precision=0)
    _, dE32, du32, _ = _loop_grad(ctx, w, u_obs, u0, precision=1)
    h = 1e-5 * E0
    fd = (_J_torch_loop(ctx, w, E0 + h, u0, u_obs, 1) - _J_torch_loop(ctx, w, E0 - h, u0, u_obs, 1)) / (2 * h)
    assert abs(dE32 - fd) <= 1e-6 * abs(fd)
    assert abs(dE32 - dE64) <= 1e-5 * abs(dE64)
    assert np.abs(du32 - du64).max() <= 1e-5 * np.abs(du64).max()


def test_explicit_loop_full_plate_matches_device_loop(ctx):
    """The differentiable loop on the full 400x200 plate (its kernels and torch's ops share torch's default
    stream: the launches must be ordered with torch's work) against the fused device loop, 30 steps."""
    torch, dev = _torch()
    import perix_b200 as px
    from bench import plate_setup
    from perix_b200.autograd import BcPlan, elastic_constants_t, explicit_loop, set_constants
    w = plate_setup(px)
    L = w["L"]
    ctx.set_geometry(L.coords, L.vols, w["off"], w["ids"], w["delta"], L.dxyz[0], 2, mirror=L.mirror)
    C11, C12, C66 = w["C"]
    ctx.epf_setup(C11, C12, C66, w["rho"], (0.0, 0.0), 0.0, True, health0=w["health0"])
    ctx.epf_set_bcs(w["bcs"])
    ctx.epf_start(np.zeros(2 * L.n), None, w["dt"])
    ctx.epf_advance(30, chunk=10)
    ref = ctx.epf_state()[0]
    C = elastic_constants_t(2, False, torch.tensor(w["E"], dtype=torch.float64, device=dev), w["nu"])
    set_constants(ctx, C, w["rho"])
    with torch.no_grad():
        uN, _ = explicit_loop(ctx, torch.zeros(2 * L.n, dtype=torch.float64, device=dev), None, w["dt"], 30, C,
                              BcPlan(w["bcs"], L.coords, L.mirror, 2, dev))
    assert np.abs(uN.cpu().numpy() - ref).max() <= 1e-10 * np.abs(ref).max()


def test_dJ_dE_3d_slab_against_finite_differences(ctx):
    """3D: a 16x16x6 slab with an edge notch and +-2 m/s pins, 40 steps, checkpoints every 10."""
    torch, dev = _torch()
    import perix_b200 as px
    from bench import slab_setup
    from perix_b200.autograd import BcPlan, elastic_constants_t, explicit_loop, set_constants
    w = slab_setup(px, nx=16, ny=16, nz=6)
    L = w["L"]
    nsteps = 40
    ctx.set_geometry(L.coords, L.vols, w["off"], w["ids"], w["delta"], L.dxyz[0], 3, mirror=L.mirror)

    def device_final(E):
        c = px.elastic_constants(3, False, E, w["nu"])
        ctx.epf_setup(c[0], c[1], c[2], w["rho"], (0.0, 0.0, 0.0), 0.0, True, health0=w["health0"])
        ctx.epf_set_bcs(w["bcs"])
        ctx.epf_start(np.zeros(3 * L.n), None, w["dt"])
        ctx.epf_advance(nsteps, chunk=10)
        return ctx.epf_state()[0]

    u_obs = device_final(1.02 * w["E"])
    J = lambda u: 0.5 * float(((u - u_obs) ** 2).sum())  # noqa: E731
    h = 1e-5 * w["E"]
    fd = (J(device_final(w["E"] + h)) - J(device_final(w["E"] - h))) / (2 * h)
    device_final(w["E"])
    E = torch.tensor(w["E"], dtype=torch.float64, device=dev, requires_grad=True)
    C = elastic_constants_t(3, False, E, w["nu"])
    set_constants(ctx, C, w["rho"])
    uN, _ = explicit_loop(ctx, torch.zeros(3 * L.n, dtype=torch.float64, device=dev), None, w["dt"], nsteps, C,
                          BcPlan(w["bcs"], L.coords, L.mirror, 3, dev), checkpoint_every=10)
    (0.5 * ((uN - torch.from_numpy(u_obs).to(dev)) ** 2).sum()).backward()
    assert abs(float(E.grad) - fd) <= 1e-6 * abs(fd)
