"""The device adjoint of the explicit loop (pxb_epf_adjoint_d through perix_b200.autograd.explicit_run) against the
torch-taped loop (explicit_loop around the bond-force adjoint, itself checked against finite differences and an
FP64 restatement in test_gpu_adjoint.py) on the notched plate, frozen damage mask:

* dJ/du0, dJ/dv0 and dJ/dE within 1e-10 of the taped loop, for the direct-pin BC program and for one with
  reflected walls (the BC transpose's +-1 entries), with all states kept and with checkpoints every 7 steps;
* dJ/dE within 1e-6 of a central finite difference of the device loop itself;
* a backward pass after a later run (which replaced the context's recording) gives the same gradients."""
import numpy as np
import pytest

from test_gpu_adjoint import E0, NSTEPS, NU, RHO, _ctx, _device_final, _torch, plate  # noqa: F401

pytestmark = pytest.mark.gpu


def _bcs(w, kind):
    import perix_b200 as px
    if kind == "pins":
        return w["bcs"]
    L = w["L"]
    bcs = [px.BC("neumann", [0, 1], L.group(g + "nodes_ghost")) for g in ("left", "right", "bottom")]
    bcs.append(px.BC("dirichlet", [1], L.group("topnodes_ghost"), value=[0.0, 1e-7], velocity=[0.0, 0.3]))
    bcs.append(px.BC("neumann", [0], L.group("topnodes_ghost")))
    bcs.append(px.BC("dirichlet", [0], L.group("leftnodes_ghost"), value=[0.0, 0.0], velocity=[5.0, 0.0],
                     box=[1.0, -1.0, 0.25 * L.coords[1::3].max(), 0.75 * L.coords[1::3].max(), 1.0, -1.0]))
    return bcs


def _grads(ctx, w, bcs, u0, v0, u_obs, device_run, checkpoint_every, schedule=-1):
    torch, dev = _torch()
    from perix_b200.autograd import BcPlan, elastic_constants_t, explicit_loop, explicit_run, set_constants
    _ctx(ctx, w, E0)
    ctx.epf_set_adjoint_schedule(schedule)
    ctx.epf_set_bcs(bcs)
    E = torch.tensor(E0, dtype=torch.float64, device=dev, requires_grad=True)
    u0t = torch.tensor(u0, device=dev, requires_grad=True)
    v0t = torch.tensor(v0, device=dev, requires_grad=True)
    C = elastic_constants_t(2, False, E, NU)
    set_constants(ctx, C, RHO)
    if device_run:
        uN, uNm1 = explicit_run(ctx, u0t, v0t, C, w["dt"], NSTEPS, checkpoint_every=checkpoint_every)
    else:
        plan = BcPlan(bcs, w["L"].coords, w["L"].mirror, 2, dev)
        uN, uNm1 = explicit_loop(ctx, u0t, v0t, w["dt"], NSTEPS, C, plan, checkpoint_every=0)
    obs = torch.tensor(u_obs, device=dev)
    J = 0.5 * ((uN - obs) ** 2).sum() + 0.25 * ((uNm1 - obs) ** 2).sum()
    J.backward()
    return float(J), float(E.grad), u0t.grad.cpu().numpy(), v0t.grad.cpu().numpy(), uN.detach().cpu().numpy()


@pytest.mark.parametrize("schedule", [0, 1, 2, 3, 4])
@pytest.mark.parametrize("checkpoint_every", [0, 7])
@pytest.mark.parametrize("kind", ["pins", "reflect"])
def test_device_adjoint_matches_taped_loop(ctx, plate, kind, checkpoint_every, schedule):  # noqa: F811
    w = plate
    n = w["L"].n
    rng = np.random.default_rng(8)
    u0 = rng.standard_normal(2 * n) * 1e-7
    v0 = rng.standard_normal(2 * n) * 1e-2
    bcs = _bcs(w, kind)
    u_obs = rng.standard_normal(2 * n) * 1e-7
    J1, dE1, du1, dv1, uN1 = _grads(ctx, w, bcs, u0, v0, u_obs, True, checkpoint_every, schedule)
    J2, dE2, du2, dv2, uN2 = _grads(ctx, w, bcs, u0, v0, u_obs, False, 0)
    assert np.abs(uN1 - uN2).max() <= 1e-10 * np.abs(uN2).max()
    assert abs(J1 - J2) <= 1e-10 * abs(J2)
    assert abs(dE1 - dE2) <= 1e-10 * abs(dE2)
    assert np.abs(du1 - du2).max() <= 1e-10 * np.abs(du2).max()
    assert np.abs(dv1 - dv2).max() <= 1e-10 * np.abs(dv2).max()


def test_device_adjoint_dJ_dE_against_finite_differences(ctx, plate):  # noqa: F811
    w = plate
    n = w["L"].n
    rng = np.random.default_rng(5)
    u0 = rng.standard_normal(2 * n) * 1e-7
    u_obs = _device_final(ctx, w, 1.02 * E0, u0)
    torch, dev = _torch()
    from perix_b200.autograd import elastic_constants_t, explicit_run, set_constants
    _ctx(ctx, w, E0)
    ctx.epf_set_bcs(w["bcs"])
    E = torch.tensor(E0, dtype=torch.float64, device=dev, requires_grad=True)
    C = elastic_constants_t(2, False, E, NU)
    set_constants(ctx, C, RHO)
    uN, _ = explicit_run(ctx, torch.tensor(u0, device=dev), None, C, w["dt"], NSTEPS, checkpoint_every=10)
    (0.5 * ((uN - torch.tensor(u_obs, device=dev)) ** 2).sum()).backward()

    def J(Ev):
        uf = _device_final(ctx, w, Ev, u0)
        return 0.5 * float(((uf - u_obs) ** 2).sum())

    h = 1e-5 * E0
    fd = (J(E0 + h) - J(E0 - h)) / (2 * h)
    assert abs(float(E.grad) - fd) <= 1e-6 * abs(fd)


def test_backward_after_a_later_run_rerecords(ctx, plate):  # noqa: F811
    """The context keeps one recorded forward loop; a backward pass whose recording a later run replaced records its
    own loop again, so its gradients equal those of the run taken alone."""
    torch, dev = _torch()
    from perix_b200.autograd import elastic_constants_t, explicit_run, set_constants
    w = plate
    n = w["L"].n
    rng = np.random.default_rng(21)
    u0 = rng.standard_normal(2 * n) * 1e-7
    u0b = rng.standard_normal(2 * n) * 1e-7
    u_obs = rng.standard_normal(2 * n) * 1e-7

    def grads(with_second_run):
        _ctx(ctx, w, E0)
        ctx.epf_set_bcs(w["bcs"])
        E = torch.tensor(E0, dtype=torch.float64, device=dev, requires_grad=True)
        u0t = torch.tensor(u0, device=dev, requires_grad=True)
        C = elastic_constants_t(2, False, E, NU)
        set_constants(ctx, C, RHO)
        uN, _ = explicit_run(ctx, u0t, None, C, w["dt"], NSTEPS, checkpoint_every=5)
        if with_second_run:
            explicit_run(ctx, torch.tensor(u0b, device=dev), None, C, w["dt"], NSTEPS // 2, checkpoint_every=0)
        (0.5 * ((uN - torch.tensor(u_obs, device=dev)) ** 2).sum()).backward()
        return float(E.grad), u0t.grad.cpu().numpy()

    dE1, du1 = grads(False)
    dE2, du2 = grads(True)
    # dJ/dC is summed with one atomic per block, so its last bit may differ from run to run
    assert abs(dE1 - dE2) <= 1e-13 * abs(dE1)
    assert np.abs(du1 - du2).max() <= 1e-13 * np.abs(du1).max()
