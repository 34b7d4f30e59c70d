"""Host logic of perix_b200.autograd (no GPU): the BC plan used by the differentiable explicit loop applies
the reference's preset (DirichletBC.cpp:107-147, NeumannBC.cpp:88-105 in list order) exactly like the
oracle's restatement, and its torch ops carry gradients to the mirrored bulk nodes."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")


def _plate():
    import perix_b200 as px
    h = 5e-4
    L = px.lattice(2, 24, 12, 0, [0.0, 24 * h, 0.0, 12 * h])
    y1, y2 = 4 * h, 8 * h
    bcs = [px.BC("neumann", [0, 1], L.group(w + "nodes_ghost")) for w in ("left", "right", "bottom", "top")]
    bcs.append(px.BC("dirichlet", [0], L.group("leftnodes_ghost"), value=[0, 0], velocity=[16.5, 0], direct=True,
                     box=[-1, 1, y1, y2, -1, 1]))
    bcs.append(px.BC("dirichlet", [1], L.group("rightnodes_ghost"), value=[1e-6, -2e-6], velocity=[0, 3.0]))
    bcs.append(px.BC("dirichlet", [0, 1], np.arange(1, L.n + 1), value=[0, 0], velocity=[0, 2.0], direct=True,
                     box=[-1, 1, 11 * h, 1, -1, 1]))
    return px, L, bcs


@pytest.mark.parametrize("t", [0.0, 3.5e-6])
def test_bc_plan_matches_oracle_preset(port, t):
    from perix_b200.autograd import BcPlan
    px, L, bcs = _plate()
    rng = np.random.default_rng(1)
    u = rng.standard_normal(2 * L.n) * 1e-6
    ref = port.bc_preset(2, L.coords, L.mirror, [b.as_dict() for b in bcs], t, u.copy())
    plan = BcPlan(bcs, L.coords, L.mirror, 2, torch.device("cpu"))
    got = plan.apply(torch.from_numpy(u.copy()), t).numpy()
    assert np.array_equal(got, ref)


def test_bc_plan_gradient_flows_to_mirrors():
    from perix_b200.autograd import BcPlan
    px, L, bcs = _plate()
    plan = BcPlan(bcs[:4], L.coords, L.mirror, 2, torch.device("cpu"))
    u = torch.zeros(2 * L.n, dtype=torch.float64, requires_grad=True)
    v = plan.apply(u, 0.0)
    g = L.group("leftnodes_ghost")[0]
    v[(g - 1) * 2].backward()
    mb = int(L.mirror[g - 1])
    grad = u.grad.numpy()
    assert grad[(mb - 1) * 2] == 1.0 and grad[(g - 1) * 2] == 0.0 and grad.sum() == 1.0
