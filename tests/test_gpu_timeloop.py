"""The explicit loop's time control against the reference loop (oracle/_ref: the reference element and BC objects
under a restatement of TimeStepping::solveExplicitDynamics, TimeStepping.cpp:479-599):

* an end time that is not a multiple of dt: the last step is clamped to land on it and takes the variable-step
  central difference u + (dt/dt_prev)(u - u_prev) + dt (dt + dt_prev)/2 a (TimeStepping.cpp:537-545);
* the blow-up guard (50-step window, x1e3 growth or non-finite U, TimeStepping.cpp:550-573): an unstable time step
  and a non-finite start must stop the run at the step the reference names."""
import numpy as np
import pytest

from conftest import load_golden
from oracle import ref_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not ref_available(), reason="reference harness not built")]


def _plate():
    import perix_b200 as px
    from oracle import RefMesh
    d = load_golden("epf2d")
    nx, ny, h = 40, 20, 5e-4
    y1, y2 = d["y_band"]
    cracks = [[0.0, y1, 5 * h, y1], [0.0, y2, 5 * h, y2]]
    m = RefMesh.structured(2, nx, ny, 0, [0, nx * h, 0, ny * h], 3.015, 2, cracks=cracks, force_only=True)
    bcs = [px.BC("neumann", [0, 1], m.group(g + "nodes_ghost")) for g in ("left", "right", "bottom", "top")]
    bcs.append(px.BC("dirichlet", [0], m.group("leftnodes_ghost"), value=[0, 0], velocity=[16.5, 0], direct=True,
                     box=[-1, 1, y1, y2, -1, 1]))
    health0 = 1 - px.crack_cut_mask(m.coords, m.mirror, m.off, m.ids, cracks=cracks)
    return d, m, bcs, health0.astype(np.uint8)


def _ref(m, d, damage_on=True):
    from oracle import RefEpf
    el = RefEpf(m, 190e9, 0.3, 8000.0, float(d["G0"]), damage_on=damage_on)
    el.rate(np.zeros(2 * m.n))
    return el, el.constants()


def _device(ctx, m, d, k, bcs, health0, variant, sc):
    ctx.set_geometry(m.coords, m.vols, m.off, m.ids, m.delta, m.dx_char, 2, mirror=m.mirror)
    ctx.epf_setup(k["C11"], k["C12"], k["C66"], 8000.0, (0.0, 0.0), sc, True, health0=health0)
    ctx.epf_set_variant(variant)
    ctx.epf_set_bcs(bcs)


@pytest.mark.parametrize("variant", [1, 8, 11])
@pytest.mark.parametrize("nsteps_frac", [37.37, 40.0, 40.0000001])
def test_end_time_lands_like_reference(ctx, variant, nsteps_frac):
    d, m, bcs, health0 = _plate()
    el, k = _ref(m, d)
    dt = float(d["dt"])
    t_end = dt * nsteps_frac
    rng = np.random.default_rng(3)
    u0 = rng.standard_normal(2 * m.n) * 1e-6
    u_r, uo_r, h_r, steps_r, trip, t_r = el.run_to(u0, None, dt, t_end, [b.as_dict() for b in bcs])
    assert trip == 0
    _device(ctx, m, d, k, bcs, health0, variant, k["sc"])
    ctx.epf_start(u0, None, dt)
    steps = ctx.epf_advance_to(t_end, chunk=16)
    u, uo, h, t = ctx.epf_state()
    assert steps == steps_r
    assert t == t_r
    assert np.array_equal(h, (h_r > 0).astype(np.uint8))
    scale = np.abs(u_r).max()
    assert np.abs(u - u_r).max() <= 1e-10 * scale
    assert np.abs(uo - uo_r).max() <= 1e-10 * scale


def test_clamped_last_step_differs_from_a_uniform_one(ctx):
    """The clamped step's variable form is not the uniform formula applied with the short dt: the two end states
    differ by much more than round-off (so the landing test above does test the variable form)."""
    d, m, bcs, health0 = _plate()
    _, k = _ref(m, d)
    dt = float(d["dt"])
    rng = np.random.default_rng(3)
    u0 = rng.standard_normal(2 * m.n) * 1e-6
    # each run from a fresh element (the damage a run commits stays in the context's health)
    _device(ctx, m, d, k, bcs, health0, 1, k["sc"])
    ctx.epf_start(u0, None, dt)
    ctx.epf_advance_to(dt * 37.37)
    u_var = ctx.epf_state()[0]
    _device(ctx, m, d, k, bcs, health0, 1, k["sc"])
    ctx.epf_start(u0, None, dt)
    ctx.epf_advance(37)
    ctx.epf_advance_to(dt * 37.37)  # the same clamped step after 37 uniform ones: identical
    assert np.array_equal(ctx.epf_state()[0], u_var)
    _device(ctx, m, d, k, bcs, health0, 1, k["sc"])
    ctx.epf_start(u0, None, dt)
    ctx.epf_advance(38)
    assert np.abs(ctx.epf_state()[0] - u_var).max() > 1e-6 * np.abs(u_var).max()


@pytest.mark.parametrize("variant", [1, 11])
def test_blowup_guard_trips_at_the_reference_step(ctx, variant):
    """dt at 2.5x the bench's CFL-limited step, no damage: the displacement grows by more than 1e3 within the guard's
    50-step window; the run stops with PXB_ERR_BLOWUP at the step where the reference guard trips."""
    import perix_b200 as px
    d, m, bcs, health0 = _plate()
    el, k = _ref(m, d, damage_on=False)
    dt = 2.5 * float(d["dt"])
    t_end = dt * 400.5
    _, _, _, steps_r, trip, _ = el.run_to(np.zeros(2 * m.n), None, dt, t_end, [b.as_dict() for b in bcs])
    assert trip > 0 and steps_r == trip - 1
    _device(ctx, m, d, k, bcs, health0, variant, 0.0)
    ctx.epf_start(np.zeros(2 * m.n), None, dt)
    with pytest.raises(px.PxbError) as e:
        ctx.epf_advance_to(t_end, chunk=16)
    assert e.value.status == 5
    assert e.value.bad_step == trip


@pytest.mark.parametrize("variant", [1, 11])
def test_non_finite_start_trips_at_step_one(ctx, variant):
    """A NaN in u0 makes every later state non-finite: the guard stops the run at step 1, as the reference's."""
    import perix_b200 as px
    d, m, bcs, health0 = _plate()
    el, k = _ref(m, d)
    dt = float(d["dt"])
    u0 = np.zeros(2 * m.n)
    u0[2 * 137] = np.nan
    _, _, _, _, trip, _ = el.run_to(u0, None, dt, dt * 10.5, [b.as_dict() for b in bcs])
    assert trip == 1
    _device(ctx, m, d, k, bcs, health0, variant, k["sc"])
    ctx.epf_start(u0, None, dt)
    with pytest.raises(px.PxbError) as e:
        ctx.epf_advance(10, chunk=4)
    assert e.value.status == 5 and e.value.bad_step == 1
