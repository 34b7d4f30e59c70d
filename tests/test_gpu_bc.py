"""The fused ghost-BC pass of the explicit step against the reference itself: the reference's
ExplicitPDDOFracElement, central difference and its own DirichletBC / NeumannBC objects applied in list order
(oracle/_ref/libperix_ref.so), on the full 400x200 notched plate and on a notched 3D slab.

The BC programs use the reference's default Dirichlet form, the reflection u_ghost = 2 g(t) - u_bulk
(DirichletBC.cpp:141-143), with a velocity ramp g(t) = value + velocity t and a box with unconstrained axes
(DirichletBC.cpp:89-98), behind zero-Neumann walls.  Every step schedule runs the same 30 steps from a seeded
random field that breaks bonds; damage sets must be identical and u within 1e-10 of its magnitude.  The plate also
runs with tension_only = false (bonds break under compression too, ExplicitPDDOFracElement.cpp:239-266)."""
import math

import numpy as np
import pytest

from oracle import ref_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not ref_available(), reason="reference harness not built")]

NSTEPS = 30
N_VARIANTS = 21
INACTIVE = [1.0, -1.0]  # min > max: the box leaves this axis unconstrained


def _plate_program(px, m, y1, y2):
    g = {w: m.group(w + "nodes_ghost") for w in ("left", "right", "bottom", "top")}
    bcs = [px.BC("neumann", [0, 1], g[w]) for w in ("left", "right", "bottom", "top")]
    # the pulled band of the left wall: reflection of a 16.5 m/s ramp in x and of a zero y, boxed in y only
    bcs.append(px.BC("dirichlet", [0, 1], g["left"], value=[0.0, 0.0], velocity=[16.5, 0.0],
                     box=INACTIVE + [y1, y2] + INACTIVE))
    # the top wall held at zero normal displacement by reflection
    bcs.append(px.BC("dirichlet", [1], g["top"], value=[0.0, 0.0]))
    return bcs


def _slab_program(px, m, Lx, Ly, h):
    g = {w: m.group(w + "nodes_ghost") for w in ("left", "right", "bottom", "top", "back", "front")}
    bcs = [px.BC("neumann", [0, 1, 2], g[w]) for w in g]
    # top and bottom walls pulled apart by reflected +-2 m/s ramps over the half of the span away from the notch
    bcs.append(px.BC("dirichlet", [1], g["top"], value=[0, 0, 0], velocity=[0, 2.0, 0],
                     box=[0.5 * Lx, 2 * Lx] + INACTIVE + INACTIVE))
    bcs.append(px.BC("dirichlet", [1], g["bottom"], value=[0, 0, 0], velocity=[0, -2.0, 0],
                     box=[0.5 * Lx, 2 * Lx] + INACTIVE + INACTIVE))
    # the back wall held at zero out-of-plane displacement by reflection
    bcs.append(px.BC("dirichlet", [2], g["back"], value=[0, 0, 0]))
    return bcs


def _case(kind, tension_only):
    import perix_b200 as px
    from oracle import RefEpf, RefMesh
    if kind == "plate":
        nx, ny, h = 400, 200, 5e-4
        Lx, Ly = nx * h, ny * h
        y1, y2 = Ly / 2 - 25 * h, Ly / 2 + 25 * h
        cracks = [[0.0, y1, 50 * h, y1], [0.0, y2, 50 * h, y2]]
        m = RefMesh.structured(2, nx, ny, 0, [0, Lx, 0, Ly], 3.015, 2, cracks=cracks, force_only=True)
        E, nu, rho = 190e9, 0.3, 8000.0
        G0 = 0.01 ** 2 * 12 * E * m.delta / (5 * math.pi)
        bcs = _plate_program(px, m, y1, y2)
        amp = 2e-6
        health0 = 1 - px.crack_cut_mask(m.coords, m.mirror, m.off, m.ids, cracks=cracks)
    else:
        nx, ny, nz, h = 40, 40, 12, 1e-3
        Lx, Ly, Lz = nx * h, ny * h, nz * h
        plane = [0.0, Ly / 2, -1.0, 10 * h, Ly / 2, -1.0, 10 * h, Ly / 2, 1.0, 0.0, Ly / 2, 1.0]
        m = RefMesh.structured(3, nx, ny, nz, [0, Lx, 0, Ly, 0, Lz], 3.015, 2, planes=[plane], force_only=True)
        E, nu, rho = 72e9, 0.22, 2440.0
        G0 = 0.004 ** 2 * 6 * E * m.delta / 5
        bcs = _slab_program(px, m, Lx, Ly, h)
        amp = 1.5e-6
        health0 = 1 - px.crack_cut_mask(m.coords, m.mirror, m.off, m.ids, planes=[plane])
    el = RefEpf(m, E, nu, rho, G0, tension_only=tension_only)
    dim = m.dim
    rng = np.random.default_rng(11 if kind == "plate" else 12)
    u0 = rng.standard_normal(m.n * dim) * amp
    el.rate(np.zeros(m.n * dim))  # the element's first preprocess derives its constants (no damage at rest)
    k = el.constants()
    dt = 0.8 * h / math.sqrt(k["C11"] / rho)
    u, uo, hh, _ = el.run(u0, None, dt, NSTEPS, [b.as_dict() for b in bcs])
    return dict(m=m, bcs=bcs, u0=u0, dt=dt, k=k, rho=rho, health0=health0.astype(np.uint8), tension_only=tension_only,
                u=u, uo=uo, h=(hh > 0).astype(np.uint8))


_CASES = {}


def case(kind, tension_only=True):
    key = (kind, tension_only)
    if key not in _CASES:
        _CASES[key] = _case(kind, tension_only)
    return _CASES[key]


def _run(ctx, c, variant, precision=0):
    import perix_b200 as px
    m, k = c["m"], c["k"]
    ctx.set_geometry(m.coords, m.vols, m.off, m.ids, m.delta, m.dx_char, m.dim, mirror=m.mirror)
    ctx.epf_setup(k["C11"], k["C12"], k["C66"], c["rho"], (0.0,) * m.dim, k["sc"], c["tension_only"],
                  health0=c["health0"], precision=precision)
    try:
        ctx.epf_set_variant(variant)
    except px.PxbError as e:
        assert e.status == 7
        pytest.skip("variant %d does not fit these families" % variant)
    ctx.epf_set_bcs(c["bcs"])
    ctx.epf_start(c["u0"], None, c["dt"])
    ctx.epf_advance(NSTEPS, chunk=10)
    return ctx.epf_state()


def _check(c, got, tol=1e-10):
    u, uo, h, _ = got
    assert (c["h"] == 0).sum() > (c["health0"] == 0).sum() + 100  # the random start breaks bonds
    assert np.array_equal(h, c["h"])
    scale = np.abs(c["u"]).max()
    assert np.abs(u - c["u"]).max() <= tol * scale
    assert np.abs(uo - c["uo"]).max() <= tol * scale


@pytest.mark.parametrize("variant", list(range(N_VARIANTS)))
@pytest.mark.parametrize("tension_only", [True, False])
def test_plate_reflection_bcs_match_reference(ctx, variant, tension_only):
    c = case("plate", tension_only)
    _check(c, _run(ctx, c, variant))


def test_plate_compression_breaks_bonds():
    """With tension_only = false more bonds break than with tension only, from the same start."""
    assert (case("plate", False)["h"] == 0).sum() > (case("plate", True)["h"] == 0).sum()


@pytest.mark.parametrize("variant", list(range(N_VARIANTS)))
def test_slab_reflection_bcs_match_reference(ctx, variant):
    c = case("slab")
    _check(c, _run(ctx, c, variant))


@pytest.mark.parametrize("kind,variant", [("plate", 1), ("plate", 11), ("slab", 1), ("slab", 7)])
def test_reflection_bcs_mixed_within_1e6(ctx, kind, variant):
    c = case(kind)
    u, _, h, _ = _run(ctx, c, variant, precision=1)
    assert np.abs(u - c["u"]).max() <= 1e-6 * np.abs(c["u"]).max()
    assert (h != c["h"]).sum() <= 1e-4 * h.size


def test_tension_only_false_rate_matches_reference(ctx):
    """One rate call (damage then force) with compression failure on, against the reference element at a field that
    breaks bonds in compression and in tension."""
    from oracle import RefEpf
    c = case("plate", False)
    m, k = c["m"], c["k"]
    E, nu = 190e9, 0.3
    G0 = 0.01 ** 2 * 12 * E * m.delta / (5 * math.pi)
    el = RefEpf(m, E, nu, c["rho"], G0, tension_only=False)
    u = c["u0"] * 4.0
    a_ref, h_ref, _ = el.rate(u)
    ctx.set_geometry(m.coords, m.vols, m.off, m.ids, m.delta, m.dx_char, 2, mirror=m.mirror)
    ctx.epf_setup(k["C11"], k["C12"], k["C66"], c["rho"], (0.0, 0.0), k["sc"], False, health0=c["health0"])
    a, nbk = ctx.epf_rate(u)
    h = ctx.epf_state()[2]
    assert np.array_equal(h, (h_ref > 0).astype(np.uint8))
    assert nbk == int(c["health0"].sum() - h.sum())
    assert np.abs(a - a_ref).max() <= 1e-12 * np.abs(a_ref).max()
