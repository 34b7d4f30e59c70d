"""The full 3D slab (120x120x24 bulk nodes + ghosts = 385,920 nodes, 44,189,344 directed bonds, central edge notch
of depth 20h as a force-only crack plane) against the reference itself (oracle/_ref/libperix_ref.so: the
reference's mesh generator, createNeighborNodes, ExplicitPDDOFracElement and its DirichletBC / NeumannBC objects,
with the harness's central difference).

* Families built on the device (pxb_set_geometry_points) equal the reference's createNeighborNodes at full size.
* Eight explicit steps from a seeded random field (std 1 um against a 4 um critical extension of the shortest
  bonds, so thousands of bonds break) on several step schedules: FP64 with identical damage sets and u within
  1e-10 of its magnitude; mixed within 1e-6 with damage sets identical but for bonds at the threshold."""
import math

import numpy as np
import pytest

from oracle import ref_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not ref_available(), reason="reference harness not built")]

NSTEPS = 8


@pytest.fixture(scope="module")
def slab():
    import perix_b200 as px
    from oracle import RefEpf, RefMesh
    nx, ny, nz, h = 120, 120, 24, 1e-3
    Lx, Ly, Lz = nx * h, ny * h, nz * h
    plane = [0.0, Ly / 2, -1.0, 20 * h, Ly / 2, -1.0, 20 * h, Ly / 2, 1.0, 0.0, Ly / 2, 1.0]
    m = RefMesh.structured(3, nx, ny, nz, [0, Lx, 0, Ly, 0, Lz], 3.015, 2, planes=[plane], force_only=True)
    E, nu, rho = 72e9, 0.22, 2440.0
    G0 = 0.004 ** 2 * 6 * E * m.delta / 5
    el = RefEpf(m, E, nu, rho, G0)
    el.rate(np.zeros(3 * m.n))  # seeds the notch, derives s_c and the elastic constants
    k = el.constants()
    dt = 0.8 * h / math.sqrt(k["C11"] / rho)
    bcs = [px.BC("neumann", [0, 1, 2], m.group(w + "nodes_ghost"))
           for w in ("left", "right", "bottom", "top", "back", "front")]
    alld = m.group("alldomain")
    bcs.append(px.BC("dirichlet", [1], alld, value=[0, 0, 0], velocity=[0, 2.0, 0], direct=True,
                     box=[-1, 1, Ly - 3 * h, 1, -1, 1]))
    bcs.append(px.BC("dirichlet", [1], alld, value=[0, 0, 0], velocity=[0, -2.0, 0], direct=True,
                     box=[-1, 1, -1, 3 * h, -1, 1]))
    health0 = (1 - px.crack_cut_mask(m.coords, m.mirror, m.off, m.ids, planes=[plane])).astype(np.uint8)
    rng = np.random.default_rng(2024)
    u0 = rng.standard_normal(3 * m.n) * 1e-6
    u, uo, hh, _ = el.run(u0, None, dt, NSTEPS, [b.as_dict() for b in bcs])
    return dict(m=m, k=k, rho=rho, dt=dt, bcs=bcs, health0=health0, u0=u0, u=u, uo=uo, h=(hh > 0).astype(np.uint8),
                E=E, nu=nu, G0=G0)


def test_slab_families_built_on_device_equal_reference(ctx, slab):
    m = slab["m"]
    assert m.n == 385920 and m.nb == 44189344
    ctx.set_geometry_points(m.coords, m.vols, m.delta, m.delta, m.dx_char, 3, mirror=m.mirror)
    off, ids = ctx.get_families()
    assert np.array_equal(off, m.off)
    assert np.array_equal(ids, m.ids)


def _run(ctx, s, variant, precision):
    import perix_b200 as px
    m, k = s["m"], s["k"]
    ctx.set_geometry(m.coords, m.vols, m.off, m.ids, m.delta, m.dx_char, 3, mirror=m.mirror)
    ctx.epf_setup(k["C11"], k["C12"], k["C66"], s["rho"], (0.0, 0.0, 0.0), k["sc"], True, health0=s["health0"],
                  precision=precision)
    try:
        ctx.epf_set_variant(variant)
    except px.PxbError as e:
        assert e.status == 7
        pytest.skip("variant %d does not fit these families" % variant)
    ctx.epf_set_bcs(s["bcs"])
    ctx.epf_start(s["u0"], None, s["dt"])
    ctx.epf_advance(NSTEPS, chunk=NSTEPS)
    return ctx.epf_state()


@pytest.mark.parametrize("variant", [1, 5, 6, 7, 8, 9, 10, 11, 12, 13, 16, 17, 18, 19, 20])
def test_slab_fp64_steps_match_reference(ctx, slab, variant):
    u, uo, h, _ = _run(ctx, slab, variant, 0)
    assert (slab["h"] == 0).sum() > (slab["health0"] == 0).sum() + 1000
    assert np.array_equal(h, slab["h"])
    scale = np.abs(slab["u"]).max()
    assert np.abs(u - slab["u"]).max() <= 1e-10 * scale
    assert np.abs(uo - slab["uo"]).max() <= 1e-10 * scale


@pytest.mark.parametrize("variant", [1, 7, 8, 10, 12, 13, 17, 19])
def test_slab_mixed_steps_within_1e6(ctx, slab, variant):
    u, _, h, _ = _run(ctx, slab, variant, 1)
    assert np.abs(u - slab["u"]).max() <= 1e-6 * np.abs(slab["u"]).max()
    assert (h != slab["h"]).sum() <= 1e-5 * h.size


@pytest.mark.parametrize("variant,chunks", [(1, -1), (13, -1), (13, 8)])
def test_slab_rate_call_matches_reference(ctx, slab, variant, chunks):
    """The per-step rate call at full size: variant 1 runs one kernel; the staged variant 13 runs the pipelined call
    with pinned buffers (node chunks, 3 by default or 8, whose kernels start as their neighbours' u arrives and whose
    accelerations go down while the next chunk computes), through pageable arrays and through pinned ones (repeated calls with the same pinned buffers
    capture, then replay, the call as a graph; the bonds broken by the first call stay broken, so the later calls
    break none and return the same accelerations)."""
    import ctypes as C

    import torch
    from oracle import RefEpf
    m, k = slab["m"], slab["k"]
    el = RefEpf(m, slab["E"], slab["nu"], slab["rho"], slab["G0"])
    el.rate(np.zeros(3 * m.n))  # seeds the notch
    acc_ref, h_ref, _ = el.rate(slab["u0"])
    h_ref = (h_ref > 0).astype(np.uint8)
    broken_ref = int((slab["health0"] > 0).sum() - h_ref.sum())
    assert broken_ref > 100
    scale = np.abs(acc_ref).max()
    ctx.set_geometry(m.coords, m.vols, m.off, m.ids, m.delta, m.dx_char, 3, mirror=m.mirror)

    def setup():
        ctx.epf_setup(k["C11"], k["C12"], k["C66"], slab["rho"], (0.0, 0.0, 0.0), k["sc"], True,
                      health0=slab["health0"])
        ctx.epf_set_variant(variant)
        ctx.epf_set_rate_chunks(chunks)

    setup()
    acc, nbroken = ctx.epf_rate(slab["u0"])
    assert np.abs(acc - acc_ref).max() <= 1e-10 * scale
    assert np.array_equal(ctx.epf_state()[2], h_ref) and nbroken == broken_ref
    setup()
    uh = torch.from_numpy(slab["u0"].copy()).pin_memory()
    ah = torch.zeros(3 * m.n, dtype=torch.float64).pin_memory()
    for call in range(3):
        ah.zero_()
        nb = C.c_longlong(-1)
        assert ctx.L.pxb_epf_rate(ctx.h, C.c_void_p(uh.data_ptr()), C.c_void_p(ah.data_ptr()), C.byref(nb)) == 0
        assert np.abs(ah.numpy() - acc_ref).max() <= 1e-10 * scale
        assert nb.value == (broken_ref if call == 0 else 0)
        assert np.array_equal(ctx.epf_state()[2], h_ref)
