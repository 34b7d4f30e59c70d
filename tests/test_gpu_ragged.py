"""Explicit fracture on ragged inputs: every schedule variant of the step kernel's per-step call against the
oracle (C restatement of ExplicitPDDOFracElement.cpp:239-299 on the oracle's own g-functions).

The cloud is a jittered lattice (U(+-0.2h)) with random holes, so families are boundary-truncated and uneven, the
node count is no multiple of any tile size, a tenth of the bonds start broken, and the displacement field breaks
part of the rest.  A cloud with an isolated node is rejected by the setup with the node's 1-based id: its moment
matrix is singular, and the reference's g-function build aborts on such a family (CalcPDOperators.cpp:196-225).
Repeated calls with the same pinned host buffers (the captured-graph replay of the per-step call) are checked the
same way.

Tolerances: damage sets identical; FP64 accelerations within 1e-12 of the largest, mixed (FP32 operator storage)
within 1e-6."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N_VARIANTS = 21
E, NU, RHO, SC = 190e9, 0.3, 8000.0, 0.01


def ragged_cloud(dim, seed):
    rng = np.random.default_rng(seed)
    side = (11, 9) if dim == 2 else (7, 5, 5)
    grid = np.stack(np.meshgrid(*[np.arange(s) for s in side], indexing="ij"), -1).reshape(-1, dim).astype(float)
    pts = grid + 0.5 + rng.uniform(-0.2, 0.2, grid.shape)
    pts = pts[rng.random(len(pts)) > 0.08]
    coords = np.zeros((len(pts), 3))
    coords[:, :dim] = pts
    return coords, rng


def navier_columns(dim, ops):
    """(Gxx, Gyy, Gxy) in 2D, (Gxx, Gyy, Gzz, Gxy, Gxz, Gyz) in 3D from the q-list order of PDOperators.cpp:51-111."""
    return ops[:, [2, 4, 3]] if dim == 2 else ops[:, [3, 6, 8, 4, 5, 7]]


@pytest.fixture(scope="module", params=[2, 3])
def case(request, port):
    import perix_b200 as px
    dim = request.param
    coords, rng = ragged_cloud(dim, 5 + dim)
    n = len(coords)
    delta = 3.015
    off, ids = px.families(coords, delta, dim == 3)
    vols = np.ones(n)
    ops, deg = port.gbuild(dim, 2, coords, vols, off, ids, delta, 1.0)
    assert deg.sum() == 0
    nb = int(off[-1])
    sizes = np.diff(off)
    assert sizes.min() < sizes.max() // 2      # boundary-truncated families next to full ones
    assert all(n % t for t in (8, 16, 32, 64))  # the last tile of every schedule is partial
    h0 = (rng.random(nb) > 0.1).astype(np.uint8)
    u = 0.012 * rng.standard_normal(n * dim)
    b = np.array([3.0, -2.0, 1.0])[:dim]
    Cv = px.elastic_constants(dim, False, E, NU)
    a_ref, h_ref = port.epf_rate(dim, coords, off, ids, navier_columns(dim, ops), Cv, RHO, b, SC, u,
                                 h0.astype(float))
    h_ref = (h_ref > 0).astype(np.uint8)
    nbreak = int(h0.sum() - h_ref.sum())
    assert 0 < nbreak < int(h0.sum())
    return dict(dim=dim, coords=coords, off=off, ids=ids, vols=vols, delta=delta, h0=h0, u=u, b=b, Cv=Cv,
                a_ref=a_ref, h_ref=h_ref, nbreak=nbreak)


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("variant", list(range(N_VARIANTS)))
def test_ragged_rate_every_variant(ctx, case, variant, precision):
    import perix_b200 as px
    c = case
    dim = c["dim"]
    ctx.set_geometry(c["coords"], c["vols"], c["off"], c["ids"], c["delta"], 1.0, dim)
    C11, C12, C66 = c["Cv"]
    ctx.epf_setup(C11, C12, C66, RHO, tuple(c["b"]), SC, True, health0=c["h0"], precision=precision)
    try:
        ctx.epf_set_variant(variant)
    except px.PxbError as e:
        assert e.status == 7  # families too large for this tile size
        pytest.skip("variant %d does not fit these families" % variant)
    a, nbk = ctx.epf_rate(c["u"])
    _, _, h, _ = ctx.epf_state()
    assert np.array_equal(h, c["h_ref"])
    assert nbk == c["nbreak"]
    tol = 1e-12 if precision == 0 else 1e-6
    assert np.abs(a - c["a_ref"]).max() <= tol * np.abs(c["a_ref"]).max()


@pytest.mark.parametrize("dim", [2, 3])
def test_isolated_node_rejected_with_its_id(ctx, dim):
    import perix_b200 as px
    coords, _ = ragged_cloud(dim, 5 + dim)
    far = np.zeros((1, 3))
    far[0, :dim] = 100.0
    coords = np.vstack([coords, far])
    n = len(coords)
    off, ids = px.families(coords, 3.015, dim == 3)
    assert off[-1] == off[-2]  # the added node has an empty family
    ctx.set_geometry(coords, np.ones(n), off, ids, 3.015, 1.0, dim)
    C11, C12, C66 = px.elastic_constants(dim, False, E, NU)
    with pytest.raises(px.PxbError) as ei:
        ctx.epf_setup(C11, C12, C66, RHO, (0, 0, 0), SC, True)
    assert ei.value.status == 3
    assert "node %d" % n in str(ei.value)


@pytest.mark.parametrize("variant", list(range(N_VARIANTS)))
def test_rate_repeated_on_pinned_buffers(ctx, case, port, variant):
    """The per-step call made repeatedly with the same pinned host buffers, as a time loop does: the second and
    later calls replay one captured graph that reads the buffers' contents at each call.  Call 1 breaks bonds,
    call 2 (same u) breaks none and gives the same acceleration (within the FP64 tolerance: some
    schedules sum a family in a different order from call to call), call 3 (new u in the same buffer) matches the
    oracle from the health after call 1."""
    import ctypes as C

    import perix_b200 as px
    import torch
    c = case
    dim = c["dim"]
    ctx.set_geometry(c["coords"], c["vols"], c["off"], c["ids"], c["delta"], 1.0, dim)
    C11, C12, C66 = c["Cv"]
    ctx.epf_setup(C11, C12, C66, RHO, tuple(c["b"]), SC, True, health0=c["h0"])
    try:
        ctx.epf_set_variant(variant)
    except px.PxbError as e:
        assert e.status == 7
        pytest.skip("variant %d does not fit these families" % variant)
    nd = c["u"].size
    u_h = torch.empty(nd, dtype=torch.float64, pin_memory=True)
    a_h = torch.empty(nd, dtype=torch.float64, pin_memory=True)
    up = C.cast(C.c_void_p(u_h.data_ptr()), C.POINTER(C.c_double))
    ap = C.cast(C.c_void_p(a_h.data_ptr()), C.POINTER(C.c_double))
    nbk = C.c_longlong(0)

    def call():
        st = ctx.L.pxb_epf_rate(ctx.h, up, ap, C.byref(nbk))
        assert st == 0, ctx.L.pxb_last_error().decode()
        return a_h.numpy().copy(), nbk.value

    u_h.copy_(torch.from_numpy(c["u"]))
    a1, n1 = call()
    assert n1 == c["nbreak"]
    assert np.abs(a1 - c["a_ref"]).max() <= 1e-12 * np.abs(c["a_ref"]).max()
    a2, n2 = call()
    assert n2 == 0
    assert np.abs(a2 - c["a_ref"]).max() <= 1e-12 * np.abs(c["a_ref"]).max()
    u3 = 1.5 * c["u"]
    u_h.copy_(torch.from_numpy(u3))
    a3, n3 = call()
    ops, _ = port.gbuild(dim, 2, c["coords"], c["vols"], c["off"], c["ids"], c["delta"], 1.0)
    a_ref3, h_ref3 = port.epf_rate(dim, c["coords"], c["off"], c["ids"], navier_columns(dim, ops), c["Cv"], RHO,
                                   c["b"], SC, u3, c["h_ref"].astype(float))
    _, _, h, _ = ctx.epf_state()
    assert np.array_equal(h, (h_ref3 > 0).astype(np.uint8))
    assert n3 == int(c["h_ref"].sum() - (h_ref3 > 0).sum()) and n3 > 0
    assert np.abs(a3 - a_ref3).max() <= 1e-12 * np.abs(a_ref3).max()
    # another schedule on the same buffers: queued once, then captured and replayed again
    ctx.epf_set_variant(1 if variant != 1 else 5)
    for _ in range(3):
        a4, n4 = call()
        assert n4 == 0
        assert np.abs(a4 - a_ref3).max() <= 1e-12 * np.abs(a_ref3).max()
