"""The CSR sparsity pattern built on the device (pxb_csr_build_pattern) against the host build (pxb_csr_pattern,
the restatement of SparseMatrix::initFromPDMesh, src/MathUtils/SparseMatrix.cpp:73-185, pinned bit-exact to the
reference's own pattern by the oracle tests): identical rowptr and cols on 2D and 3D lattices with mirror ghosts
and on a jittered cloud without them, for 1 to 3 dof per node; an implicit Cahn-Hilliard run and its adjoint give
bitwise the same results on either pattern; node lists above the device sort's capacity are refused."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _geometry(ctx, kind):
    import perix_b200 as px
    if kind == "2d":
        L = px.lattice(2, 32, 24, 0, [0.0, 1.0, 0.0, 0.75])
        coords, vols, mirror, h = L.coords, L.vols, L.mirror, L.dxyz[0]
        delta = 3.015 * h * (1.0 + 1e-6)
        off, ids = px.families(coords, delta, False, mirror=mirror)
        dim = 2
    elif kind == "3d":
        L = px.lattice(3, 10, 9, 8, [0.0, 1.0, 0.0, 0.9, 0.0, 0.8])
        coords, vols, mirror, h = L.coords, L.vols, L.mirror, L.dxyz[0]
        delta = 3.015 * h * (1.0 + 1e-6)
        off, ids = px.families(coords, delta, True, mirror=mirror)
        dim = 3
    else:
        rng = np.random.default_rng(5)
        n, h = 3000, 1.0 / 50
        pts = rng.uniform(0.0, 1.0, (n, 2))
        coords = np.zeros((n, 3))
        coords[:, :2] = pts
        coords = coords.reshape(-1)
        vols = np.full(n, h * h)
        mirror = None
        delta = 3.015 * h
        off, ids = px.families(coords, delta, False)
        dim = 2
    ctx.set_geometry(coords, vols, off, ids, delta, h, dim, mirror=mirror)
    return off, ids, mirror


@pytest.mark.parametrize("kind,ndofs", [("2d", (1, 2, 3)), ("3d", (1, 3)), ("cloud", (1, 2))])
def test_device_pattern_matches_host(ctx, kind, ndofs):
    import perix_b200 as px
    off, ids, mirror = _geometry(ctx, kind)
    for nd in ndofs:
        rowptr, cols = px.csr_pattern(off, ids, mirror, nd)
        nnz = ctx.csr_build_pattern(nd)
        assert nnz == cols.size
        r, c = ctx.csr_get_pattern()
        assert np.array_equal(r, rowptr)
        assert np.array_equal(c, cols)


def test_device_pattern_ch_gradient_identical():
    import perix_b200 as px
    from perix_b200.build import build
    build()
    out = []
    for device_pattern in (False, True):
        ctx = px.Context(0)
        try:
            L = px.lattice(2, 24, 24, 0, [0.0, 1.0, 0.0, 1.0])
            delta = 3.015 * L.dxyz[0] * (1.0 + 1e-6)
            off, ids = px.families(L.coords, delta, False, mirror=L.mirror)
            ctx.set_geometry(L.coords, L.vols, off, ids, delta, L.dxyz[0], 2, mirror=L.mirror)
            ctx.gbuild(2, px.FP64)
            ctx.ch_build_geometry()
            if device_pattern:
                ctx.csr_build_pattern(2)
            else:
                ctx.csr_set_pattern(*px.csr_pattern(off, ids, L.mirror, 2), 2)
            c0 = 0.5 + np.random.default_rng(3).uniform(-0.01, 0.01, L.n)
            out.append(ctx.ch_gradient(c0, 2.5, 1e-4, 1.0, 1e-6, 3))
        finally:
            ctx.close()
    (E0, dk0, g0, s0), (E1, dk1, g1, s1) = out
    assert E0 == E1 and dk0 == dk1 and np.array_equal(g0, g1)
    assert s0["lin_iters"] == s1["lin_iters"]


def test_device_pattern_refuses_long_lists(ctx):
    import perix_b200 as px
    L = px.lattice(2, 40, 40, 0, [0.0, 1.0, 0.0, 1.0])
    delta = 9.5 * L.dxyz[0]  # about 280 neighbours per node
    off, ids = px.families(L.coords, delta, False, mirror=L.mirror)
    assert int(np.diff(off).max()) + 1 > 256
    ctx.set_geometry(L.coords, L.vols, off, ids, delta, L.dxyz[0], 2, mirror=L.mirror)
    with pytest.raises(px.PxbError, match="more than 256"):
        ctx.csr_build_pattern(1)
