"""pxb_gbuild_noalloc_d: the g-build entry point for callers that cannot call cudaMalloc (their device memory
belongs to another allocator, or they cannot afford its implicit synchronisation).  The test owns every
buffer (allocated here with torch, outside the entry point); the entry point's only working memory is the
library's fixed 4 MiB device array.  Calls in a row (a 2D lattice, then a 3D lattice, FP64 and mixed) must each
match the regular allocating entry point (pxb_gbuild) within the g-function tolerance.  A call that reports a
degenerate family is followed by a clean call that must report none, which shows that the counters the shared
array keeps from one call are reset for the next."""
import ctypes as C

import numpy as np
import pytest

from conftest import load_golden, scaled_err

pytestmark = pytest.mark.gpu


def _noalloc(lib, torch, dim, off, ids1, coords, vols, delta, dx_char, precision=0, layer=None, expect=0):
    """Run the entry point on torch-owned device copies; returns (status, ops[nb, nop], defect or None, deg, nd,
    first)."""
    dev = torch.device("cuda", 0)
    n = coords.size // 3
    nb = int(off[-1])
    nop = 5 if dim == 2 else 9
    t_off = torch.from_numpy(np.ascontiguousarray(off, dtype=np.int32)).to(dev)
    t_ids = torch.from_numpy(np.ascontiguousarray(ids1 - 1, dtype=np.int32)).to(dev)
    t_xyz = torch.from_numpy(np.ascontiguousarray(coords, dtype=np.float64)).to(dev)
    t_vol = torch.from_numpy(np.ascontiguousarray(vols, dtype=np.float64)).to(dev)
    t_lay = None if layer is None else torch.from_numpy(np.ascontiguousarray(layer, dtype=np.int32)).to(dev)
    odt = torch.float32 if precision else torch.float64
    ops = torch.full((max(nb, 1) * nop,), float("nan"), dtype=odt, device=dev)
    nd_def = (nop - dim) * dim
    defect = torch.full((n * nd_def,), float("nan"), dtype=torch.float32, device=dev) if precision else None
    deg = torch.zeros(n, dtype=torch.uint8, device=dev)
    nd, first = C.c_int(-1), C.c_int(-1)
    stream = torch.cuda.current_stream(dev).cuda_stream
    st = lib.pxb_gbuild_noalloc_d(dim, 2, precision, n, C.c_longlong(nb), C.c_void_p(t_off.data_ptr()),
                                  C.c_void_p(t_ids.data_ptr()), C.c_void_p(t_xyz.data_ptr()),
                                  C.c_void_p(t_vol.data_ptr()), None if t_lay is None else C.c_void_p(t_lay.data_ptr()),
                                  C.c_double(delta), C.c_double(dx_char), C.c_void_p(ops.data_ptr()),
                                  None if defect is None else C.c_void_p(defect.data_ptr()),
                                  C.c_void_p(deg.data_ptr()), C.byref(nd), C.byref(first), C.c_void_p(stream))
    assert st == expect, lib.pxb_last_error().decode()
    g = ops.double().cpu().numpy()[: nb * nop].reshape(nb, nop)
    dfc = None if defect is None else defect.double().cpu().numpy().reshape(n, nop - dim, dim)
    return g, dfc, deg.cpu().numpy(), nd.value, first.value


def _call(lib, torch, d, dim, precision=0):
    s = d["scalars"]
    g, dfc, deg, nd, first = _noalloc(lib, torch, dim, d["off"], d["ids"], d["coords"], d["vols"], float(s[0]),
                                      float(s[4]), precision)
    assert nd == 0 and first == 0 and not deg.any()
    return g, dfc


def _regular(ctx, d, dim, precision=0):
    s = d["scalars"]
    ctx.set_geometry(d["coords"], d["vols"], d["off"], d["ids"], s[0], s[4], dim, mirror=d["mirror"])
    ctx.gbuild(2, precision)
    return ctx.get_ops()


def _first_moments(g, d, dim):
    """sum_j g^k_j xi_j[m] of the second-derivative slots k >= dim, per node, and its magnitude scale."""
    x = d["coords"].reshape(-1, 3)[:, :dim]
    off = d["off"]
    n = off.size - 1
    node = np.repeat(np.arange(n), np.diff(off))
    xi = x[d["ids"] - 1] - x[node]
    m = np.zeros((n, g.shape[1] - dim, dim))
    sc = np.zeros_like(m)
    for k in range(dim, g.shape[1]):
        for c in range(dim):
            np.add.at(m[:, k - dim, c], node, g[:, k] * xi[:, c])
            np.add.at(sc[:, k - dim, c], node, np.abs(g[:, k] * xi[:, c]))
    return m, sc


def _apply_mixed(g, dfc, d, dim, u):
    """All derivatives of u with the FP32-operator defect correction D^k -= sum_m defect[k][m] D^m."""
    off = d["off"]
    n = off.size - 1
    node = np.repeat(np.arange(n), np.diff(off))
    du = u[d["ids"] - 1] - u[node]
    out = np.zeros((n, g.shape[1]))
    for k in range(g.shape[1]):
        np.add.at(out[:, k], node, g[:, k] * du)
    out[:, dim:] -= np.einsum("nkm,nm->nk", dfc, out[:, :dim])
    return out


def test_noalloc_gbuild_matches_regular_entry_point_twice(ctx):
    import torch
    lib = ctx.L
    first = load_golden("poisson16")
    second = load_golden("lattice3d")
    g1, _ = _call(lib, torch, first, 2)
    g2, _ = _call(lib, torch, second, 3)
    assert scaled_err(g1, _regular(ctx, first, 2), first["off"]) <= 1e-12
    assert scaled_err(g2, _regular(ctx, second, 3), second["off"]) <= 1e-12
    # and against the reference's own g-functions
    assert scaled_err(g1, first["ops"], first["off"]) <= 1e-12
    assert scaled_err(g2, second["ops"], second["off"]) <= 1e-12


@pytest.mark.parametrize("name,dim", [("poisson16", 2), ("lattice3d", 3)])
def test_noalloc_mixed_matches_regular_mixed_with_defects(ctx, name, dim):
    """PXB_MIXED: the FP32 operators equal the regular mixed build's; the defects are the first moments of those
    stored operators; the corrected apply equals the regular mixed apply and stays within 1e-6 of FP64."""
    import torch
    lib = ctx.L
    d = load_golden(name)
    g, dfc = _call(lib, torch, d, dim, precision=1)
    g_reg = _regular(ctx, d, dim, precision=1)
    assert scaled_err(g, g_reg, d["off"]) <= 1e-6
    assert np.isfinite(dfc).all()
    m, sc = _first_moments(g, d, dim)
    assert np.all(np.abs(dfc - m) <= 1e-6 * sc + 1e-300)
    rng = np.random.default_rng(7)
    u = rng.standard_normal(d["coords"].size // 3)
    nop = g.shape[1]
    ours = _apply_mixed(g, dfc, d, dim, u)
    regular = ctx.apply(u, list(range(nop))).reshape(-1, nop)
    off = d["off"]
    node = np.repeat(np.arange(off.size - 1), np.diff(off))
    du = np.abs(u[d["ids"] - 1] - u[node])
    scale = np.zeros_like(ours)
    for k in range(nop):
        np.add.at(scale[:, k], node, np.abs(g[:, k]) * du)
    assert np.all(np.abs(ours - regular) <= 1e-10 * scale + 1e-300)
    exact = _apply_mixed(d["ops"], np.zeros_like(dfc), d, dim, u)  # FP64 reference operators, no correction
    assert np.all(np.abs(ours - exact) <= 1e-6 * scale + 1e-300)


def _truncate_family(d, node, keep):
    """Families of d with node `node` (0-based) cut to its first `keep` members."""
    off, ids = d["off"], d["ids"]
    lens = np.diff(off).copy()
    parts = [ids[off[i]:off[i + 1]] if i != node else ids[off[i]:off[i] + keep] for i in range(off.size - 1)]
    lens[node] = keep
    return np.concatenate([[0], np.cumsum(lens)]).astype(np.int32), np.concatenate(parts).astype(np.int32)


def test_noalloc_degenerate_family_then_clean_call(ctx):
    """A family too small for order 2 is reported with its 1-based id; a ghost of layer 2 with that family gets zero
    operators instead; the next clean call reports nothing left over from the failed one."""
    import torch
    lib = ctx.L
    d = load_golden("poisson16")
    s = d["scalars"]
    bad = 40
    off, ids = _truncate_family(d, bad, 3)
    _, _, deg, nd, first = _noalloc(lib, torch, 2, off, ids, d["coords"], d["vols"], float(s[0]), float(s[4]),
                                    expect=3)
    assert nd == 1 and first == bad + 1 and deg[bad] == 1 and deg.sum() == 1
    layer = np.zeros(d["coords"].size // 3, dtype=np.int32)
    layer[bad] = 2
    g, _, deg, nd, first = _noalloc(lib, torch, 2, off, ids, d["coords"], d["vols"], float(s[0]), float(s[4]),
                                    layer=layer)
    assert nd == 0 and first == 0
    assert np.all(g[off[bad]:off[bad + 1]] == 0.0)
    g1, _ = _call(lib, torch, d, 2)
    assert scaled_err(g1, d["ops"], d["off"]) <= 1e-12


def test_noalloc_rejects_malformed_families(ctx):
    import torch
    lib = ctx.L
    d = load_golden("poisson16")
    s = d["scalars"]
    n = d["coords"].size // 3
    ids = d["ids"].copy()
    ids[17] = n + 1  # 0-based n: one past the last node
    _noalloc(lib, torch, 2, d["off"], ids, d["coords"], d["vols"], float(s[0]), float(s[4]), expect=1)
    assert b"malformed" in lib.pxb_last_error()
    off = d["off"].copy()
    off[5], off[6] = off[6], off[5]
    _noalloc(lib, torch, 2, off, d["ids"], d["coords"], d["vols"], float(s[0]), float(s[4]), expect=1)
    assert b"malformed" in lib.pxb_last_error()


def test_noalloc_rejects_sizes_beyond_its_scratch(ctx):
    import torch
    lib = ctx.L
    limit = lib.pxb_gbuild_noalloc_max_nodes(2)
    assert limit == ((4 << 20) - 256) // 16
    dev = torch.device("cuda", 0)
    buf = torch.zeros(16, dtype=torch.float64, device=dev)
    p = C.c_void_p(buf.data_ptr())
    st = lib.pxb_gbuild_noalloc_d(2, 2, 0, limit + 1, C.c_longlong(0), p, p, p, p, None, C.c_double(1.0),
                                  C.c_double(0.0), p, None, None, None, None, None)
    assert st == 1
    assert b"exceed" in lib.pxb_last_error()
