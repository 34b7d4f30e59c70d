"""pxb_gbuild_noalloc_d: the g-build entry point for callers that cannot call cudaMalloc (their device memory
belongs to another allocator, or they cannot afford its implicit synchronisation).  The test owns every
buffer (allocated here with torch, outside the entry point); the entry point's only working memory is the
library's fixed 4 MiB device array.  Two calls in a row (a 2D lattice, then a 3D lattice) must each match the
regular allocating entry point (pxb_gbuild) within the g-function tolerance, which also shows that the shared
array's leftovers from the first call do not leak into the second."""
import ctypes as C

import numpy as np
import pytest

from conftest import load_golden, scaled_err

pytestmark = pytest.mark.gpu


def _noalloc(lib, d, dim, torch, precision=0):
    dev = torch.device("cuda", 0)
    n = d["coords"].size // 3
    nb = int(d["off"][-1])
    nop = 5 if dim == 2 else 9
    off = torch.from_numpy(d["off"].astype(np.int32)).to(dev)
    ids0 = torch.from_numpy((d["ids"] - 1).astype(np.int32)).to(dev)
    xyz = torch.from_numpy(d["coords"].astype(np.float64)).to(dev)
    vol = torch.from_numpy(d["vols"].astype(np.float64)).to(dev)
    ops = torch.full((nb * nop,), float("nan"), dtype=torch.float64, device=dev)
    deg = torch.zeros(n, dtype=torch.uint8, device=dev)
    nd, first = C.c_int(-1), C.c_int(-1)
    stream = torch.cuda.current_stream(dev).cuda_stream
    st = lib.pxb_gbuild_noalloc_d(dim, 2, precision, n, C.c_longlong(nb), C.c_void_p(off.data_ptr()),
                                  C.c_void_p(ids0.data_ptr()), C.c_void_p(xyz.data_ptr()), C.c_void_p(vol.data_ptr()),
                                  C.c_double(float(d["scalars"][0])), C.c_double(float(d["scalars"][4])),
                                  C.c_void_p(ops.data_ptr()), C.c_void_p(deg.data_ptr()), C.byref(nd), C.byref(first),
                                  C.c_void_p(stream))
    assert st == 0, lib.pxb_last_error().decode()
    assert nd.value == 0 and first.value == 0
    return ops.cpu().numpy().reshape(nb, nop), deg.cpu().numpy()


def _regular(ctx, d, dim):
    s = d["scalars"]
    ctx.set_geometry(d["coords"], d["vols"], d["off"], d["ids"], s[0], s[4], dim, mirror=d["mirror"])
    ctx.gbuild(2, 0)
    return ctx.get_ops()


def test_noalloc_gbuild_matches_regular_entry_point_twice(ctx):
    import torch
    lib = ctx.L
    first = load_golden("poisson16")
    second = load_golden("lattice3d")
    g1, deg1 = _noalloc(lib, first, 2, torch)
    g2, deg2 = _noalloc(lib, second, 3, torch)
    assert not deg1.any() and not deg2.any()
    assert scaled_err(g1, _regular(ctx, first, 2), first["off"]) <= 1e-12
    assert scaled_err(g2, _regular(ctx, second, 3), second["off"]) <= 1e-12
    # and against the reference's own g-functions
    assert scaled_err(g1, first["ops"], first["off"]) <= 1e-12
    assert scaled_err(g2, second["ops"], second["off"]) <= 1e-12


def test_noalloc_rejects_sizes_beyond_its_scratch(ctx):
    import torch
    lib = ctx.L
    limit = lib.pxb_gbuild_noalloc_max_nodes(2)
    assert limit == ((4 << 20) - 256) // 16
    dev = torch.device("cuda", 0)
    buf = torch.zeros(16, dtype=torch.float64, device=dev)
    p = C.c_void_p(buf.data_ptr())
    st = lib.pxb_gbuild_noalloc_d(2, 2, 0, limit + 1, C.c_longlong(0), p, p, p, p, C.c_double(1.0), C.c_double(0.0),
                                  p, None, None, None, None)
    assert st == 1
    assert b"exceed" in lib.pxb_last_error()
