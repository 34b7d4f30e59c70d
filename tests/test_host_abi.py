"""CPU tests of the product library: it loads, exports every C-ABI symbol declared in include/*.h, its host
utilities (lattice + ghosts, reference-order families, crack seeding, CSR pattern) reproduce the reference's
own outputs bit for bit, and it fails cleanly (no crash, no CPU fallback) where no GPU is present."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT, gpu_available, load_golden


@pytest.fixture(scope="module")
def px():
    from perix_b200.build import build
    build()
    import perix_b200
    return perix_b200


def declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(pxb_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol(px):
    lib = px.lib()
    names = declared("perix_b200.h")
    assert len(names) >= 40
    headers = sorted(h for h in os.listdir(os.path.join(ROOT, "include")) if h.startswith("perix_b200") and h.endswith(".h"))
    assert "perix_b200_measure.h" in headers
    for h in headers:
        names = declared(h)
        assert names, h
        missing = [n for n in names if not hasattr(lib, n)]
        assert not missing, (h, missing)


def test_dropin_symbols_exported(px):
    out = subprocess.run(["nm", "-D", "-C", "--defined-only", px.lib_path()], capture_output=True, text=True).stdout
    for fn in ("perix_cuda::assemble(", "perix_cuda::assembleCahnHilliard(", "perix_cuda::assembleStressCahnHilliard(",
               "perix_cuda::assembleCached(", "perix_cuda::assembleExplicitPDDOFracAccel(", "perix_cuda::shutdown()"):
        assert fn in out, fn


def test_version_and_null_context_errors(px):
    lib = px.lib()
    assert lib.pxb_version() == 1
    assert lib.pxb_set_geometry(None, 0, 2, None, None, None, None, C.c_double(1.0), C.c_double(0.0), None, None) == 1
    assert b"NULL context" in lib.pxb_last_error()
    assert lib.pxb_gbuild(None, 2, 0, None, None) == 1


@pytest.mark.skipif(gpu_available(), reason="checks the no-GPU failure path")
def test_no_gpu_fails_loudly(px):
    with pytest.raises(px.PxbError) as e:
        px.Context(0)
    assert e.value.status == 2


LATTICES = {
    "poisson16": (2, 16, 16, 0, [0, 1, 0, 1]),
    "lattice3d": (3, 5, 5, 4, [0, 0.5, 0, 0.5, 0, 0.4]),
    "epf2d": (2, 40, 20, 0, [0, 40 * 5e-4, 0, 20 * 5e-4]),
    "epf3d": (3, 10, 10, 4, [0, 1e-2, 0, 1e-2, 0, 4e-3]),
}


@pytest.mark.parametrize("name", sorted(LATTICES))
def test_lattice_matches_reference(px, name):
    d = load_golden(name)
    L = px.lattice(*LATTICES[name])
    assert np.array_equal(L.coords, d["coords"])
    assert np.array_equal(L.vols, d["vols"])
    assert np.array_equal(L.mirror, d["mirror"])
    delta = 3.015 * L.dxyz[0] * (1 + 1e-6)
    assert delta == d["scalars"][0]
    assert max(L.dxyz) == d["scalars"][4]


@pytest.mark.parametrize("name", ["poisson16", "lattice3d", "cloud2d", "cloud3d", "epf2d", "epf3d"])
def test_families_match_reference(px, name):
    d = load_golden(name)
    dim = 3 if d["scalars"][3] > 0 else 2
    cracks = d["cracks"] if "cracks" in d else None
    planes = d["plane"].reshape(1, -1) if "plane" in d else None
    mirror = d["mirror"] if d["mirror"].any() else None
    off, ids = px.families(d["coords"], d["scalars"][0], dim == 3, cracks=cracks, planes=planes, mirror=mirror,
                           force_only=cracks is not None or planes is not None)
    assert np.array_equal(off, d["off"]) and np.array_equal(ids, d["ids"])


@pytest.mark.parametrize("name", ["epf2d", "epf3d"])
def test_crack_seed_matches_reference(px, name):
    d = load_golden(name)
    cracks = d["cracks"] if "cracks" in d else None
    planes = d["plane"].reshape(1, -1) if "plane" in d else None
    cut = px.crack_cut_mask(d["coords"], d["mirror"], d["off"], d["ids"], cracks=cracks, planes=planes)
    assert np.array_equal(1 - cut, d["health0"])


@pytest.mark.parametrize("name,ndof", [("poisson16", 1), ("poisson16", 2), ("lattice3d", 1)])
def test_csr_pattern_matches_reference(px, name, ndof):
    d = load_golden(name)
    rp, cols = px.csr_pattern(d["off"], d["ids"], d["mirror"], ndof)
    assert np.array_equal(rp, d["rowptr%d" % ndof]) and np.array_equal(cols, d["cols%d" % ndof])


def test_lattice_groups_and_errors(px):
    L = px.lattice(2, 6, 4, 0, [0, 6, 0, 4])
    assert L.n == 24 + 2 * 4 + 2 * 6
    assert np.array_equal(L.group("leftnodes_ghost"), np.arange(25, 29))
    assert np.array_equal(L.group("leftnodes"), np.array([1, 7, 13, 19]))
    with pytest.raises(px.PxbError):
        px.lattice(4, 2, 2, 2, [0, 1, 0, 1])


def test_multi_index_table_matches_reference_order(px):
    assert px.multi_indices(2, 2) == [(1, 0, 0), (0, 1, 0), (2, 0, 0), (1, 1, 0), (0, 2, 0)]
    assert px.multi_indices(3, 2)[3:] == [(2, 0, 0), (1, 1, 0), (1, 0, 1), (0, 2, 0), (0, 1, 1), (0, 0, 2)]
