"""The ghost BC preset of the oracle's C restatement (oracle/pddo_oracle.c orc_bc_preset) against the reference's
own DirichletBC / NeumannBC objects (compiled into oracle/_ref/libperix_ref.so, applied in list order like
BCSystem::presetSolution, BCSystem.cpp:114-129).

The programs cover the reference's default reflection form 2 g(t) - u_bulk (DirichletBC.cpp:141-143) with a
velocity ramp, direct pins, boxes with an unconstrained axis (min > max, DirichletBC.cpp:89-98), a z window in 2D,
a reflection off a directly pinned bulk node (the closed form 2G - G') and Neumann copies of pinned bulk nodes."""
import numpy as np
import pytest

from oracle import ref_available

pytestmark = pytest.mark.skipif(not ref_available(), reason="reference harness not built")


def bc_programs(m, dim):
    """BC lists (dicts in the oracle layout) exercising every closed form of the preset."""
    g = {w: m.group(w + "nodes_ghost") for w in ("left", "right", "bottom", "top")}
    if dim == 3:
        g.update({w: m.group(w + "nodes_ghost") for w in ("back", "front")})
    comps = list(range(dim))
    xyz = m.coords.reshape(-1, 3)
    ymid = 0.5 * (xyz[:, 1].min() + xyz[:, 1].max())
    v = [0.3, -0.2, 0.1][:dim]
    w = [16.5, 2.0, -1.0][:dim]
    inactive = [1.0, -1.0]  # min > max: the axis is not constrained
    progs = []
    # 1. reflection with a ramp on the left wall, boxed in y (x and z unconstrained), Neumann elsewhere
    p = [dict(kind="dirichlet", comps=comps, nodes=g["left"], value=v, velocity=w,
              box=inactive + [xyz[:, 1].min() - 1, ymid] + inactive)]
    p += [dict(kind="neumann", comps=comps, nodes=g[s]) for s in g if s != "left"]
    progs.append(p)
    # 2. pin the left bulk column directly, then reflect the left ghosts off it (2G - G'), then copy its value to the
    #    bottom ghosts (a Neumann copy reads the mirror's latest value), a direct pin of the right wall in a z window
    #    that holds z = 0 in 2D (and the lower half in 3D)
    zlo, zhi = (-1.0, 1.0) if dim == 2 else (xyz[:, 2].min() - 1, 0.5 * (xyz[:, 2].min() + xyz[:, 2].max()))
    p = [dict(kind="dirichlet", comps=[0], nodes=m.group("leftnodes"), value=v, velocity=w, direct=True),
         dict(kind="dirichlet", comps=comps, nodes=g["left"], value=[-x for x in v], velocity=[0.5 * x for x in w]),
         dict(kind="neumann", comps=comps, nodes=g["bottom"]),
         dict(kind="dirichlet", comps=[dim - 1], nodes=g["right"], value=v, velocity=w, direct=True,
              box=inactive + inactive + [zlo, zhi])]
    progs.append(p)
    # 3. a box that excludes everything through its z window in 2D (z = 0 outside [1, 2]), then a reflection of the
    #    top wall without a box
    p = [dict(kind="dirichlet", comps=comps, nodes=g["top"], value=v, velocity=w, box=inactive + inactive + [1.0, 2.0]),
         dict(kind="dirichlet", comps=[0], nodes=g["top"], value=v, velocity=w)]
    progs.append(p)
    return progs


@pytest.mark.parametrize("dim", [2, 3])
def test_bc_preset_restatement_matches_reference_objects(port, dim):
    from oracle import RefMesh
    if dim == 2:
        m = RefMesh.structured(2, 16, 8, 0, [0, 1.6, 0, 0.8], 3.015)
    else:
        m = RefMesh.structured(3, 8, 7, 6, [0, 0.8, 0, 0.7, 0, 0.6], 3.015)
    rng = np.random.default_rng(3 + dim)
    for prog in bc_programs(m, dim):
        for t in (0.0, 1.7e-3):
            u = rng.standard_normal(m.n * dim)
            ref = m.bc_preset(prog, t, u)
            ours = port.bc_preset(dim, m.coords, m.mirror, prog, t, u)
            assert np.array_equal(ours, ref)
            assert not np.array_equal(ref, u)  # the program wrote something
