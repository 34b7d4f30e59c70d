"""ctypes mirror of the perix_b200 C-ABI (include/perix_b200.h).

Names and argument meanings follow the reference's CUDA-assembly boundary and element semantics
(reference include/PDSystem/CudaAssemble.h, src/ElmtSystem/ExplicitPDDOFracElement.cpp); see the header for
the per-function contract.  Host arrays are numpy; device arrays may be passed as raw pointers (ints), e.g.
``torch.Tensor.data_ptr()``.
"""
import ctypes as C
import math
import os
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

FP64 = 0
MIXED = 1

_PKG = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_PKG, "libperix_b200.so")
_LIB = None

_STATUS = {0: "OK", 1: "INVALID", 2: "CUDA", 3: "DEGENERATE", 4: "OOM", 5: "BLOWUP", 6: "STATE", 7: "UNSUPPORTED"}


class PxbError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__("%s: %s" % (_STATUS.get(status, str(status)), msg))
        self.status = status


def lib_path():
    return _LIB_PATH


def lib():
    """Load libperix_b200.so (built in-tree by perix_b200.build); raise if it is absent."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(_LIB_PATH):
            raise PxbError(6, "libperix_b200.so is not built (run `python -m perix_b200.build`)")
        L = C.CDLL(_LIB_PATH)
        L.pxb_last_error.restype = C.c_char_p
        L.pxb_version.restype = C.c_int
        _LIB = L
    return _LIB


def _p(a, ct=C.c_double):
    if a is None:
        return None
    if isinstance(a, int):
        return C.cast(C.c_void_p(a), C.POINTER(ct))
    return a.ctypes.data_as(C.POINTER(ct))


def _vp(a):
    return None if a is None else C.c_void_p(a)


def _check(status):
    if status != 0:
        raise PxbError(status, lib().pxb_last_error().decode(errors="replace"))


def _check_step(status, bad):
    if status != 0:
        e = PxbError(status, lib().pxb_last_error().decode(errors="replace"))
        e.bad_step = bad.value
        raise e


def _f64(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64)


def _i32(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.int32)


def _u8(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.uint8)


# ---------------------------------------------------------------------------------------------- host helpers
def multi_indices(dim, order):
    """Reference multi-index list (PDOperators.cpp:51-75): list of (p,q,r)."""
    out = []
    for o in range(1, order + 1):
        for p in range(o, -1, -1):
            if dim == 3:
                for q in range(o - p, -1, -1):
                    out.append((p, q, o - p - q))
            else:
                out.append((p, o - p, 0))
    return out


def elastic_constants(dim, plane_stress, E, nu):
    """Navier constants C11, C12, C66 (reference ExplicitPDDOFracElement.cpp:38-53)."""
    if dim >= 3 or not plane_stress:
        d = (1.0 + nu) * (1.0 - 2.0 * nu)
        return E * (1.0 - nu) / d, E * nu / d, E / (2.0 * (1.0 + nu))
    d = 1.0 - nu * nu
    return E / d, E * nu / d, E / (2.0 * (1.0 + nu))


def critical_stretch(dim, plane_stress, G0, E, delta):
    """s_c from the fracture energy (reference include/ElmtSystem/FractureCriterion.h:30-43)."""
    if G0 <= 0 or E <= 0 or delta <= 0:
        return 0.0
    if dim >= 3:
        s2 = 5.0 * G0 / (6.0 * E * delta)
    elif plane_stress:
        s2 = 4.0 * math.pi * G0 / (9.0 * E * delta)
    else:
        s2 = 5.0 * math.pi * G0 / (12.0 * E * delta)
    return math.sqrt(s2)


@dataclass
class LatticeMesh:
    dim: int
    n: int
    coords: np.ndarray        # (3n,) xyz interleaved
    vols: np.ndarray
    mirror: np.ndarray        # 1-based mirror bulk id, 0 for bulk
    ghost_group: np.ndarray   # -1 bulk, else index into GROUPS_2D / GROUPS_3D
    dxyz: np.ndarray
    nbulk: int = 0

    def group(self, name):
        """Node ids (1-based) of a reference physical group: '<wall>nodes_ghost', '<wall>nodes', 'alldomain'."""
        names = GROUPS_3D if self.dim == 3 else GROUPS_2D
        if name == "alldomain":
            return np.arange(1, self.n + 1, dtype=np.int32)
        for g, w in enumerate(names):
            if name == w + "nodes_ghost":
                return np.nonzero(self.ghost_group == g)[0].astype(np.int32) + 1
            if name == w + "nodes":
                ids = self.mirror[self.ghost_group == g]
                return np.unique(ids[ids > 0]).astype(np.int32)
        return np.zeros(0, np.int32)


GROUPS_2D = ("left", "right", "bottom", "top")
GROUPS_3D = ("left", "right", "bottom", "top", "back", "front")


def lattice(dim, nx, ny, nz, box):
    """Structured PD lattice + mirror ghosts as PeriX's createPDMesh builds it (pxb_lattice)."""
    L = lib()
    b = _f64(list(box) + [0.0] * (6 - len(box)))
    n = C.c_int(0)
    dxyz = np.zeros(3, np.float64)
    _check(L.pxb_lattice(int(dim), int(nx), int(ny), int(nz), _p(b), C.byref(n), None, None, None, None, _p(dxyz)))
    coords = np.zeros(3 * n.value, np.float64)
    vols = np.zeros(n.value, np.float64)
    mirror = np.zeros(n.value, np.int32)
    grp = np.zeros(n.value, np.int32)
    _check(L.pxb_lattice(int(dim), int(nx), int(ny), int(nz), _p(b), C.byref(n), _p(coords), _p(vols),
                         _p(mirror, C.c_int), _p(grp, C.c_int), _p(dxyz)))
    nbulk = nx * ny * (nz if dim == 3 else 1)
    return LatticeMesh(dim, n.value, coords, vols, mirror, grp, dxyz, nbulk)


def families(coords3, radius, is3d, cracks=None, planes=None, mirror=None, force_only=False):
    """Family CSR (off, 1-based ids) in the reference visit order (pxb_families)."""
    L = lib()
    c = _f64(coords3).reshape(-1)
    n = c.size // 3
    cr = None if cracks is None or len(cracks) == 0 else _f64(cracks).reshape(-1)
    pl = None if planes is None or len(planes) == 0 else _f64(planes).reshape(-1)
    mir = _i32(mirror)
    off = np.zeros(n + 1, np.int32)
    nb = C.c_longlong(0)
    args = (n, _p(c), C.c_double(radius), int(is3d), 0 if cr is None else cr.size // 4, _p(cr),
            0 if pl is None else pl.size // 12, _p(pl), _p(mir, C.c_int), int(force_only))
    _check(L.pxb_families(*args, _p(off, C.c_int), None, C.byref(nb)))
    ids = np.zeros(max(1, nb.value), np.int32)
    _check(L.pxb_families(*args, _p(off, C.c_int), _p(ids, C.c_int), C.byref(nb)))
    return off, ids[:nb.value]


def families_vh(coords3, node_horizon, is3d, cracks=None, planes=None, mirror=None, force_only=False):
    """Dual families of a variable horizon (pxb_families_vh): pairs within max(delta_i, delta_j)."""
    L = lib()
    c = _f64(coords3).reshape(-1)
    n = c.size // 3
    h = _f64(node_horizon)
    cr = None if cracks is None or len(cracks) == 0 else _f64(cracks).reshape(-1)
    pl = None if planes is None or len(planes) == 0 else _f64(planes).reshape(-1)
    mir = _i32(mirror)
    off = np.zeros(n + 1, np.int32)
    nb = C.c_longlong(0)
    args = (n, _p(c), _p(h), int(is3d), 0 if cr is None else cr.size // 4, _p(cr),
            0 if pl is None else pl.size // 12, _p(pl), _p(mir, C.c_int), int(force_only))
    _check(L.pxb_families_vh(*args, _p(off, C.c_int), None, C.byref(nb)))
    ids = np.zeros(max(1, nb.value), np.int32)
    _check(L.pxb_families_vh(*args, _p(off, C.c_int), _p(ids, C.c_int), C.byref(nb)))
    return off, ids[:nb.value]


def variable_horizon(dim, vols, horizon, dx_char, mirror=None):
    """Per-node horizon and spacing from the node volumes (pxb_variable_horizon)."""
    v = _f64(vols)
    d = np.zeros(v.size, np.float64)
    sp = np.zeros(v.size, np.float64)
    _check(lib().pxb_variable_horizon(v.size, int(dim), _p(v), _p(_i32(mirror), C.c_int), C.c_double(horizon),
                                      C.c_double(dx_char), _p(d), _p(sp)))
    return d, sp


def crack_cut_mask(coords3, mirror, off, ids, cracks=None, planes=None):
    L = lib()
    c = _f64(coords3).reshape(-1)
    cr = None if cracks is None or len(cracks) == 0 else _f64(cracks).reshape(-1)
    pl = None if planes is None or len(planes) == 0 else _f64(planes).reshape(-1)
    out = np.zeros(max(1, int(off[-1])), np.uint8)
    _check(L.pxb_crack_cut_mask(c.size // 3, _p(c), _p(_i32(mirror), C.c_int), _p(_i32(off), C.c_int),
                                _p(_i32(ids), C.c_int), 0 if cr is None else cr.size // 4, _p(cr),
                                0 if pl is None else pl.size // 12, _p(pl), _p(out, C.c_ubyte)))
    return out[:int(off[-1])]


def csr_pattern(off, ids, mirror=None, ndof=1):
    L = lib()
    off = _i32(off)
    ids = _i32(ids)
    n = off.size - 1
    rowptr = np.zeros(n * ndof + 1, np.int32)
    nnz = C.c_longlong(0)
    _check(L.pxb_csr_pattern(n, int(ndof), _p(off, C.c_int), _p(ids, C.c_int), _p(_i32(mirror), C.c_int),
                             _p(rowptr, C.c_int), None, C.byref(nnz)))
    cols = np.zeros(max(1, nnz.value), np.int32)
    _check(L.pxb_csr_pattern(n, int(ndof), _p(off, C.c_int), _p(ids, C.c_int), _p(_i32(mirror), C.c_int),
                             _p(rowptr, C.c_int), _p(cols, C.c_int), C.byref(nnz)))
    return rowptr, cols[:nnz.value]


# ------------------------------------------------------------------------------------------------- BCs
@dataclass
class BC:
    """One boundary condition in the reference's list semantics (DirichletBC / NeumannBC)."""
    kind: str                      # "dirichlet" | "neumann"
    comps: Sequence[int]           # 0-based components
    nodes: np.ndarray              # 1-based node ids
    value: Sequence[float] = field(default_factory=lambda: [0.0, 0.0, 0.0])
    velocity: Sequence[float] = field(default_factory=lambda: [0.0, 0.0, 0.0])
    direct: bool = False
    box: Optional[Sequence[float]] = None   # xlo,xhi,ylo,yhi,zlo,zhi

    def as_dict(self):
        return dict(kind=self.kind, comps=list(self.comps), nodes=self.nodes, value=list(self.value),
                    velocity=list(self.velocity), direct=self.direct, box=self.box)


def _bc_arrays(bcs: List[BC], dim):
    nbc = len(bcs)
    kind = np.zeros(max(1, nbc), np.int32)
    mask = np.zeros(max(1, nbc), np.int32)
    direct = np.zeros(max(1, nbc), np.int32)
    val = np.zeros(max(1, nbc) * dim, np.float64)
    vel = np.zeros(max(1, nbc) * dim, np.float64)
    has_box = np.zeros(max(1, nbc), np.int32)
    box = np.zeros(max(1, nbc) * 6, np.float64)
    off = np.zeros(nbc + 1, np.int32)
    nodes = []
    for e, bc in enumerate(bcs):
        kind[e] = 0 if bc.kind == "dirichlet" else 1
        for c in bc.comps:
            mask[e] |= 1 << int(c)
        direct[e] = int(bool(bc.direct))
        for a in range(dim):
            val[e * dim + a] = bc.value[a] if a < len(bc.value) else 0.0
            vel[e * dim + a] = bc.velocity[a] if a < len(bc.velocity) else 0.0
        if bc.box is not None:
            has_box[e] = 1
            box[6 * e:6 * e + 6] = np.asarray(list(bc.box) + [0.0] * (6 - len(bc.box)), np.float64)
        nodes.extend(int(x) for x in np.asarray(bc.nodes).reshape(-1))
        off[e + 1] = len(nodes)
    return nbc, kind, mask, direct, val, vel, has_box, box, off, np.asarray(nodes if nodes else [1], np.int32)


# ---------------------------------------------------------------------------------------------- context
class StressChParams(C.Structure):
    """pxb_stress_ch_params (include/perix_b200.h)."""
    _fields_ = [(k, C.c_double) for k in ("C11", "C12", "C66", "A", "Kh", "Ch", "Omega", "cref", "chi", "kappa",
                                          "dt", "kres", "rho")]
    DEFAULTS = {"dt": 1.0, "kres": 1e-8}


class ChRunParams(C.Structure):
    """pxb_ch_run_params (include/perix_b200.h)."""
    _fields_ = [("chi", C.c_double), ("kappa", C.c_double), ("M0", C.c_double), ("dt", C.c_double),
                ("nsteps", C.c_int), ("newton_rtol", C.c_double), ("newton_max", C.c_int), ("lin_rtol", C.c_double),
                ("lin_max", C.c_int)]


class ChRunStats(C.Structure):
    """pxb_ch_run_stats (include/perix_b200.h)."""
    _fields_ = [("steps", C.c_int), ("newton_iters", C.c_int), ("lin_iters", C.c_int), ("max_residual", C.c_double),
                ("max_lin_relres", C.c_double), ("energy", C.c_double)]


class CachedParams(C.Structure):
    """pxb_cached_params (include/perix_b200.h)."""
    _fields_ = [("C11", C.c_double), ("C12", C.c_double), ("C66", C.c_double), ("rho", C.c_double),
                ("dt", C.c_double), ("b", C.c_double * 3)]


class Context:
    """A perix_b200 device context (one GPU, one stream).  Mirrors the pxb_* entry points."""

    def __init__(self, device=0):
        L = lib()
        h = C.c_void_p()
        _check(L.pxb_ctx_create(int(device), C.byref(h)))
        self.h = h
        self.L = L
        self.n = 0
        self.dim = 0
        self.nb = 0
        self.nop = 0

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self.L.pxb_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- plumbing
    def set_stream(self, stream_ptr):
        """Run on an external CUDA stream.  A handle of 0 (torch's default stream) means the legacy default
        stream and is passed as cudaStreamLegacy; None restores the context's own (non-blocking) stream."""
        if stream_ptr is not None and int(stream_ptr) == 0:
            stream_ptr = 1  # cudaStreamLegacy
        _check(self.L.pxb_ctx_set_stream(self.h, _vp(stream_ptr)))

    def synchronize(self):
        _check(self.L.pxb_ctx_synchronize(self.h))

    def device_bytes(self):
        v = C.c_size_t(0)
        _check(self.L.pxb_ctx_device_bytes(self.h, C.byref(v)))
        return v.value

    def launch_count(self):
        v = C.c_longlong(0)
        _check(self.L.pxb_ctx_launch_count(self.h, C.byref(v)))
        return v.value

    # -- geometry
    def set_geometry(self, coords3, vols, off, ids, delta, dx_char, dim, mirror=None, layer=None):
        c = _f64(coords3).reshape(-1)
        self._keep = (c, _f64(vols), _i32(off), _i32(ids), _i32(mirror), _i32(layer))
        c, v, o, i, m, l_ = self._keep
        self.n = c.size // 3
        self.dim = dim
        self.nb = int(o[-1])
        _check(self.L.pxb_set_geometry(self.h, self.n, int(dim), _p(c), _p(v), _p(o, C.c_int), _p(i, C.c_int),
                                       C.c_double(delta), C.c_double(dx_char), _p(m, C.c_int), _p(l_, C.c_int)))

    # -- g-functions
    def set_geometry_points(self, coords3, vols, radius, delta, dx_char, dim, mirror=None, layer=None):
        """Geometry with the families built on the device (reference order, equal to ``families``)."""
        c = _f64(coords3).reshape(-1)
        n = c.size // 3
        nb = C.c_longlong(0)
        _check(self.L.pxb_set_geometry_points(self.h, n, int(dim), _p(c), _p(_f64(vols)), C.c_double(radius),
                                              C.c_double(delta), C.c_double(dx_char), _p(_i32(mirror), C.c_int),
                                              _p(_i32(layer), C.c_int), C.byref(nb)))
        self.n, self.dim, self.nb = n, int(dim), nb.value
        return nb.value

    def set_node_horizons(self, node_delta, node_spacing=None):
        """Variable horizon: per-node delta and rim spacing (None clears)."""
        self._vh = (_f64(node_delta), _f64(node_spacing))
        _check(self.L.pxb_set_node_horizons(self.h, _p(self._vh[0]), _p(self._vh[1])))

    def epf_set_variable_horizon_stretch(self, G0, E, plane_stress=False):
        """Per-bond critical stretch s_c(0.5 (delta_i + delta_j)) (pxb_epf_set_variable_horizon_stretch)."""
        _check(self.L.pxb_epf_set_variable_horizon_stretch(self.h, C.c_double(G0), C.c_double(E), int(plane_stress)))

    def get_families(self):
        off = np.zeros(self.n + 1, np.int32)
        ids = np.zeros(max(1, self.nb), np.int32)
        _check(self.L.pxb_get_families(self.h, _p(off, C.c_int), _p(ids, C.c_int)))
        return off, ids[:self.nb]

    def gbuild_set_schedule(self, schedule):
        """-1 default, 0 lane groups, 1 one warp per node, 2 one warp per node with the FP64 tensor-core tiles
        (pxb_gbuild_set_schedule)."""
        _check(self.L.pxb_gbuild_set_schedule(self.h, int(schedule)))

    def epf_set_rate_chunks(self, chunks):
        """Node chunks of the pipelined per-step rate call (pinned buffers): -1 by mesh size, 1 off, 2..8
        (pxb_epf_set_rate_chunks)."""
        _check(self.L.pxb_epf_set_rate_chunks(self.h, int(chunks)))

    def epf_set_adjoint_schedule(self, schedule):
        """The recorded reverse sweep's kernel: -1 default, 0 both operator streams, 1 reverse-only, 2-4 reverse-only
        staged through shared memory in three launch configurations (pxb_epf_set_adjoint_schedule)."""
        _check(self.L.pxb_epf_set_adjoint_schedule(self.h, int(schedule)))

    def gbuild(self, order=2, precision=FP64, allow_degenerate=False):
        nd = C.c_int(0)
        first = C.c_int(0)
        st = self.L.pxb_gbuild(self.h, int(order), int(precision), C.byref(nd), C.byref(first))
        if st == 3 and allow_degenerate:
            pass
        else:
            _check(st)
        n = C.c_int(0)
        _check(self.L.pxb_gbuild_info(self.h, C.byref(n), None))
        self.nop = n.value
        return nd.value, first.value

    def get_ops(self):
        out = np.zeros(self.nb * self.nop, np.float64)
        _check(self.L.pxb_get_ops(self.h, _p(out)))
        return out.reshape(-1, self.nop)

    def apply(self, u, slots):
        s = _i32(slots)
        u = _f64(u)
        out = np.zeros(self.n * s.size, np.float64)
        _check(self.L.pxb_apply(self.h, _p(u), int(s.size), _p(s, C.c_int), _p(out)))
        return out.reshape(self.n, s.size)

    def apply_d(self, u_ptr, slots, out_ptr):
        s = _i32(slots)
        _check(self.L.pxb_apply_d(self.h, _p(u_ptr), int(s.size), _p(s, C.c_int), _p(out_ptr)))

    def apply_adjoint(self, ybar, slots):
        s = _i32(slots)
        y = _f64(ybar).reshape(-1)
        out = np.zeros(self.n, np.float64)
        _check(self.L.pxb_apply_adjoint(self.h, _p(y), int(s.size), _p(s, C.c_int), _p(out)))
        return out

    def apply_adjoint_d(self, ybar_ptr, slots, out_ptr):
        s = _i32(slots)
        _check(self.L.pxb_apply_adjoint_d(self.h, _p(ybar_ptr), int(s.size), _p(s, C.c_int), _p(out_ptr)))

    # -- explicit fracture
    def epf_setup(self, C11, C12, C66, rho, b=(0.0, 0.0, 0.0), sc=0.0, tension_only=True, health0=None,
                  precision=FP64):
        bb = _f64(list(b) + [0.0] * (3 - len(b)))
        h = _u8(health0)
        _check(self.L.pxb_epf_setup(self.h, int(precision), C.c_double(C11), C.c_double(C12), C.c_double(C66),
                                    C.c_double(rho), _p(bb), C.c_double(sc), int(bool(tension_only)),
                                    _p(h, C.c_ubyte)))

    def epf_rate(self, u):
        u = _f64(u)
        a = np.zeros(self.n * self.dim, np.float64)
        nbk = C.c_longlong(0)
        _check(self.L.pxb_epf_rate(self.h, _p(u), _p(a), C.byref(nbk)))
        return a, nbk.value

    def epf_set_bcs(self, bcs: List[BC]):
        nbc, kind, mask, direct, val, vel, has_box, box, off, nodes = _bc_arrays(bcs, self.dim)
        self._bc_keep = (kind, mask, direct, val, vel, has_box, box, off, nodes)
        _check(self.L.pxb_epf_set_bcs(self.h, nbc, _p(kind, C.c_int), _p(mask, C.c_int), _p(direct, C.c_int),
                                      _p(val), _p(vel), _p(has_box, C.c_int), _p(box), _p(off, C.c_int),
                                      _p(nodes, C.c_int)))

    def epf_start(self, u0, v0, dt):
        _check(self.L.pxb_epf_start(self.h, _p(_f64(u0)), _p(_f64(v0)), C.c_double(dt)))

    def epf_advance(self, nsteps, chunk=0):
        """nsteps uniform steps; a tripped blow-up guard raises PxbError (status 5) with .bad_step set."""
        bad = C.c_int(0)
        _check_step(self.L.pxb_epf_advance(self.h, int(nsteps), int(chunk), C.byref(bad)), bad)

    def epf_advance_to(self, t_end, chunk=0):
        """Advance to t_end with the reference's clamped variable-dt last step; returns the number of steps."""
        bad = C.c_int(0)
        steps = C.c_longlong(0)
        _check_step(self.L.pxb_epf_advance_to(self.h, C.c_double(t_end), int(chunk), C.byref(bad), C.byref(steps)),
                    bad)
        return steps.value

    def set_memory_limit(self, nbytes):
        """Cap the device bytes this context may hold (0: none); allocations past it raise PxbError (status 4)."""
        _check(self.L.pxb_ctx_set_memory_limit(self.h, C.c_size_t(int(nbytes))))

    def epf_set_wait_budget(self, tries):
        """Fault-path test hook (include/perix_b200_measure.h): try_wait calls a staged consumer wait may make; -1
        restores the default."""
        _check(self.L.pxb_epf_set_wait_budget(self.h, int(tries)))

    def epf_state(self):
        u = np.zeros(self.n * self.dim, np.float64)
        up = np.zeros(self.n * self.dim, np.float64)
        h = np.zeros(max(1, self.nb), np.uint8)
        t = C.c_double(0)
        _check(self.L.pxb_epf_get_state(self.h, _p(u), _p(up), _p(h, C.c_ubyte), C.byref(t)))
        return u, up, h[:self.nb], t.value

    def epf_set_state(self, u=None, u_prev=None, health=None, t=0.0):
        _check(self.L.pxb_epf_set_state(self.h, _p(_f64(u)), _p(_f64(u_prev)), _p(_u8(health), C.c_ubyte),
                                        C.c_double(t)))

    def epf_broken(self):
        v = C.c_longlong(0)
        _check(self.L.pxb_epf_broken_count(self.h, C.byref(v)))
        return v.value

    def epf_set_variant(self, variant):
        _check(self.L.pxb_epf_set_variant(self.h, int(variant)))

    def epf_variant(self):
        v, lpn = C.c_int(0), C.c_int(0)
        _check(self.L.pxb_epf_get_variant(self.h, C.byref(v), C.byref(lpn)))
        return v.value, lpn.value

    def epf_autotune(self, steps=10, flush_bytes=256 << 20, use_cache=False):
        best = C.c_int(0)
        ms = np.zeros(self.L.pxb_epf_variant_count(), np.float32)
        _check(self.L.pxb_epf_autotune(self.h, int(steps), C.c_size_t(flush_bytes), int(bool(use_cache)),
                                       C.byref(best), ms.ctypes.data_as(C.POINTER(C.c_float))))
        return best.value, ms

    def epf_force_adjoint(self, u, abar):
        ub = np.zeros(self.n * self.dim, np.float64)
        dC = np.zeros(3, np.float64)
        _check(self.L.pxb_epf_force_adjoint(self.h, _p(_f64(u)), _p(_f64(abar)), _p(ub), _p(dC)))
        return ub, dC

    def epf_force_adjoint_d(self, u_ptr, abar_ptr, ubar_ptr, dC_ptr):
        _check(self.L.pxb_epf_force_adjoint_d(self.h, _p(u_ptr), _p(abar_ptr), _p(ubar_ptr), _p(dC_ptr)))

    def epf_set_constants(self, C11, C12, C66, rho):
        _check(self.L.pxb_epf_set_constants(self.h, C.c_double(C11), C.c_double(C12), C.c_double(C66),
                                            C.c_double(rho)))

    def epf_force_frozen_d(self, u_ptr, a_ptr):
        _check(self.L.pxb_epf_force_frozen_d(self.h, _p(u_ptr), _p(a_ptr)))

    # -- batched clouds
    def batch_set(self, clouds):
        """clouds: list of dicts with dim, coords3 (n x 3), vols, off, ids (1-based within the cloud), delta,
        dx_char.  Concatenates them into the batch numbering."""
        dims = _i32([c["dim"] for c in clouds])
        node_off = np.zeros(len(clouds) + 1, np.int64)
        node_off[1:] = np.cumsum([int(np.asarray(c["vols"]).size) for c in clouds])
        coords = np.concatenate([_f64(c["coords3"]).reshape(-1) for c in clouds])
        vols = np.concatenate([_f64(c["vols"]) for c in clouds])
        offs, base = [np.zeros(1, np.int64)], 0
        for c in clouds:
            o = np.asarray(c["off"], np.int64)
            offs.append(o[1:] + base)
            base += int(o[-1])
        neigh_off = np.concatenate(offs)
        if base >= 2 ** 31 or node_off[-1] >= 2 ** 31:
            raise ValueError("batch too large for 32-bit offsets")
        ids = np.concatenate([_i32(c["ids"]) for c in clouds])
        delta = _f64([c["delta"] for c in clouds])
        dxc = _f64([c["dx_char"] for c in clouds])
        _check(self.L.pxb_batch_set(self.h, len(clouds), _p(dims, C.c_int), _p(_i32(node_off), C.c_int), _p(coords),
                                    _p(vols), _p(_i32(neigh_off), C.c_int), _p(ids, C.c_int), _p(delta), _p(dxc)))
        self.batch_dims = [int(c["dim"]) for c in clouds]
        self.batch_node_off = node_off
        n, nb, ol, opl = C.c_longlong(0), C.c_longlong(0), C.c_longlong(0), C.c_longlong(0)
        _check(self.L.pxb_batch_info(self.h, C.byref(n), C.byref(nb), C.byref(ol), C.byref(opl)))
        self.batch_n, self.batch_nb, self.batch_out_len, self.batch_ops_len = n.value, nb.value, ol.value, opl.value
        self.batch_bond_counts = [int(np.asarray(c["off"])[-1]) for c in clouds]

    def batch_set_points(self, clouds):
        """clouds: list of dicts with dim, coords3, vols, delta, dx_char (and optionally radius, default delta);
        the families are built on the device."""
        dims = _i32([c["dim"] for c in clouds])
        node_off = np.zeros(len(clouds) + 1, np.int64)
        node_off[1:] = np.cumsum([int(np.asarray(c["vols"]).size) for c in clouds])
        coords = np.concatenate([_f64(c["coords3"]).reshape(-1) for c in clouds])
        vols = np.concatenate([_f64(c["vols"]) for c in clouds])
        radius = _f64([c.get("radius", c["delta"]) for c in clouds])
        delta = _f64([c["delta"] for c in clouds])
        dxc = _f64([c["dx_char"] for c in clouds])
        _check(self.L.pxb_batch_set_points(self.h, len(clouds), _p(dims, C.c_int), _p(_i32(node_off), C.c_int),
                                           _p(coords), _p(vols), _p(radius), _p(delta), _p(dxc)))
        self.batch_dims = [int(c["dim"]) for c in clouds]
        self.batch_node_off = node_off
        n, nb, ol, opl = C.c_longlong(0), C.c_longlong(0), C.c_longlong(0), C.c_longlong(0)
        _check(self.L.pxb_batch_info(self.h, C.byref(n), C.byref(nb), C.byref(ol), C.byref(opl)))
        self.batch_n, self.batch_nb, self.batch_out_len, self.batch_ops_len = n.value, nb.value, ol.value, opl.value
        counts = []
        for k in range(len(clouds)):
            off = np.zeros(int(node_off[k + 1] - node_off[k]) + 1, np.int32)
            _check(self.L.pxb_batch_get_families(self.h, k, _p(off, C.c_int), None))
            counts.append(int(off[-1]))
        self.batch_bond_counts = counts

    def batch_get_families(self, cloud):
        n = int(self.batch_node_off[cloud + 1] - self.batch_node_off[cloud])
        off = np.zeros(n + 1, np.int32)
        ids = np.zeros(max(1, self.batch_bond_counts[cloud]), np.int32)
        _check(self.L.pxb_batch_get_families(self.h, int(cloud), _p(off, C.c_int), _p(ids, C.c_int)))
        return off, ids[:self.batch_bond_counts[cloud]]

    def batch_gbuild(self, precision=FP64):
        nd, first = C.c_int(0), C.c_int(0)
        _check(self.L.pxb_batch_gbuild(self.h, int(precision), C.byref(nd), C.byref(first)))
        return nd.value, first.value

    def batch_apply(self, u):
        out = np.zeros(self.batch_out_len, np.float64)
        _check(self.L.pxb_batch_apply(self.h, _p(_f64(u)), _p(out)))
        return out

    def batch_apply_d(self, u_ptr, out_ptr):
        _check(self.L.pxb_batch_apply_d(self.h, _p(u_ptr), _p(out_ptr)))

    def batch_split(self, out):
        """Per-cloud views (n_k x nop_k) of a batch apply output."""
        res, pos = [], 0
        for k, d in enumerate(self.batch_dims):
            n = int(self.batch_node_off[k + 1] - self.batch_node_off[k])
            nop = 9 if d == 3 else 5
            res.append(out[pos:pos + n * nop].reshape(n, nop))
            pos += n * nop
        return res

    def batch_get_ops(self, cloud):
        nop = 9 if self.batch_dims[cloud] == 3 else 5
        ops = np.zeros(max(1, self.batch_bond_counts[cloud] * nop), np.float64)
        _check(self.L.pxb_batch_get_ops(self.h, int(cloud), _p(ops)))
        return ops[:self.batch_bond_counts[cloud] * nop].reshape(-1, nop)

    def batch_set_variant(self, which, variant):
        _check(self.L.pxb_batch_set_variant(self.h, int(which), int(variant)))

    def batch_variant(self, which):
        v = C.c_int(0)
        _check(self.L.pxb_batch_get_variant(self.h, int(which), C.byref(v)))
        return v.value

    def batch_time(self, what, reps, flush_bytes=256 << 20, u_ptr=0, out_ptr=0):
        ms = np.zeros(reps, np.float32)
        _check(self.L.pxb_batch_time(self.h, int(what), int(reps), C.c_size_t(flush_bytes), _vp(u_ptr), _vp(out_ptr),
                                     ms.ctypes.data_as(C.POINTER(C.c_float))))
        return ms

    def batch_autotune(self, what, reps=3, flush_bytes=256 << 20, u_ptr=0, out_ptr=0):
        best = C.c_int(0)
        ms = np.zeros(self.L.pxb_batch_variant_count(), np.float32)
        _check(self.L.pxb_batch_autotune(self.h, int(what), int(reps), C.c_size_t(flush_bytes), _vp(u_ptr),
                                         _vp(out_ptr), C.byref(best), ms.ctypes.data_as(C.POINTER(C.c_float))))
        return best.value, ms

    # -- CSR assembly
    def csr_set_pattern(self, rowptr, cols, ndof=1):
        r = _i32(rowptr)
        c = _i32(cols)
        self._csr_keep = (r, c)
        _check(self.L.pxb_csr_set_pattern(self.h, int(ndof), _p(r, C.c_int), _p(c, C.c_int), C.c_longlong(c.size)))
        self.nnz = c.size
        self._csr_ndof = int(ndof)

    def csr_build_pattern(self, ndof=1):
        """The pattern of csr_pattern, built on the device from the context's families and mirror map and set as
        the context's pattern (pxb_csr_build_pattern); returns nnz."""
        nnz = C.c_longlong(0)
        _check(self.L.pxb_csr_build_pattern(self.h, int(ndof), C.byref(nnz)))
        self._csr_keep = None
        self.nnz = int(nnz.value)
        self._csr_ndof = int(ndof)
        return self.nnz

    def csr_get_pattern(self):
        """(rowptr, cols) of the context's pattern, copied from the device."""
        rowptr = np.zeros(self.n * self._csr_ndof + 1, np.int32)
        cols = np.zeros(self.nnz, np.int32)
        _check(self.L.pxb_csr_get_pattern(self.h, _p(rowptr, C.c_int), _p(cols, C.c_int)))
        return rowptr, cols

    def assemble_scalar(self, type_, coef, u, f=0.0, f_node=None, dt=0.0, uold=None):
        kv = np.zeros(self.nnz, np.float64)
        rhs = np.zeros(self.n, np.float64)
        _check(self.L.pxb_assemble_scalar(self.h, int(type_), C.c_double(coef), C.c_double(f), _p(_f64(f_node)),
                                          C.c_double(dt), _p(_f64(u)), _p(_f64(uold)), _p(kv), _p(rhs)))
        return kv, rhs

    def ch_set_geometry(self, rev, lapbond, isghost=None):
        g = None if isghost is None else np.ascontiguousarray(isghost, np.int8)
        _check(self.L.pxb_ch_set_geometry(self.h, _p(_i32(rev), C.c_int), _p(_f64(lapbond)), _p(g, C.c_char)))

    def ch_build_geometry(self):
        _check(self.L.pxb_ch_build_geometry(self.h))

    def ch_get_geometry(self):
        rev = np.zeros(max(1, self.nb), np.int32)
        lap = np.zeros(max(1, self.nb), np.float64)
        ghost = np.zeros(self.n, np.int8)
        _check(self.L.pxb_ch_get_geometry(self.h, _p(rev, C.c_int), _p(lap), _p(ghost, C.c_char)))
        return rev[:self.nb], lap[:self.nb], ghost

    def ch_mobility_d(self, M0, u_ptr, mnode_ptr):
        _check(self.L.pxb_ch_mobility_d(self.h, C.c_double(M0), _p(u_ptr), _p(mnode_ptr)))

    def assemble_ch_d(self, kappa, chi, dt, mnode_ptr, u_ptr, uold_ptr, kvals_ptr, rhs_ptr):
        _check(self.L.pxb_assemble_ch_d(self.h, C.c_double(kappa), C.c_double(chi), C.c_double(dt), _p(mnode_ptr),
                                        _p(u_ptr), _p(uold_ptr), _p(kvals_ptr), _p(rhs_ptr)))

    def assemble_stress_ch(self, params, mnode, u, uold=None, health=None, vel=None):
        """Stress-coupled Cahn-Hilliard (ndof = dim + 2) K and rhs; params: dict with the fields of
        StressChParams (C11 C12 C66 A Kh Ch Omega cref chi kappa dt kres rho)."""
        p = StressChParams(**{k: float(params.get(k, StressChParams.DEFAULTS.get(k, 0.0)))
                              for k, _ in StressChParams._fields_})
        kv = np.zeros(self.nnz, np.float64)
        rhs = np.zeros((self.dim + 2) * self.n, np.float64)
        _check(self.L.pxb_assemble_stress_ch(self.h, C.byref(p), _p(_f64(mnode)), _p(None if health is None else _f64(health)),
                                             _p(None if vel is None else _f64(vel)), _p(_f64(u)),
                                             _p(None if uold is None else _f64(uold)), _p(kv), _p(rhs)))
        return kv, rhs

    def assemble_stress_ch_d(self, params, mnode_ptr, u_ptr, uold_ptr, kvals_ptr, rhs_ptr, health_ptr=None,
                             vel_ptr=None):
        p = StressChParams(**{k: float(params.get(k, StressChParams.DEFAULTS.get(k, 0.0)))
                              for k, _ in StressChParams._fields_})
        _check(self.L.pxb_assemble_stress_ch_d(self.h, C.byref(p), _p(mnode_ptr), _p(health_ptr), _p(vel_ptr),
                                               _p(u_ptr), _p(uold_ptr), _p(kvals_ptr), _p(rhs_ptr)))

    def _ch_params(self, chi, kappa, M0, dt, nsteps, newton_rtol, newton_max, lin_rtol, lin_max):
        return ChRunParams(chi=float(chi), kappa=float(kappa), M0=float(M0), dt=float(dt), nsteps=int(nsteps),
                           newton_rtol=float(newton_rtol), newton_max=int(newton_max), lin_rtol=float(lin_rtol),
                           lin_max=int(lin_max))

    def ch_run(self, c0, chi, kappa, M0, dt, nsteps, newton_rtol=1e-13, newton_max=40, lin_rtol=1e-12,
               lin_max=2000):
        """Backward-Euler Cahn-Hilliard run on the device (pxb_ch_run): returns (u_final [2n], E, stats dict)."""
        p = self._ch_params(chi, kappa, M0, dt, nsteps, newton_rtol, newton_max, lin_rtol, lin_max)
        u = np.zeros(2 * self.n, np.float64)
        E = C.c_double(0.0)
        st = ChRunStats()
        _check(self.L.pxb_ch_run(self.h, C.byref(p), _p(_f64(c0)), _p(u), C.byref(E), C.byref(st)))
        return u, E.value, {k: getattr(st, k) for k, _ in ChRunStats._fields_}

    def ch_gradient(self, c0, chi, kappa, M0, dt, nsteps, newton_rtol=1e-13, newton_max=40, lin_rtol=1e-12,
                    lin_max=2000):
        """(E, dE/dkappa, dE/dc0 [n], stats) by the discrete adjoint of the run (pxb_ch_gradient)."""
        p = self._ch_params(chi, kappa, M0, dt, nsteps, newton_rtol, newton_max, lin_rtol, lin_max)
        g = np.zeros(self.n, np.float64)
        E, dk = C.c_double(0.0), C.c_double(0.0)
        st = ChRunStats()
        _check(self.L.pxb_ch_gradient(self.h, C.byref(p), _p(_f64(c0)), C.byref(E), C.byref(dk), _p(g), C.byref(st)))
        return E.value, dk.value, g, {k: getattr(st, k) for k, _ in ChRunStats._fields_}

    def ch_energy(self, kappa, chi, u):
        E = C.c_double(0.0)
        g = np.zeros(2 * self.n, np.float64)
        _check(self.L.pxb_ch_energy(self.h, C.c_double(kappa), C.c_double(chi), _p(_f64(u)), C.byref(E), _p(g)))
        return E.value, g

    def epf_project(self, u=None, plane_strain=True):
        """Damage, von Mises, stress and strain (3x3 per node) of u (None: the current state) with the current
        bond health (pxb_epf_project)."""
        n = self.n
        dmg, vm = np.zeros(n), np.zeros(n)
        st, ep = np.zeros(9 * n), np.zeros(9 * n)
        _check(self.L.pxb_epf_project(self.h, _p(None if u is None else _f64(u)), int(bool(plane_strain)), _p(dmg),
                                      _p(vm), _p(st), _p(ep)))
        return dict(damage=dmg, vonMises=vm, stress=st.reshape(n, 9), strain=ep.reshape(n, 9))

    def assemble_cached(self, params, u, uold=None, nodecache=None, ncache=3, bondcache=None, nbcache=1):
        """Implicit PDDO dynamic fracture (ndof = dim) K and rhs; params: dict with C11 C12 C66 rho dt and b
        (3 values); nodecache [n*ncache] committed velocity, bondcache [nb*nbcache] frozen bond health."""
        p = CachedParams(C11=float(params["C11"]), C12=float(params["C12"]), C66=float(params["C66"]),
                         rho=float(params["rho"]), dt=float(params["dt"]),
                         b=(C.c_double * 3)(*[float(x) for x in params.get("b", (0.0, 0.0, 0.0))]))
        kv = np.zeros(self.nnz, np.float64)
        rhs = np.zeros(self.dim * self.n, np.float64)
        _check(self.L.pxb_assemble_cached(self.h, C.byref(p), _p(None if nodecache is None else _f64(nodecache)),
                                          int(ncache), _p(None if bondcache is None else _f64(bondcache)),
                                          int(nbcache), _p(_f64(u)), _p(None if uold is None else _f64(uold)),
                                          _p(kv), _p(rhs)))
        return kv, rhs

    def assemble_ch(self, kappa, chi, dt, mnode, u, uold):
        kv = np.zeros(self.nnz, np.float64)
        rhs = np.zeros(2 * self.n, np.float64)
        _check(self.L.pxb_assemble_ch(self.h, C.c_double(kappa), C.c_double(chi), C.c_double(dt), _p(_f64(mnode)),
                                      _p(_f64(u)), _p(_f64(uold)), _p(kv), _p(rhs)))
        return kv, rhs
