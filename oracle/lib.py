"""ctypes bindings for the two oracle libraries (test infrastructure only, see ``oracle/__init__.py``)."""
import ctypes as C
import math
import os

import numpy as np

ORACLE_DIR = os.path.dirname(os.path.abspath(__file__))
_PORT_SO = os.path.join(ORACLE_DIR, "_ref", "libpddo_oracle.so")
_REF_SO = os.path.join(ORACLE_DIR, "_ref", "libperix_ref.so")
_DROPIN_SO = os.path.join(ORACLE_DIR, "_ref", "libperix_ref_dropin.so")

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")


def _ptr(a, ctype):
    return None if a is None else a.ctypes.data_as(C.POINTER(ctype))


def port_available():
    return os.path.exists(_PORT_SO)


def ref_available():
    return os.path.exists(_REF_SO)


def bc_program_arrays(bcs, dim):
    """Encode a BC list (dicts with kind/comps/direct/value/velocity/box/nodes) in the harness' C layout.

    kind: "dirichlet" | "neumann"; comps: list of 0-based components; nodes: 1-based ids.
    """
    nbc = len(bcs)
    kind = np.zeros(nbc, np.int32)
    mask = np.zeros(nbc, np.int32)
    direct = np.zeros(nbc, np.int32)
    val = np.zeros(max(1, nbc) * dim, np.float64)
    vel = np.zeros(max(1, nbc) * dim, np.float64)
    has_box = np.zeros(nbc, np.int32)
    box = np.zeros(max(1, nbc) * 6, np.float64)
    off = np.zeros(nbc + 1, np.int32)
    nodes = []
    for e, bc in enumerate(bcs):
        kind[e] = 0 if bc["kind"] == "dirichlet" else 1
        for c in bc["comps"]:
            mask[e] |= 1 << c
        direct[e] = int(bc.get("direct", False))
        v = bc.get("value", [0.0] * dim)
        w = bc.get("velocity", [0.0] * dim)
        for a in range(dim):
            val[e * dim + a] = v[a]
            vel[e * dim + a] = w[a]
        if bc.get("box") is not None:
            has_box[e] = 1
            box[6 * e:6 * e + 6] = np.asarray(bc["box"], np.float64)
        nodes.extend(int(x) for x in bc["nodes"])
        off[e + 1] = len(nodes)
    return dict(nbc=nbc, kind=kind, mask=mask, direct=direct, val=val, vel=vel, has_box=has_box, box=box,
                off=off, nodes=np.asarray(nodes if nodes else [0], np.int32))


class PortOracle:
    """The plain-C restatement (oracle/pddo_oracle.c)."""

    def __init__(self):
        if not port_available():
            raise RuntimeError("oracle not built: run `make -C oracle port`")
        L = C.CDLL(_PORT_SO)
        L.orc_qindices.restype = C.c_int
        L.orc_families.restype = C.c_longlong
        L.orc_crack_cuts.restype = C.c_int
        L.orc_gbuild.restype = C.c_int
        L.orc_csr_pattern.restype = C.c_longlong
        L.orc_critical_stretch.restype = C.c_double
        self.L = L

    def qindices(self, dim, order):
        pqr = np.zeros(3 * 64, np.int32)
        fact = np.zeros(64, np.int32)
        nop = self.L.orc_qindices(dim, order, _ptr(pqr, C.c_int), _ptr(fact, C.c_int))
        return pqr[:3 * nop].reshape(nop, 3).copy(), fact[:nop].copy()

    def families(self, coords3, radius, is3d, cracks=None, planes=None, mirror=None, force_only=False):
        coords3 = np.ascontiguousarray(coords3, np.float64).reshape(-1)
        n = coords3.size // 3
        cr = None if cracks is None or len(cracks) == 0 else np.ascontiguousarray(cracks, np.float64).reshape(-1)
        pl = None if planes is None or len(planes) == 0 else np.ascontiguousarray(planes, np.float64).reshape(-1)
        mir = None if mirror is None else np.ascontiguousarray(mirror, np.int32)
        off = np.zeros(n + 1, np.int32)
        args = (n, _ptr(coords3, C.c_double), C.c_double(radius), int(is3d), 0 if cr is None else cr.size // 4,
                _ptr(cr, C.c_double), 0 if pl is None else pl.size // 12, _ptr(pl, C.c_double),
                _ptr(mir, C.c_int), int(force_only))
        nb = self.L.orc_families(*args, _ptr(off, C.c_int), None)
        ids = np.zeros(max(1, nb), np.int32)
        self.L.orc_families(*args, _ptr(off, C.c_int), _ptr(ids, C.c_int))
        return off, ids[:nb]

    def crack_cuts(self, coords3, mirror, cracks, planes, i1, j1):
        coords3 = np.ascontiguousarray(coords3, np.float64).reshape(-1)
        cr = None if cracks is None or len(cracks) == 0 else np.ascontiguousarray(cracks, np.float64).reshape(-1)
        pl = None if planes is None or len(planes) == 0 else np.ascontiguousarray(planes, np.float64).reshape(-1)
        mir = None if mirror is None else np.ascontiguousarray(mirror, np.int32)
        return bool(self.L.orc_crack_cuts(coords3.size // 3, _ptr(coords3, C.c_double), _ptr(mir, C.c_int),
                                          0 if cr is None else cr.size // 4, _ptr(cr, C.c_double),
                                          0 if pl is None else pl.size // 12, _ptr(pl, C.c_double), int(i1), int(j1)))

    def gbuild(self, dim, order, coords3, vols, off, ids, delta, dx_char, volume_correction=True):
        coords3 = np.ascontiguousarray(coords3, np.float64).reshape(-1)
        n = coords3.size // 3
        nop = self.qindices(dim, order)[0].shape[0]
        ops = np.zeros(int(off[-1]) * nop, np.float64)
        deg = np.zeros(n, np.uint8)
        self.L.orc_gbuild(n, dim, order, _ptr(coords3, C.c_double), _ptr(np.ascontiguousarray(vols, np.float64),
                          C.c_double), _ptr(off, C.c_int), _ptr(ids, C.c_int), C.c_double(delta),
                          C.c_double(dx_char), int(volume_correction), _ptr(ops, C.c_double), _ptr(deg, C.c_ubyte))
        return ops.reshape(-1, nop), deg

    def apply(self, off, ids, ops, u):
        n = off.size - 1
        nop = ops.shape[1]
        out = np.zeros(n * nop, np.float64)
        self.L.orc_apply(n, nop, _ptr(off, C.c_int), _ptr(ids, C.c_int),
                         _ptr(np.ascontiguousarray(ops, np.float64), C.c_double),
                         _ptr(np.ascontiguousarray(u, np.float64), C.c_double), _ptr(out, C.c_double))
        return out.reshape(n, nop)

    def csr_pattern(self, off, ids, mirror, ndof=1):
        n = off.size - 1
        rowptr = np.zeros(n * ndof + 1, np.int32)
        mir = None if mirror is None else np.ascontiguousarray(mirror, np.int32)
        nnz = self.L.orc_csr_pattern(n, ndof, _ptr(off, C.c_int), _ptr(ids, C.c_int), _ptr(mir, C.c_int),
                                     _ptr(rowptr, C.c_int), None)
        cols = np.zeros(max(1, nnz), np.int32)
        self.L.orc_csr_pattern(n, ndof, _ptr(off, C.c_int), _ptr(ids, C.c_int), _ptr(mir, C.c_int),
                               _ptr(rowptr, C.c_int), _ptr(cols, C.c_int))
        return rowptr, cols[:nnz]

    def poisson_assemble(self, dim, off, ids, ops, lapslots, sigma, f, u, rowptr, cols):
        n = off.size - 1
        kv = np.zeros(int(rowptr[-1]), np.float64)
        rhs = np.zeros(n, np.float64)
        ls = np.ascontiguousarray(lapslots, np.int32)
        self.L.orc_poisson_assemble(n, dim, ops.shape[1], _ptr(ls, C.c_int), _ptr(off, C.c_int), _ptr(ids, C.c_int),
                                    _ptr(np.ascontiguousarray(ops, np.float64), C.c_double), C.c_double(sigma),
                                    _ptr(None if f is None else np.ascontiguousarray(f, np.float64), C.c_double),
                                    _ptr(np.ascontiguousarray(u, np.float64), C.c_double), _ptr(rowptr, C.c_int),
                                    _ptr(cols, C.c_int), _ptr(kv, C.c_double), _ptr(rhs, C.c_double))
        return kv, rhs

    def elastic_constants(self, dim, plane_stress, E, nu):
        Cv = np.zeros(3, np.float64)
        self.L.orc_elastic_constants(dim, int(plane_stress), C.c_double(E), C.c_double(nu), _ptr(Cv, C.c_double))
        return Cv

    def critical_stretch(self, dim, plane_stress, G0, E, delta):
        return self.L.orc_critical_stretch(dim, int(plane_stress), C.c_double(G0), C.c_double(E), C.c_double(delta))

    def epf_rate(self, dim, coords3, off, ids, navier, Cv, rho, b, sc, u, health, tension_only=True,
                 damage_on=True):
        coords3 = np.ascontiguousarray(coords3, np.float64).reshape(-1)
        n = coords3.size // 3
        h = np.ascontiguousarray(health, np.float64).copy()
        acc = np.zeros(n * dim, np.float64)
        self.L.orc_epf_rate(n, dim, _ptr(coords3, C.c_double), _ptr(off, C.c_int), _ptr(ids, C.c_int),
                            _ptr(np.ascontiguousarray(navier, np.float64), C.c_double), C.c_double(Cv[0]),
                            C.c_double(Cv[1]), C.c_double(Cv[2]), C.c_double(rho),
                            _ptr(np.ascontiguousarray(b, np.float64), C.c_double), C.c_double(sc), int(tension_only),
                            int(damage_on), _ptr(np.ascontiguousarray(u, np.float64), C.c_double),
                            _ptr(h, C.c_double), _ptr(acc, C.c_double))
        return acc, h

    def bc_preset(self, dim, coords3, mirror, bcs, t, u):
        coords3 = np.ascontiguousarray(coords3, np.float64).reshape(-1)
        p = bc_program_arrays(bcs, dim)
        uu = np.ascontiguousarray(u, np.float64).copy()
        mir = None if mirror is None else np.ascontiguousarray(mirror, np.int32)
        self.L.orc_bc_preset(coords3.size // 3, dim, _ptr(coords3, C.c_double), _ptr(mir, C.c_int), p["nbc"],
                             _ptr(p["kind"], C.c_int), _ptr(p["mask"], C.c_int), _ptr(p["direct"], C.c_int),
                             _ptr(p["val"], C.c_double), _ptr(p["vel"], C.c_double), _ptr(p["has_box"], C.c_int),
                             _ptr(p["box"], C.c_double), _ptr(p["off"], C.c_int), _ptr(p["nodes"], C.c_int),
                             C.c_double(t), _ptr(uu, C.c_double))
        return uu

    def epf_run(self, dim, coords3, mirror, off, ids, navier, Cv, rho, b, sc, u0, v0, dt, nsteps, bcs, health,
                tension_only=True, damage_on=True):
        coords3 = np.ascontiguousarray(coords3, np.float64).reshape(-1)
        n = coords3.size // 3
        p = bc_program_arrays(bcs, dim)
        u = np.zeros(n * dim, np.float64)
        uo = np.zeros(n * dim, np.float64)
        h = np.ascontiguousarray(health, np.float64).copy()
        mir = None if mirror is None else np.ascontiguousarray(mirror, np.int32)
        self.L.orc_epf_run(n, dim, _ptr(coords3, C.c_double), _ptr(mir, C.c_int), _ptr(off, C.c_int),
                           _ptr(ids, C.c_int), _ptr(np.ascontiguousarray(navier, np.float64), C.c_double),
                           C.c_double(Cv[0]), C.c_double(Cv[1]), C.c_double(Cv[2]), C.c_double(rho),
                           _ptr(np.ascontiguousarray(b, np.float64), C.c_double), C.c_double(sc), int(tension_only),
                           int(damage_on), _ptr(np.ascontiguousarray(u0, np.float64), C.c_double),
                           _ptr(None if v0 is None else np.ascontiguousarray(v0, np.float64), C.c_double),
                           C.c_double(dt), int(nsteps), p["nbc"], _ptr(p["kind"], C.c_int), _ptr(p["mask"], C.c_int),
                           _ptr(p["direct"], C.c_int), _ptr(p["val"], C.c_double), _ptr(p["vel"], C.c_double),
                           _ptr(p["has_box"], C.c_int), _ptr(p["box"], C.c_double), _ptr(p["off"], C.c_int),
                           _ptr(p["nodes"], C.c_int), _ptr(u, C.c_double), _ptr(uo, C.c_double), _ptr(h, C.c_double))
        return u, uo, h


_REFCU_SO = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_ref", "libperix_ref_cuda.so")


def ref_cuda_available():
    return os.path.exists(_REFCU_SO)


def ref_cuda_epf_bench(dim, coords3, vols, off, ids, delta, dx_char, Cv, rho, sc, u, health, reps=20,
                       flush_bytes=256 << 20, tension_only=True):
    """Times the reference's own GPU explicit path (oracle/ref_cuda_harness.cu): per-step call, force kernel
    alone, operator build.  Returns (call_ms, kernel_ms, opbuild_ms, accel)."""
    L = C.CDLL(_REFCU_SO)
    coords3 = np.ascontiguousarray(coords3, np.float64).reshape(-1)
    n = coords3.size // 3
    if dim == 2:
        q = [(1, 0, 0), (0, 1, 0), (2, 0, 0), (1, 1, 0), (0, 2, 0)]
    else:
        q = [(1, 0, 0), (0, 1, 0), (0, 0, 1), (2, 0, 0), (1, 1, 0), (1, 0, 1), (0, 2, 0), (0, 1, 1), (0, 0, 2)]
    qp = np.array([a for a, _, _ in q], np.int32)
    qq = np.array([b for _, b, _ in q], np.int32)
    qr = np.array([c for _, _, c in q], np.int32)
    fact = np.array([math.factorial(a) * math.factorial(b) * math.factorial(c) for a, b, c in q], np.float64)
    h = np.ascontiguousarray(health, np.float64).copy()
    out = np.zeros(4, np.float64)
    acc = np.zeros(n * dim, np.float64)
    L.refcu_epf_bench.restype = C.c_int
    st = L.refcu_epf_bench(n, dim, _ptr(coords3, C.c_double), _ptr(np.ascontiguousarray(vols, np.float64), C.c_double),
                           _ptr(np.ascontiguousarray(off, np.int32), C.c_int),
                           _ptr(np.ascontiguousarray(ids, np.int32), C.c_int), _ptr(qp, C.c_int), _ptr(qq, C.c_int),
                           _ptr(qr, C.c_int), _ptr(fact, C.c_double), len(q), C.c_double(delta), C.c_double(dx_char),
                           C.c_double(Cv[0]), C.c_double(Cv[1]), C.c_double(Cv[2]), C.c_double(rho), C.c_double(sc),
                           int(tension_only), _ptr(np.ascontiguousarray(u, np.float64), C.c_double), _ptr(h, C.c_double),
                           int(reps), C.c_size_t(flush_bytes), _ptr(out, C.c_double), _ptr(acc, C.c_double))
    if st:
        raise RuntimeError("reference GPU harness failed with status %d" % st)
    return float(out[0]), float(out[1]), float(out[2]), acc


_REF = None


def ref_cuda_stress_ch(dim, coords3, vols, off, ids, delta, dx_char, rowptr, cols, p13, rev, lapbond, isghost,
                       mnode, u, uold, health=None, vel=None):
    """The reference's own GPU stress-coupled CH assembler (its CUDA TU built for sm_100a); returns K, rhs."""
    L = C.CDLL(_REFCU_SO)
    pqr = []
    for o in (1, 2):
        for p in range(o, -1, -1):
            if dim == 3:
                for q in range(o - p, -1, -1):
                    pqr.append((p, q, o - p - q))
            else:
                pqr.append((p, o - p, 0))
    qp = np.array([x[0] for x in pqr], np.int32)
    qq = np.array([x[1] for x in pqr], np.int32)
    qr = np.array([x[2] for x in pqr], np.int32)
    fact = np.array([math.factorial(a) * math.factorial(b) * math.factorial(c) for a, b, c in pqr], np.float64)
    nd = dim + 2
    n = np.asarray(vols).size
    kv = np.zeros(np.asarray(cols).size, np.float64)
    rhs = np.zeros(n * nd, np.float64)
    f64 = lambda a: np.ascontiguousarray(a, np.float64)
    i32 = lambda a: np.ascontiguousarray(a, np.int32)
    st = L.refcu_stress_ch(int(n), int(dim), _ptr(f64(coords3), C.c_double), _ptr(f64(vols), C.c_double),
                           _ptr(i32(off), C.c_int), _ptr(i32(ids), C.c_int), _ptr(qp, C.c_int), _ptr(qq, C.c_int),
                           _ptr(qr, C.c_int), _ptr(fact, C.c_double), int(len(pqr)), C.c_double(delta),
                           C.c_double(dx_char), _ptr(i32(rowptr), C.c_int), _ptr(i32(cols), C.c_int), int(kv.size),
                           _ptr(f64(p13), C.c_double), _ptr(i32(rev), C.c_int), _ptr(f64(lapbond), C.c_double),
                           _ptr(np.ascontiguousarray(isghost, np.int8), C.c_char), _ptr(f64(mnode), C.c_double),
                           None if health is None else _ptr(f64(health), C.c_double),
                           None if vel is None else _ptr(f64(vel), C.c_double), _ptr(f64(u), C.c_double),
                           _ptr(f64(uold), C.c_double), _ptr(kv, C.c_double), _ptr(rhs, C.c_double))
    if st:
        raise RuntimeError("reference stress-CH GPU assembly failed")
    return kv, rhs


def ref_cuda_assemble_bench(dim, coords3, vols, off, ids, delta, dx_char, rowptr, cols, sigma, f, u, reps=10,
                            flush_bytes=256 << 20):
    """Times the reference's own implicit GPU path (oracle/ref_cuda_harness.cu) on a Poisson assembly: the
    perix_cuda::assemble call, its one-off opsBuildKernel and assembleKernel alone.  The child process should set
    PERIX_CUDA_OPCACHE=1 so that the reference keeps an operator cache at nop 5 too.  Returns (call_ms,
    opsbuild_ms, kernel_ms, kvals, rhs)."""
    L = C.CDLL(_REFCU_SO)
    coords3 = np.ascontiguousarray(coords3, np.float64).reshape(-1)
    n = coords3.size // 3
    if dim == 2:
        q = [(1, 0, 0), (0, 1, 0), (2, 0, 0), (1, 1, 0), (0, 2, 0)]
    else:
        q = [(1, 0, 0), (0, 1, 0), (0, 0, 1), (2, 0, 0), (1, 1, 0), (1, 0, 1), (0, 2, 0), (0, 1, 1), (0, 0, 2)]
    qp = np.array([a for a, _, _ in q], np.int32)
    qq = np.array([b for _, b, _ in q], np.int32)
    qr = np.array([c for _, _, c in q], np.int32)
    fact = np.array([math.factorial(a) * math.factorial(b) * math.factorial(c) for a, b, c in q], np.float64)
    rowptr = np.ascontiguousarray(rowptr, np.int32)
    cols = np.ascontiguousarray(cols, np.int32)
    out = np.zeros(4, np.float64)
    kv = np.zeros(cols.size, np.float64)
    rhs = np.zeros(n, np.float64)
    L.refcu_assemble_bench.restype = C.c_int
    st = L.refcu_assemble_bench(n, dim, _ptr(coords3, C.c_double), _ptr(np.ascontiguousarray(vols, np.float64), C.c_double),
                                _ptr(np.ascontiguousarray(off, np.int32), C.c_int),
                                _ptr(np.ascontiguousarray(ids, np.int32), C.c_int), _ptr(qp, C.c_int),
                                _ptr(qq, C.c_int), _ptr(qr, C.c_int), _ptr(fact, C.c_double), len(q), C.c_double(delta),
                                C.c_double(dx_char), _ptr(rowptr, C.c_int), _ptr(cols, C.c_int), int(cols.size),
                                C.c_double(sigma), C.c_double(f), _ptr(np.ascontiguousarray(u, np.float64), C.c_double),
                                int(reps), C.c_size_t(flush_bytes), _ptr(out, C.c_double), _ptr(kv, C.c_double),
                                _ptr(rhs, C.c_double))
    if st:
        raise RuntimeError("reference GPU assembly harness failed with status %d" % st)
    return float(out[0]), float(out[1]), float(out[2]), kv, rhs


_DROPIN = None


def dropin_available():
    return os.path.exists(_DROPIN_SO)


def _ref_lib(dropin=False):
    """The reference harness library; dropin=True loads the build whose reference callers (compiled with
    -DPERIX_CUDA_ASSEMBLE) are linked to libperix_b200.so."""
    global _REF, _DROPIN
    if dropin:
        if _DROPIN is None:
            if not dropin_available():
                raise RuntimeError("drop-in harness not built: run `make -C oracle dropin` where the reference is present")
            _DROPIN = _bind_ref(C.CDLL(_DROPIN_SO))
        return _DROPIN
    if _REF is None:
        if not ref_available():
            raise RuntimeError("reference harness not built: run `make -C oracle ref` where the reference is present")
        _REF = _bind_ref(C.CDLL(_REF_SO))
    return _REF


def _bind_ref(L):
    vp = C.c_void_p
    L.ref_mesh_structured.restype = vp
    L.ref_mesh_cloud.restype = vp
    L.ref_mesh_cloud_vh.restype = vp
    L.ref_mesh_nodes.restype = C.c_int
    L.ref_mesh_bonds.restype = C.c_longlong
    L.ref_group_size.restype = C.c_int
    L.ref_crack_cuts.restype = C.c_int
    L.ref_gbuild_time.restype = C.c_double
    L.ref_csr_nnz.restype = C.c_int
    L.ref_poisson_assemble.restype = C.c_double
    L.ref_ch_assemble.restype = C.c_double
    L.ref_stress_ch_assemble.restype = C.c_double
    L.ref_dynfrac_assemble.restype = C.c_double
    L.ref_epf_create.restype = vp
    L.ref_epf_rate.restype = C.c_double
    L.ref_epf_run.restype = C.c_double
    L.ref_max_threads.restype = C.c_int
    for name in ("ref_mesh_free", "ref_mesh_nodes", "ref_mesh_bonds", "ref_mesh_scalars", "ref_mesh_get",
                 "ref_group_size", "ref_group_get", "ref_crack_cuts", "ref_qindices", "ref_gbuild",
                 "ref_gbuild_time", "ref_apply", "ref_csr_nnz", "ref_csr_pattern", "ref_poisson_assemble",
                 "ref_epf_free", "ref_epf_rate", "ref_epf_set_health", "ref_epf_constants", "ref_epf_opcache",
                 "ref_bc_preset", "ref_epf_run"):
        getattr(L, name).argtypes = None
    L.ref_system_assemble.restype = C.c_double
    L.ref_epf_run_to.restype = C.c_int
    L.ref_epf_use_cuda.restype = C.c_int
    L.ref_is_dropin.restype = C.c_int
    return L


class RefMesh:
    """A PD mesh built by the reference's own generators/createPDMesh/createNeighborNodes."""

    def __init__(self, handle, dim, order, dropin=False):
        self.L = _ref_lib(dropin)
        self.dropin = dropin
        self.h = C.c_void_p(handle)
        self.dim = dim
        self.order = order
        self.n = self.L.ref_mesh_nodes(self.h)
        self.nb = self.L.ref_mesh_bonds(self.h)
        sc = np.zeros(6, np.float64)
        self.L.ref_mesh_scalars(self.h, _ptr(sc, C.c_double))
        self.delta, self.dx, self.dy, self.dz, self.dx_char, nop = sc
        self.nop = int(nop)
        self.coords = np.zeros(3 * self.n, np.float64)
        self.vols = np.zeros(self.n, np.float64)
        self.off = np.zeros(self.n + 1, np.int32)
        self.ids = np.zeros(max(1, self.nb), np.int32)
        self.mirror = np.zeros(self.n, np.int32)
        self.L.ref_mesh_get(self.h, _ptr(self.coords, C.c_double), _ptr(self.vols, C.c_double),
                            _ptr(self.off, C.c_int), _ptr(self.ids, C.c_int), _ptr(self.mirror, C.c_int))
        self.ids = self.ids[:self.nb]

    @classmethod
    def structured(cls, dim, nx, ny, nz, box, factor, order=2, cracks=None, planes=None, force_only=False,
                   dropin=False):
        L = _ref_lib(dropin)
        b = np.ascontiguousarray(list(box) + [0.0] * (6 - len(box)), np.float64)
        cr = None if not cracks else np.ascontiguousarray(cracks, np.float64).reshape(-1)
        pl = None if not planes else np.ascontiguousarray(planes, np.float64).reshape(-1)
        h = L.ref_mesh_structured(int(dim), int(nx), int(ny), int(nz), _ptr(b, C.c_double), C.c_double(factor),
                                  int(order), int(force_only), 0 if cr is None else cr.size // 4,
                                  _ptr(cr, C.c_double), 0 if pl is None else pl.size // 12, _ptr(pl, C.c_double))
        m = cls(h, dim, order, dropin)
        m.cracks = cr
        m.planes = pl
        m.force_only = force_only
        return m

    @classmethod
    def cloud(cls, dim, coords3, vols, dx, dy, dz, horizon, order=2, volume_correction=True):
        L = _ref_lib()
        c = np.ascontiguousarray(coords3, np.float64).reshape(-1)
        v = np.ascontiguousarray(vols, np.float64)
        h = L.ref_mesh_cloud(int(dim), c.size // 3, _ptr(c, C.c_double), _ptr(v, C.c_double), C.c_double(dx),
                             C.c_double(dy), C.c_double(dz), C.c_double(horizon), int(order), int(volume_correction))
        m = cls(h, dim, order)
        m.cracks = None
        m.planes = None
        m.force_only = False
        return m

    @classmethod
    def cloud_vh(cls, dim, coords3, vols, dx, dy, dz, horizon, order=2, volume_correction=True, dropin=False):
        """A cloud with the reference's variable horizon on (NodeHorizon / NodeSpacing from the node volumes, dual
        families)."""
        L = _ref_lib(dropin)
        c = np.ascontiguousarray(coords3, np.float64).reshape(-1)
        v = np.ascontiguousarray(vols, np.float64)
        h = L.ref_mesh_cloud_vh(int(dim), c.size // 3, _ptr(c, C.c_double), _ptr(v, C.c_double), C.c_double(dx),
                                C.c_double(dy), C.c_double(dz), C.c_double(horizon), int(order), int(volume_correction))
        m = cls(h, dim, order, dropin)
        m.cracks = None
        m.planes = None
        m.force_only = False
        m.node_delta = np.zeros(m.n)
        m.node_spacing = np.zeros(m.n)
        L.ref_mesh_node_horizon(m.h, _ptr(m.node_delta, C.c_double), _ptr(m.node_spacing, C.c_double))
        return m

    def group(self, name):
        k = self.L.ref_group_size(self.h, name.encode())
        out = np.zeros(max(1, k), np.int32)
        self.L.ref_group_get(self.h, name.encode(), _ptr(out, C.c_int))
        return out[:k]

    def crack_cuts(self, i1, j1):
        return bool(self.L.ref_crack_cuts(self.h, int(i1), int(j1)))

    def qindices(self):
        pqr = np.zeros(3 * self.nop, np.int32)
        fact = np.zeros(self.nop, np.int32)
        self.L.ref_qindices(self.h, _ptr(pqr, C.c_int), _ptr(fact, C.c_int))
        return pqr.reshape(-1, 3), fact

    def gbuild(self, nthreads=0):
        ops = np.zeros(self.nb * self.nop, np.float64)
        deg = np.zeros(self.n, np.uint8)
        self.L.ref_gbuild(self.h, _ptr(ops, C.c_double), _ptr(deg, C.c_ubyte), int(nthreads or os.cpu_count()))
        return ops.reshape(-1, self.nop), deg

    def gbuild_time(self, nthreads=0, reps=1):
        return self.L.ref_gbuild_time(self.h, int(nthreads or os.cpu_count()), int(reps))

    def apply(self, u, nthreads=0):
        out = np.zeros(self.n * self.nop, np.float64)
        self.L.ref_apply(self.h, _ptr(np.ascontiguousarray(u, np.float64), C.c_double), _ptr(out, C.c_double),
                         int(nthreads or os.cpu_count()))
        return out.reshape(self.n, self.nop)

    def csr_pattern(self, ndof=1):
        nnz = self.L.ref_csr_nnz(self.h, int(ndof))
        rowptr = np.zeros(self.n * ndof + 1, np.int32)
        cols = np.zeros(nnz, np.int32)
        self.L.ref_csr_pattern(self.h, int(ndof), _ptr(rowptr, C.c_int), _ptr(cols, C.c_int))
        return rowptr, cols

    def poisson_assemble(self, sigma, f, u, nthreads=0):
        nnz = self.L.ref_csr_nnz(self.h, 1)
        kv = np.zeros(nnz, np.float64)
        rhs = np.zeros(self.n, np.float64)
        t = self.L.ref_poisson_assemble(self.h, C.c_double(sigma),
                                        _ptr(None if f is None else np.ascontiguousarray(f, np.float64), C.c_double),
                                        _ptr(np.ascontiguousarray(u, np.float64), C.c_double), _ptr(kv, C.c_double),
                                        _ptr(rhs, C.c_double), int(nthreads or os.cpu_count()))
        return kv, rhs, t

    def ch_assemble(self, chi, kappa, M0, dt, u, uold, nthreads=0):
        """Cahn-Hilliard (2 dof) K/rhs through the reference element, plus its geometry (lambda-corrected
        Laplacian per bond, reverse-bond index, ghost flags) and Picard mobility."""
        nnz = self.L.ref_csr_nnz(self.h, 2)
        nb = int(self.off[-1])
        kv = np.zeros(nnz, np.float64)
        rhs = np.zeros(2 * self.n, np.float64)
        lap = np.zeros(nb, np.float64)
        rev = np.zeros(nb, np.int32)
        ghost = np.zeros(self.n, np.int8)
        mnode = np.zeros(self.n, np.float64)
        t = self.L.ref_ch_assemble(self.h, C.c_double(chi), C.c_double(kappa), C.c_double(M0), C.c_double(dt),
                                   _ptr(np.ascontiguousarray(u, np.float64), C.c_double),
                                   _ptr(np.ascontiguousarray(uold, np.float64), C.c_double), _ptr(kv, C.c_double),
                                   _ptr(rhs, C.c_double), _ptr(lap, C.c_double), _ptr(rev, C.c_int),
                                   _ptr(ghost, C.c_char), _ptr(mnode, C.c_double), int(nthreads or os.cpu_count()))
        return kv, rhs, dict(lapbond=lap, rev=rev, isghost=ghost, mnode=mnode), t

    def stress_ch_assemble(self, E, nu, plane_stress, Omega, cref, D, chi, kappa, dt, u, uold, nthreads=0):
        """StressCahnHilliardElement (ndof = dim + 2) K, rhs and its own geometry / mobility / derived constants
        (C11, C12, C66, A, Kh, Ch)."""
        nd = self.dim + 2
        nnz = self.L.ref_csr_nnz(self.h, nd)
        kv = np.zeros(nnz, np.float64)
        rhs = np.zeros(self.n * nd, np.float64)
        lap = np.zeros(max(1, self.nb), np.float64)
        rev = np.zeros(max(1, self.nb), np.int32)
        ghost = np.zeros(self.n, np.int8)
        mnode = np.zeros(self.n, np.float64)
        consts = np.zeros(6, np.float64)
        t = self.L.ref_stress_ch_assemble(self.h, C.c_double(E), C.c_double(nu), int(plane_stress), C.c_double(Omega),
                                          C.c_double(cref), C.c_double(D), C.c_double(chi), C.c_double(kappa),
                                          C.c_double(dt), _ptr(np.ascontiguousarray(u, np.float64), C.c_double),
                                          _ptr(np.ascontiguousarray(uold, np.float64), C.c_double),
                                          _ptr(kv, C.c_double), _ptr(rhs, C.c_double), _ptr(lap, C.c_double),
                                          _ptr(rev, C.c_int), _ptr(ghost, C.c_char), _ptr(mnode, C.c_double),
                                          _ptr(consts, C.c_double), int(nthreads or os.cpu_count()))
        return kv, rhs, dict(lapbond=lap[:self.nb], rev=rev[:self.nb], isghost=ghost, mnode=mnode,
                             consts=consts), t

    def dynfrac_assemble(self, E, nu, rho, G0, dt, uprev, uold, u, plane_stress=False, tension_only=True,
                         b=(0.0, 0.0, 0.0)):
        """PDDODynamicFracElement (ndof = dim): initialised from uprev, committed at uold, assembled at u.
        Returns K, rhs, the committed velocity [n*dim], bond health [nb] and (C11, C12, C66)."""
        nd = self.dim
        nnz = self.L.ref_csr_nnz(self.h, nd)
        kv = np.zeros(nnz, np.float64)
        rhs = np.zeros(self.n * nd, np.float64)
        vel = np.zeros(self.n * nd, np.float64)
        health = np.zeros(max(1, self.nb), np.float64)
        consts = np.zeros(3, np.float64)
        f64 = lambda a: np.ascontiguousarray(a, np.float64)
        self.L.ref_dynfrac_assemble(self.h, C.c_double(E), C.c_double(nu), C.c_double(rho), C.c_double(G0),
                                    int(plane_stress), int(tension_only), C.c_double(b[0]), C.c_double(b[1]),
                                    C.c_double(b[2]), C.c_double(dt), _ptr(f64(uprev), C.c_double),
                                    _ptr(f64(uold), C.c_double), _ptr(f64(u), C.c_double), _ptr(kv, C.c_double),
                                    _ptr(rhs, C.c_double), _ptr(vel, C.c_double), _ptr(health, C.c_double),
                                    _ptr(consts, C.c_double))
        return kv, rhs, vel, health[:self.nb], consts

    def system_assemble(self, type_, coef, f, u, dt=0.0, uold=None, use_cuda=False):
        """K (CSR values on the reference pattern) and rhs of a single PoissonElement (type 0: sigma = coef) or
        DiffusionElement (type 1: D = coef, transient with dt and uold) through the reference's
        PDSystem::formResidualAndJacobian, or with use_cuda through its formResidualAndJacobianCUDA caller (the
        drop-in build, where that caller runs this backend's perix_cuda::assemble).  Returns kv, rhs, seconds."""
        nnz = self.L.ref_csr_nnz(self.h, 1)
        kv = np.zeros(nnz, np.float64)
        rhs = np.zeros(self.n, np.float64)
        f64 = lambda a: np.ascontiguousarray(a, np.float64)
        t = self.L.ref_system_assemble(self.h, int(type_), C.c_double(coef), C.c_double(f), C.c_double(dt),
                                       _ptr(f64(u), C.c_double), _ptr(None if uold is None else f64(uold), C.c_double),
                                       _ptr(kv, C.c_double), _ptr(rhs, C.c_double), int(bool(use_cuda)))
        if t < 0:
            raise RuntimeError("use_cuda needs the drop-in build of the reference harness")
        return kv, rhs, t

    def bc_preset(self, bcs, t, u):
        p = bc_program_arrays(bcs, self.dim)
        uu = np.ascontiguousarray(u, np.float64).copy()
        self.L.ref_bc_preset(self.h, p["nbc"], _ptr(p["kind"], C.c_int), _ptr(p["mask"], C.c_int),
                             _ptr(p["direct"], C.c_int), _ptr(p["val"], C.c_double), _ptr(p["vel"], C.c_double),
                             _ptr(p["has_box"], C.c_int), _ptr(p["box"], C.c_double), _ptr(p["off"], C.c_int),
                             _ptr(p["nodes"], C.c_int), C.c_double(t), _ptr(uu, C.c_double))
        return uu

    def __del__(self):
        try:
            self.L.ref_mesh_free(self.h)
        except Exception:
            pass


class RefEpf:
    """The reference ExplicitPDDOFracElement bound to a RefMesh."""

    def __init__(self, mesh, E, nu, rho, G0, plane_stress=False, tension_only=True, damage_on=True, b=(0, 0, 0)):
        self.L = _ref_lib(getattr(mesh, "dropin", False))
        self.mesh = mesh
        self.h = C.c_void_p(self.L.ref_epf_create(mesh.h, C.c_double(E), C.c_double(nu), C.c_double(rho),
                                                  C.c_double(G0), int(plane_stress), int(tension_only),
                                                  int(damage_on), C.c_double(b[0]), C.c_double(b[1]),
                                                  C.c_double(b[2])))

    def rate(self, u, nthreads=0):
        m = self.mesh
        acc = np.zeros(m.n * m.dim, np.float64)
        h = np.zeros(m.nb, np.float64)
        t = self.L.ref_epf_rate(self.h, _ptr(np.ascontiguousarray(u, np.float64), C.c_double), _ptr(acc, C.c_double),
                                _ptr(h, C.c_double), int(nthreads or os.cpu_count()))
        return acc, h, t

    def project(self, which, u):
        """computeNodalProjection at u for every node: "damage", "vonMises" (n values), "stress", "strain"
        (n x 9, row-major 3x3)."""
        k = {"damage": 0, "vonMises": 1, "stress": 2, "strain": 3}[which]
        out = np.zeros(self.mesh.n * (1 if k < 2 else 9), np.float64)
        self.L.ref_epf_project(self.h, k, _ptr(np.ascontiguousarray(u, np.float64), C.c_double), _ptr(out, C.c_double))
        return out if k < 2 else out.reshape(-1, 9)

    def use_cuda(self, on=True):
        """LocalElmtInfo::UseCuda of the following rate calls: the reference element then runs its
        perix_cuda::assembleExplicitPDDOFracAccel branch (drop-in build only)."""
        if self.L.ref_epf_use_cuda(self.h, int(bool(on))) != 0:
            raise RuntimeError("use_cuda needs the drop-in build of the reference harness")

    def set_health(self, h):
        self.L.ref_epf_set_health(self.h, _ptr(np.ascontiguousarray(h, np.float64), C.c_double))

    def constants(self):
        out = np.zeros(5, np.float64)
        self.L.ref_epf_constants(self.h, _ptr(out, C.c_double))
        return dict(sc=out[0], C11=out[1], C12=out[2], C66=out[3], stable_dt=out[4])

    def opcache(self):
        nops = 9 if self.mesh.dim == 3 else 5
        out = np.zeros(self.mesh.nb * nops, np.float64)
        self.L.ref_epf_opcache(self.h, _ptr(out, C.c_double))
        return out.reshape(-1, nops)

    def run(self, u0, v0, dt, nsteps, bcs, nthreads=0):
        m = self.mesh
        p = bc_program_arrays(bcs, m.dim)
        u = np.zeros(m.n * m.dim, np.float64)
        uo = np.zeros(m.n * m.dim, np.float64)
        h = np.zeros(m.nb, np.float64)
        t = self.L.ref_epf_run(self.h, _ptr(np.ascontiguousarray(u0, np.float64), C.c_double),
                               _ptr(None if v0 is None else np.ascontiguousarray(v0, np.float64), C.c_double),
                               C.c_double(dt), int(nsteps), p["nbc"], _ptr(p["kind"], C.c_int),
                               _ptr(p["mask"], C.c_int), _ptr(p["direct"], C.c_int), _ptr(p["val"], C.c_double),
                               _ptr(p["vel"], C.c_double), _ptr(p["has_box"], C.c_int), _ptr(p["box"], C.c_double),
                               _ptr(p["off"], C.c_int), _ptr(p["nodes"], C.c_int), _ptr(u, C.c_double),
                               _ptr(uo, C.c_double), _ptr(h, C.c_double), int(nthreads or os.cpu_count()))
        return u, uo, h, t

    def run_to(self, u0, v0, dt, t_end, bcs, nthreads=0):
        """The reference loop to t_end (clamped variable-dt last step, BC preset, blow-up guard); returns u, uold,
        health, the number of completed steps, the 1-based step at which the guard tripped (0 if none), and t."""
        m = self.mesh
        p = bc_program_arrays(bcs, m.dim)
        u = np.zeros(m.n * m.dim, np.float64)
        uo = np.zeros(m.n * m.dim, np.float64)
        h = np.zeros(m.nb, np.float64)
        trip = C.c_int(0)
        t = C.c_double(0.0)
        steps = self.L.ref_epf_run_to(self.h, _ptr(np.ascontiguousarray(u0, np.float64), C.c_double),
                                      _ptr(None if v0 is None else np.ascontiguousarray(v0, np.float64), C.c_double),
                                      C.c_double(dt), C.c_double(t_end), p["nbc"], _ptr(p["kind"], C.c_int),
                                      _ptr(p["mask"], C.c_int), _ptr(p["direct"], C.c_int),
                                      _ptr(p["val"], C.c_double), _ptr(p["vel"], C.c_double),
                                      _ptr(p["has_box"], C.c_int), _ptr(p["box"], C.c_double),
                                      _ptr(p["off"], C.c_int), _ptr(p["nodes"], C.c_int), _ptr(u, C.c_double),
                                      _ptr(uo, C.c_double), _ptr(h, C.c_double), C.byref(trip), C.byref(t),
                                      int(nthreads or os.cpu_count()))
        return u, uo, h, int(steps), trip.value, t.value

    def __del__(self):
        try:
            self.L.ref_epf_free(self.h)
        except Exception:
            pass
