"""The drop-in boundary exercised by the reference's own callers: oracle/_ref/libperix_ref_dropin.so holds the
reference's PDSystem::formResidualAndJacobianCUDA (FormResidualAndJacobianCUDA.cpp) and ExplicitPDDOFracElement's
UseCuda branch (ExplicitPDDOFracElement.cpp:174-235), compiled unchanged with -DPERIX_CUDA_ASSEMBLE against this
backend's perix_cuda:: header and linked to libperix_b200.so.  Each call below goes reference caller ->
perix_cuda:: shim -> pxb_* C-ABI -> kernels, and is compared with the reference's CPU path on the same inputs
(PDSystem::formResidualAndJacobian; the element's OpenMP loop).  The diffusion branch of the scalar assembly is also
checked directly through the C-ABI against the reference's DiffusionElement."""
import math

import numpy as np
import pytest

from oracle import dropin_available, ref_available

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not (ref_available() and dropin_available()), reason="drop-in harness not built")]


@pytest.fixture(autouse=True)
def fresh_shim():
    """The shim keeps one default context keyed by the problem sizes, like the reference's file-static device
    state; each test starts from a released one."""
    import perix_b200 as px
    px.lib().pxb_cuda_shutdown()
    yield
    px.lib().pxb_cuda_shutdown()


def _mesh(dim, dropin):
    from oracle import RefMesh
    if dim == 2:
        return RefMesh.structured(2, 32, 24, 0, [0, 1.0, 0, 0.75], 3.015, 2, dropin=dropin)
    return RefMesh.structured(3, 10, 8, 6, [0, 1.0, 0, 0.8, 0, 0.6], 3.015, 2, dropin=dropin)


def _close(a, b, tol=1e-12):
    return np.abs(a - b).max() <= tol * np.abs(b).max()


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("type_", [0, 1])
def test_form_residual_and_jacobian_cuda_through_shim(dim, type_):
    """PDSystem::formResidualAndJacobianCUDA -> perix_cuda::assemble (Poisson, type 0; transient diffusion, type 1)
    against PDSystem::formResidualAndJacobian on the CPU."""
    m = _mesh(dim, dropin=True)
    rng = np.random.default_rng(5 + dim + 10 * type_)
    u = rng.standard_normal(m.n)
    uold = u + 0.1 * rng.standard_normal(m.n)
    coef, f, dt = (1.7, 0.3, 0.0) if type_ == 0 else (0.8, -0.4, 2.5e-3)
    kv_cpu, rhs_cpu, _ = m.system_assemble(type_, coef, f, u, dt=dt, uold=uold)
    kv_gpu, rhs_gpu, _ = m.system_assemble(type_, coef, f, u, dt=dt, uold=uold, use_cuda=True)
    assert _close(kv_gpu, kv_cpu) and _close(rhs_gpu, rhs_cpu)
    # a second call with new values reuses the resident structure
    u2 = rng.standard_normal(m.n)
    kv_cpu, rhs_cpu, _ = m.system_assemble(type_, coef, f, u2, dt=dt, uold=uold)
    kv_gpu, rhs_gpu, _ = m.system_assemble(type_, coef, f, u2, dt=dt, uold=uold, use_cuda=True)
    assert _close(kv_gpu, kv_cpu) and _close(rhs_gpu, rhs_cpu)


@pytest.mark.parametrize("dim", [2, 3])
def test_diffusion_assembly_matches_reference_element(ctx, dim):
    """pxb_assemble_scalar type 1 (transient diffusion, dt > 0 with u_old) against the reference's DiffusionElement in
    PDSystem::formResidualAndJacobian."""
    m = _mesh(dim, dropin=False)
    rng = np.random.default_rng(40 + dim)
    u = rng.standard_normal(m.n)
    uold = u + 0.05 * rng.standard_normal(m.n)
    D, f, dt = 0.8, -0.4, 2.5e-3
    kv_ref, rhs_ref, _ = m.system_assemble(1, D, f, u, dt=dt, uold=uold)
    ctx.set_geometry(m.coords, m.vols, m.off, m.ids, m.delta, m.dx_char, dim, mirror=m.mirror)
    ctx.gbuild(2, 0)
    rowptr, cols = m.csr_pattern(1)
    ctx.csr_set_pattern(rowptr, cols, 1)
    kv, rhs = ctx.assemble_scalar(1, D, u, f=f, dt=dt, uold=uold)
    assert _close(kv, kv_ref) and _close(rhs, rhs_ref)


def _plate(dropin):
    import perix_b200 as px
    from oracle import RefMesh
    nx, ny, h = 200, 100, 5e-4
    Lx, Ly = nx * h, ny * h
    y1, y2 = Ly / 2 - 12.5 * h, Ly / 2 + 12.5 * h
    cracks = [[0.0, y1, 25 * h, y1], [0.0, y2, 25 * h, y2]]
    m = RefMesh.structured(2, nx, ny, 0, [0, Lx, 0, Ly], 3.015, 2, cracks=cracks, force_only=True, dropin=dropin)
    return m, px


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("tension_only", [True, False])
def test_explicit_element_use_cuda_through_shim(monkeypatch, precision, tension_only):
    """ExplicitPDDOFracElement::preprocessIteration with LocalElmtInfo::UseCuda (the element hands damage and force to
    perix_cuda::assembleExplicitPDDOFracAccel) against the same element on the CPU, over calls at growing
    displacements that break bonds: health identical and acceleration within 1e-12 (FP64) or 1e-6 (mixed,
    PERIX_B200_PRECISION=mixed)."""
    from oracle import RefEpf
    if precision == "mixed":
        monkeypatch.setenv("PERIX_B200_PRECISION", "mixed")
    else:
        monkeypatch.delenv("PERIX_B200_PRECISION", raising=False)
    m, _ = _plate(dropin=True)
    E, nu, rho = 190e9, 0.3, 8000.0
    G0 = 0.01 ** 2 * 12 * E * m.delta / (5 * math.pi)
    gpu = RefEpf(m, E, nu, rho, G0, tension_only=tension_only)
    cpu = RefEpf(m, E, nu, rho, G0, tension_only=tension_only)
    gpu.use_cuda(True)
    rng = np.random.default_rng(17)
    base = rng.standard_normal(m.n * 2) * 1e-6
    broke = 0
    for scale in (0.0, 1.0, 2.0, 3.0):
        u = base * scale
        a_c, h_c, _ = cpu.rate(u)
        a_g, h_g, _ = gpu.rate(u)
        if precision == "fp64":
            assert np.array_equal(h_g, h_c)
            assert _close(a_g, a_c) if np.abs(a_c).max() > 0 else np.abs(a_g).max() == 0
        else:
            assert (h_g != h_c).sum() <= 1e-4 * h_c.size
            assert np.abs(a_g - a_c).max() <= 1e-6 * max(np.abs(a_c).max(), 1e-300)
        broke = int((h_c == 0).sum())
    assert broke > 100


def test_explicit_c_entry_matches_element():
    """pxb_cuda_explicit_accel (the C entry over the same shim call, used by FFI callers and the benchmark) gives the
    reference element's acceleration and health."""
    import ctypes as C

    import perix_b200 as px
    from oracle import RefEpf
    m, _ = _plate(dropin=False)
    E, nu, rho = 190e9, 0.3, 8000.0
    G0 = 0.01 ** 2 * 12 * E * m.delta / (5 * math.pi)
    cpu = RefEpf(m, E, nu, rho, G0)
    cpu.rate(np.zeros(2 * m.n))  # seeds the notch health, derives the constants
    k = cpu.constants()
    health = np.ascontiguousarray(cpu.rate(np.zeros(2 * m.n))[1])
    rng = np.random.default_rng(23)
    u = rng.standard_normal(2 * m.n) * 3e-6
    a_ref, h_ref, _ = cpu.rate(u)
    L = px.lib()
    acc = np.zeros(2 * m.n)
    changed = C.c_int(-1)
    f64 = lambda a: np.ascontiguousarray(a, np.float64).ctypes.data_as(C.POINTER(C.c_double))
    i32 = lambda a: np.ascontiguousarray(a, np.int32).ctypes.data_as(C.POINTER(C.c_int))
    body = np.zeros(3)
    ok = L.pxb_cuda_explicit_accel(m.n, 2, i32(m.off), i32(m.ids), f64(m.coords), f64(m.vols), C.c_double(m.delta),
                                   C.c_double(m.dx_char), C.c_double(k["C11"]), C.c_double(k["C12"]),
                                   C.c_double(k["C66"]), C.c_double(rho), f64(body), C.c_double(k["sc"]), 1, 1, f64(u),
                                   health.ctypes.data_as(C.POINTER(C.c_double)),
                                   acc.ctypes.data_as(C.POINTER(C.c_double)), C.byref(changed))
    assert ok == 1
    assert changed.value == 1
    assert np.array_equal(health, h_ref)
    assert _close(acc, a_ref)
