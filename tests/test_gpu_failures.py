"""Failure paths that leave the context usable, made without faulting the GPU:

* an allocation that exceeds the context's device-memory cap (pxb_ctx_set_memory_limit) fails with PXB_ERR_OOM
  before it reaches the driver; raising the cap lets the same call succeed;
* a staged step kernel whose consumer mbarrier waits are given no tries (pxb_epf_set_wait_budget(ctx, 0)) gives up
  on every tile, drains its bulk copies with the normal budget and reports the failure (PXB_ERR_CUDA, "wait ran
  out"); with the default budget restored the same context reproduces the reference trajectory;
* the staged reverse sweep of the device adjoint (adjoint schedule 2) with no tries fails the same way, and with the
  default budget restored gives the gradient of the unstaged reverse-only sweep."""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


def test_memory_cap_gives_oom_and_context_recovers():
    import perix_b200 as px
    d = load_golden("epf2d")
    s = d["scalars"]
    with px.Context(0) as c:
        c.set_memory_limit(64 << 10)
        with pytest.raises(px.PxbError) as e:
            c.set_geometry(d["coords"], d["vols"], d["off"], d["ids"], s[0], s[4], 2, mirror=d["mirror"])
        assert e.value.status == 4 and "limit" in str(e.value)
        c.set_memory_limit(0)
        c.set_geometry(d["coords"], d["vols"], d["off"], d["ids"], s[0], s[4], 2, mirror=d["mirror"])
        c.gbuild(2, px.FP64)
        before = c.device_bytes()
        c.set_memory_limit(before + 1024)
        sc, C11, C12, C66 = d["consts"][:4]
        with pytest.raises(px.PxbError) as e:
            c.epf_setup(C11, C12, C66, float(d["rho"]), (0, 0), sc, True, health0=d["health0"])
        assert e.value.status == 4


@pytest.mark.parametrize("variant", [8, 11])
def test_wait_budget_exhausted_reports_error_and_context_recovers(ctx, variant):
    import perix_b200 as px
    from test_gpu_parity import epf_context, plate_bcs
    d = load_golden("epf2d")
    n = d["coords"].size // 3
    epf_context(ctx, d, 2)
    ctx.epf_set_variant(variant)
    ctx.epf_set_bcs(plate_bcs(d, px))
    ctx.epf_start(np.zeros(n * 2), None, float(d["dt"]))
    ctx.epf_set_wait_budget(0)
    with pytest.raises(px.PxbError) as e:
        ctx.epf_advance(3, chunk=3)
    assert e.value.status == 2 and "wait ran out" in str(e.value)
    with pytest.raises(px.PxbError) as e:
        ctx.epf_rate(np.zeros(n * 2))
    assert e.value.status == 2 and "wait ran out" in str(e.value)
    # default budget: the same context runs the reference trajectory again
    ctx.epf_set_wait_budget(-1)
    epf_context(ctx, d, 2)
    ctx.epf_set_variant(variant)
    ctx.epf_set_bcs(plate_bcs(d, px))
    ctx.epf_start(np.zeros(n * 2), None, float(d["dt"]))
    ctx.epf_advance(int(d["nsteps"]), chunk=16)
    u, _, h, _ = ctx.epf_state()
    assert np.array_equal(h, d["health"])
    assert np.abs(u - d["u"]).max() <= 1e-10 * np.abs(d["u"]).max()


def test_staged_adjoint_wait_budget_exhausted_reports_error_and_recovers(ctx):
    import ctypes as C

    import perix_b200 as px
    import torch
    from test_gpu_parity import epf_context, plate_bcs
    d = load_golden("epf2d")
    n = d["coords"].size // 3
    epf_context(ctx, d, 2)
    ctx.epf_set_variant(11)
    ctx.epf_set_bcs(plate_bcs(d, px))
    dev = torch.device("cuda", 0)
    ctx.set_stream(torch.cuda.current_stream(dev).cuda_stream)
    rng = np.random.default_rng(5)
    u0 = torch.tensor(rng.standard_normal(2 * n) * 1e-7, device=dev)
    gN = torch.tensor(rng.standard_normal(2 * n), device=dev)
    p = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    assert ctx.L.pxb_epf_record_d(ctx.h, p(u0), None, C.c_double(float(d["dt"])), 20, 0, None, None) == 0

    def sweep(schedule):
        ctx.epf_set_adjoint_schedule(schedule)
        u0b, v0b = torch.empty_like(u0), torch.empty_like(u0)
        dC = torch.zeros(3, dtype=torch.float64, device=dev)
        st = ctx.L.pxb_epf_adjoint_recorded_d(ctx.h, p(gN), None, p(u0b), p(v0b), p(dC))
        torch.cuda.synchronize(dev)
        return st, u0b.cpu().numpy(), dC.cpu().numpy()

    ctx.epf_set_wait_budget(0)
    st, _, _ = sweep(2)
    assert st == 2 and "wait ran out" in ctx.L.pxb_last_error().decode()
    ctx.epf_set_wait_budget(-1)
    st, g2, c2 = sweep(2)
    assert st == 0
    st, g1, c1 = sweep(1)
    assert st == 0
    assert np.abs(g2 - g1).max() <= 1e-12 * np.abs(g1).max()
    assert np.abs(c2 - c1).max() <= 1e-12 * np.abs(c1).max()
