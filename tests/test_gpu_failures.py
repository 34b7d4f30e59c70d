"""Failure paths that leave the context usable, made without faulting the GPU:

* an allocation that exceeds the context's device-memory cap (pxb_ctx_set_memory_limit) fails with PXB_ERR_OOM
  before it reaches the driver; raising the cap lets the same call succeed;
* a staged step kernel whose consumer mbarrier waits are given no tries (pxb_epf_set_wait_budget(ctx, 0)) gives up
  on every tile, drains its bulk copies with the normal budget and reports the failure (PXB_ERR_CUDA, "wait ran
  out"); with the default budget restored the same context reproduces the reference trajectory."""
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
