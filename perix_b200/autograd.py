"""torch.autograd wrappers over the adjoint kernels of the C-ABI.

- ``pddo_apply(ctx, u, slots)``: the family-sum derivative apply D^k u (reference PoissonElement.cpp:67-105,
  ExplicitPDDOFracElement.cpp:348-366); its backward is the transpose family-scatter ``pxb_apply_adjoint_d``.
- ``frozen_force(ctx, u, C)``: the explicit element's acceleration a = (L(u) + b)/rho with the damage mask held
  fixed (reference ExplicitPDDOFracElement.cpp:239-299 without the breaking test); its backward is the
  bond-force adjoint ``pxb_epf_force_adjoint_d``, which returns dJ/du and dJ/d(C11, C12, C66).
- ``explicit_loop(ctx, u0, v0, dt, nsteps, C, plan)``: the central-difference loop of the reference
  (TimeStepping.cpp:479-536) with the ghost BC preset after every step (DirichletBC.cpp:107-147,
  NeumannBC.cpp:88-105), written in torch around ``frozen_force``.  Segments of ``checkpoint_every`` steps are
  wrapped in torch.utils.checkpoint, so the backward pass keeps one state per segment and recomputes the
  steps inside a segment.
- ``explicit_run(ctx, u0, v0, C, dt, nsteps)``: the same loop run entirely on the device (the context's fused
  step kernels and its BC program); its backward is the device adjoint ``pxb_epf_adjoint_d`` (per step the BC
  transpose and one fused bond-force / central-difference adjoint kernel, forward states recomputed from
  checkpoints), which returns dJ/du0, dJ/dv0 and dJ/dC.
- ``elastic_constants_t``: C11, C12, C66 as torch functions of E and nu (ExplicitPDDOFracElement.cpp:38-53).
- ``ch_free_energy(ctx, c0, kappa, ...)``: the total free energy after a backward-Euler Cahn-Hilliard run on the
  device (CahnHilliardElement.cpp:66-292 per step); its backward is the discrete adjoint of the run
  (``pxb_ch_gradient``), which returns dE/dkappa and dE/dc0 together.

The perix context does the arithmetic; torch supplies the tape, the device memory and the stream (each call
puts the context on torch's current stream).  All tensors are float64 on the context's GPU.
"""
import numpy as np
import torch
from torch.utils.checkpoint import checkpoint

from .api import BC, Context  # noqa: F401  (BC for type hints in callers)


def _on_stream(pctx, t):
    pctx.set_stream(torch.cuda.current_stream(t.device).cuda_stream)


def _f64c(t):
    return t.detach().to(torch.float64).contiguous()


class _Apply(torch.autograd.Function):
    @staticmethod
    def forward(fctx, u, pctx, slots):
        u = _f64c(u)
        out = torch.empty((u.numel(), len(slots)), dtype=torch.float64, device=u.device)
        _on_stream(pctx, u)
        pctx.apply_d(u.data_ptr(), slots, out.data_ptr())
        fctx.pctx, fctx.slots = pctx, list(slots)
        return out

    @staticmethod
    def backward(fctx, gout):
        g = _f64c(gout)
        ub = torch.empty(g.shape[0], dtype=torch.float64, device=g.device)
        _on_stream(fctx.pctx, g)
        fctx.pctx.apply_adjoint_d(g.data_ptr(), fctx.slots, ub.data_ptr())
        return ub, None, None


def pddo_apply(pctx, u, slots):
    """(N,) scalar field -> (N, len(slots)) derivatives for the multi-index slots (0-based) of the context's
    operator cache; differentiable in u."""
    return _Apply.apply(u, pctx, list(slots))


class _FrozenForce(torch.autograd.Function):
    @staticmethod
    def forward(fctx, u, C, pctx):
        u = _f64c(u)
        a = torch.empty_like(u)
        _on_stream(pctx, u)
        pctx.epf_force_frozen_d(u.data_ptr(), a.data_ptr())
        fctx.save_for_backward(u)
        fctx.pctx = pctx
        return a

    @staticmethod
    def backward(fctx, abar):
        (u,) = fctx.saved_tensors
        ab = _f64c(abar)
        ub = torch.empty_like(u)
        dC = torch.empty(3, dtype=torch.float64, device=u.device)
        _on_stream(fctx.pctx, u)
        fctx.pctx.epf_force_adjoint_d(u.data_ptr(), ab.data_ptr(), ub.data_ptr(), dC.data_ptr())
        return ub, dC, None


def frozen_force(pctx, u, C):
    """a = (L(u) + b)/rho (N*dim, interleaved) with the context's current health mask held fixed.  C is the
    (3,) tensor (C11, C12, C66) that the context was set up with (``epf_set_constants``); it only routes the
    gradient dJ/dC."""
    return _FrozenForce.apply(u, C, pctx)


def elastic_constants_t(dim, plane_stress, E, nu):
    """(C11, C12, C66) as a (3,) tensor, differentiable in E (and nu)."""
    if dim >= 3 or not plane_stress:
        d = (1.0 + nu) * (1.0 - 2.0 * nu)
        return torch.stack([E * (1.0 - nu) / d, E * nu / d, E / (2.0 * (1.0 + nu))])
    d = 1.0 - nu * nu
    return torch.stack([E / d, E * nu / d, E / (2.0 * (1.0 + nu))])


class BcPlan:
    """The BC list compiled to index tensors: entries are applied in list order (reference semantics); within
    an entry every target is written from values read before the entry (no target of an entry is the mirror of
    another of its targets, which holds for ghost layers and boxed groups; checked here).

    Dirichlet: u[g,a] = 2 G(t) - u[mirror(g),a] (reflection) or G(t) (direct or no mirror), G = value + velocity*t,
    nodes filtered by the optional box; Neumann: u[g,a] = u[mirror(g),a] for ghosts with a mirror."""

    def __init__(self, bcs, coords3, mirror, dim, device):
        xyz = np.asarray(coords3, np.float64).reshape(-1, 3)
        mir = np.zeros(xyz.shape[0], np.int64) if mirror is None else np.asarray(mirror, np.int64)
        self.dim = dim
        self.ops = []
        for bc in bcs:
            ids = np.unique(np.asarray(bc.nodes, np.int64))  # 1-based; a repeated id writes the same value
            comps = [int(c) for c in bc.comps]
            if bc.kind == "dirichlet":
                if bc.box is not None:
                    # DirichletBC::insideBox: all three axes, an axis with min > max unconstrained
                    box = np.asarray(list(bc.box) + [0.0] * (6 - len(bc.box)), np.float64)
                    inside = np.ones(ids.size, bool)
                    for a in range(3):
                        if box[2 * a] > box[2 * a + 1]:
                            continue
                        x = xyz[ids - 1, a]
                        inside &= (x >= box[2 * a]) & (x <= box[2 * a + 1])
                    ids = ids[inside]
                mb = mir[ids - 1]
                refl = (mb >= 1) & (not bc.direct)
                for kind, sel in (("reflect", refl), ("direct", ~refl)):
                    if not sel.any():
                        continue
                    tg, sr, va, ve = [], [], [], []
                    for a in comps:
                        tg.append((ids[sel] - 1) * dim + a)
                        sr.append((mb[sel] - 1) * dim + a)
                        va.append(np.full(sel.sum(), float(bc.value[a])))
                        ve.append(np.full(sel.sum(), float(bc.velocity[a])))
                    tgt, src = np.concatenate(tg), np.concatenate(sr)
                    if kind == "reflect":
                        assert not np.intersect1d(tgt, src).size, "a BC target mirrors another target"
                    self.ops.append((kind, torch.from_numpy(tgt).to(device), torch.from_numpy(src).to(device),
                                     torch.from_numpy(np.concatenate(va)).to(device),
                                     torch.from_numpy(np.concatenate(ve)).to(device)))
            else:
                mb = mir[ids - 1]
                ids, mb = ids[mb >= 1], mb[mb >= 1]
                if not ids.size:
                    continue
                tgt = np.concatenate([(ids - 1) * dim + a for a in comps])
                src = np.concatenate([(mb - 1) * dim + a for a in comps])
                assert not np.intersect1d(tgt, src).size, "a BC target mirrors another target"
                self.ops.append(("copy", torch.from_numpy(tgt).to(device), torch.from_numpy(src).to(device),
                                 None, None))

    def apply(self, u, t):
        for kind, tgt, src, val, vel in self.ops:
            if kind == "copy":
                u = u.index_put((tgt,), u[src])
            else:
                g = val + vel * t
                u = u.index_put((tgt,), 2.0 * g - u[src] if kind == "reflect" else g)
        return u


def _segment(pctx, C, plan, dt2, times, force, u, uold):
    for tn in times:
        a = force(pctx, u, C)
        un = 2.0 * u - uold + dt2 * a
        un = plan.apply(un, tn)
        uold, u = u, un
    return u, uold


def explicit_loop(pctx, u0, v0, dt, nsteps, C, plan, checkpoint_every=100, t0=0.0, force=None):
    """nsteps central-difference steps from (u0, v0) at t0 with a frozen damage mask; returns (u^N, u^{N-1}).

    u^{-1} = u0 - dt v0 + dt^2/2 a(u0); u^{n+1} = 2u^n - u^{n-1} + dt^2 a(u^n), then the BC preset at t_{n+1}
    (t accumulated as t + dt like the reference loop).  The context's constants must equal C (see
    ``set_constants``).  With checkpoint_every > 0 each segment of that many steps is recomputed in the
    backward pass instead of stored.  ``force(pctx, u, C)`` replaces ``frozen_force`` (e.g. by a plain-torch
    restatement for reference gradients)."""
    force = force or frozen_force
    a0 = force(pctx, u0, C)
    if v0 is None:
        v0 = torch.zeros_like(u0)
    uold = u0 - dt * v0 + (0.5 * dt * dt) * a0
    u = u0
    dt2 = dt * dt
    t = t0
    done = 0
    while done < nsteps:
        k = min(checkpoint_every if checkpoint_every > 0 else nsteps, nsteps - done)
        times = []
        for _ in range(k):
            t = t + dt
            times.append(t)
        if checkpoint_every > 0 and torch.is_grad_enabled():
            u, uold = checkpoint(_segment, pctx, C, plan, dt2, times, force, u, uold, use_reentrant=False)
        else:
            u, uold = _segment(pctx, C, plan, dt2, times, force, u, uold)
        done += k
    return u, uold


def _record(pctx, u0, v0, dt, nsteps, ck, uN=None, uNm1=None):
    import ctypes as Ct
    p = lambda t: None if t is None else Ct.c_void_p(t.data_ptr())  # noqa: E731
    _on_stream(pctx, u0)
    st = pctx.L.pxb_epf_record_d(pctx.h, p(u0), p(v0), Ct.c_double(dt), int(nsteps), int(ck), p(uN), p(uNm1))
    if st:
        from .api import PxbError
        raise PxbError(st, pctx.L.pxb_last_error().decode(errors="replace"))
    pctx._recording = token = object()  # the context keeps one recording: the latest
    return token


class _ExplicitRun(torch.autograd.Function):
    @staticmethod
    def forward(fctx, u0, C, v0, pctx, dt, nsteps, checkpoint_every):
        u0c = _f64c(u0)
        v0c = None if v0 is None else _f64c(v0)
        uN = torch.empty_like(u0c)
        uNm1 = torch.empty_like(u0c)
        fctx.token = _record(pctx, u0c, v0c, dt, nsteps, checkpoint_every, uN, uNm1)
        fctx.save_for_backward(u0c, *(() if v0c is None else (v0c,)))
        fctx.pctx, fctx.dt, fctx.nsteps, fctx.ck, fctx.has_v0 = pctx, dt, nsteps, checkpoint_every, v0c is not None
        return uN, uNm1

    @staticmethod
    def backward(fctx, gN, gNm1):
        import ctypes as Ct
        saved = fctx.saved_tensors
        u0 = saved[0]
        v0 = saved[1] if fctx.has_v0 else None
        if getattr(fctx.pctx, "_recording", None) is not fctx.token:  # a later run replaced this one's recording
            fctx.token = _record(fctx.pctx, u0, v0, fctx.dt, fctx.nsteps, fctx.ck)
        gN = torch.zeros_like(u0) if gN is None else _f64c(gN)
        gNm1 = None if gNm1 is None else _f64c(gNm1)
        u0bar = torch.empty_like(u0)
        v0bar = torch.empty_like(u0)
        dC = torch.zeros(3, dtype=torch.float64, device=u0.device)
        _on_stream(fctx.pctx, u0)
        p = lambda t: None if t is None else Ct.c_void_p(t.data_ptr())  # noqa: E731
        st = fctx.pctx.L.pxb_epf_adjoint_recorded_d(fctx.pctx.h, p(gN), p(gNm1), p(u0bar), p(v0bar), p(dC))
        if st:
            from .api import PxbError
            raise PxbError(st, fctx.pctx.L.pxb_last_error().decode(errors="replace"))
        return u0bar, dC, (v0bar if fctx.has_v0 else None), None, None, None, None


def explicit_run(pctx, u0, v0, C, dt, nsteps, checkpoint_every=0):
    """(u^N, u^{N-1}) of nsteps central-difference steps from (u0, v0) run on the device with the context's BC program
    (pxb_epf_record_d, which keeps the forward states the backward pass needs), differentiable in u0, v0 and C through
    the device adjoint (pxb_epf_adjoint_recorded_d).  The damage mask is frozen at the context's current health (no
    bond breaks; the context's explicit state is left as it is), and the context's constants must equal C
    (``set_constants``).  checkpoint_every > 0 keeps a state every that many steps and recomputes the others in the
    backward pass; 0 keeps them all (nsteps * N * dim doubles on the device)."""
    return _ExplicitRun.apply(u0, C, v0, pctx, float(dt), int(nsteps), int(checkpoint_every))


def set_constants(pctx, C, rho):
    """Puts the values of the (3,) tensor C into the context (one device-to-host read)."""
    c11, c12, c66 = (float(x) for x in C.detach().cpu())
    pctx.epf_set_constants(c11, c12, c66, rho)


class _ChEnergy(torch.autograd.Function):
    @staticmethod
    def forward(fctx, c0, kappa, pctx, chi, M0, dt, nsteps):
        c = _f64c(c0).cpu().numpy()
        k = float(kappa)
        E, dk, g, _ = pctx.ch_gradient(c, chi, k, M0, dt, nsteps)
        fctx.save_for_backward(torch.from_numpy(g).to(c0.device), torch.tensor(dk, dtype=torch.float64,
                                                                               device=c0.device))
        return torch.tensor(E, dtype=torch.float64, device=c0.device)

    @staticmethod
    def backward(fctx, gE):
        g, dk = fctx.saved_tensors
        return gE * g, gE * dk, None, None, None, None, None


def ch_free_energy(pctx, c0, kappa, chi, M0, dt, nsteps):
    """Total free energy of the final state of an implicit Cahn-Hilliard run from c0 (one value per node; ghost
    entries follow their mirror nodes) as a differentiable function of c0 and kappa (a 0-d tensor).  The forward
    pass already runs the adjoint (pxb_ch_gradient) and keeps the gradient for the backward pass."""
    if not torch.is_tensor(kappa):
        kappa = torch.tensor(float(kappa), dtype=torch.float64, device=c0.device)
    return _ChEnergy.apply(c0, kappa, pctx, float(chi), float(M0), float(dt), int(nsteps))

