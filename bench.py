"""Benchmark: explicit PDDO fracture bond-updates/s (and g-build nodes/s).

Headline workload: the 3D notched slab (120x120x24 bulk nodes + one ghost layer per face = 385,920 PD nodes,
44,189,344 directed bonds, h = 1 mm, delta = 3.015h, E = 72 GPa, nu = 0.22, rho = 2440, s_c = 0.004, a central edge
notch of depth 20h as a force-only crack plane, +-2 m/s pins on the top and bottom three-node layers,
dt = 0.8 h / sqrt(C11/rho)).  The 2D notched plate (400x200 nodes, h = 0.5 mm, E = 190 GPa, nu = 0.3, rho = 8000,
s_c = 0.01, two force-only slits of 50h, 16.5 m/s pull) is reported under "plate_2d".

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl perix|reference] [--headline-only]

A step is one explicit time step (damage + Navier force + central difference + BC pass, one fused kernel),
timed alone with CUDA events on the launching stream; the L2 is flushed (256 MiB write, then read back) before
every timed step (the slab's bond streams, 1.3-2.4 GB, exceed the L2 anyway), and the state is restored from a
snapshot taken 100 steps into the run every 100 steps, so every timed step works on the same physical regime.
Multi-GPU runs (torchrun) are independent replicas of the slab (weak scaling); the time is the max over ranks.
Prints one JSON line on rank 0.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

FLUSH_BYTES = 256 << 20
EPISODE = 100          # steps between snapshot restores
S0 = 100               # steps run before the snapshot is taken


# ------------------------------------------------------------------------------------------------- workload
def plate_setup(px):
    nx, ny, h = 400, 200, 5e-4
    L = px.lattice(2, nx, ny, 0, [0.0, nx * h, 0.0, ny * h])
    delta = 3.015 * L.dxyz[0] * (1.0 + 1e-6)
    y1, y2 = 0.05 - 25 * h, 0.05 + 25 * h
    cracks = [[0.0, y1, 50 * h, y1], [0.0, y2, 50 * h, y2]]
    off, ids = px.families(L.coords, delta, False, cracks=cracks, mirror=L.mirror, force_only=True)
    health0 = (1 - px.crack_cut_mask(L.coords, L.mirror, off, ids, cracks=cracks)).astype(np.uint8)
    E, nu, rho = 190e9, 0.3, 8000.0
    C11, C12, C66 = px.elastic_constants(2, False, E, nu)
    sc_target = 0.01
    G0 = sc_target ** 2 * 12.0 * E * delta / (5.0 * math.pi)
    sc = px.critical_stretch(2, False, G0, E, delta)
    dt = 0.8 * h / math.sqrt(C11 / rho)
    bcs = [px.BC("neumann", [0, 1], L.group(w + "nodes_ghost")) for w in ("left", "right", "bottom", "top")]
    bcs.append(px.BC("dirichlet", [0], L.group("leftnodes_ghost"), value=[0, 0], velocity=[16.5, 0], direct=True,
                     box=[-1, 1, y1, y2, -1, 1]))
    return dict(L=L, off=off, ids=ids, delta=delta, health0=health0, C=(C11, C12, C66), rho=rho, sc=sc, dt=dt,
                bcs=bcs, E=E, nu=nu, G0=G0, cracks=cracks, n=L.n, nb=int(off[-1]), h=h, dim=2, kind="plate")


def slab_setup(px, nx=120, ny=120, nz=24):
    """3D slab (120x120x24 bulk nodes + one ghost layer per face = 385,920 nodes), h = 1 mm, delta = 3.015h,
    E = 72 GPa, nu = 0.22, rho = 2440, s_c = 0.004 (G0 = s_c^2 6 E delta / 5), central edge notch of depth 20h
    as a force-only crack plane at y = Ly/2, zero Neumann on every ghost wall, then +-2 m/s y-velocity pins on
    the top and bottom three-node layers (box on all nodes), dt = 0.8 h / sqrt(C11 / rho)."""
    h = 1e-3
    Lx, Ly, Lz = nx * h, ny * h, nz * h
    L = px.lattice(3, nx, ny, nz, [0.0, Lx, 0.0, Ly, 0.0, Lz])
    delta = 3.015 * L.dxyz[0] * (1.0 + 1e-6)
    plane = [0.0, Ly / 2, -1.0, 20 * h, Ly / 2, -1.0, 20 * h, Ly / 2, 1.0, 0.0, Ly / 2, 1.0]
    off, ids = px.families(L.coords, delta, True, planes=[plane], mirror=L.mirror, force_only=True)
    health0 = (1 - px.crack_cut_mask(L.coords, L.mirror, off, ids, planes=[plane])).astype(np.uint8)
    E, nu, rho, sc_t = 72e9, 0.22, 2440.0, 0.004
    C11, C12, C66 = px.elastic_constants(3, False, E, nu)
    G0 = sc_t ** 2 * 6.0 * E * delta / 5.0
    sc = px.critical_stretch(3, False, G0, E, delta)
    dt = 0.8 * h / math.sqrt(C11 / rho)
    bcs = [px.BC("neumann", [0, 1, 2], L.group(w + "nodes_ghost"))
           for w in ("left", "right", "bottom", "top", "back", "front")]
    alld = L.group("alldomain")
    bcs.append(px.BC("dirichlet", [1], alld, value=[0, 0, 0], velocity=[0, 2.0, 0], direct=True,
                     box=[-1, 1, Ly - 3 * h, 1, -1, 1]))
    bcs.append(px.BC("dirichlet", [1], alld, value=[0, 0, 0], velocity=[0, -2.0, 0], direct=True,
                     box=[-1, 1, -1, 3 * h, -1, 1]))
    return dict(L=L, off=off, ids=ids, delta=delta, health0=health0, C=(C11, C12, C66), rho=rho, sc=sc, dt=dt,
                bcs=bcs, E=E, nu=nu, G0=G0, plane=plane, n=L.n, nb=int(off[-1]), h=h, dim=3, kind="slab",
                size=(nx, ny, nz))


def slab_adjoint(px, device=0, adjoint_steps=1000, checkpoint_every=100):
    """The 3D slab's frozen-mask adjoint: d(misfit)/dE over the first `adjoint_steps` steps with checkpointed
    recomputation, checked against central finite differences of the device loop."""
    import torch
    from perix_b200.autograd import elastic_constants_t, explicit_run, set_constants
    t0 = time.perf_counter()
    w = slab_setup(px)
    res = {"workload": "3D slab 120x120x24 (+ghosts), edge notch 20h", "nodes": w["n"], "bonds": w["nb"],
           "host_setup_s": time.perf_counter() - t0}
    L = w["L"]
    # adjoint: misfit against the displacement of a 2 % stiffer slab, frozen damage mask (damage off)
    dev = torch.device("cuda", device)
    ctx = px.Context(device)
    ctx.set_geometry(L.coords, L.vols, w["off"], w["ids"], w["delta"], L.dxyz[0], 3, mirror=L.mirror)

    tuned = {}

    def device_final(E):
        c = px.elastic_constants(3, False, E, w["nu"])
        ctx.epf_setup(c[0], c[1], c[2], w["rho"], (0.0, 0.0, 0.0), 0.0, True, health0=w["health0"])
        ctx.epf_set_bcs(w["bcs"])
        ctx.epf_start(np.zeros(3 * L.n), None, w["dt"])
        if not tuned:  # the step schedule of this frozen-mask loop, timed once (state unchanged)
            tuned.update(autotune(ctx))
        ctx.epf_set_variant(tuned["variant"])
        ctx.epf_advance(adjoint_steps, chunk=100)
        return ctx.epf_state()[0]

    u_obs = device_final(1.02 * w["E"])
    J = lambda uN: 0.5 * float(((uN - u_obs) ** 2).sum())  # noqa: E731
    def cfd(rel):
        hE = rel * w["E"]
        return (J(device_final(w["E"] + hE)) - J(device_final(w["E"] - hE))) / (2 * hE)

    # central differences at two steps; their Richardson extrapolation removes the O(h^2) truncation term,
    # which 1000 steps of wave propagation make visible at h = 1e-5 E
    fd1, fd2 = cfd(1e-5), cfd(5e-6)
    fd = (4.0 * fd2 - fd1) / 3.0
    # the forward loop alone: start + adjoint_steps graph-captured steps on the set-up context (set-up and the state
    # read-back outside the timed region, as the gradient's set-up is)
    device_final(w["E"])
    ctx.epf_start(np.zeros(3 * L.n), None, w["dt"])
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    ctx.epf_advance(adjoint_steps, chunk=100)
    torch.cuda.synchronize(dev)
    fwd_secs = time.perf_counter() - t0
    def gradient(ck):
        E = torch.tensor(w["E"], dtype=torch.float64, device=dev, requires_grad=True)
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        C = elastic_constants_t(3, False, E, w["nu"])
        set_constants(ctx, C, w["rho"])
        uN, _ = explicit_run(ctx, torch.zeros(3 * L.n, dtype=torch.float64, device=dev), None, C, w["dt"],
                             adjoint_steps, checkpoint_every=ck)
        Jt = 0.5 * ((uN - torch.from_numpy(u_obs).to(dev)) ** 2).sum()
        Jt.backward()
        torch.cuda.synchronize(dev)
        secs = time.perf_counter() - t0
        return {"steps": adjoint_steps, "checkpoint_every": ck, "precision": "fp64", "dJ_dE": float(E.grad),
                "dJ_dE_central_fd": {"h=1e-5E": fd1, "h=5e-6E": fd2, "richardson": fd},
                "rel_err_vs_fd": abs(float(E.grad) - fd) / abs(fd),
                "rel_err_vs_fd_h5e-6": abs(float(E.grad) - fd2) / abs(fd2), "seconds_forward_and_backward": secs,
                "seconds_forward_loop_alone": fwd_secs, "over_forward": secs / fwd_secs}

    how = ("forward: the frozen-mask device loop keeping its checkpoints (pxb_epf_record_d); backward: per step the BC "
           "transpose and one fused bond-force / central-difference adjoint kernel (pxb_epf_adjoint_recorded_d)")
    res["forward_step_variant"] = tuned.get("variant")
    gradient(checkpoint_every)  # warm-up: the first gradient call carries one-off set-up (reverse maps, buffers)
    res["adjoint"] = gradient(checkpoint_every)
    res["adjoint"]["method"] = how + ", states recomputed segment by segment from the checkpoints"
    gradient(0)  # warm-up of the all-states buffers
    res["adjoint_all_states_kept"] = gradient(0)
    res["adjoint_all_states_kept"]["method"] = how + ", every state kept (%.1f GB), nothing recomputed" % (
        adjoint_steps * 3 * L.n * 8 / 1e9)
    ctx.close()
    return res


def poisson_solve(px, kvals, rhs, L, rowptr, cols):
    """One static solve of the assembled 64x64 Poisson system (K dU = RHS from U = 0, the Newton step of a linear problem)
    after the reference's Dirichlet row replacement on the ghost layer (DirichletBC.cpp:176-231: ghost row g
    becomes s*(dU_g + dU_b) = s*(2*0 - U_g - U_b), reflecting through the wall).  Host direct solve (the solve is
    not on the hot path); returns U and the relative L2 error against sin(pi x) sin(pi y) over the bulk nodes."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla
    n = L.n
    K = sp.csr_matrix((np.asarray(kvals, np.float64), np.asarray(cols), np.asarray(rowptr)), shape=(n, n)).tolil()
    b = np.asarray(rhs, np.float64).copy()
    for g in np.nonzero(L.mirror > 0)[0]:
        K.rows[g] = [g, int(L.mirror[g]) - 1]
        K.data[g] = [1.0, 1.0]
        b[g] = 0.0
    U = spla.spsolve(K.tocsr(), b)
    x, y = L.coords[0::3], L.coords[1::3]
    bulk = L.mirror == 0
    ex = np.sin(math.pi * x) * np.sin(math.pi * y)
    err = math.sqrt(float(((U - ex)[bulk] ** 2 * L.vols[bulk]).sum()) / float((ex[bulk] ** 2 * L.vols[bulk]).sum()))
    return U, err


def poisson_measure(px, device=0, reps=20):
    """The 64x64 Poisson workload: 64x64 cell-centred lattice on the unit square, delta = 3.015h, order 2, sigma = 1,
    f = 2 pi^2 sin(pi x) sin(pi y), reflected Dirichlet 0 on the four ghost groups.  FP64 g-build and Poisson
    assembly on the GPU (CUDA events), one host solve, L2 error; the reference's OpenMP assembly of the same
    system through oracle/_ref is timed beside it when present."""
    import torch
    L = px.lattice(2, 64, 64, 0, [0.0, 1.0, 0.0, 1.0])
    delta = 3.015 * L.dxyz[0] * (1.0 + 1e-6)
    off, ids = px.families(L.coords, delta, False, mirror=L.mirror)
    rowptr, cols = px.csr_pattern(off, ids, L.mirror, 1)
    ctx = px.Context(device)
    ctx.set_geometry(L.coords, L.vols, off, ids, delta, L.dxyz[0], 2, mirror=L.mirror)
    gb, gb_ms = gbuild_rate(px, ctx, "fp64", reps=5)
    ctx.gbuild(2, px.FP64)
    ctx.csr_set_pattern(rowptr, cols, 1)
    x, y = L.coords[0::3], L.coords[1::3]
    f = 2 * math.pi ** 2 * np.sin(math.pi * x) * np.sin(math.pi * y)
    dev = torch.device("cuda", device)
    ctx.set_stream(torch.cuda.current_stream(dev).cuda_stream)
    fd = torch.from_numpy(f).to(dev)
    ud = torch.zeros(L.n, dtype=torch.float64, device=dev)
    kd = torch.empty(int(rowptr[-1]), dtype=torch.float64, device=dev)
    rd = torch.empty(L.n, dtype=torch.float64, device=dev)
    import ctypes as C

    def assemble():
        st = ctx.L.pxb_assemble_scalar_d(ctx.h, 0, C.c_double(1.0), C.c_double(0.0), C.c_void_p(fd.data_ptr()),
                                         C.c_double(0.0), C.c_void_p(ud.data_ptr()), None, C.c_void_p(kd.data_ptr()),
                                         C.c_void_p(rd.data_ptr()))
        if st:
            raise RuntimeError(ctx.L.pxb_last_error().decode())

    for _ in range(3):
        assemble()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    ev[0].record()
    for _ in range(reps):
        assemble()
    ev[1].record()
    torch.cuda.synchronize(dev)
    asm_ms = ev[0].elapsed_time(ev[1]) / reps
    U, err = poisson_solve(px, kd.cpu().numpy(), rd.cpu().numpy(), L, rowptr, cols)
    res = {"nodes": L.n, "bonds": int(off[-1]), "nnz": int(rowptr[-1]), "gbuild_ms": gb_ms,
           "assembly_ms": asm_ms, "l2_rel_error_vs_exact": err}
    try:
        from oracle import RefMesh, ref_available
        if ref_available():
            m = RefMesh.structured(2, 64, 64, 0, [0, 1, 0, 1], 3.015, 2)
            m.gbuild()
            _, _, t = m.poisson_assemble(1.0, f, np.zeros(m.n))
            res["reference_cpu_assembly_ms"] = t * 1e3
            res["reference_cpu_gbuild_ms"] = m.gbuild_time(reps=3) * 1e3
            res["reference_cpu_threads"] = os.cpu_count()
    except Exception as e:  # noqa: BLE001
        res["reference_cpu_assembly_ms"] = "unavailable: %s" % e
    ctx.close()
    return res


def ch_measure(px, device=0, nside=256, nsteps=200, reps=20, fd=True):
    """The 256x256 Cahn-Hilliard spinodal-decomposition workload: h = 1/256, delta = 3.015h, c0 = 0.5 + U(+-0.01)
    (seeded), chi = 2.5, M0 = 1, kappa = 1e-4, backward Euler dt = 1e-6 for 200 steps, mobility frozen per Newton
    iteration, zero Neumann on the four ghost walls.  Times the CH assembly kernel (CUDA events, L2 flushed) with
    its HBM roofline, the whole run on the device (wall clock: each Newton iteration reads its residual norm back,
    each BiCGStab solve its device-side status once per batch of iterations) and the adjoint gradient of the final
    free energy in kappa and c0, and checks both against central differences and their Richardson extrapolation."""
    import ctypes as C

    import torch
    L = px.lattice(2, nside, nside, 0, [0.0, 1.0, 0.0, 1.0])
    delta = 3.015 * L.dxyz[0] * (1.0 + 1e-6)
    off, ids = px.families(L.coords, delta, False, mirror=L.mirror)
    t0 = time.perf_counter()
    rowptr, cols = px.csr_pattern(off, ids, L.mirror, 2)
    t_host_pattern = time.perf_counter() - t0
    ctx = px.Context(device)
    ctx.set_geometry(L.coords, L.vols, off, ids, delta, L.dxyz[0], 2, mirror=L.mirror)
    ctx.gbuild(2, px.FP64)
    ctx.ch_build_geometry()
    ctx.csr_build_pattern(2)  # warm-up
    t_dev = []
    for _ in range(3):  # the pattern of the run: built on the device, slot map included (best of 3 builds)
        t0 = time.perf_counter()
        ctx.csr_build_pattern(2)
        t_dev.append(time.perf_counter() - t0)
    t_dev_pattern = min(t_dev)
    r_d, c_d = ctx.csr_get_pattern()
    pattern_match = bool(np.array_equal(r_d, rowptr) and np.array_equal(c_d, cols))
    chi, kappa, M0, dt = 2.5, 1e-4, 1.0, 1e-6
    rng = np.random.default_rng(2024)
    c0 = 0.5 + rng.uniform(-0.01, 0.01, L.n)
    nb, nnz = int(off[-1]), int(rowptr[-1])
    res = {"nodes": L.n, "bonds": nb, "rows": 2 * L.n, "nnz": nnz, "steps": nsteps,
           "pattern_host_ms": t_host_pattern * 1e3, "pattern_device_ms": t_dev_pattern * 1e3,
           "pattern_device_ms_runs": [t * 1e3 for t in t_dev],
           "pattern_device_matches_host": pattern_match}
    # the assembly kernel alone at the initial state
    dev = torch.device("cuda", device)
    ctx.set_stream(torch.cuda.current_stream(dev).cuda_stream)
    u = np.zeros(2 * L.n)
    u[0::2] = np.where(L.mirror > 0, c0[np.maximum(L.mirror, 1) - 1], c0)
    ud = torch.from_numpy(u).to(dev)
    mn = torch.empty(L.n, dtype=torch.float64, device=dev)
    ctx.ch_mobility_d(M0, ud.data_ptr(), mn.data_ptr())
    kd = torch.empty(nnz, dtype=torch.float64, device=dev)
    rd = torch.empty(2 * L.n, dtype=torch.float64, device=dev)
    flush = torch.empty(FLUSH_BYTES // 8, dtype=torch.float64, device=dev)
    ms = []
    for r in range(reps + 3):
        flush.fill_(float(r))
        flush.sum()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        ctx.assemble_ch_d(kappa, chi, dt, mn.data_ptr(), ud.data_ptr(), ud.data_ptr(), kd.data_ptr(), rd.data_ptr())
        b.record()
        torch.cuda.synchronize(dev)
        if r >= 3:
            ms.append(a.elapsed_time(b))
    asm_ms = float(np.mean(ms))
    # bytes per assembly: per bond id 4 + g2 8 + reverse index 4 + 4 slot ids 16 + 4 K values 32; per node the
    # state (c, mu, c_old: 24), mobility 8, volume 8, rhs 16, and the zeroing of the node's two rows
    B = nb * (4 + 8 + 4 + 16 + 32) + L.n * (24 + 8 + 8 + 16)
    hbm, _ = peaks()
    res["assembly_ms"] = asm_ms
    res["assembly_algorithmic_bytes"] = B
    res["assembly_achieved_gbs"] = B / (asm_ms * 1e-3) / 1e9
    res["assembly_frac_of_measured_hbm"] = B / (asm_ms * 1e-3) / 1e9 / hbm
    ctx.set_stream(None)
    t0 = time.perf_counter()
    _, E, st = ctx.ch_run(c0, chi, kappa, M0, dt, nsteps)
    t_run = time.perf_counter() - t0
    res.update(run_s=t_run, steps_per_s=nsteps / t_run, energy=E, newton_iters=st["newton_iters"],
               bicgstab_iters=st["lin_iters"], max_bicgstab_relres=st["max_lin_relres"])
    t0 = time.perf_counter()
    E2, dk, g, st2 = ctx.ch_gradient(c0, chi, kappa, M0, dt, nsteps)
    res.update(gradient_s=time.perf_counter() - t0, dE_dkappa=dk, dE_dc0_norm=float(np.linalg.norm(g)),
               energy_gradient_run_matches=abs(E2 - E) <= 1e-14 * abs(E))
    try:
        from oracle import RefMesh, ref_available
        if ref_available():
            # the reference's OpenMP assembly of the same system (its element preprocess excluded)
            m = RefMesh.structured(2, nside, nside, 0, [0, 1, 0, 1], 3.015, 2)
            _, _, _, t = m.ch_assemble(chi, kappa, M0, dt, u, u)
            res["reference_cpu_assembly_ms"] = t * 1e3
            res["reference_cpu_threads"] = os.cpu_count()
    except Exception as e:  # noqa: BLE001
        res["reference_cpu_assembly_ms"] = "unavailable: %s" % e
    if fd:
        # central differences with steps h and 2h; their Richardson combination removes the h^2 term, which at
        # 200 steps of spinodal growth is not small against 1e-6 (the growth rate depends strongly on kappa)
        def central(f, h):
            return (f(h) - f(-h)) / (2 * h)

        fk = lambda e: ctx.ch_run(c0, chi, kappa + e, M0, dt, nsteps)[1]
        d1, d2 = central(fk, 1e-6), central(fk, 2e-6)
        rk = (4 * d1 - d2) / 3
        v = np.where(L.mirror == 0, np.random.default_rng(7).standard_normal(L.n), 0.0)
        fc = lambda e: ctx.ch_run(c0 + e * v, chi, kappa, M0, dt, nsteps)[1]
        # E moves by ~1e-12 per 1e-6 of c0 along v, near its rounding noise: larger steps, Richardson-combined
        e1, e2 = central(fc, 1e-4), central(fc, 2e-4)
        rc = (4 * e1 - e2) / 3
        ad = float(g @ v)
        res.update(dE_dkappa_central_fd_1e6=d1, dE_dkappa_rel_err_vs_fd_1e6=abs(dk - d1) / abs(d1),
                   dE_dkappa_richardson=rk, dE_dkappa_rel_err_vs_richardson=abs(dk - rk) / abs(rk),
                   dE_dc0_dir=ad, dE_dc0_dir_central_fd_1e4=e1, dE_dc0_dir_rel_err_vs_fd_1e4=abs(ad - e1) / abs(e1),
                   dE_dc0_dir_rel_err_vs_richardson=abs(ad - rc) / abs(rc))
    ctx.close()
    return res


def clouds_generate(px, nclouds=256, nmin=1000, nmax=200000, seed=2024, families=True):
    """Batched-cloud workload: clouds alternate 2D / 3D (half each), node counts log-uniform in [nmin, nmax]
    (seeded), cell-centred lattice of spacing h = 1 mm jittered by U(-0.2h, 0.2h) per coordinate, no ghosts
    (families truncated at the cloud boundary), delta = 3.015h, unit-cell volumes, dx_char = h."""
    rng = np.random.default_rng(seed)
    h = 1e-3
    clouds = []
    for k in range(nclouds):
        dim = 2 if k % 2 == 0 else 3
        target = math.exp(rng.uniform(math.log(nmin), math.log(nmax)))
        if dim == 2:
            nx = max(2, int(round(math.sqrt(target))))
            ny = max(2, int(round(target / nx)))
            g = np.stack(np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij"), -1).reshape(-1, 2)
            xyz = np.zeros((g.shape[0], 3))
            xyz[:, :2] = (g + 0.5) * h
        else:
            m = max(2, int(round(target ** (1.0 / 3.0))))
            g = np.stack(np.meshgrid(np.arange(m), np.arange(m), np.arange(m), indexing="ij"), -1).reshape(-1, 3)
            xyz = (g + 0.5) * h
        xyz[:, :dim] += rng.uniform(-0.2 * h, 0.2 * h, size=(xyz.shape[0], dim))
        delta = 3.015 * h * (1.0 + 1e-6)
        c = dict(dim=dim, coords3=xyz, vols=np.full(xyz.shape[0], h ** dim), delta=delta, dx_char=h)
        if families:  # host families (reference order); the device builds them itself (batch_set_points)
            c["off"], c["ids"] = px.families(xyz, delta, dim == 3)
        clouds.append(c)
    return clouds


def cubic_field(clouds, seed=7):
    """Random cubic polynomial per cloud (N(0,1) coefficients on coordinates scaled to the cloud's extent) and
    its exact order-2 derivatives in the multi-index order of the operators."""
    rng = np.random.default_rng(seed)
    u, exact = [], []
    for c in clouds:
        dim = c["dim"]
        x = c["coords3"][:, :dim]
        L = float(x.max() - x.min())
        xs = x / L
        exps = [e for e in np.ndindex(*(4,) * dim) if sum(e) <= 3]
        coef = rng.standard_normal(len(exps))
        f = np.zeros(x.shape[0])
        for a, e in zip(coef, exps):
            f += a * np.prod(xs ** np.asarray(e), axis=1)
        slots = [(1, 0), (0, 1), (2, 0), (1, 1), (0, 2)] if dim == 2 else \
            [(1, 0, 0), (0, 1, 0), (0, 0, 1), (2, 0, 0), (1, 1, 0), (1, 0, 1), (0, 2, 0), (0, 1, 1), (0, 0, 2)]
        d = np.zeros((x.shape[0], len(slots)))
        for s, q in enumerate(slots):
            for a, e in zip(coef, exps):
                if all(ei >= qi for ei, qi in zip(e, q)):
                    term = np.full(x.shape[0], a)
                    for ax in range(dim):
                        for r in range(q[ax]):
                            term = term * (e[ax] - r)
                        term = term * xs[:, ax] ** (e[ax] - q[ax])
                    d[:, s] += term / L ** sum(q)
        u.append(f)
        exact.append(d)
    return u, exact


def algorithmic_bytes(n, nb, dim, prec):
    """Per step: nb*(4 B id + c*s B operators + 1 B health) + N*(x, u^n, u^{n-1}, u^{n+1}: 4*dim*8 B)."""
    c = 6 if dim == 3 else 3
    s = 4 if prec == "mixed" else 8
    return nb * (4 + c * s + 1) + n * (4 * dim * 8)


# ------------------------------------------------------------------------------------------------- helpers
class ClockSampler:
    """nvidia-smi samples (SM clock, max clock, throttle reasons) while the timed region runs."""

    def __init__(self, index):
        self.index = index
        self.samples = []
        self.proc = None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap,utilization.gpu")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.samples.append(parts)

    def __exit__(self, *exc):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no-samples"], "samples": 0}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in self.samples for k in range(4) if s[4 + k].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def reduce_max(value, ws):
    """Max over ranks (the slowest rank sets the job time)."""
    if ws <= 1:
        return value
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


PROFILE_FILES = {"plate": "epf_step_plate.md", "slab": "epf_step_slab.md"}


def read_traffic(kind, prec, variant=None):
    """DRAM bytes per step-kernel launch from the committed ncu summary of this workload: the line of this precision
    whose "(variant N)" names the schedule the autotuner picked (None until that one is captured)."""
    path = os.path.join(ROOT, "profiles", PROFILE_FILES[kind])
    if not os.path.exists(path):
        return None
    key = "traffic_bytes_per_launch_%s:" % prec
    for line in open(path):
        if line.strip().startswith(key):
            rest = line.split(":", 1)[1].strip()
            if variant is not None and "(variant %d)" % variant not in rest:
                continue
            try:
                return float(rest.split()[0])
            except ValueError:
                return None
    return None


def kernel_name(dim, prec, tuned):
    """The step kernel the autotuner picked (variants 0-2 lane groups, 3-4 CSR tiles, 5 and up TMA-staged)."""
    v, lpn = tuned["variant"], tuned["lanes_per_node"]
    mixed = "true" if prec == "mixed" else "false"
    if v >= 5:
        return "pxb::epf_tma_kernel<%d,%s,LPN=%d,...> (variant %d)" % (dim, mixed, lpn, v)
    if v >= 3:
        return "pxb::epf_stream_kernel<%d,%s,EPF_STEP,...> (variant %d)" % (dim, mixed, v)
    return "pxb::epf_kernel<%d,%s,EPF_STEP,LPN=%d,...> (variant %d)" % (dim, mixed, lpn, v)


def peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"], "measured"
    except Exception:
        return 6650.0, "fallback"


def workload_name(kind, n, nb):
    """The workload name both arms report."""
    if kind == "plate":
        return ("explicit_pddo_frac 2D notched plate 400x200 (%d PD nodes, %d directed bonds), dt=0.8h/c" % (n, nb))
    return ("explicit_pddo_frac 3D notched slab 120x120x24 (+ghosts: %d PD nodes, %d directed bonds), edge notch 20h, "
            "+-2 m/s pins, dt=0.8h/c" % (n, nb))


# --------------------------------------------------------------------------------------------- reference arm
def ref_workload(kind):
    """The same workload built only from the reference's own code (oracle/_ref): its mesh generator,
    createNeighborNodes and crack seeding, ExplicitPDDOFracElement (constants and s_c from G0), and the BC list as
    DirichletBC / NeumannBC entries on its node groups.  Returns None when the harness is not built."""
    from oracle import RefEpf, RefMesh, ref_available
    if not ref_available():
        return None
    if kind == "plate":
        nx, ny, h = 400, 200, 5e-4
        Lx, Ly = nx * h, ny * h
        y1, y2 = 0.05 - 25 * h, 0.05 + 25 * h
        cracks = [[0.0, y1, 50 * h, y1], [0.0, y2, 50 * h, y2]]
        m = RefMesh.structured(2, nx, ny, 0, [0, Lx, 0, Ly], 3.015, 2, cracks=cracks, force_only=True)
        E, nu, rho = 190e9, 0.3, 8000.0
        G0 = 0.01 ** 2 * 12.0 * E * m.delta / (5.0 * math.pi)
        bcs = [dict(kind="neumann", comps=[0, 1], nodes=m.group(g + "nodes_ghost"))
               for g in ("left", "right", "bottom", "top")]
        bcs.append(dict(kind="dirichlet", comps=[0], nodes=m.group("leftnodes_ghost"), value=[0, 0],
                        velocity=[16.5, 0], direct=True, box=[-1, 1, y1, y2, -1, 1]))
    else:
        nx, ny, nz, h = 120, 120, 24, 1e-3
        Lx, Ly, Lz = nx * h, ny * h, nz * h
        plane = [0.0, Ly / 2, -1.0, 20 * h, Ly / 2, -1.0, 20 * h, Ly / 2, 1.0, 0.0, Ly / 2, 1.0]
        m = RefMesh.structured(3, nx, ny, nz, [0, Lx, 0, Ly, 0, Lz], 3.015, 2, planes=[plane], force_only=True)
        E, nu, rho = 72e9, 0.22, 2440.0
        G0 = 0.004 ** 2 * 6.0 * E * m.delta / 5.0
        bcs = [dict(kind="neumann", comps=[0, 1, 2], nodes=m.group(g + "nodes_ghost"))
               for g in ("left", "right", "bottom", "top", "back", "front")]
        alld = m.group("alldomain")
        bcs.append(dict(kind="dirichlet", comps=[1], nodes=alld, value=[0, 0, 0], velocity=[0, 2.0, 0], direct=True,
                        box=[-1, 1, Ly - 3 * h, 1, -1, 1]))
        bcs.append(dict(kind="dirichlet", comps=[1], nodes=alld, value=[0, 0, 0], velocity=[0, -2.0, 0], direct=True,
                        box=[-1, 1, -1, 3 * h, -1, 1]))
    probe = RefEpf(m, E, nu, rho, G0)
    probe.rate(np.zeros(m.dim * m.n), nthreads=1 if m.n < 100000 else 0)  # derives C11 (and s_c) from the element
    dt = 0.8 * h / math.sqrt(probe.constants()["C11"] / rho)
    return dict(kind=kind, m=m, E=E, nu=nu, rho=rho, G0=G0, bcs=bcs, dt=dt, n=m.n, nb=m.nb, dim=m.dim)


def cpu_reference(kind, steps, warmup, threads=None):
    """The reference's own OpenMP CPU path (oracle/_ref, built from the reference sources) on the workload: per step
    the element sweep (damage + force) plus the central difference and the BC preset (reference BC objects).  Only
    the stepping loop is timed: the start's rate call, which on a fresh element also builds its operator cache and
    starts the OpenMP pool, stays outside; on the plate a separate warm-up run of `warmup` steps comes first."""
    from oracle import RefEpf
    r = ref_workload(kind)
    if r is None:
        return None
    m = r["m"]
    threads = threads or os.cpu_count()
    if kind == "plate" and warmup > 0:
        el = RefEpf(m, r["E"], r["nu"], r["rho"], r["G0"], plane_stress=False)
        el.run(np.zeros(m.dim * m.n), None, r["dt"], warmup, r["bcs"], nthreads=threads)
    el = RefEpf(m, r["E"], r["nu"], r["rho"], r["G0"], plane_stress=False)
    _, _, _, t = el.run(np.zeros(m.dim * m.n), None, r["dt"], steps, r["bcs"], nthreads=threads)
    t = max(t, 1e-9)
    return dict(value=m.nb * steps / t, seconds=t, steps=steps, cores=threads, nb=m.nb, n=m.n)


def reference_gpu():
    """The reference's own CUDA explicit path on this GPU (bench.py --profile refgpu, in a child process so that
    its device state and runtime stay apart from this process's)."""
    try:
        r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--profile", "refgpu"], capture_output=True,
                           text=True, timeout=600)
        line = [x for x in r.stdout.splitlines() if x.startswith("{")]
        if r.returncode != 0 or not line:
            return {"unavailable": "reference GPU run failed: " + (r.stderr.strip().splitlines() or ["?"])[-1][:200]}
        d = json.loads(line[-1])
        d.pop("profile", None)
        d["what"] = ("perix_cuda::assembleExplicitPDDOFracAccel from the reference's CudaAssembleKernels.cu built for "
                     "sm_100a: call = H2D u + force kernel + D2H accel per step; force kernel alone with CUDA events, "
                     "L2 flushed; opbuild = its one-off operator build; assembly: perix_cuda::assemble (Poisson) "
                     "with its opsBuildKernel and assembleKernel timed alone beside this backend's g-build and "
                     "assembly on the same mesh")
        return d
    except Exception as e:  # noqa: BLE001
        return {"unavailable": "reference GPU run failed: %s" % e}


def single_cloud(px, dim, nside, seed=11):
    """One cloud of the batched-cloud workload's recipe at a fixed size: nside^dim cell-centred nodes of spacing
    h = 1 mm jittered by U(-0.2h, 0.2h), delta = 3.015h, unit-cell volumes, no ghosts."""
    rng = np.random.default_rng(seed)
    h = 1e-3
    g = np.stack(np.meshgrid(*(np.arange(nside),) * dim, indexing="ij"), -1).reshape(-1, dim)
    xyz = np.zeros((g.shape[0], 3))
    xyz[:, :dim] = (g + 0.5) * h + rng.uniform(-0.2 * h, 0.2 * h, size=(g.shape[0], dim))
    delta = 3.015 * h * (1.0 + 1e-6)
    off, ids = px.families(xyz, delta, dim == 3)
    return dict(dim=dim, coords3=xyz, vols=np.full(g.shape[0], h ** dim), delta=delta, dx_char=h, off=off, ids=ids)


def reference_cpu_gbuild_clouds(px):
    """The reference's own order-2 g-build (PDOperators::buildGeometryCache, OpenMP on all host cores) on the largest
    2D and 3D clouds of the batched-cloud recipe, families from its own createNeighborNodes (oracle/_ref).  The
    same clouds' device g-build is in reference_gpu.assembly."""
    res = {}
    try:
        from oracle import RefMesh, ref_available
        if not ref_available():
            return {"unavailable": "oracle/_ref not built"}
        for name, dim, nside, reps in (("cloud_2d_447x447", 2, 447, 2), ("cloud_3d_58x58x58", 3, 58, 1)):
            c = single_cloud(px, dim, nside)
            h = c["dx_char"]
            m = RefMesh.cloud(dim, c["coords3"], c["vols"], h, h, h if dim == 3 else 0.0, 3.015 * h)
            secs = m.gbuild_time(reps=reps)
            res[name] = {"nodes": int(c["vols"].size), "ms": secs * 1e3, "nodes_per_s": c["vols"].size / secs,
                         "threads": os.cpu_count()}
    except Exception as e:  # noqa: BLE001
        res["unavailable"] = "reference g-build failed: %s" % e
    return res


def assembly_pair(px, c, mirror=None, reps=10):
    """Order-2 g-build + Poisson assembly (sigma = 1, f = 1, u = 0) on one mesh: this backend's g-build and
    assembly kernels (CUDA events, L2 flushed before each g-build) beside the reference's own GPU path on the same
    mesh (oracle/_ref/libperix_ref_cuda.so: opsBuildKernel and assembleKernel with CUDA events, L2 flushed, and the
    whole perix_cuda::assemble call on host buffers).  The two CSR value arrays are compared."""
    import ctypes as C
    import torch
    from oracle import ref_cuda_assemble_bench
    dim, n = c["dim"], c["vols"].size
    rowptr, cols = px.csr_pattern(c["off"], c["ids"], mirror, 1)
    ctx = px.Context(0)
    ctx.set_geometry(c["coords3"].reshape(-1), c["vols"], c["off"], c["ids"], c["delta"], c["dx_char"], dim,
                     mirror=mirror)
    _, gb_ms = gbuild_rate(px, ctx, "fp64", reps=5)
    ctx.gbuild(2, px.FP64)
    ctx.csr_set_pattern(rowptr, cols, 1)
    dev = torch.device("cuda", 0)
    ctx.set_stream(torch.cuda.current_stream(dev).cuda_stream)
    ud = torch.zeros(n, dtype=torch.float64, device=dev)
    kd = torch.empty(int(rowptr[-1]), dtype=torch.float64, device=dev)
    rd = torch.empty(n, dtype=torch.float64, device=dev)

    def assemble():
        st = ctx.L.pxb_assemble_scalar_d(ctx.h, 0, C.c_double(1.0), C.c_double(1.0), None, C.c_double(0.0),
                                         C.c_void_p(ud.data_ptr()), None, C.c_void_p(kd.data_ptr()),
                                         C.c_void_p(rd.data_ptr()))
        if st:
            raise RuntimeError(ctx.L.pxb_last_error().decode())

    for _ in range(3):
        assemble()
    flush = torch.empty(FLUSH_BYTES // 8, dtype=torch.float64, device=dev)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    tot = 0.0
    for r in range(reps):
        flush.fill_(float(r))
        ev[0].record()
        assemble()
        ev[1].record()
        torch.cuda.synchronize(dev)
        tot += ev[0].elapsed_time(ev[1])
    asm_ms = tot / reps
    ours = kd.cpu().numpy()
    ctx.close()
    del flush
    torch.cuda.empty_cache()
    call_ms, ob_ms, ak_ms, kv, _ = ref_cuda_assemble_bench(dim, c["coords3"], c["vols"], c["off"], c["ids"], c["delta"],
                                                           c["dx_char"], rowptr, cols, 1.0, 1.0, np.zeros(n),
                                                           reps=reps, flush_bytes=FLUSH_BYTES)
    scale = float(np.abs(kv).max()) or 1.0
    return {"nodes": n, "bonds": int(c["off"][-1]), "nnz": int(rowptr[-1]), "gbuild_ms": gb_ms, "assembly_ms": asm_ms,
            "ref_call_ms": call_ms, "ref_opsbuild_ms": ob_ms, "ref_assemble_kernel_ms": ak_ms,
            "gbuild_speedup_vs_ref_opsbuild": ob_ms / gb_ms, "assembly_speedup_vs_ref_kernel": ak_ms / asm_ms,
            "kvals_max_rel_diff": float(np.abs(ours - kv).max()) / scale}


REF_MAX_STEPS = 40     # bound on the reference arm's timed steps (about 0.2-0.4 s each on the slab)


def run_reference_arm(args):
    """The reference's own CPU implementation of the path (oracle/_ref) on the headline workload; nothing of this
    backend is loaded.  Rank 0 alone runs it under torchrun."""
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    steps = max(1, min(args.steps, REF_MAX_STEPS))
    r = cpu_reference("slab", steps, min(args.warmup, 3))
    if r is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref (reference sources) not built"}))
        return
    sample = ("%d explicit steps of the 3D slab (element sweep + central difference + BC preset), %d threads"
              % (steps, r["cores"]))
    line = {"impl": "reference", "metric": "bond-updates/s (explicit frac)", "value": r["value"],
            "unit": "bond-updates/s", "n_gpus": ws, "steps": steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * r["seconds"] / steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": workload_name("slab", r["n"], r["nb"]), "nodes": r["n"], "bonds": r["nb"],
                       "threads": r["cores"]},
            "cpu_baseline": {"value": r["value"], "unit": "bond-updates/s", "cores": r["cores"], "kind": "reference",
                             "sample": sample},
            "e2e": {"value": r["value"], "unit": "bond-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


# ------------------------------------------------------------------------------------------------ perix arm
def explicit_context(px, w, prec, device):
    """A context holding the workload's explicit element (FP64 or mixed) with its BC program."""
    ctx = px.Context(device)
    L, dim = w["L"], w["dim"]
    ctx.set_geometry(L.coords, L.vols, w["off"], w["ids"], w["delta"], L.dxyz[0], dim, mirror=L.mirror)
    C11, C12, C66 = w["C"]
    ctx.epf_setup(C11, C12, C66, w["rho"], (0.0,) * dim, w["sc"], True, health0=w["health0"],
                  precision=px.MIXED if prec == "mixed" else px.FP64)
    ctx.epf_set_bcs(w["bcs"])
    return ctx


def measure_precision(px, w, prec, steps, warmup, ws, device):
    ctx = explicit_context(px, w, prec, device)
    ctx.epf_start(np.zeros(w["dim"] * w["n"]), None, w["dt"])
    ctx.epf_advance(S0)
    snap(ctx)
    tuned = autotune(ctx, steps=20 if w["kind"] == "plate" else 5)
    ms = np.zeros(max(warmup, 1), np.float32)
    time_steps(ctx, max(warmup, 1), ms)
    restore(ctx)
    barrier(ws)
    launches0 = ctx.launch_count()
    t_wall = time.perf_counter()
    ms = np.zeros(steps, np.float32)
    time_steps(ctx, steps, ms)
    t_wall = time.perf_counter() - t_wall
    launches = ctx.launch_count() - launches0
    barrier(ws)
    tuned["launch_floor"] = launch_floor(ctx) if tuned["variant"] >= 5 else None
    return ctx, ms, launches, t_wall, tuned


def launch_floor(ctx, reps=20):
    """The fixed cost inside each timed step: an empty kernel with the tuned step kernel's launch shape, after
    the same L2 flush, timed with CUDA events like a step (pxb_epf_launch_floor)."""
    import ctypes as C
    ms = np.zeros(reps, np.float32)
    g, b, sm = C.c_int(0), C.c_int(0), C.c_size_t(0)
    st = ctx.L.pxb_epf_launch_floor(ctx.h, C.c_size_t(FLUSH_BYTES), reps, ms.ctypes.data_as(C.POINTER(C.c_float)),
                                    C.byref(g), C.byref(b), C.byref(sm))
    if st:
        raise RuntimeError(ctx.L.pxb_last_error().decode())
    return {"ms": float(np.mean(ms[1:])), "grid": g.value, "block": b.value, "smem_bytes": sm.value}


def autotune(ctx, steps=20):
    """pxb_epf_autotune: time each schedule variant on this plate from the snapshot state, keep the fastest."""
    import ctypes as C
    best = C.c_int(0)
    ms = np.zeros(ctx.L.pxb_epf_variant_count(), np.float32)
    st = ctx.L.pxb_epf_autotune(ctx.h, steps, C.c_size_t(FLUSH_BYTES), 0, C.byref(best),
                                ms.ctypes.data_as(C.POINTER(C.c_float)))
    if st:
        raise RuntimeError(ctx.L.pxb_last_error().decode())
    lpn = C.c_int(0)
    v = C.c_int(0)
    ctx.L.pxb_epf_get_variant(ctx.h, C.byref(v), C.byref(lpn))
    return {"variant": best.value, "lanes_per_node": lpn.value, "ms_per_variant": [round(float(x), 5) for x in ms]}


def snap(ctx):
    import ctypes as C
    st = ctx.L.pxb_epf_snapshot(ctx.h)
    if st:
        raise RuntimeError(ctx.L.pxb_last_error().decode())


def restore(ctx):
    st = ctx.L.pxb_epf_restore(ctx.h)
    if st:
        raise RuntimeError(ctx.L.pxb_last_error().decode())


def time_steps(ctx, nsteps, ms_out):
    import ctypes as C
    st = ctx.L.pxb_epf_time_steps(ctx.h, int(nsteps), C.c_size_t(FLUSH_BYTES), EPISODE,
                                  ms_out.ctypes.data_as(C.POINTER(C.c_float)))
    if st:
        raise RuntimeError(ctx.L.pxb_last_error().decode())


def gbuild_rate(px, ctx, prec, reps=5):
    import ctypes as C
    p = px.MIXED if prec == "mixed" else px.FP64
    ctx.gbuild(2, p)
    ms = np.zeros(reps, np.float32)
    st = ctx.L.pxb_gbuild_time(ctx.h, 2, p, reps, C.c_size_t(FLUSH_BYTES), ms.ctypes.data_as(C.POINTER(C.c_float)))
    if st:
        raise RuntimeError(ctx.L.pxb_last_error().decode())
    return ctx.n / (float(np.mean(ms)) * 1e-3), float(np.mean(ms))


def e2e_rate(px, ctx, w, steps):
    """The drop-in per-step call (reference assembleExplicitPDDOFracAccel semantics): pinned host u in,
    pinned host acceleration out, every step.  After one second of untimed calls, five timed batches of steps/5
    calls; the median batch rate (the host's wait on each call varies with the load of the shared machine, the
    device work does not)."""
    import torch
    n2 = w["dim"] * w["n"]
    u_h = torch.empty(n2, dtype=torch.float64, pin_memory=True)
    a_h = torch.empty(n2, dtype=torch.float64, pin_memory=True)
    u, _, _, _ = ctx.epf_state()
    u_h.copy_(torch.from_numpy(u))
    import ctypes as C
    nbk = C.c_longlong(0)
    up = C.cast(C.c_void_p(u_h.data_ptr()), C.POINTER(C.c_double))
    ap = C.cast(C.c_void_p(a_h.data_ptr()), C.POINTER(C.c_double))
    # untimed warm-up of at least one second of calls: after the device idled, calls start up to 1.6x slower and
    # speed up over the first ~0.3 s of back-to-back calls (the GPU is mostly waiting on PCIe meanwhile)
    t_w = time.perf_counter()
    k = 0
    while k < 50 or time.perf_counter() - t_w < 1.0:
        ctx.L.pxb_epf_rate(ctx.h, up, ap, C.byref(nbk))
        k += 1
    per = max(2, steps // 5)
    rates = []
    for _ in range(5):
        t = time.perf_counter()
        for _ in range(per):
            st = ctx.L.pxb_epf_rate(ctx.h, up, ap, C.byref(nbk))
            if st:
                raise RuntimeError(ctx.L.pxb_last_error().decode())
        rates.append(w["nb"] * per / (time.perf_counter() - t))
    return float(np.median(rates)), n2 * 8, n2 * 8 + 16


def pageable_call_us(ctx, w, calls=50):
    """Median time of the per-step call made with pageable host arrays (numpy), as the reference element passes
    its std::vector data: the copies go through the driver's staging buffers and no graph is used."""
    import ctypes as C
    u, _, _, _ = ctx.epf_state()
    u = np.ascontiguousarray(u, np.float64)
    a = np.zeros_like(u)
    nbk = C.c_longlong(0)
    up, ap = u.ctypes.data_as(C.POINTER(C.c_double)), a.ctypes.data_as(C.POINTER(C.c_double))
    ts = []
    for k in range(calls + 10):
        t = time.perf_counter()
        st = ctx.L.pxb_epf_rate(ctx.h, up, ap, C.byref(nbk))
        if st:
            raise RuntimeError(ctx.L.pxb_last_error().decode())
        if k >= 10:
            ts.append(time.perf_counter() - t)
    return float(np.median(ts)) * 1e6


def pcie_copy_us(nbytes, device, reps=20):
    """Device time (CUDA events, median of reps) of one pinned host->device and one device->host copy of nbytes:
    the transfers inside each per-step call, measured alone on this machine's link."""
    import torch
    dev = torch.device("cuda", device)
    h = torch.empty(nbytes // 8, dtype=torch.float64, pin_memory=True)
    d = torch.empty(nbytes // 8, dtype=torch.float64, device=dev)
    out = {}
    for name, dst, src in (("h2d", d, h), ("d2h", h, d)):
        ts = []
        for _ in range(reps + 3):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            dst.copy_(src, non_blocking=True)
            b.record()
            torch.cuda.synchronize(dev)
            ts.append(a.elapsed_time(b) * 1e3)
        out[name] = float(np.median(ts[3:]))
    return out


def shim_call_us(px, w, calls=30):
    """Median time of the reference boundary's own drop-in call, perix_cuda::assembleExplicitPDDOFracAccel (through
    its C entry pxb_cuda_explicit_accel), made as the reference element makes it: pageable host arrays (numpy, the
    element's std::vector data), 1-based families, double health in/out.  The shim's first call of the problem
    uploads the mesh, builds the operators and times its schedules; the timed calls are the per-step calls that
    follow, at the displacement of the state after 100 steps.  Returns (us per call, calls whose health changed)."""
    import ctypes as C
    L, dim = w["L"], w["dim"]
    ctx = explicit_context(px, w, "fp64", 0)
    ctx.epf_start(np.zeros(dim * w["n"]), None, w["dt"])
    ctx.epf_advance(S0)
    u, _, h8, _ = ctx.epf_state()
    ctx.close()
    lib = px.lib()
    f64 = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))  # noqa: E731
    i32 = lambda a: a.ctypes.data_as(C.POINTER(C.c_int))  # noqa: E731
    off = np.ascontiguousarray(w["off"], np.int32)
    ids = np.ascontiguousarray(w["ids"], np.int32)
    coords = np.ascontiguousarray(L.coords, np.float64)
    vols = np.ascontiguousarray(L.vols, np.float64)
    u = np.ascontiguousarray(u, np.float64)
    health = h8.astype(np.float64)
    acc = np.zeros_like(u)
    body = np.zeros(3)
    changed = C.c_int(0)
    C11, C12, C66 = w["C"]
    args = (w["n"], dim, i32(off), i32(ids), f64(coords), f64(vols), C.c_double(w["delta"]), C.c_double(L.dxyz[0]),
            C.c_double(C11), C.c_double(C12), C.c_double(C66), C.c_double(w["rho"]), f64(body), C.c_double(w["sc"]),
            1, 1, f64(u), f64(health), f64(acc), C.byref(changed))
    lib.pxb_cuda_shutdown()
    ts, nchanged = [], 0
    for k in range(calls + 5):
        t = time.perf_counter()
        if lib.pxb_cuda_explicit_accel(*args) != 1:
            raise RuntimeError("pxb_cuda_explicit_accel failed: " + lib.pxb_last_error().decode())
        if k >= 5:
            ts.append(time.perf_counter() - t)
            nchanged += int(changed.value)
    lib.pxb_cuda_shutdown()
    return float(np.median(ts)) * 1e6, nchanged


def mixed_error(px, w, device):
    """max|u_mixed - u_fp64| / max|u_fp64| after 100 graph-captured steps from the same 100-step state, and the
    number of bonds whose health differs."""
    res = {}
    for prec in ("fp64", "mixed"):
        ctx = explicit_context(px, w, prec, device)
        ctx.epf_start(np.zeros(w["dim"] * w["n"]), None, w["dt"])
        ctx.epf_advance(2 * S0)
        res[prec] = ctx.epf_state()
        ctx.close()
    u64, u32 = res["fp64"][0], res["mixed"][0]
    return float(np.abs(u32 - u64).max() / np.abs(u64).max()), int((res["fp64"][2] != res["mixed"][2]).sum())


def explicit_workload(px, w, steps, warmup, ws, local, e2e_calls):
    """Both precisions of one explicit workload: CUDA-event step times (L2 flushed), the L2-warm 100-step graph
    chunk, the g-build rate, and for the headline precision (mixed when within 1e-6 of FP64 after 100 steps) the
    roofline and the per-step calls from host memory.  Returns the JSON block and the headline's timed launches."""
    hbm, peak_kind = peaks()
    out = {}
    for prec in ("fp64", "mixed"):
        with ClockSampler(local) as clk:
            ctx, ms, launches, wall, tuned = measure_precision(px, w, prec, steps, warmup, ws, local)
        t = reduce_max(float(ms.sum()) * 1e-3, ws)
        # graph-captured chunk from the snapshot (L2-warm, the production loop); the first advance captures and
        # instantiates the graph for the tuned variant, the next five are timed
        restore(ctx)
        ctx.epf_advance(EPISODE, chunk=EPISODE)
        chunks = []
        for _ in range(5):
            restore(ctx)
            t0 = time.perf_counter()
            ctx.epf_advance(EPISODE, chunk=EPISODE)
            chunks.append(time.perf_counter() - t0)
        steady = w["nb"] * EPISODE / float(np.median(chunks))
        gb, gb_ms = gbuild_rate(px, ctx, prec, reps=3)
        out[prec] = dict(ctx=ctx, ms=ms, t=t, launches=launches, wall=wall, clocks=clk.summary(), steady=steady,
                         gbuild=gb, gbuild_ms=gb_ms, tuned=tuned)
    err, hdiff = mixed_error(px, w, local)
    head = "mixed" if err <= 1e-6 else "fp64"
    r = out[head]
    mean_s = float(np.mean(r["ms"])) * 1e-3
    B = algorithmic_bytes(w["n"], w["nb"], w["dim"], head)
    achieved = B / mean_s / 1e9
    e2e, h2d, d2h = e2e_rate(px, r["ctx"], w, e2e_calls)
    copies = pcie_copy_us(h2d, local)
    pageable_us = pageable_call_us(r["ctx"], w)
    for p in out.values():
        p["ctx"].close()
    shim_us, shim_changed = shim_call_us(px, w)
    block = {
        "value": ws * w["nb"] * steps / r["t"],
        "ms_per_step": 1e3 * r["t"] / steps,
        "precision": head,
        "dtype": "mixed(f32-storage,f64-arith)" if head == "mixed" else "f64",
        "nodes": w["n"], "bonds": w["nb"],
        "workload": workload_name(w["kind"], w["n"], w["nb"]),
        "e2e": {"value": ws * e2e, "unit": "bond-updates/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "call_us": 1e6 * w["nb"] / e2e,
                "call_us_pageable_buffers": pageable_us,
                "drop_in_call_us": shim_us,
                "drop_in_calls_with_health_changed": shim_changed,
                "pcie_copy_us": {"h2d": copies["h2d"], "d2h": copies["d2h"],
                                 "note": "one pinned copy of the call's u (h2d) or acceleration (d2h) bytes alone, "
                                         "CUDA events, median of 20: the link speed this machine gave"},
                "api": "pxb_epf_rate (per-step call, pinned host u in / acceleration out, headline precision); "
                       "drop_in_call_us: perix_cuda::assembleExplicitPDDOFracAccel via pxb_cuda_explicit_accel with "
                       "pageable arrays and double health in/out (FP64, the shim's default)"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "traffic": read_traffic(w["kind"], head, r["tuned"]["variant"]), "peak_kind": peak_kind,
                     "algorithmic_bytes_per_launch": B, "kernel": kernel_name(w["dim"], head, r["tuned"]),
                     "launch_floor_ms": (r["tuned"]["launch_floor"] or {}).get("ms"),
                     "note": "achieved = algorithmic bytes / CUDA-event step time; launch_floor_ms is an empty "
                             "kernel of the same launch shape timed the same way (flush, events)"},
        "gpu_launches": int(r["launches"]),
        "clocks": {k: r["clocks"][k] for k in ("sm_mhz", "sm_max_mhz", "reasons")},
        "fp64": {"value": ws * w["nb"] * steps / out["fp64"]["t"], "ms_per_step": 1e3 * out["fp64"]["t"] / steps,
                 "frac_of_measured_hbm": algorithmic_bytes(w["n"], w["nb"], w["dim"], "fp64") /
                 (float(np.mean(out["fp64"]["ms"])) * 1e-3) / 1e9 / hbm,
                 "autotune": out["fp64"]["tuned"]},
        "mixed": {"value": ws * w["nb"] * steps / out["mixed"]["t"], "ms_per_step": 1e3 * out["mixed"]["t"] / steps,
                  "frac_of_measured_hbm": algorithmic_bytes(w["n"], w["nb"], w["dim"], "mixed") /
                  (float(np.mean(out["mixed"]["ms"])) * 1e-3) / 1e9 / hbm,
                  "rel_err_vs_fp64_after_100_steps": err, "health_differs": hdiff, "autotune": out["mixed"]["tuned"]},
        "mixed_over_fp64": out["fp64"]["t"] / out["mixed"]["t"],
        "steady_state_graph": {"fp64": out["fp64"]["steady"], "mixed": out["mixed"]["steady"],
                               "note": "100-step CUDA-graph chunk, L2-warm (wall clock incl. host sync, median of 5 chunks)"},
        "gbuild_nodes_per_s": {"fp64": out["fp64"]["gbuild"], "mixed": out["mixed"]["gbuild"],
                               "ms": {"fp64": out["fp64"]["gbuild_ms"], "mixed": out["mixed"]["gbuild_ms"]},
                               "workload": "order-2 g-build of the same mesh (all operators stored)"},
    }
    return block


def run_perix(args):
    ws, rank, local = dist_env()
    if ws > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    import perix_b200 as px
    steps = args.steps
    slab = explicit_workload(px, slab_setup(px), steps, args.warmup, ws, local, max(10, min(steps, 100)))
    plate = None
    cpu = None
    clouds = refgpu = poisson = ch = adjoint = None
    if rank == 0 and ws == 1:
        cpu = cpu_reference("slab", 10, 2)
        if not args.headline_only:
            plate = explicit_workload(px, plate_setup(px), steps, args.warmup, ws, local, max(10, min(steps, 200)))
            plate["cpu_baseline"] = cpu_reference("plate", 20, 2)
            clouds = clouds_measure(px, device=local)
            clouds["reference_cpu_gbuild"] = reference_cpu_gbuild_clouds(px)
            adjoint = slab_adjoint(px, device=local)
            refgpu = reference_gpu()
            poisson = poisson_measure(px, device=local)
            ch = ch_measure(px, device=local)
    if rank != 0:
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    line = {
        "metric": "bond-updates/s (explicit frac)",
        "value": slab["value"],
        "unit": "bond-updates/s",
        "n_gpus": ws,
        "steps": steps,
        "warmup": args.warmup,
        "ms_per_step": slab["ms_per_step"],
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": slab["dtype"],
        "precision": slab["precision"] + (" (f32 Navier-coefficient storage; f64 arithmetic, state and stretch "
                                          "decisions)" if slab["precision"] == "mixed" else ""),
        "data": "synthetic",
        "config": {"workload": slab["workload"], "nodes": slab["nodes"], "bonds": slab["bonds"],
                   "parallelism": "replicas" if ws > 1 else "single-gpu",
                   "l2": "flushed before every timed step (256 MiB write, then the same 256 MiB read back); the "
                         "step's bond streams exceed the 126 MB L2",
                   "state": "snapshot after %d steps, restored every %d steps" % (S0, EPISODE)},
        "e2e": slab["e2e"],
        "roofline": slab["roofline"],
        "cpu_baseline": ({"value": cpu["value"], "unit": "bond-updates/s", "cores": cpu["cores"], "kind": "reference",
                          "sample": "10 explicit steps of the same slab through the reference's OpenMP CPU path "
                                    "(element sweep + central difference + BC preset)"} if cpu else None),
        "gpu_launches": slab["gpu_launches"],
        "clocks": slab["clocks"],
        "fp64": slab["fp64"],
        "mixed": slab["mixed"],
        "mixed_over_fp64": slab["mixed_over_fp64"],
        "steady_state_graph": slab["steady_state_graph"],
        "gbuild_nodes_per_s": slab["gbuild_nodes_per_s"],
        "slab_adjoint": adjoint,
        "plate_2d": plate,
        "batched_clouds": clouds,
        "reference_gpu": refgpu,
        "poisson_64x64": poisson,
        "cahn_hilliard_256x256": ch,
    }
    print(json.dumps(line))
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def clouds_measure(px, nclouds=256, reps=3, device=0):
    """Batched clouds: one context holds every cloud; the g-build (FP64, then mixed) and the all-derivative apply
    are autotuned over their schedules and timed with CUDA events (L2 flushed before each launch).  Errors: the
    mixed g-functions and derivatives against the FP64 ones, and the FP64 derivatives of the random cubics
    against the exact ones (order-2 truncation error, reported, not a precision claim)."""
    import torch
    t0 = time.perf_counter()
    clouds = clouds_generate(px, nclouds=nclouds, families=False)
    fields, exact = cubic_field(clouds)
    t_setup = time.perf_counter() - t0
    ctx = px.Context(device)
    t0 = time.perf_counter()
    ctx.batch_set_points(clouds)  # families of every cloud built on the device
    t_fam = time.perf_counter() - t0
    dev = torch.device("cuda", device)
    ctx.set_stream(torch.cuda.current_stream(dev).cuda_stream)
    u = torch.from_numpy(np.concatenate(fields)).to(dev)
    out = torch.empty(ctx.batch_out_len, dtype=torch.float64, device=dev)
    res = {"clouds": nclouds, "nodes": ctx.batch_n, "bonds": ctx.batch_nb,
           "dims": {"2d": sum(1 for c in clouds if c["dim"] == 2), "3d": sum(1 for c in clouds if c["dim"] == 3)},
           "host_setup_s": t_setup, "batch_set_points_s": t_fam}
    derivs = {}
    for prec, p in (("fp64", px.FP64), ("mixed", px.MIXED)):
        ctx.batch_gbuild(p)
        gbest, gms = ctx.batch_autotune(0, reps=reps, flush_bytes=FLUSH_BYTES)
        ctx.batch_gbuild(p)
        abest, ams = ctx.batch_autotune(1, reps=reps, flush_bytes=FLUSH_BYTES, u_ptr=u.data_ptr(), out_ptr=out.data_ptr())
        ctx.batch_apply_d(u.data_ptr(), out.data_ptr())
        torch.cuda.synchronize(dev)
        derivs[prec] = out.cpu().numpy()
        g_ms, a_ms = float(gms[gbest]), float(ams[abest])
        s_b = 4 if prec == "mixed" else 8
        # apply bytes per launch: nb*(4 B id + nop*s B g) + N*(8 B u + 8*nop B out) per cloud (u_j gathers: L2);
        # mixed adds the per-node FP32 first-moment defects of the second-derivative operators
        a_bytes = sum(ctx.batch_bond_counts[k] * (4 + (9 if c["dim"] == 3 else 5) * s_b) +
                      c["vols"].size * (8 + 8 * (9 if c["dim"] == 3 else 5)) +
                      (c["vols"].size * (18 if c["dim"] == 3 else 6) * 4 if prec == "mixed" else 0)
                      for k, c in enumerate(clouds))
        hbm, _ = peaks()
        res[prec] = {"gbuild_nodes_per_s": ctx.batch_n / (g_ms * 1e-3), "gbuild_ms": g_ms, "gbuild_schedule": gbest,
                     "gbuild_ms_per_schedule": [round(float(x), 4) for x in gms],
                     "apply_ms": a_ms, "apply_schedule": abest, "apply_algorithmic_bytes": a_bytes,
                     "apply_achieved_gbs": a_bytes / (a_ms * 1e-3) / 1e9,
                     "apply_frac_of_measured_hbm": a_bytes / (a_ms * 1e-3) / 1e9 / hbm,
                     "apply_ms_per_schedule": [round(float(x), 4) for x in ams]}
    d64 = ctx.batch_split(derivs["fp64"])
    d32 = ctx.batch_split(derivs["mixed"])
    trunc = {"2d": [0.0, 0.0], "3d": [0.0, 0.0]}
    # mixed vs FP64, first / second derivatives: max |error| over the cloud relative to (a) the same slot's max
    # |value| over the cloud, (b) the max over the slots of that order (gradient / Hessian magnitude), (c) L2
    errs = {"per_slot": [0.0, 0.0], "per_order": [0.0, 0.0], "l2": [0.0, 0.0]}
    worst = None
    for k, c in enumerate(clouds):
        dim = c["dim"]
        diff = np.abs(d32[k] - d64[k])
        for o, sl in enumerate((slice(0, dim), slice(dim, None))):
            a, b = diff[:, sl], np.abs(d64[k][:, sl])
            ps = float((a.max(axis=0) / b.max(axis=0)).max())
            po = float(a.max() / b.max())
            l2 = float(np.sqrt((a ** 2).sum() / (b ** 2).sum()))
            if o == 0 and (worst is None or ps > worst[0]):
                worst = (ps, k, dim, int(c["vols"].size))
            for key, v in (("per_slot", ps), ("per_order", po), ("l2", l2)):
                errs[key][o] = max(errs[key][o], v)
    for k, c in enumerate(clouds):
        dim = c["dim"]
        esc = np.abs(exact[k]).max(axis=0)
        e = np.abs(d64[k] - exact[k]).max(axis=0) / esc
        key = "%dd" % dim
        trunc[key][0] = max(trunc[key][0], float(e[:dim].max()))
        trunc[key][1] = max(trunc[key][1], float(e[dim:].max()))
    res["mixed_rel_err_vs_fp64"] = {key: {"first": v[0], "second": v[1]} for key, v in errs.items()}
    res["mixed_rel_err_vs_fp64"]["worst_first_per_slot_cloud"] = {"cloud": worst[1], "dim": worst[2], "nodes": worst[3]}
    res["truncation_err_vs_exact_cubics"] = {k: {"first": v[0], "second": v[1]} for k, v in trunc.items()}
    ctx.close()
    return res


def run_profile(args):
    """One kernel family on the plate, for profiler captures.  --profile step: the plate runs 100 steps with
    variant 1, then --steps timed steps of variant --variant from that state (so that variant's step kernel is
    the only kernel of its name launched); --profile gbuild: --steps order-2 g-builds."""
    import perix_b200 as px
    w = plate_setup(px)
    ctx = px.Context(0)
    L = w["L"]
    ctx.set_geometry(L.coords, L.vols, w["off"], w["ids"], w["delta"], L.dxyz[0], 2, mirror=L.mirror)
    if args.profile == "slab":
        print(json.dumps({"profile": "slab", **slab_adjoint(px)}))
        ctx.close()
        return
    if args.profile == "ch":
        ctx.close()
        print(json.dumps({"profile": "ch", **ch_measure(px, nsteps=args.steps)}))
        return
    if args.profile == "refgpu":
        # the reference's own GPU explicit path (oracle/_ref/libperix_ref_cuda.so) on the plate and the slab,
        # from the state after 100 steps; run in a child process of the main bench
        from oracle import ref_cuda_available, ref_cuda_epf_bench
        ctx.close()
        # the reference keeps its operator cache at nop 5 (2D implicit) only when PERIX_CUDA_OPCACHE=1; it reads
        # the variable once, at its first call (this is a child process of the main bench)
        os.environ["PERIX_CUDA_OPCACHE"] = "1"
        if not ref_cuda_available():
            print(json.dumps({"profile": "refgpu", "unavailable": "oracle/_ref/libperix_ref_cuda.so not built"}))
            return
        res = {"profile": "refgpu"}
        for name, setup, dim in (("plate_2d", plate_setup, 2), ("slab_3d", slab_setup, 3)):
            wv = setup(px)
            Lv = wv["L"]
            c = px.Context(0)
            c.set_geometry(Lv.coords, Lv.vols, wv["off"], wv["ids"], wv["delta"], Lv.dxyz[0], dim, mirror=Lv.mirror)
            C11, C12, C66 = wv["C"]
            c.epf_setup(C11, C12, C66, wv["rho"], (0.0,) * dim, wv["sc"], True, health0=wv["health0"])
            c.epf_set_bcs(wv["bcs"])
            c.epf_start(np.zeros(dim * Lv.n), None, wv["dt"])
            c.epf_advance(S0)
            u, _, hh, _ = c.epf_state()
            c.close()
            call_ms, kern_ms, ob_ms, _ = ref_cuda_epf_bench(dim, Lv.coords, Lv.vols, wv["off"], wv["ids"], wv["delta"],
                                                            Lv.dxyz[0], wv["C"], wv["rho"], wv["sc"], u,
                                                            hh.astype(np.float64), reps=20, flush_bytes=FLUSH_BYTES)
            res[name] = {"nodes": Lv.n, "bonds": wv["nb"], "call_ms": call_ms, "force_kernel_ms": kern_ms,
                         "opbuild_ms": ob_ms, "force_kernel_bond_updates_per_s": wv["nb"] / (kern_ms * 1e-3),
                         "call_bond_updates_per_s": wv["nb"] / (call_ms * 1e-3)}
        # the implicit path: order-2 g-build + Poisson assembly on the 64x64 Poisson lattice and on the largest 2D
        # and 3D clouds of the batched-cloud workload
        L = px.lattice(2, 64, 64, 0, [0.0, 1.0, 0.0, 1.0])
        delta = 3.015 * L.dxyz[0] * (1.0 + 1e-6)
        off, ids = px.families(L.coords, delta, False, mirror=L.mirror)
        asm = {"poisson_64x64": assembly_pair(px, dict(dim=2, coords3=L.coords, vols=L.vols, delta=delta,
                                                       dx_char=L.dxyz[0], off=off, ids=ids), mirror=L.mirror)}
        asm["cloud_2d_447x447"] = assembly_pair(px, single_cloud(px, 2, 447))
        asm["cloud_3d_58x58x58"] = assembly_pair(px, single_cloud(px, 3, 58))
        res["assembly"] = asm
        print(json.dumps(res))
        return
    if args.profile == "slabadjoint":
        # the slab at --size x --size x 24: a recorded frozen-mask forward of --steps steps with every state kept,
        # then its reverse sweep (the adjoint kernels a capture looks at), with adjoint schedule --variant (-1: default)
        import ctypes as C
        import torch
        ctx.close()
        ws = slab_setup(px, nx=args.size, ny=args.size)
        Ls = ws["L"]
        dev = torch.device("cuda", 0)
        c = px.Context(0)
        c.set_geometry(Ls.coords, Ls.vols, ws["off"], ws["ids"], ws["delta"], Ls.dxyz[0], 3, mirror=Ls.mirror)
        k3 = px.elastic_constants(3, False, ws["E"], ws["nu"])
        c.epf_setup(k3[0], k3[1], k3[2], ws["rho"], (0.0, 0.0, 0.0), 0.0, True, health0=ws["health0"])
        c.epf_set_bcs(ws["bcs"])
        c.epf_set_adjoint_schedule(args.variant if 0 <= args.variant <= 4 else -1)  # (the default 8: -1)
        c.set_stream(torch.cuda.current_stream(dev).cuda_stream)
        rng = np.random.default_rng(3)
        u0 = torch.tensor(rng.standard_normal(3 * Ls.n) * 1e-6, device=dev)
        gN = torch.tensor(rng.standard_normal(3 * Ls.n), device=dev)
        u0b, v0b = torch.empty_like(u0), torch.empty_like(u0)
        dC = torch.zeros(3, dtype=torch.float64, device=dev)
        p = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
        if c.L.pxb_epf_record_d(c.h, p(u0), None, C.c_double(ws["dt"]), args.steps, 0, None, None):
            raise RuntimeError(c.L.pxb_last_error().decode())
        t0 = time.perf_counter()
        if c.L.pxb_epf_adjoint_recorded_d(c.h, p(gN), None, p(u0b), p(v0b), p(dC)):
            raise RuntimeError(c.L.pxb_last_error().decode())
        torch.cuda.synchronize(dev)
        print(json.dumps({"profile": "slabadjoint", "size": args.size, "nodes": Ls.n, "bonds": ws["nb"],
                          "steps": args.steps, "sweep_s": time.perf_counter() - t0, "dC": dC.tolist()}))
        c.close()
        return
    if args.profile == "slabstep":
        # the 3D slab at --size x --size x 24: 100 steps of variant 1, then --steps timed steps of --variant
        ctx.close()
        w5 = slab_setup(px, nx=args.size, ny=args.size, nz=24)
        L5 = w5["L"]
        ctx = px.Context(0)
        ctx.set_geometry(L5.coords, L5.vols, w5["off"], w5["ids"], w5["delta"], L5.dxyz[0], 3, mirror=L5.mirror)
        C11, C12, C66 = w5["C"]
        ctx.epf_setup(C11, C12, C66, w5["rho"], (0.0, 0.0, 0.0), w5["sc"], True, health0=w5["health0"],
                      precision=px.MIXED if args.precision == "mixed" else px.FP64)
        ctx.epf_set_bcs(w5["bcs"])
        ctx.epf_start(np.zeros(3 * L5.n), None, w5["dt"])
        ctx.epf_set_variant(1)
        ctx.epf_advance(S0)
        snap(ctx)
        ctx.epf_set_variant(args.variant)
        ms = np.zeros(args.steps, np.float32)
        time_steps(ctx, args.steps, ms)
        print(json.dumps({"profile": "slabstep", "size": args.size, "nodes": L5.n, "bonds": w5["nb"],
                          "precision": args.precision, "variant": args.variant, "ms_per_step": float(np.mean(ms[1:] if
                          ms.size > 1 else ms))}))
        ctx.close()
        return
    if args.profile == "cloudsapply":
        # --steps clouds (log-uniform 1k..200k nodes), one FP64 or mixed g-build, then 3 applies of schedule --variant
        ctx.close()
        import torch
        clouds = clouds_generate(px, nclouds=args.steps, families=False)
        fields, _ = cubic_field(clouds)
        ctx = px.Context(0)
        ctx.batch_set_points(clouds)
        dev = torch.device("cuda", 0)
        ctx.set_stream(torch.cuda.current_stream(dev).cuda_stream)
        ctx.batch_gbuild(px.MIXED if args.precision == "mixed" else px.FP64)
        ctx.batch_set_variant(1, args.variant)
        u = torch.from_numpy(np.concatenate(fields)).to(dev)
        out = torch.empty(ctx.batch_out_len, dtype=torch.float64, device=dev)
        ms = ctx.batch_time(1, 3, FLUSH_BYTES, u.data_ptr(), out.data_ptr())
        print(json.dumps({"profile": "cloudsapply", "clouds": args.steps, "nodes": ctx.batch_n, "bonds": ctx.batch_nb,
                          "precision": args.precision, "schedule": args.variant, "ms": [float(x) for x in ms]}))
        ctx.close()
        return
    if args.profile == "cloudsgbuild":
        # --steps clouds (log-uniform 1k..200k nodes), then 3 FP64 or mixed order-2 g-builds with schedule --variant
        ctx.close()
        import torch
        clouds = clouds_generate(px, nclouds=args.steps, families=False)
        ctx = px.Context(0)
        ctx.batch_set_points(clouds)
        dev = torch.device("cuda", 0)
        ctx.set_stream(torch.cuda.current_stream(dev).cuda_stream)
        ctx.batch_set_variant(0, args.variant)
        prec = px.MIXED if args.precision == "mixed" else px.FP64
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        ms = []
        for _ in range(3):
            ev[0].record()
            ctx.batch_gbuild(prec)
            ev[1].record()
            torch.cuda.synchronize(dev)
            ms.append(ev[0].elapsed_time(ev[1]))
        print(json.dumps({"profile": "cloudsgbuild", "clouds": args.steps, "nodes": ctx.batch_n, "bonds": ctx.batch_nb,
                          "precision": args.precision, "schedule": args.variant, "ms": ms}))
        ctx.close()
        return
    if args.profile == "clouds":
        print(json.dumps({"profile": "clouds", **clouds_measure(px, nclouds=args.steps)}))
        ctx.close()
        return
    if args.profile == "gbuild":
        gb, ms = gbuild_rate(px, ctx, args.precision, reps=args.steps)
        print(json.dumps({"profile": "gbuild", "precision": args.precision, "nodes_per_s": gb, "ms": ms}))
        ctx.close()
        return
    C11, C12, C66 = w["C"]
    p = px.MIXED if args.precision == "mixed" else px.FP64
    ctx.epf_setup(C11, C12, C66, w["rho"], (0.0, 0.0), w["sc"], True, health0=w["health0"], precision=p)
    ctx.epf_set_bcs(w["bcs"])
    ctx.epf_start(np.zeros(2 * L.n), None, w["dt"])
    ctx.epf_set_variant(1)
    ctx.epf_advance(S0)
    snap(ctx)
    ctx.epf_set_variant(args.variant)
    ms = np.zeros(args.steps, np.float32)
    time_steps(ctx, args.steps, ms)
    print(json.dumps({"profile": "step", "precision": args.precision, "variant": args.variant,
                      "ms_per_step": float(np.mean(ms)), "bond_updates_per_s": w["nb"] / (float(np.mean(ms)) * 1e-3)}))
    ctx.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="perix", choices=["perix", "reference"])
    ap.add_argument("--profile", choices=["step", "gbuild", "clouds", "slab", "slabstep", "slabadjoint", "cloudsapply", "cloudsgbuild", "refgpu", "ch"], default=None,
                    help="run one kernel family only (for profiler captures); prints its own JSON line")
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="mixed")
    ap.add_argument("--variant", type=int, default=8)
    ap.add_argument("--size", type=int, default=120, help="--profile c5step: slab of size x size x 24 nodes")
    ap.add_argument("--headline-only", action="store_true",
                    help="the slab step line alone (no plate, batched-cloud, adjoint, reference-GPU, Poisson and CH keys)")
    args = ap.parse_args()
    if args.profile:
        run_profile(args)
    elif args.impl == "reference":
        run_reference_arm(args)
    else:
        run_perix(args)


if __name__ == "__main__":
    main()
