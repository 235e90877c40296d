#!/usr/bin/env python
"""Headline benchmark: plain FP64 compressible Navier-Stokes RHS + RK stage update
on a 256^3 periodic Taylor-Green box (Mach 0.1, Re 1600, gamma 1.4, Pr 0.71,
1e-4 seeded density noise, CFL 0.5 with dt recomputed on the device every step).

A step is one RK step = 4 RK stages over the whole box.  Throughput is
grid-point RK-stage updates per second (Mpts*RK-stages/s), whole job.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Timed regions (all on the device with CUDA events, barrier + synchronize on
both sides, max over ranks):
  value     K graph-replayed steps on a device-resident state;
  roofline  K eager steps with CUDA events around every pass (same workload);
  e2e       K steps through cs_solver_step_host: pinned host state -> device,
            step, device -> host, every step.
The state (5 x 134 MB) and the gradient scratch (12 x 134 MB) are far larger
than the 126 MB L2, so no flush is needed between steps.
With --gpus N > 1 every rank advances its own independent 256^3 box (replicas,
weak scaling; the only collective is the timing max).
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mpts*RK-stages/s at 256^3: mixed vs plain FP64 at <=1e-6 rel err; adjoint/fwd time"
UNIT = "Mpts*RK-stages/s"
MACH, RE, CFL = 0.1, 1600.0, 0.5
# Algorithmic bytes per grid point per launch of each pass (FP64, constant
# metrics): gradient pass reads q (5) and writes 4 gradients; flux x reads q
# and 12 gradients and writes R; flux y also reads R; flux z + RK reads q,
# 12 gradients, R and q^n and writes q (stage 0: q^n is the stage input).
ALG_BYTES = {"grad_x": 72, "grad_y": 72, "grad_z": 72, "flux_x": 176, "flux_y": 216,
             "flux_z_rk": 8 * (5 + 12 + 5 + 5 + 5)}
STAGE_BYTES = 864  # sum of the passes above per point per stage


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=60)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--n", type=int, default=256)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-mixed", action="store_true")
    p.add_argument("--no-ensemble", action="store_true")
    p.add_argument("--no-adjoint", action="store_true")
    p.add_argument("--no-curvilinear", action="store_true")
    p.add_argument("--no-reference-kernels", action="store_true")
    p.add_argument("--no-config1", action="store_true")
    p.add_argument("--no-dropin", action="store_true")
    p.add_argument("--no-filter", action="store_true")
    p.add_argument("--schedule", default="auto", choices=["auto", "tma", "onephase"],
                   help="auto: the autotuner picks each pass's schedule (default); tma / onephase: fixed, no "
                        "autotuning (used for ncu launch lists, where the autotuner's own timings are distorted)")
    return p.parse_args()


FIELDS = ["rho", "rho_u", "rho_v", "rho_w", "rho_E"]


def state_errors(q, qref, lmx):
    """Per-field error of a state against a reference state: relative to each
    field's maximum, and for the momenta also relative to the largest momentum."""
    errs, errs_m = {}, {}
    mmax = max(float(qref[i * lmx:(i + 1) * lmx].abs().max()) for i in (1, 2, 3))
    for i, name in enumerate(FIELDS):
        a, b = q[i * lmx:(i + 1) * lmx], qref[i * lmx:(i + 1) * lmx]
        d = float((a - b).abs().max())
        errs[name] = d / float(b.abs().max())
        if 1 <= i <= 3:
            errs_m[name] = d / mmax
    return errs, errs_m


def mixed_512_gcbc_section(args, steps=6):
    """Mixed forms of the Taylor-Green box at 512^3 with non-reflective GCBC x
    faces and periodic y/z, all autotuned: ms per step, and the per-field error
    of each mixed state against the FP64 state after the same steps from the
    same initial state.  `mixed` is the FP32-interior form (CS_PREC_MIXED_F32:
    its x lines have physical closures and run the table solve; y and z the
    ChunkFactors solve); `mixed_refinement_sweep_on` adds the FP64-residual
    refinement sweep to it; `mixed_fp64_rhs` forms every right-hand side and
    flux in FP64 (CS_PREC_MIXED)."""
    import torch
    import compact_schemes_b200 as cs
    from compact_schemes_b200.solver import PREC_MIXED, PREC_MIXED_F32, REFINE_ALL
    n = 512
    lmx = n ** 3
    nbc = [[cs.BC_NON_REFLECTIVE, cs.BC_PERIODIC, cs.BC_PERIODIC]] * 2
    variants = [("plain", 0, 0), ("mixed", PREC_MIXED_F32, 0), ("mixed_refinement_sweep_on", PREC_MIXED_F32, REFINE_ALL),
                ("mixed_fp64_rhs", PREC_MIXED, 0)]
    out, qref = {}, None
    for key, prec, refine in variants:
        s = cs.Solver(cs.tgv_config(n, mach=MACH, re=RE, cfl=CFL, use_graph=True, nbc=nbc, gcbc=True,
                                    precision=prec, refine=refine))
        q = torch.empty(5 * lmx, dtype=torch.float64, device="cuda")
        cs.tgv_init(q, (n, n, n), MACH, 1e-4, 0)
        choice = s.autotune(q, reps=1)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.step(q)  # graph capture (counted in the error comparison, not in the timing)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(steps):
            s.step(q)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        out[key] = {"ms_per_step": ms, "value": lmx * 4 / (ms * 1e-3) / 1e6,
                    "schedule": {"%s_%s" % ("grad" if k == 0 else "flux", "xyz"[a]): v
                                 for (k, a), v in choice.items()}}
        if qref is None:
            qref = q
        else:
            out[key]["speedup_vs_plain"] = out["plain"]["ms_per_step"] / ms
            out[key]["rel_err_vs_fp64_per_field"], out[key]["rel_err_momentum_vs_max_momentum"] = \
                state_errors(q, qref, lmx)
            del q
        s.close()
        torch.cuda.empty_cache()
    del qref
    torch.cuda.empty_cache()
    return dict(out, workload="taylor_green_512^3, GCBC non-reflective x faces, periodic y/z",
                speedup_mixed_vs_plain=out["plain"]["ms_per_step"] / out["mixed"]["ms_per_step"],
                steps_compared=steps + 1, unit=UNIT)


CURV_STAGE_BYTES = 864 + 3 * 80 + 80 // 4  # + metrics in the 3 flux passes and the dt pass of stage 0


def curvilinear_section(args, uniform_ms, steps=20):
    """The Taylor-Green state on a curvilinear periodic 256^3 grid
    (x = xi + A sin(eta) sin(zeta) and cyclic, A = 0.1): metrics from
    cs.grid.metrics, the fused FP64 step reading them per point."""
    import torch
    import compact_schemes_b200 as cs
    n = args.n
    dims = (n, n, n)
    lmx = n ** 3
    h = 2 * math.pi / n
    ax = torch.arange(n, dtype=torch.float64, device="cuda") * h
    X, Y, Z = ax.view(1, 1, n), ax.view(1, n, 1), ax.view(n, 1, 1)
    amp = 0.1
    xyz = torch.stack([(X + amp * torch.sin(Y) * torch.sin(Z)).expand(n, n, n).reshape(-1),
                       (Y + amp * torch.sin(Z) * torch.sin(X)).expand(n, n, n).reshape(-1),
                       (Z + amp * torch.sin(X) * torch.sin(Y)).expand(n, n, n).reshape(-1)]).reshape(-1)
    nbc = [[cs.BC_PERIODIC] * 3] * 2
    nm = cs.numerics_pc(dims, nbc)
    nm.deriv_setup()
    g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    g0.record()
    met = cs.grid.metrics(nm, xyz, [[2 * math.pi, 0, 0], [0, 2 * math.pi, 0], [0, 0, 2 * math.pi]])
    g1.record()
    torch.cuda.synchronize()
    metrics_ms = g0.elapsed_time(g1)
    nm.close()
    del xyz
    s = cs.Solver(cs.tgv_config(n, mach=MACH, re=RE, cfl=CFL, use_graph=True))
    s.set_metrics(*met)
    q = torch.empty(5 * lmx, dtype=torch.float64, device="cuda")
    cs.tgv_init(q, dims, MACH, 1e-4, 0)
    choice = s.autotune(q, reps=1)
    for _ in range(args.warmup):
        s.step(q)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        s.step(q)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    s.profile_begin()
    for _ in range(2):
        s.step(q)
    prof = s.profile_end()
    hbm, _ = peaks()
    stage_ms = sum(v[0] for v in prof.values()) / 8
    s.close()
    del met, q
    torch.cuda.empty_cache()
    return {"workload": "taylor_green_%d^3 on a curvilinear periodic grid (amplitude 0.1), FP64" % n,
            "value": lmx * 4 / (ms * 1e-3) / 1e6, "unit": UNIT, "ms_per_step": ms, "steps": steps,
            "slowdown_vs_uniform": ms / uniform_ms, "grid_metrics_ms": metrics_ms,
            "schedule": {"%s_%s" % ("grad" if k == 0 else "flux", "xyz"[a]): v for (k, a), v in choice.items()},
            "passes_ms_per_launch": {k: v[0] / v[1] for k, v in prof.items() if v[1]},
            "stage_model": {"bytes_per_point": CURV_STAGE_BYTES, "ms_per_stage": stage_ms,
                            "frac": CURV_STAGE_BYTES * lmx / (stage_ms * 1e-3) / 1e9 / hbm}}


def ensemble_section(args):
    """64 seeded Taylor-Green boxes, each axis in {32,48,64,96,128}, Mach in
    [0.05,0.3), Re in [400,3200), FP64: the autotuned ensemble step against
    looping one graph-replayed Solver per box, both on device-resident state."""
    import torch
    import compact_schemes_b200 as cs
    boxes = cs.draw_boxes(64, 0)
    npts = cs.ensemble.ensemble_points(boxes)
    cfgs = cs.ensemble_tgv(boxes)
    ens = cs.Ensemble(cfgs)
    q = torch.zeros(ens.state_size(), dtype=torch.float64, device="cuda")
    for b, (d, m, _) in enumerate(boxes):
        cs.tgv_init(ens.box_view(q, b), d, m, 1e-4, b)
    tuning, tune_ms = ens.autotune(q, reps=2)
    steps = 5
    for _ in range(2):
        ens.step(q)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        ens.step(q)
    e1.record()
    torch.cuda.synchronize()
    ens.last_dt()  # raises on a dependency-wait timeout
    t_ens = e0.elapsed_time(e1) / steps
    solvers = [cs.Solver(c) for c in cfgs]
    views = [ens.box_view(q, b) for b in range(len(boxes))]
    for sv, v in zip(solvers, views):
        sv.step(v)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(steps):
        for sv, v in zip(solvers, views):
            sv.step(v)
    e1.record()
    torch.cuda.synchronize()
    t_loop = e0.elapsed_time(e1) / steps
    for sv in solvers:
        sv.close()
    ens.close()
    rate = lambda ms: npts * 4 / (ms * 1e-3) / 1e6
    return {"workload": "64 seeded TGV boxes, axes in {32,48,64,96,128}, FP64", "points": npts,
            "value": rate(t_ens), "unit": UNIT, "ms_per_step": t_ens,
            "loop_per_box_value": rate(t_loop), "loop_ms_per_step": t_loop,
            "speedup_vs_loop": t_loop / t_ens, "tuning": tuning, "autotune_ms_per_step": tune_ms,
            "launches_per_step": 4, "steps": steps}


def adjoint_section(args):
    """Gradient of the kinetic energy after 50 steps of the 128^3 Taylor-Green
    box with respect to the initial density (velocity, pressure fixed),
    checkpoint every 10 steps, time steps frozen at the CFL trajectory's."""
    import torch
    import compact_schemes_b200 as cs
    n, nsteps, every = 128, 50, 10
    lmx = n ** 3
    cfg = cs.tgv_config(n, mach=MACH, re=RE, cfl=CFL, use_graph=False)
    s = cs.Solver(cfg)
    free0 = torch.cuda.mem_get_info()[0]
    a = cs.Adjoint(cfg)
    free1 = torch.cuda.mem_get_info()[0]
    q0 = torch.empty(5 * lmx, dtype=torch.float64, device="cuda")
    cs.tgv_init(q0, (n, n, n), MACH, 1e-4, 0)
    qr, dts = q0.clone(), []
    for _ in range(nsteps):
        s.step(qr, 0.0)
        dts.append(s.last_dt())
    ev = lambda: torch.cuda.Event(enable_timing=True)
    e0, e1 = ev(), ev()
    qf = q0.clone()
    e0.record()
    for dt in dts:
        s.step(qf, dt)
    e1.record()
    torch.cuda.synchronize()
    t_fwd = e0.elapsed_time(e1)
    lam = torch.empty_like(q0)
    a.gradient(q0, dts, every, lam)
    e0.record()
    J = a.gradient(q0, dts, every, lam)
    e1.record()
    torch.cuda.synchronize()
    t_grad = e0.elapsed_time(e1)
    # one reverse step: stage recomputation + step adjoint, against one forward step
    st = [torch.empty_like(q0) for _ in range(4)]
    out = torch.empty_like(q0)
    e0.record()
    for _ in range(5):
        a.stages(q0, dts[0], st)
        a.step_vjp(st, dts[0], lam, out)
    e1.record()
    torch.cuda.synchronize()
    t_rev_step = e0.elapsed_time(e1) / 5
    sweep_bytes = a.gradient_bytes(nsteps, every)
    # d J / d rho0 and central differences along 8 seeded Gaussian directions
    lv = lam.view(5, -1)
    u = q0.view(5, -1)[1:4] / q0.view(5, -1)[0]
    g = lv[0] + (lv[1:4] * u).sum(0) + 0.5 * lv[4] * (u * u).sum(0)
    gen = torch.Generator(device="cuda").manual_seed(0)
    eps, fd_err = 1e-6, []

    def j_of(rho):
        qq = q0.clone().view(5, -1)
        p = 0.4 * (qq[4] - 0.5 * qq[0] * (u * u).sum(0))
        qq[0] = rho
        qq[1:4] = rho * u
        qq[4] = p / 0.4 + 0.5 * rho * (u * u).sum(0)
        qq = qq.reshape(-1)
        for dt in dts:
            s.step(qq, dt)
        return a.kinetic_energy(qq)

    rho0 = q0.view(5, -1)[0].clone()
    for _ in range(8):
        v = torch.randn(lmx, dtype=torch.float64, device="cuda", generator=gen)
        fd = (j_of(rho0 + eps * v) - j_of(rho0 - eps * v)) / (2 * eps)
        fd_err.append(abs(float((g * v).sum()) - fd) / abs(fd))
    # forward/adjoint dot product for the 50-step map
    x = torch.randn(5 * lmx, dtype=torch.float64, device="cuda", generator=gen)
    y = torch.randn(5 * lmx, dtype=torch.float64, device="cuda", generator=gen)
    q, dx = q0.clone(), x.clone()
    for dt in dts:
        a.stages(q, dt, st)
        a.step_jvp(st, dt, dx, out)
        dx, out = out, dx
        s.step(q, dt)
    lam_y = torch.empty_like(q0)
    a_grad_dot = _adjoint_map(a, s, q0, dts, every, y, lam_y)
    lhs, rhs = float((y * dx).sum()), float((lam_y * x).sum())
    a.close()
    s.close()
    return {"workload": "128^3 TGV, 50 steps, checkpoint every 10, dJ/drho0 of J = kinetic energy", "J": J,
            "forward_ms": t_fwd, "gradient_ms": t_grad, "gradient_over_forward": t_grad / t_fwd,
            "reverse_step_ms": t_rev_step, "forward_step_ms": t_fwd / nsteps,
            "adjoint_step_over_forward_step": t_rev_step / (t_fwd / nsteps),
            "memory_bytes": {"adjoint_scratch": free0 - free1, "checkpoint_sweep": sweep_bytes,
                             "peak": free0 - free1 + sweep_bytes},
            "fd_rel_err_8_dirs": fd_err, "fd_eps": eps,
            "dot_product_rel_err": abs(lhs - rhs) / abs(lhs), "dt": "frozen at the CFL trajectory's"}


def _adjoint_map(a, s, q0, dts, every, y, lam_out):
    """lam_out = A^T y for the tangent A of len(dts) steps (recomputing stages)."""
    import torch
    traj, q = [], q0.clone()
    for dt in dts:
        traj.append(q.clone())
        s.step(q, dt)
    st = [torch.empty_like(q0) for _ in range(4)]
    lam, out = y.clone(), torch.empty_like(q0)
    for k in reversed(range(len(dts))):
        a.stages(traj[k], dts[k], st)
        a.step_vjp(st, dts[k], lam, out)
        lam, out = out, lam
    lam_out.copy_(lam)
    return True


REF_GPU = os.path.join(ROOT, "oracle", "_ref", "libref_gpu.so")


class _Raw:
    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f8", "data": (int(ptr), False),
                                         "version": 3}


def device_view(ptr, n):
    """torch float64 view of n doubles at a raw device address owned by the library."""
    import torch
    return torch.as_tensor(_Raw(ptr, n), device="cuda")


def reference_kernels_section(args):
    """The reference's own sm_100a kernels for the derivative and flux steps,
    compiled from its sources into oracle/_ref/libref_gpu.so, timed beside
    this library's on the same 256^3 FP64 inputs (CUDA events, one stream,
    after warm-up; inputs larger than L2):
      deriv_kernel_2d<Axis,double> (src/cuda/kernels/numerics_pc.hpp:174-249)
        against cs_deriv, y and z lines, physical (ndf 0) and periodic (ndf 1)
        closures; 16 B/pt (one field read, one written).  The reference's x
        kernel is valid only for lze = 1 and is not timed;
      calc_fluxes_pre_compute_kernel<true,double>
        (src/cuda/kernels/physics.hpp:42-193) against cs_calc_fluxes_pre:
        reads qa 5, p, de 5, metrics 9, tau 6, heat 3, writes 15 fluxes and
        de[4]: 45 words = 360 B/pt."""
    import ctypes
    import torch
    import compact_schemes_b200 as cs
    if not os.path.exists(REF_GPU):
        return {"unavailable": "oracle/_ref/libref_gpu.so not built (make -C oracle ref needs the reference sources)"}
    R = ctypes.CDLL(REF_GPU)
    vp = ctypes.c_void_p
    R.ref_gpu_deriv2d.argtypes = [ctypes.c_int, vp, vp, vp, vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                  ctypes.c_int, ctypes.c_int, ctypes.c_uint, ctypes.c_uint, vp]
    R.ref_gpu_fluxes_pre_time.argtypes = [vp] * 9 + [ctypes.c_double] * 3 + [ctypes.c_uint, vp, ctypes.c_int, vp,
                                                                             ctypes.POINTER(ctypes.c_float)]
    dev = torch.device("cuda", torch.cuda.current_device())
    stream = torch.cuda.current_stream()
    sp = vp(stream.cuda_stream)
    reps, warm = 20, 3
    hbm, _ = peaks()
    n = 256
    dims = (n, n, n)
    lmx = n ** 3

    def timed(fn):
        for _ in range(warm):
            fn()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    rows = []
    for axis in (1, 2):
        for ndf in (0, 1):
            b = cs.BC_PERIODIC if ndf else cs.BC_NON_REFLECTIVE
            nm = cs.numerics_pc(dims, [[b] * 3] * 2)
            nm.deriv_setup()
            g = torch.Generator(device=dev).manual_seed(1)
            f = torch.randn(lmx, dtype=torch.float64, device=dev, generator=g)
            if ndf:
                blk = torch.zeros(15 * lmx, dtype=torch.float64, device=dev)
                blk[axis * lmx:(axis + 1) * lmx] = f
                nm.fill_buffers(blk, 0, 1, 0, dims)
                nm.mpigo(dims, None, 1, 0)
                del blk
            ours = torch.empty(3 * lmx, dtype=torch.float64, device=dev)
            theirs = torch.empty(3 * lmx, dtype=torch.float64, device=dev)
            _, _, recv = nm.buffers(axis)
            scratch = torch.zeros(10 * n * n, dtype=torch.float64, device=dev)
            _, pbci = nm.coeffs()
            dpbci = torch.tensor(pbci, dtype=torch.float64, device=dev)
            t_ours = timed(lambda: nm.deriv2d(axis, f, ours, ndf, ndf, dims, 0, 0, stream=stream))

            def run_ref():
                rc = R.ref_gpu_deriv2d(axis, vp(f.data_ptr()), vp(theirs.data_ptr()), vp(recv),
                                       vp(dpbci.data_ptr()), vp(scratch.data_ptr()), ndf, ndf, *dims, 0, 0, sp)
                if rc:
                    raise RuntimeError("reference deriv kernel launch failed: %d" % rc)
            t_ref = timed(run_ref)
            a, t = ours[axis * lmx:(axis + 1) * lmx], theirs[axis * lmx:(axis + 1) * lmx]
            gbs = lambda ms: 16.0 * lmx / (ms * 1e-3) / 1e9
            rows.append({"kernel": "deriv", "axis": "xyz"[axis], "ndf": ndf, "ours_ms": t_ours,
                         "reference_ms": t_ref, "speedup": t_ref / t_ours, "ours_frac": gbs(t_ours) / hbm,
                         "reference_frac": gbs(t_ref) / hbm,
                         "max_rel_diff": float((a - t).abs().max() / t.abs().max())})
            nm.close()
            del f, ours, theirs, scratch
            torch.cuda.empty_cache()
    # flux pre-compute on a smooth state with per-point metrics
    g = torch.Generator(device=dev).manual_seed(2)
    rnd = lambda k: torch.rand(k * lmx, dtype=torch.float64, device=dev, generator=g)
    rho = 1.0 + 0.1 * rnd(1)
    vel = 0.3 * (rnd(3) - 0.5)
    p = 1 / 1.4 + 0.05 * rnd(1)
    v3 = vel.view(3, -1)
    qa = torch.cat([rho, rho * v3[0], rho * v3[1], rho * v3[2], p / 0.4 + 0.5 * rho * (v3 ** 2).sum(0)])
    de = torch.cat([1 / rho, v3[0], v3[1], v3[2], 1.4 * p / rho])
    h = 2 * math.pi / n
    met = [torch.zeros(3 * lmx, dtype=torch.float64, device=dev) for _ in range(3)]
    for a in range(3):
        met[a][a * lmx:(a + 1) * lmx] = h * h * (1 + 0.01 * rnd(1))
    tau, heat = 1e-3 * rnd(6), 1e-3 * rnd(3)
    ph = cs.physics(dims, True)
    ph.umf = (0.0, 0.0, 0.0)
    b0, _, dtau, dheat = ph.buffers()
    device_view(dtau, 6 * lmx).copy_(tau)
    device_view(dheat, 3 * lmx).copy_(heat)
    de_o = de.clone()
    t_ours = timed(lambda: ph.calc_fluxes_pre(qa, p, de_o, met[0], met[1], met[2], stream=stream))
    theirs = torch.zeros(15 * lmx, dtype=torch.float64, device=dev)
    de_r = de.clone()
    structs = torch.zeros(16, dtype=torch.float64, device=dev)
    ms = ctypes.c_float()
    ptrs = [vp(x.data_ptr()) for x in (theirs, qa, p, de_r, met[0], met[1], met[2], tau, heat)]
    for _ in range(2):
        rc = R.ref_gpu_fluxes_pre_time(*ptrs, 0.0, 0.0, 0.0, lmx, vp(structs.data_ptr()), warm, sp, ctypes.byref(ms))
    rc = R.ref_gpu_fluxes_pre_time(*ptrs, 0.0, 0.0, 0.0, lmx, vp(structs.data_ptr()), reps, sp, ctypes.byref(ms))
    if rc:
        raise RuntimeError("reference flux kernel failed: %d" % rc)
    t_ref = float(ms.value)
    torch.cuda.synchronize()
    ours_buf = device_view(b0, 15 * lmx)
    diff = max(float((ours_buf[c * lmx:(c + 1) * lmx] - theirs[c * lmx:(c + 1) * lmx]).abs().max() /
                     theirs[c * lmx:(c + 1) * lmx].abs().max()) for c in range(15))
    gbs = lambda ms_: 360.0 * lmx / (ms_ * 1e-3) / 1e9
    rows.append({"kernel": "fluxes_pre", "ours_ms": t_ours, "reference_ms": t_ref, "speedup": t_ref / t_ours,
                 "ours_frac": gbs(t_ours) / hbm, "reference_frac": gbs(t_ref) / hbm, "max_rel_diff": diff})
    ph.close()
    del qa, de, de_o, de_r, met, tau, heat, theirs
    torch.cuda.empty_cache()
    return {"workload": "256^3 FP64 fields, one launch per kernel", "reps": reps,
            "deriv_bytes_per_point": 16, "fluxes_pre_bytes_per_point": 360, "rows": rows}


def dropin_section(args, fused_ms_per_step, stages=8):
    """The reference-shaped call sequence through the drop-in API, the path a
    caller of physics / numerics_pc gets: per RK stage thermo,
    calc_viscous_shear_stress, thermo, calc_fluxes (15 single-field solves
    plus the interface sums) and rk_update, on the 256^3 Taylor-Green state
    with per-point metric arrays of the uniform grid.  Unfused pointwise
    kernels; timed with CUDA events over `stages` stages."""
    import torch
    import compact_schemes_b200 as cs
    n = args.n
    dims = (n, n, n)
    lmx = n ** 3
    dev = torch.device("cuda", torch.cuda.current_device())
    nbc = [[cs.BC_PERIODIC] * 3] * 2
    nm = cs.numerics_pc(dims, nbc)
    nm.deriv_setup()
    ph = cs.physics(dims, True)
    q = torch.empty(5 * lmx, dtype=torch.float64, device=dev)
    cs.tgv_init(q, dims, MACH, 1e-4, 0)
    qn = q.clone()
    h = 2 * math.pi / n
    met = [torch.zeros(3 * lmx, dtype=torch.float64, device=dev) for _ in range(3)]
    for a in range(3):
        met[a][a * lmx:(a + 1) * lmx] = h * h
    yaco = torch.full((lmx,), 1.0 / h ** 3, dtype=torch.float64, device=dev)
    de = torch.zeros(5 * lmx, dtype=torch.float64, device=dev)
    p = torch.zeros(lmx, dtype=torch.float64, device=dev)
    ssk = torch.full((lmx,), MACH / RE, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream()
    dt = 1e-3

    def stage(k):
        cs.thermo(q, de, p, stream=stream)
        ph.calc_viscous_shear_stress(de, ssk, met[0], met[1], met[2], yaco, dims, None, nm, streams=stream)
        cs.thermo(q, de, p, stream=stream)
        ph.calc_fluxes(q, p, de, met[0], met[1], met[2], dims, None, nm, streams=stream)
        cs.rk_update(qn, de, yaco, dt / (4 - k % 4), q, stream=stream)

    for k in range(2):
        stage(k)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for k in range(stages):
        stage(k)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / stages
    ph.close()
    nm.close()
    del q, qn, met, yaco, de, p, ssk
    torch.cuda.empty_cache()
    return {"workload": "256^3 Taylor-Green, FP64, drop-in physics / numerics_pc call sequence per RK stage "
                        "(metric arrays of the uniform grid)",
            "value": lmx / (ms * 1e-3) / 1e6, "unit": UNIT, "ms_per_stage": ms,
            "fused_ms_per_stage": fused_ms_per_step / 4, "fused_speedup": ms / (fused_ms_per_step / 4),
            "stages": stages}


def filter_section(args, plain_ms_per_step, steps=20):
    """The compact filter inside the time step (CS_FILTER_STEP: after every RK
    step, alpha_f 0.45, all five conserved fields along x, y and z) on the
    headline 256^3 workload: step time against the plain step, and each
    filter pass against 80 B/pt (five fields read and written)."""
    import torch
    import compact_schemes_b200 as cs
    from compact_schemes_b200.solver import FILTER_STEP
    n = args.n
    lmx = n ** 3
    s = cs.Solver(cs.tgv_config(n, mach=MACH, re=RE, cfl=CFL, use_graph=True, filter=FILTER_STEP, alpha_f=0.45))
    q = torch.empty(5 * lmx, dtype=torch.float64, device="cuda")
    cs.tgv_init(q, (n, n, n), MACH, 1e-4, 0)
    s.autotune(q, reps=1)
    for _ in range(args.warmup):
        s.step(q)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        s.step(q)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    s.profile_begin()
    for _ in range(2):
        s.step(q)
    prof = s.profile_end()
    s.close()
    del q
    torch.cuda.empty_cache()
    hbm, _ = peaks()
    fms, fl = prof["filter"]
    per = fms / fl
    return {"workload": "taylor_green_%d^3 FP64, filter after every RK step (alpha_f 0.45)" % n,
            "ms_per_step": ms, "plain_ms_per_step": plain_ms_per_step, "filter_share": 1 - plain_ms_per_step / ms,
            "value": lmx * 4 / (ms * 1e-3) / 1e6, "unit": UNIT,
            "filter_pass_ms_per_launch": per, "filter_pass_bytes_per_point": 80,
            "filter_pass_frac": 80 * lmx / (per * 1e-3) / 1e9 / hbm}


def config1_section(args, reps=20):
    """The derivative-and-filter workload: the 64^3 non-periodic [0,1]^3
    field of 8 Fourier modes (MT19937-64 seed 0), physical closures on all
    faces; index-space compact derivatives along x, y, z and the filter
    (alpha_f 0.45) along x then y then z.  GPU: 6 line-solve launches per
    pass (the field is L2-resident, 2 MB: latency-bound, not an HBM case);
    CPU: the oracle on the host cores.  Error: GPU against the oracle."""
    import numpy as np
    import torch
    import compact_schemes_b200 as cs
    import oracle as O
    dims = (64, 64, 64)
    nm = cs.numerics_pc(dims, [[cs.BC_NON_REFLECTIVE] * 3] * 2)
    nm.deriv_setup()
    f = cs.grid.fourier_field(dims, 0, 8)
    d = [torch.empty_like(f) for _ in range(3)]
    a, b = torch.empty_like(f), torch.empty_like(f)
    stream = torch.cuda.current_stream()

    def gpu_pass():
        for ax in range(3):
            nm.deriv1d(ax, f, d[ax], 0, 0, dims, 0, halo=cs.HALO_SELF, stream=stream)
        nm.filter(0, f, a, 0.45, dims, stream=stream)
        nm.filter(1, a, b, 0.45, dims, stream=stream)
        nm.filter(2, b, a, 0.45, dims, stream=stream)

    for _ in range(3):
        gpu_pass()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        gpu_pass()
    e1.record(stream)
    torch.cuda.synchronize()
    gpu_ms = e0.elapsed_time(e1) / reps
    fh = f.cpu().numpy()
    t0 = time.perf_counter()
    for _ in range(3):
        ref_d = [O.deriv(fh, dims, ax, 0, 0) for ax in range(3)]
        r = fh
        for ax in range(3):
            r = O.filt(r, dims, ax, 0, 0, 0.45)
    cpu_ms = (time.perf_counter() - t0) * 1e3 / 3
    rel = lambda x, y: float(np.abs(x - y).max() / np.abs(y).max())
    errs = {"deriv_" + "xyz"[ax]: rel(d[ax].cpu().numpy(), ref_d[ax]) for ax in range(3)}
    errs["filter_xyz"] = rel(a.cpu().numpy(), r)
    nm.close()
    return {"workload": "64^3 Fourier-mode field (8 modes, MT19937-64 seed 0), non-periodic [0,1]^3: "
                        "d/dx, d/dy, d/dz and filter x->y->z", "gpu_ms_per_pass": gpu_ms,
            "cpu_ms_per_pass": cpu_ms, "cpu_cores": O.num_threads(), "cpu_kind": "port (FP64 oracle)",
            "speedup_gpu_vs_cpu": cpu_ms / gpu_ms, "rel_err_gpu_vs_oracle": errs, "tolerance": 1e-12}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms during a region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        self.p.wait()
        self.f.flush()
        self.f.seek(0)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f:
            c = [x.strip() for x in line.split(",")]
            if len(c) < 9:
                continue
            try:
                sm.append(float(c[1]))
                smax.append(float(c[2]))
            except ValueError:
                continue
            for nm, v in zip(names, c[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.f.name)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(args):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(0)
    return world, rank, local


def max_over_ranks(x, world, device="cuda"):
    """Max of a per-rank timing over the process group (the job's time)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world, cuda=True):
    import torch
    if cuda:
        torch.cuda.synchronize()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    if cuda:
        torch.cuda.synchronize()


def cpu_oracle_stage_rate(n, stages=1):
    """Oracle (FP64 C++/OpenMP restatement) RK stages at n^3 on the host cores."""
    import numpy as np
    import oracle as O
    dims = (n, n, n)
    q = O.tgv_init(dims, MACH, 1e-4, 0)
    q1 = np.empty_like(q)
    m = O.uniform_metrics(*dims)
    nbc = [[45] * 3, [45] * 3]
    de, _ = O.thermo(q)
    dt = O.time_step_m(de, m, MACH / RE, (0.0, 0.0, 0.0), CFL)
    del de
    t0 = time.perf_counter()
    for k in range(stages):
        O.rk_stage(q, q if k == 0 else q1, q1, k % 4, dt, MACH / RE, m, dims, nbc)
    t = time.perf_counter() - t0
    return n ** 3 * stages / t / 1e6, t, O.num_threads()


def workload_config(n, world):
    """The workload both arms print (the same keys and values)."""
    return {"workload": "taylor_green_%d^3_fp64_plain" % n, "n": n, "mach": MACH, "re": RE, "cfl": CFL,
            "rk": "4-stage, q^(k) = q^n - dt/(4-k) J R", "bc": "periodic (quasi-disjoint closure)",
            "l2": "inputs larger than L2 (state 671 MB + gradients 1.6 GB), no flush",
            "parallelism": "replicas" if world > 1 else "single GPU"}


def run_reference(args):
    """Reference arm: the reference has no CPU implementation of the path, so its
    CPU path is the oracle port of its kernels, timed on the host cores."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import numpy as np
    import oracle as O
    n = args.n
    dims = (n, n, n)
    q = O.tgv_init(dims, MACH, 1e-4, 0)
    q1 = np.empty_like(q)
    m = O.uniform_metrics(*dims)
    nbc = [[45] * 3, [45] * 3]
    de, _ = O.thermo(q)
    dt = O.time_step_m(de, m, MACH / RE, (0.0, 0.0, 0.0), CFL)
    del de
    for k in range(args.warmup):
        O.rk_stage(q, q if k == 0 else q1, q1, k % 4, dt, MACH / RE, m, dims, nbc)
    t0 = time.perf_counter()
    for k in range(args.steps):
        O.rk_stage(q, q1, q1, (k + 1) % 4, dt, MACH / RE, m, dims, nbc)
    t = time.perf_counter() - t0
    value = n ** 3 * args.steps / t / 1e6
    cores = O.num_threads()
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": workload_config(n, world),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": "%d RK stages of the %d^3 Taylor-Green box (FP64 oracle, "
                                       "C++/OpenMP restatement of the reference kernels; a step of this "
                                       "arm is one RK stage, dt from the initial state)" % (args.steps, n)},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def run_ours(args):
    import torch
    import compact_schemes_b200 as cs

    world, rank, local = dist_setup(args)
    n = args.n
    dims = (n, n, n)
    lmx = n ** 3
    pts_stages_per_step = lmx * 4
    from compact_schemes_b200.solver import SCHED_AUTO, SCHED_ONEPHASE, SCHED_TMA
    sched = {"auto": SCHED_AUTO, "tma": SCHED_TMA, "onephase": SCHED_ONEPHASE}[args.schedule]
    cfg = cs.tgv_config(n, mach=MACH, re=RE, cfl=CFL, use_graph=True, schedule=sched)
    s = cs.Solver(cfg)
    q = torch.empty(5 * lmx, dtype=torch.float64, device="cuda")
    cs.tgv_init(q, dims, MACH, 1e-4, rank)
    stream = torch.cuda.current_stream()

    # per-pass schedule (the state is not modified)
    tuned = s.autotune(q, reps=1) if args.schedule == "auto" else s.schedule()
    for _ in range(args.warmup):
        s.step(q, 0.0)
    barrier(world)

    # --- value: graph-replayed steps on the device-resident state -------------
    clk = ClockSampler(local)
    clk.start()
    time.sleep(0.3)
    barrier(world)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        s.step(q, 0.0)
    e1.record(stream)
    barrier(world)
    clocks = clk.stop()
    t_ms = max_over_ranks(e0.elapsed_time(e1), world)
    value = world * pts_stages_per_step * args.steps / (t_ms * 1e-3) / 1e6

    # --- roofline: eager steps with per-pass events ------------------------------
    s.profile_begin()
    for _ in range(args.steps):
        s.step(q, 0.0)
    prof = s.profile_end()
    barrier(world)
    hbm, peak_kind = peaks()
    per_pass = {}
    for k, (ms, cnt) in prof.items():
        if cnt:
            b = ALG_BYTES.get(k)
            if k == "flux_z_rk":  # stage 0 reads q^n only once: stage-averaged bytes
                b = (3 * ALG_BYTES[k] + (ALG_BYTES[k] - 40)) / 4
            per_pass[k] = {"ms_per_launch": ms / cnt, "launches": cnt, "total_ms": ms}
            if b:
                gbs = b * lmx / (ms / cnt * 1e-3) / 1e9
                per_pass[k].update({"alg_bytes_per_point": b, "achieved_gbs": gbs, "frac": gbs / hbm})
    top = max(per_pass, key=lambda k: per_pass[k]["total_ms"])
    alg = per_pass[top]["alg_bytes_per_point"] * lmx
    achieved = alg / (per_pass[top]["ms_per_launch"] * 1e-3) / 1e9
    stage_ms = sum(v["total_ms"] for v in per_pass.values()) / (4 * args.steps)
    traffic, traffic_src = None, None
    try:
        # DRAM bytes of one launch per stage kind of this pass at 256^3
        # (ncu dram__bytes_read.sum + dram__bytes_write.sum, profiles/)
        with open(os.path.join(ROOT, "profiles", "traffic_%s_256.json" % top)) as f:
            tj = json.load(f)
        if n == 256:
            traffic = (tj["stage0_bytes"] + 3 * tj["stage1_bytes"]) / 4
            traffic_src = {"file": "profiles/traffic_%s_256.json" % top, "stage0_bytes": tj["stage0_bytes"],
                           "stage1_bytes": tj["stage1_bytes"],
                           "stage0_alg_bytes": (ALG_BYTES[top] - 40) * lmx if top == "flux_z_rk" else None,
                           "stage1_alg_bytes": ALG_BYTES[top] * lmx}
    except Exception:
        pass
    roofline = {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                "frac": achieved / hbm, "traffic": traffic, "kernel": top,
                "peak_source": peak_kind,
                "alg_bytes_per_launch": alg, "traffic_detail": traffic_src}

    # --- e2e: host buffers through cs_solver_step_host ------------------------------
    qh_in = torch.empty(5 * lmx, dtype=torch.float64, pin_memory=True)
    qh_out = torch.empty(5 * lmx, dtype=torch.float64, pin_memory=True)
    qh_in.copy_(q.cpu())
    s.step_host(qh_in, qh_out, 0.0)  # first call allocates the solver-owned state
    barrier(world)
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for _ in range(args.steps):
        s.step_host(qh_in, qh_out, 0.0)
        qh_in, qh_out = qh_out, qh_in
    f1.record(stream)
    barrier(world)
    te_ms = max_over_ranks(f0.elapsed_time(f1), world)
    e2e = {"value": world * pts_stages_per_step * args.steps / (te_ms * 1e-3) / 1e6, "unit": UNIT,
           "h2d_bytes_per_step": 5 * lmx * 8, "d2h_bytes_per_step": 5 * lmx * 8,
           "ms_per_step": te_ms / args.steps}

    # --- mixed form: same workload and timing, error against the FP64 path -------
    mixed = None
    if not args.no_mixed:
        # the mixed forms, each autotuned, timed like `value`; state error
        # against the FP64 path after 100 steps from the same initial state
        from compact_schemes_b200.solver import PREC_MIXED, PREC_MIXED_F32, REFINE_ALL
        acc_steps = 100
        qp = torch.empty(5 * lmx, dtype=torch.float64, device="cuda")
        cs.tgv_init(qp, dims, MACH, 1e-4, rank)
        for _ in range(acc_steps):
            s.step(qp, 0.0)
        variants = [("mixed", PREC_MIXED_F32, 0), ("refinement_sweep_on", PREC_MIXED_F32, REFINE_ALL),
                    ("mixed_fp64_rhs", PREC_MIXED, 0)]
        res = {}
        for key, prec, refine in variants:
            sm = cs.Solver(cs.tgv_config(n, mach=MACH, re=RE, cfl=CFL, use_graph=True, precision=prec,
                                         refine=refine))
            qm = torch.empty(5 * lmx, dtype=torch.float64, device="cuda")
            cs.tgv_init(qm, dims, MACH, 1e-4, rank)
            choice = sm.autotune(qm, reps=1)
            for _ in range(args.warmup):
                sm.step(qm, 0.0)
            barrier(world)
            g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            g0.record(stream)
            for _ in range(args.steps):
                sm.step(qm, 0.0)
            g1.record(stream)
            barrier(world)
            tm_ms = max_over_ranks(g0.elapsed_time(g1), world)
            cs.tgv_init(qm, dims, MACH, 1e-4, rank)
            for _ in range(acc_steps):
                sm.step(qm, 0.0)
            torch.cuda.synchronize()
            errs, errs_m = state_errors(qm, qp, lmx)
            mvalue = world * pts_stages_per_step * args.steps / (tm_ms * 1e-3) / 1e6
            res[key] = {"value": mvalue, "unit": UNIT, "ms_per_step": tm_ms / args.steps,
                        "speedup_vs_plain": mvalue / value,
                        "schedule": {"%s_%s" % ("grad" if k == 0 else "flux", "xyz"[a]): v
                                     for (k, a), v in choice.items()},
                        "rel_err_vs_fp64_per_field": errs, "rel_err_momentum_vs_max_momentum": errs_m,
                        "steps_compared": acc_steps}
            sm.close()
            del qm
            torch.cuda.empty_cache()
        del qp
        mixed = dict(res["mixed"],
                     arith="FP32 fluxes, interior right-hand sides and line solves (per-row factors as "
                           "constants); FP64 state, RK accumulation, thermodynamics and closure rows; "
                           "no refinement sweep",
                     mixed_fp64_rhs=dict(res["mixed_fp64_rhs"],
                                         arith="fluxes and every right-hand side formed in FP64, FP32 line "
                                               "solves from tables"),
                     refinement_sweep_on=dict(res["refinement_sweep_on"],
                                              arith="mixed plus one refinement sweep after every FP32 line "
                                                    "solve: residual of the FP32 right-hand side formed in FP64, "
                                                    "solved in FP32, added"))

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, t, cores = cpu_oracle_stage_rate(n, stages=1)
        cpu = {"value": rate, "unit": UNIT, "cores": cores, "kind": "port",
               "sample": "1 RK stage of the %d^3 Taylor-Green box in %.1f s (FP64 oracle, "
                         "C++/OpenMP restatement of the reference kernels)" % (n, t)}

    ensemble = adjoint = mixed512 = curvilinear = refk = cfg1 = dropin = filt = None
    if rank == 0 and world == 1:
        s.close()
        if not args.no_reference_kernels:
            refk = reference_kernels_section(args)
            torch.cuda.empty_cache()
        if not args.no_config1:
            cfg1 = config1_section(args)
        if not args.no_dropin:
            dropin = dropin_section(args, t_ms / args.steps)
            torch.cuda.empty_cache()
        if not args.no_filter:
            filt = filter_section(args, t_ms / args.steps)
        if not args.no_curvilinear:
            curvilinear = curvilinear_section(args, t_ms / args.steps)
            torch.cuda.empty_cache()
        if not args.no_mixed:
            mixed512 = mixed_512_gcbc_section(args)
            torch.cuda.empty_cache()
        if not args.no_ensemble:
            ensemble = ensemble_section(args)
            torch.cuda.empty_cache()
        if not args.no_adjoint:
            adjoint = adjoint_section(args)
            torch.cuda.empty_cache()

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_ms / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic",
                "config": workload_config(n, world),
                "schedule": {"%s_%s" % ("grad" if k == 0 else "flux", "xyz"[a]): v for (k, a), v in tuned.items()},
                "dt_policy": "CFL 0.5 recomputed from q^n every step, on the device",
                "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "mixed": mixed,
                "mixed_512_gcbc": mixed512, "ensemble": ensemble, "adjoint": adjoint,
                "curvilinear": curvilinear, "reference_kernels": refk, "config1": cfg1, "dropin": dropin,
                "filter": filt,
                "gpu_launches": 24 * args.steps, "clocks": clocks,
                "passes": per_pass,
                "stage_model": {"bytes_per_point": STAGE_BYTES, "ms_per_stage": stage_ms,
                                "achieved_gbs": STAGE_BYTES * lmx / (stage_ms * 1e-3) / 1e9,
                                "frac": STAGE_BYTES * lmx / (stage_ms * 1e-3) / 1e9 / hbm}}
        print(json.dumps(line))
    s.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
