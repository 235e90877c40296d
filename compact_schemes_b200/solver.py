"""Fused RHS / RK-stage solver over the C ABI (cs_solver_* in include/compact_b200.h).

Replaces the per-stage driver sequence of the reference (driver/canard.cu:132-224):
calc_time_step, calc_viscous_shear_stress, calc_fluxes, gcbc_go and the
conserved-variable update, for one block held as a single rank on a uniform
Cartesian grid.
"""
from __future__ import annotations

import ctypes
import math

from . import check, lib, ptr, stream_ptr, BC_PERIODIC


class SolverConfig(ctypes.Structure):
    _fields_ = [("lxi", ctypes.c_int), ("let", ctypes.c_int), ("lze", ctypes.c_int),
                ("nbc", ctypes.c_int * 3 * 2), ("viscous", ctypes.c_int), ("mu", ctypes.c_double),
                ("umf", ctypes.c_double * 3), ("dx", ctypes.c_double), ("dy", ctypes.c_double),
                ("dz", ctypes.c_double), ("cfl", ctypes.c_double), ("gcbc", ctypes.c_int),
                ("use_graph", ctypes.c_int), ("tile", ctypes.c_int * 3 * 2),
                ("precision", ctypes.c_int), ("refine", ctypes.c_int), ("schedule", ctypes.c_int),
                ("filter", ctypes.c_int), ("alpha_f", ctypes.c_double)]


PREC_FP64 = 0
PREC_MIXED = 1
PREC_MIXED_F32 = 2  # mixed, FP32 interior arithmetic (fluxes, interior RHS) on uniform lines
REFINE_NONE = 0  # mixed: no refinement sweep (the measured state error is the same)
REFINE_ALL = 1   # mixed: a refinement sweep after every FP32 line solve
REFINE_FLUX = 2  # mixed: refinement in the flux passes only
SCHED_AUTO = 0
SCHED_ONEPHASE = 1
SCHED_PIPELINE = 2
SCHED_TMA = 3
FILTER_NONE = 0   # no filter in the time step
FILTER_STEP = 1   # compact filter x, y, z on the state after every RK step
FILTER_STAGE = 2  # the same after every RK stage (FP64 only)


def tgv_config(n, mach=0.1, re=1600.0, cfl=0.5, viscous=True, use_graph=True, dims=None,
               nbc=None, gcbc=False, tile=None, precision=PREC_FP64, refine=REFINE_NONE, schedule=SCHED_AUTO,
               filter=FILTER_NONE, alpha_f=0.45):
    """Taylor-Green box [0,2pi)^3 in CANARD units: mu = rho0 U0 L / Re with U0 = Mach."""
    lxi, let, lze = dims if dims is not None else (n, n, n)
    c = SolverConfig()
    c.lxi, c.let, c.lze = lxi, let, lze
    nbc = nbc if nbc is not None else [[BC_PERIODIC] * 3, [BC_PERIODIC] * 3]
    for f in range(2):
        for a in range(3):
            c.nbc[f][a] = nbc[f][a]
    c.viscous = int(viscous)
    c.mu = mach / re
    c.umf[:] = (0.0, 0.0, 0.0)
    two_pi = 2.0 * math.pi
    c.dx, c.dy, c.dz = two_pi / lxi, two_pi / let, two_pi / lze
    c.cfl = cfl
    c.gcbc = int(gcbc)
    c.use_graph = int(use_graph)
    c.precision = int(precision)
    c.refine = int(refine)
    c.schedule = int(schedule)
    c.filter = int(filter)
    c.alpha_f = float(alpha_f)
    if tile is not None:
        for k in range(2):
            for a in range(3):
                c.tile[k][a] = int(tile[k][a])
    return c


class Solver:
    def __init__(self, cfg: SolverConfig):
        self.cfg = cfg
        self._h = ctypes.c_void_p()
        check(lib().cs_solver_create(ctypes.byref(self._h), ctypes.byref(cfg)))

    @property
    def lmx(self):
        return self.cfg.lxi * self.cfg.let * self.cfg.lze

    def close(self):
        if self._h:
            lib().cs_solver_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def rhs(self, q, out, stream=None):
        check(lib().cs_solver_rhs(self._h, ptr(q), ptr(out), stream_ptr(stream)))

    def stage(self, k, qn, qin, qout, dt, stream=None):
        check(lib().cs_solver_stage(self._h, k, ptr(qn), ptr(qin), ptr(qout), float(dt),
                                    stream_ptr(stream)))

    def step(self, q, dt=0.0, stream=None):
        check(lib().cs_solver_step(self._h, ptr(q), float(dt), stream_ptr(stream)))

    PASS_NAMES = ("grad_x", "grad_y", "grad_z", "flux_x", "flux_y", "flux_z_rk", "gcbc", "filter")

    def profile_begin(self):
        check(lib().cs_solver_profile_begin(self._h))

    def profile_end(self):
        """{pass name: (total ms, launches)} since profile_begin (synchronizes)."""
        ms = (ctypes.c_double * len(self.PASS_NAMES))()
        n = (ctypes.c_int * len(self.PASS_NAMES))()
        check(lib().cs_solver_profile_end(self._h, ms, n))
        return {k: (ms[i], n[i]) for i, k in enumerate(self.PASS_NAMES)}

    def step_host(self, q_in, q_out, dt=0.0, stream=None):
        """One step on host buffers (pinned torch CPU tensors or any host memory)."""
        check(lib().cs_solver_step_host(self._h, ctypes.c_void_p(q_in.data_ptr()),
                                        ctypes.c_void_p(q_out.data_ptr()), float(dt),
                                        stream_ptr(stream)))

    def schedule(self):
        """Current schedule per pass: {(kind, axis): 8 | 16 (one-phase tile
        lines) | 0 (pipelined) | 1 (TMA-staged gradient pass)}."""
        ch = (ctypes.c_int * 3 * 2)()
        check(lib().cs_solver_schedule(self._h, ctypes.byref(ch)))
        return {(k, a): ch[k][a] for k in range(2) for a in range(3)}

    def autotune(self, q, reps=2, stream=None):
        """Pick the fastest schedule per pass on a scratch copy of q; returns
        {(kind, axis): 8 | 16 (one-phase tile lines) | 0 (pipelined) |
        1 (TMA-staged gradient pass)}."""
        ch = (ctypes.c_int * 3 * 2)()
        check(lib().cs_solver_autotune(self._h, ptr(q), int(reps), ctypes.byref(ch), stream_ptr(stream)))
        return {(k, a): ch[k][a] for k in range(2) for a in range(3)}

    def set_metrics(self, xim=None, etm=None, zem=None, yaco=None):
        """Per-point metrics (torch CUDA float64: xim/etm/zem [3*lmx], yaco
        [lmx]) for every later call; no arguments returns to the uniform grid.
        The tensors are kept alive by the solver."""
        arrs = (xim, etm, zem, yaco)
        check(lib().cs_solver_set_metrics(self._h, *(None if a is None else ptr(a) for a in arrs)))
        self._metrics = arrs if xim is not None else None

    def last_dt(self):
        v = ctypes.c_double()
        check(lib().cs_solver_last_dt(self._h, ctypes.byref(v)))
        return v.value


def tgv_init(q, dims, mach=0.1, noise=1e-4, seed=0, stream=None):
    lxi, let, lze = dims
    check(lib().cs_tgv_init(ptr(q), lxi, let, lze, float(mach), float(noise), int(seed),
                            stream_ptr(stream)))


def _main(argv=None):
    """python -m compact_schemes_b200.solver --n N [--precision P] [--steps K] [--curvilinear A] [--schedule S]:
    K CFL-stepped RK steps of the N^3 Taylor-Green box (profiling driver);
    with A > 0 on the periodic wavy grid x = xi + A sin(eta) sin(zeta)
    (and cyclic), metrics read per point."""
    import argparse
    import torch
    p = argparse.ArgumentParser()
    p.add_argument("--n", type=int, default=128)
    p.add_argument("--precision", type=int, default=PREC_FP64)
    p.add_argument("--steps", type=int, default=1)
    p.add_argument("--graph", type=int, default=0)
    p.add_argument("--curvilinear", type=float, default=0.0)
    p.add_argument("--schedule", type=int, default=SCHED_AUTO)
    a = p.parse_args(argv)
    from compact_schemes_b200 import solver as S  # the package's classes, not __main__'s
    s = S.Solver(S.tgv_config(a.n, precision=a.precision, use_graph=bool(a.graph), schedule=a.schedule))
    if a.curvilinear > 0:
        import compact_schemes_b200 as cs
        n = a.n
        ax = torch.arange(n, dtype=torch.float64, device="cuda") * (2 * math.pi / n)
        X, Y, Z = ax.view(1, 1, n), ax.view(1, n, 1), ax.view(n, 1, 1)
        A = a.curvilinear
        xyz = torch.stack([(X + A * torch.sin(Y) * torch.sin(Z)).expand(n, n, n).reshape(-1),
                           (Y + A * torch.sin(Z) * torch.sin(X)).expand(n, n, n).reshape(-1),
                           (Z + A * torch.sin(X) * torch.sin(Y)).expand(n, n, n).reshape(-1)]).reshape(-1)
        nm = cs.numerics_pc((n, n, n), [[BC_PERIODIC] * 3] * 2)
        nm.deriv_setup()
        s.set_metrics(*cs.grid.metrics(nm, xyz, [[2 * math.pi, 0, 0], [0, 2 * math.pi, 0], [0, 0, 2 * math.pi]]))
        nm.close()
    q = torch.empty(5 * a.n ** 3, dtype=torch.float64, device="cuda")
    S.tgv_init(q, (a.n, a.n, a.n))
    for _ in range(a.steps):
        s.step(q)
    print("steps", a.steps, "last dt", s.last_dt())


if __name__ == "__main__":
    _main()
