"""Tangent-linear and adjoint RHS / RK step (cs_rhs_jvp, cs_rhs_vjp,
cs_step_jvp, cs_step_vjp, cs_adjoint_gradient of include/compact_b200.h).

Device arrays are torch CUDA tensors of [nf * lmx] doubles; the RK step is
linearized with its time step held fixed.
"""
from __future__ import annotations

import ctypes

from . import check, lib, ptr, stream_ptr
from .solver import SolverConfig

_d = ctypes.c_double
_P = ctypes.POINTER(ctypes.c_double)


class Adjoint:
    def __init__(self, cfg: SolverConfig):
        self.cfg = cfg
        self.lmx = cfg.lxi * cfg.let * cfg.lze
        self._h = ctypes.c_void_p()
        check(lib().cs_adjoint_create(ctypes.byref(self._h), ctypes.byref(cfg)))

    def close(self):
        if self._h:
            lib().cs_adjoint_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def deriv(self, axis, x, out, nfields=1, transpose=False, accumulate=False, stream=None):
        check(lib().cs_adjoint_deriv(self._h, int(axis), int(transpose), ptr(x), ptr(out), int(nfields),
                                     int(accumulate), stream_ptr(stream)))

    def filter(self, axis, alpha_f, x, out, nfields=1, transpose=False, accumulate=False, stream=None):
        check(lib().cs_adjoint_filter(self._h, int(axis), int(transpose), float(alpha_f), ptr(x), ptr(out),
                                      int(nfields), int(accumulate), stream_ptr(stream)))

    def rhs_jvp(self, q, dq, out, stream=None):
        check(lib().cs_rhs_jvp(self._h, ptr(q), ptr(dq), ptr(out), stream_ptr(stream)))

    def rhs_vjp(self, q, lam, out, stream=None):
        check(lib().cs_rhs_vjp(self._h, ptr(q), ptr(lam), ptr(out), stream_ptr(stream)))

    @staticmethod
    def _four(stages):
        return (ctypes.c_void_p * 4)(*[ptr(s) for s in stages])

    def stages(self, qn, dt, stages, q_next=None, stream=None):
        check(lib().cs_adjoint_stages(self._h, ptr(qn), float(dt), self._four(stages),
                                      ptr(q_next) if q_next is not None else None, stream_ptr(stream)))

    def step_jvp(self, stages, dt, dq, out, stream=None):
        check(lib().cs_step_jvp(self._h, self._four(stages), float(dt), ptr(dq), ptr(out), stream_ptr(stream)))

    def step_vjp(self, stages, dt, lam_next, out, stream=None):
        check(lib().cs_step_vjp(self._h, self._four(stages), float(dt), ptr(lam_next), ptr(out),
                                stream_ptr(stream)))

    def kinetic_energy(self, q, dJdq=None, stream=None):
        J = _d()
        check(lib().cs_kinetic_energy(self._h, ptr(q), ctypes.byref(J), ptr(dJdq) if dJdq is not None else None,
                                      stream_ptr(stream)))
        return J.value

    def gradient_bytes(self, nsteps, every):
        b = ctypes.c_size_t()
        check(lib().cs_adjoint_gradient_bytes(self._h, int(nsteps), int(every), ctypes.byref(b)))
        return b.value

    def gradient(self, q0, dts, every, grad_out, stream=None):
        """dJ/dq0 of the kinetic energy after len(dts) steps; returns J."""
        n = len(dts)
        arr = (ctypes.c_double * n)(*[float(x) for x in dts])
        J = _d()
        check(lib().cs_adjoint_gradient(self._h, ptr(q0), n, arr, int(every), ptr(grad_out), ctypes.byref(J),
                                        stream_ptr(stream)))
        return J.value


def _arr(vals, n):
    return (ctypes.c_double * n)(*[float(v) for v in vals])


def point_flux(axis, viscous, q, G, M, J, mu, umf):
    F = (ctypes.c_double * 5)()
    check(lib().cs_point_flux(axis, int(viscous), _arr(q, 5), _arr(G, 12), _arr(M, 9), float(J), float(mu),
                              _arr(umf, 3), F))
    return list(F)


def point_flux_jvp(axis, viscous, q, G, dq, dG, M, J, mu, umf):
    F = (ctypes.c_double * 5)()
    check(lib().cs_point_flux_jvp(axis, int(viscous), _arr(q, 5), _arr(G, 12), _arr(dq, 5), _arr(dG, 12), _arr(M, 9),
                                  float(J), float(mu), _arr(umf, 3), F))
    return list(F)


def point_flux_vjp(axis, viscous, q, G, Fbar, M, J, mu, umf):
    qb = (ctypes.c_double * 5)()
    gb = (ctypes.c_double * 12)()
    check(lib().cs_point_flux_vjp(axis, int(viscous), _arr(q, 5), _arr(G, 12), _arr(Fbar, 5), _arr(M, 9), float(J),
                                  float(mu), _arr(umf, 3), qb, gb))
    return list(qb), list(gb)


def point_prim(q):
    o = (ctypes.c_double * 4)()
    check(lib().cs_point_prim(_arr(q, 5), o))
    return list(o)


def point_prim_jvp(q, dq):
    o = (ctypes.c_double * 4)()
    check(lib().cs_point_prim_jvp(_arr(q, 5), _arr(dq, 5), o))
    return list(o)


def point_prim_vjp(q, pb):
    o = (ctypes.c_double * 5)()
    check(lib().cs_point_prim_vjp(_arr(q, 5), _arr(pb, 4), o))
    return list(o)


def _main(argv=None):
    """python -m compact_schemes_b200.adjoint --n N --steps K --every E: dJ/dq0
    of the kinetic energy of the N^3 Taylor-Green box (profiling driver)."""
    import argparse
    import torch
    from .solver import Solver, tgv_config, tgv_init
    p = argparse.ArgumentParser()
    p.add_argument("--n", type=int, default=64)
    p.add_argument("--steps", type=int, default=4)
    p.add_argument("--every", type=int, default=2)
    a = p.parse_args(argv)
    from compact_schemes_b200 import adjoint as A  # the package's classes, not __main__'s
    cfg = tgv_config(a.n, use_graph=False)
    s, adj = Solver(cfg), A.Adjoint(cfg)
    q0 = torch.empty(5 * a.n ** 3, dtype=torch.float64, device="cuda")
    tgv_init(q0, (a.n, a.n, a.n))
    qr, dts = q0.clone(), []
    for _ in range(a.steps):
        s.step(qr)
        dts.append(s.last_dt())
    g = torch.empty_like(q0)
    J = adj.gradient(q0, dts, a.every, g)
    print("J", J, "|dJ/dq0|", float(g.norm()))


if __name__ == "__main__":
    _main()
