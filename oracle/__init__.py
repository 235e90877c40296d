"""FP64 CPU oracle for the compact-scheme hot path -- TEST INFRASTRUCTURE ONLY.

Thin ctypes wrapper over ``oracle/liboracle.so`` (built from oracle.cpp by
``make -C oracle``).  Only tests/, ``__graft_entry__.smoke()`` and bench.py's
cpu_baseline / reference arm use it, always as the checker or the timed CPU
baseline; the product path (``compact_schemes_b200``) never imports it.

All arrays are numpy float64 in the reference's SoA layout
``q[v*lmx + i + lxi*(j + let*k)]``.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

BC_NON_REFLECTIVE = 10
BC_WALL_INVISCID = 20
BC_WALL_VISCOUS = 25
BC_INTER_CURV = 30
BC_INTER_STRAIGHT = 35
BC_INTER_SUBDOMAINS = 40
BC_PERIODIC = 45


class Metrics(ctypes.Structure):
    _fields_ = [("xim", ctypes.c_void_p), ("etm", ctypes.c_void_p), ("zem", ctypes.c_void_p),
                ("yaco", ctypes.c_void_p), ("c_xim", ctypes.c_double * 3),
                ("c_etm", ctypes.c_double * 3), ("c_zem", ctypes.c_double * 3),
                ("c_yaco", ctypes.c_double)]


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            raise RuntimeError("oracle/liboracle.so missing: run `make -C oracle`")
        L = ctypes.CDLL(path)
        vp, i32, i64, f64 = ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_double
        L.or_deriv_setup.argtypes = [vp, vp]
        L.or_fill_buffer.argtypes = [vp, vp, i32, i32, i32, i32, i32, vp]
        L.or_deriv.argtypes = [vp, vp, i32, i32, i32, i32, i32, i32, vp, vp, i32, vp, vp]
        L.or_deriv.restype = i32
        L.or_deriv_line.argtypes = [vp, vp, i32, i32, i32, vp, vp, vp]
        L.or_deriv_line.restype = i32
        L.or_filter.argtypes = [vp, vp, i32, i32, i32, i32, i32, i32, f64]
        L.or_filter.restype = i32
        L.or_filter_line.argtypes = [vp, vp, i32, i32, i32, f64]
        L.or_filter_line.restype = i32
        L.or_fluxes_pre.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, i64]
        L.or_time_step.argtypes = [vp, vp, vp, vp, vp, vp, vp, f64, i64]
        L.or_time_step.restype = f64
        L.or_time_step_m.argtypes = [vp, Metrics, f64, vp, f64, i64]
        L.or_time_step_m.restype = f64
        L.or_thermo.argtypes = [vp, vp, vp, i64]
        L.or_viscous.argtypes = [vp, f64, Metrics, i32, i32, i32, vp, vp, vp, vp, vp]
        L.or_viscous.restype = i32
        L.or_rhs.argtypes = [vp, vp, f64, Metrics, vp, i32, i32, i32, vp, i32, vp]
        L.or_rhs.restype = i32
        L.or_rhs_scaled.argtypes = [vp, vp, f64, Metrics, vp, i32, i32, i32, vp, i32, vp, vp]
        L.or_rhs_scaled.restype = i32
        L.or_gcbc_x.argtypes = [vp, vp, vp, vp, vp, vp, f64, vp, i32, i32, i32, vp]
        L.or_gcbc_x.restype = i32
        L.or_rk_step.argtypes = [vp, f64, Metrics, vp, i32, i32, i32, vp, i32, f64, f64, i32]
        L.or_rk_step.restype = f64
        L.or_rk_stage.argtypes = [vp, vp, vp, i32, f64, f64, Metrics, vp, i32, i32, i32, vp, i32]
        L.or_rk_stage.restype = f64
        L.or_grid_metrics.argtypes = [vp, vp, i32, i32, i32, vp, vp, vp, vp, vp]
        L.or_grid_metrics.restype = i32
        L.or_tgv_init.argtypes = [vp, i32, i32, i32, f64, f64, ctypes.c_uint64]
        L.or_gcbc_go.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, i32, i32, i32, f64, vp]
        L.or_gcbc_go.restype = i32
        L.or_fourier_field.argtypes = [i32, i32, i32, ctypes.c_uint64, i32, vp, vp]
        L.or_noise.argtypes = [ctypes.c_uint64, ctypes.c_uint64]
        L.or_noise.restype = f64
        L.or_num_threads.restype = i32
        L.or_set_reversed_solves.argtypes = [i32]
        _LIB = L
    return _LIB


def _p(a):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"] and a.dtype == np.float64, (a.dtype, a.flags)
    return a.ctypes.data_as(ctypes.c_void_p)


def _ip(a):
    a = np.ascontiguousarray(a, dtype=np.int32)
    return a, a.ctypes.data_as(ctypes.c_void_p)


def deriv_setup():
    pbco, pbci = np.zeros(16), np.zeros(16)
    lib().or_deriv_setup(_p(pbco), _p(pbci))
    return pbco, pbci


def uniform_metrics(lxi, let, lze, box=(2 * np.pi, 2 * np.pi, 2 * np.pi), periodic=True):
    """Constant metrics of a uniform Cartesian grid: xim = J^-1 grad(xi), yaco = J."""
    hx, hy, hz = (b / (n if periodic else n - 1) for b, n in zip(box, (lxi, let, lze)))
    m = Metrics()
    m.xim = m.etm = m.zem = m.yaco = None
    m.c_xim[:] = (hy * hz, 0.0, 0.0)
    m.c_etm[:] = (0.0, hx * hz, 0.0)
    m.c_zem[:] = (0.0, 0.0, hx * hy)
    m.c_yaco = 1.0 / (hx * hy * hz)
    return m


def field_metrics(xim, etm, zem, yaco):
    m = Metrics()
    m.xim, m.etm, m.zem, m.yaco = _p(xim), _p(etm), _p(zem), _p(yaco)
    m._keep = (xim, etm, zem, yaco)
    return m


def fill_buffer(f, dims, axis, face, pbco):
    lxi, let, lze = dims
    F = (let * lze, lxi * lze, lxi * let)[axis]
    send = np.zeros(2 * F)
    lib().or_fill_buffer(_p(f), _p(send), lxi, let, lze, axis, face, _p(pbco))
    return send


def deriv(f, dims, axis, nstart=0, nend=0, recv=None, drva=None, var=0, coeffs=None):
    lxi, let, lze = dims
    pbco, pbci = coeffs if coeffs is not None else deriv_setup()
    out = np.empty_like(f)
    rc = lib().or_deriv(_p(f), _p(out), lxi, let, lze, axis, nstart, nend, _p(recv), _p(drva),
                        var, _p(pbco), _p(pbci))
    if rc:
        raise ValueError("or_deriv failed (%d)" % rc)
    return out


def deriv_line(f, nstart=0, nend=0, recv4=None, coeffs=None):
    pbco, pbci = coeffs if coeffs is not None else deriv_setup()
    f = np.ascontiguousarray(f, dtype=np.float64)
    x = np.empty_like(f)
    r4 = None if recv4 is None else np.ascontiguousarray(recv4, dtype=np.float64)
    rc = lib().or_deriv_line(_p(f), _p(x), f.size, nstart, nend, _p(r4), _p(pbco), _p(pbci))
    if rc:
        raise ValueError("or_deriv_line failed")
    return x


def filt(f, dims, axis, nstart=0, nend=0, alpha_f=0.45):
    lxi, let, lze = dims
    out = np.empty_like(f)
    if lib().or_filter(_p(f), _p(out), lxi, let, lze, axis, nstart, nend, alpha_f):
        raise ValueError("or_filter failed")
    return out


def filter_line(f, nstart=0, nend=0, alpha_f=0.45):
    f = np.ascontiguousarray(f, dtype=np.float64)
    x = np.empty_like(f)
    if lib().or_filter_line(_p(f), _p(x), f.size, nstart, nend, alpha_f):
        raise ValueError("or_filter_line failed")
    return x


def fluxes_pre(qa, p, de, xim, etm, zem, tau=None, heat=None, umf=(0.0, 0.0, 0.0)):
    n = p.size
    buf = np.zeros(15 * n)
    de = de.copy()
    u = np.asarray(umf, dtype=np.float64)
    lib().or_fluxes_pre(_p(buf), _p(qa), _p(p), _p(de), _p(xim), _p(etm), _p(zem), _p(tau),
                        _p(heat), _p(u), n)
    return buf, de


def time_step(xim, etm, zem, de, yaco, ssk, umf, cfl):
    u = np.asarray(umf, dtype=np.float64)
    return lib().or_time_step(_p(xim), _p(etm), _p(zem), _p(de), _p(yaco), _p(ssk), _p(u), cfl,
                              yaco.size)


def time_step_m(de, metrics, mu, umf, cfl):
    u = np.asarray(umf, dtype=np.float64)
    return lib().or_time_step_m(_p(de), metrics, mu, _p(u), cfl, de.size // 5)


def thermo(q):
    n = q.size // 5
    de, p = np.zeros(5 * n), np.zeros(n)
    lib().or_thermo(_p(q), _p(de), _p(p), n)
    return de, p


def viscous(de, mu, metrics, dims, ndf):
    lxi, let, lze = dims
    n = lxi * let * lze
    tau, heat = np.zeros(6 * n), np.zeros(3 * n)
    pbco, pbci = deriv_setup()
    nd, ndp = _ip(ndf)
    rc = lib().or_viscous(_p(de), mu, metrics, lxi, let, lze, ndp, _p(pbco), _p(pbci), _p(tau),
                          _p(heat))
    if rc:
        raise ValueError("or_viscous failed")
    return tau, heat


def rhs(q, mu, metrics, dims, ndf, viscous=True, umf=(0.0, 0.0, 0.0), drva_x=None,
        with_scale=False):
    """RHS de = sum_a d_a F[m][a]; with_scale also returns, per field, the max of
    sum_a |d_a F[m][a]| (the size of the summed terms)."""
    lxi, let, lze = dims
    out = np.zeros_like(q)
    nd, ndp = _ip(ndf)
    u = np.asarray(umf, dtype=np.float64)
    scale = np.zeros(5)
    rc = lib().or_rhs_scaled(_p(q), _p(out), mu, metrics, _p(u), lxi, let, lze, ndp, int(viscous),
                             _p(drva_x), _p(scale))
    if rc:
        raise ValueError("or_rhs failed")
    return (out, scale) if with_scale else out


def gcbc_x(rhs_arr, drva_x, cm, q, sbcc, metrics, dims, nbc, umf=(0.0, 0.0, 0.0)):
    lxi, let, lze = dims
    nb, nbp = _ip(nbc)
    u = np.asarray(umf, dtype=np.float64)
    yaco = None
    rc = lib().or_gcbc_x(_p(rhs_arr), _p(drva_x), _p(cm), _p(q), yaco, _p(sbcc), metrics.c_yaco,
                         _p(u), lxi, let, lze, nbp)
    if rc:
        raise ValueError("or_gcbc_x failed")


def gcbc_go(drva, cm, drvb, qa, de, p, yaco, sbcc, umf, dudtmf, dims, dtwi, nbc):
    """In place: drva[a] -> characteristic form, drvb[a] filled, de updated
    (or_gcbc_go).  drva, cm, drvb: lists of 3 float64 arrays (or None)."""
    lxi, let, lze = dims
    arr = lambda xs: (ctypes.c_void_p * 3)(*[None if x is None else x.ctypes.data for x in xs])
    nb, nbp = _ip(nbc)
    u = np.asarray(umf, dtype=np.float64)
    du = np.asarray(dudtmf, dtype=np.float64)
    rc = lib().or_gcbc_go(arr(drva), arr(cm), arr(drvb), _p(qa), _p(de), _p(p), _p(yaco), _p(sbcc), _p(u),
                          _p(du), lxi, let, lze, float(dtwi), nbp)
    if rc:
        raise ValueError("or_gcbc_go failed (%d)" % rc)


def rk_step(q, mu, metrics, dims, nbc, viscous=True, dt=0.0, cfl=0.5, gcbc=False,
            umf=(0.0, 0.0, 0.0)):
    """In-place: q <- q^{n+1}.  Returns dt used."""
    lxi, let, lze = dims
    nb, nbp = _ip(nbc)
    u = np.asarray(umf, dtype=np.float64)
    dt = lib().or_rk_step(_p(q), mu, metrics, _p(u), lxi, let, lze, nbp, int(viscous), dt, cfl,
                          int(gcbc))
    if dt < 0:
        raise ValueError("or_rk_step failed")
    return dt


def rk_stage(qn, qin, qout, k, dt, mu, metrics, dims, nbc, viscous=True, umf=(0.0, 0.0, 0.0)):
    lxi, let, lze = dims
    nb, nbp = _ip(nbc)
    u = np.asarray(umf, dtype=np.float64)
    r = lib().or_rk_stage(_p(qn), _p(qin), _p(qout), k, dt, mu, metrics, _p(u), lxi, let, lze, nbp,
                          int(viscous))
    if r < 0:
        raise ValueError("or_rk_stage failed")


def grid_metrics(xyz, dims, nbc, period=None):
    """Metrics of the grid with coordinates xyz ([3][lmx]); returns a Metrics
    with per-point arrays (xim, etm, zem: [3][lmx], yaco: [lmx])."""
    lxi, let, lze = dims
    n = lxi * let * lze
    xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1)
    per = np.zeros((3, 3)) if period is None else np.ascontiguousarray(period, dtype=np.float64)
    ndf = (np.asarray(nbc) >= BC_INTER_STRAIGHT).astype(np.int32)
    nd, ndp = _ip(ndf)
    xim, etm, zem, yaco = np.empty(3 * n), np.empty(3 * n), np.empty(3 * n), np.empty(n)
    rc = lib().or_grid_metrics(_p(xyz), _p(per), lxi, let, lze, ndp, _p(xim), _p(etm), _p(zem), _p(yaco))
    if rc:
        raise ValueError("or_grid_metrics failed (%d)" % rc)
    return field_metrics(xim, etm, zem, yaco)


def tgv_init(dims, mach=0.1, noise=1e-4, seed=0):
    lxi, let, lze = dims
    q = np.zeros(5 * lxi * let * lze)
    lib().or_tgv_init(_p(q), lxi, let, lze, mach, noise, seed)
    return q


def fourier_field(dims, seed=0, nmodes=8):
    """(modes [nmodes][5] = A, kx, ky, kz, phi; field) of or_fourier_field."""
    lxi, let, lze = dims
    modes = np.zeros(nmodes * 5)
    f = np.zeros(lxi * let * lze)
    lib().or_fourier_field(lxi, let, lze, seed, nmodes, _p(modes), _p(f))
    return modes.reshape(nmodes, 5), f


def noise(seed, index):
    return lib().or_noise(seed, index)


class reversed_solves:
    """Context: the oracle solves its lines bottom-up (noise-floor measurement)."""

    def __enter__(self):
        lib().or_set_reversed_solves(1)

    def __exit__(self, *exc):
        lib().or_set_reversed_solves(0)


def num_threads():
    return lib().or_num_threads()


def wall_update(q, npex, dims, nbc, umf=(0.0, 0.0, 0.0)):
    """In-place wall boundary state update (or_wall_update)."""
    lxi, let, lze = dims
    npex = np.ascontiguousarray(npex, dtype=np.int32)
    nb = (ctypes.c_int * 6)(*[int(nbc[f][a]) for f in range(2) for a in range(3)])
    u = (ctypes.c_double * 3)(*umf)
    lib().or_wall_update.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                     ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
    if lib().or_wall_update(_p(q), npex.ctypes.data_as(ctypes.c_void_p), u, lxi, let, lze, nb):
        raise ValueError("or_wall_update failed")
    return q
