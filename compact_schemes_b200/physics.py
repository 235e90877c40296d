"""physics / physics_rtc and gcbc_go: the reference's physics API over the C ABI.

Mirrors src/physics_base.hpp, src/physics_pc.hpp, src/physics_rtc.hpp and
src/gcbc.hpp (method names, argument meaning, buffer layout); fields are torch
CUDA tensors; errors raise CSError.  This is the compatibility path with
per-point metric arrays; ``Solver`` is the fused fast path.
"""
from __future__ import annotations

import ctypes

from . import Dcomp, check, lib, nbc_array, ptr, stream_ptr


class physics:  # noqa: N801 - reference class name
    """physics<EnableViscous, double> (src/physics_pc.hpp:54-257)."""

    def __init__(self, dcomp, enable_viscous=True):
        self.dcomp = dcomp if isinstance(dcomp, Dcomp) else Dcomp.of(*dcomp)
        self.enable_viscous = bool(enable_viscous)
        self._h = ctypes.c_void_p()
        check(lib().cs_physics_create(ctypes.byref(self._h), self.dcomp, int(enable_viscous)))
        self._umf = (0.0, 0.0, 0.0)
        self.dudtmf = (0.0, 0.0, 0.0)

    def close(self):
        if self._h:
            lib().cs_physics_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def umf(self):
        return self._umf

    @umf.setter
    def umf(self, v):
        self._umf = tuple(float(x) for x in v)
        check(lib().cs_physics_set_umf(self._h, (ctypes.c_double * 3)(*self._umf)))

    def init(self):
        """physics::init is empty in the reference (src/physics_pc.hpp:78-81)."""

    def buffers(self):
        """(buffer, buffer_deriv, stress tensor [6][lmx], heat fluxes [3][lmx]) device pointers."""
        b = [ctypes.c_void_p() for _ in range(4)]
        check(lib().cs_physics_buffers(self._h, *[ctypes.byref(x) for x in b]))
        return tuple(x.value for x in b)

    def calc_fluxes_pre(self, qa, pressure, de, xim, etm, zem, stream=None):
        check(lib().cs_calc_fluxes_pre(self._h, ptr(qa), ptr(pressure), ptr(de), ptr(xim), ptr(etm),
                                       ptr(zem), stream_ptr(stream)))

    def calc_fluxes(self, qa, pressure, de, xim, etm, zem, dcomp, mcd, numerics_instance,
                    streams=None):
        d = dcomp if isinstance(dcomp, Dcomp) else Dcomp.of(*dcomp)
        check(lib().cs_calc_fluxes(self._h, numerics_instance.handle, ptr(qa), ptr(pressure), ptr(de),
                                   ptr(xim), ptr(etm), ptr(zem), d, stream_ptr(streams)))

    def calc_viscous_shear_stress(self, de, ssk, xim, etm, zem, yaco, dcomp, mcd,
                                  numerics_instance, streams=None):
        d = dcomp if isinstance(dcomp, Dcomp) else Dcomp.of(*dcomp)
        check(lib().cs_calc_viscous_shear_stress(self._h, numerics_instance.handle, ptr(de), ptr(ssk),
                                                 ptr(xim), ptr(etm), ptr(zem), ptr(yaco), d,
                                                 stream_ptr(streams)))

    def calc_time_step(self, xim, etm, zem, de, yaco, ssk, cfl, size, stream=None):
        """Returns dte (the reference writes it through a pointer)."""
        v = ctypes.c_double()
        check(lib().cs_calc_time_step(self._h, ptr(xim), ptr(etm), ptr(zem), ptr(de), ptr(yaco),
                                      ptr(ssk), float(cfl), ctypes.byref(v), int(size),
                                      stream_ptr(stream)))
        return v.value

    def movef(self, dtko, dtk, timo):
        """Empty in the reference (src/physics_base.hpp:147-150); see rk_update."""


physics_rtc = physics


def wall_condition_update(q, npex, dims, nbc, umf=(0.0, 0.0, 0.0), stream=None):
    """wall_condition_update (src/gcbc.hpp:188-228) on a device state q [5*lmx]
    with the int32 wall mask npex [lmx] (0 = wall point)."""
    from . import Dcomp, nbc_array
    u = (ctypes.c_double * 3)(*[float(x) for x in umf])
    check(lib().cs_wall_condition_update(ptr(q), ptr(npex), u, Dcomp.of(*dims), nbc_array(nbc), stream_ptr(stream)))


def thermo(q, de, pressure, stream=None):
    check(lib().cs_thermo(ptr(q), ptr(de), ptr(pressure), pressure.numel(), stream_ptr(stream)))


def rk_update(qn, de, yaco, dtk, qout, stream=None):
    check(lib().cs_rk_update(ptr(qn), ptr(de), ptr(yaco), float(dtk), ptr(qout), yaco.numel(),
                             stream_ptr(stream)))


def gcbc_go(*args, **kw):
    """gcbc_go (src/gcbc.hpp:86-186).

    Reference signature: gcbc_go(drva_buffer, cm_buffer, drvb_buffer, qa, de,
    pressure, yaco, sbcc, umf, dudtmf, dcomp_info, dtwi, nbc, mcd) -- every
    face code (non-reflective, walls, curvilinear interfaces; cs_gcbc_apply);
    drva_buffer / drvb_buffer / cm_buffer are lists of 3 device pointers or
    tensors (None where unused).  Also gcbc_go(numerics_instance, cm, qa, de,
    pressure, yaco, sbcc, umf, dcomp, nbc) for non-reflective faces with drva
    taken from the numerics object (cs_gcbc_go)."""
    if hasattr(args[0], "handle"):
        return _gcbc_go_numerics(*args, **kw)
    return _gcbc_apply(*args, **kw)


def _addr(x):
    if x is None:
        return None
    return x if isinstance(x, int) else x.data_ptr()


def _gcbc_apply(drva_buffer, cm_buffer, drvb_buffer, qa, de, pressure, yaco, sbcc, umf, dudtmf, dcomp, dtwi, nbc,
                mcd=None, stream=None):
    d = dcomp if isinstance(dcomp, Dcomp) else Dcomp.of(*dcomp)
    arr = lambda xs: (ctypes.c_void_p * 3)(*[_addr(x) for x in xs])
    mc = nbc_array(mcd if mcd is not None else [[0] * 3, [0] * 3])
    check(lib().cs_gcbc_apply(arr(drva_buffer), arr(cm_buffer), arr(drvb_buffer), ptr(qa), ptr(de), ptr(pressure),
                              ptr(yaco), ptr(sbcc), (ctypes.c_double * 3)(*umf), (ctypes.c_double * 3)(*dudtmf), d,
                              float(dtwi), nbc_array(nbc), mc, stream_ptr(stream)))


def _gcbc_go_numerics(numerics_instance, cm, qa, de, pressure, yaco, sbcc, umf, dcomp, nbc, mcd=None,
                      stream=None):
    d = dcomp if isinstance(dcomp, Dcomp) else Dcomp.of(*dcomp)
    cms = (ctypes.c_void_p * 3)(*[None if c is None else c.data_ptr() for c in cm])
    check(lib().cs_gcbc_go(numerics_instance.handle, cms, ptr(qa), ptr(de), ptr(pressure), ptr(yaco),
                           ptr(sbcc), (ctypes.c_double * 3)(*umf), d, nbc_array(nbc),
                           stream_ptr(stream)))
