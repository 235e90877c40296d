"""numerics_pc / numerics_rtc: the reference's compact-derivative API over the C ABI.

Mirrors src/numerics_base.hpp, src/numerics_pc.hpp and src/numerics_rtc.hpp:
same method names and argument meaning; fields are torch CUDA tensors; errors
raise CSError instead of exiting.
"""
from __future__ import annotations

import ctypes

from . import Dcomp, check, lib, nbc_array, ptr, stream_ptr, HALO_RECV, HALO_SELF


class numerics_pc:  # noqa: N801 - reference class name
    """numerics_pc<double> (src/numerics_pc.hpp:42-290)."""

    def __init__(self, dcomp, nbc):
        self.dcomp = dcomp if isinstance(dcomp, Dcomp) else Dcomp.of(*dcomp)
        self._h = ctypes.c_void_p()
        check(lib().cs_numerics_create(ctypes.byref(self._h), self.dcomp, nbc_array(nbc)))
        nd = (ctypes.c_int * 3 * 2)()
        check(lib().cs_get_ndf(self._h, nd))
        self.ndf = [[nd[f][a] for a in range(3)] for f in range(2)]

    def close(self):
        if self._h:
            lib().cs_numerics_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def deriv_setup(self):
        check(lib().cs_deriv_setup(self._h))

    def coeffs(self):
        a, b = (ctypes.c_double * 16)(), (ctypes.c_double * 16)()
        check(lib().cs_get_coeffs(self._h, a, b))
        return list(a), list(b)

    def buffers(self, axis):
        """(drva, send, recv) device pointers of numerics_base (src/numerics_base.hpp:389-395)."""
        d, s, r = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
        check(lib().cs_get_buffers(self._h, axis, ctypes.byref(d), ctypes.byref(s), ctypes.byref(r)))
        return d.value, s.value, r.value

    def deriv1d(self, axis, infield, outfield, nstart, nend, dcomp, variable_id, stream=None,
                halo=HALO_RECV):
        """numerics_pc::deriv1d<Axis> (src/numerics_pc.hpp:74-119)."""
        self._deriv(axis, infield, outfield, nstart, nend, dcomp, variable_id, 0, 0, stream, halo)

    def deriv2d(self, axis, infield, outfield, nstart, nend, dcomp, variable_id, component_id,
                stream=None, halo=HALO_RECV):
        """numerics_pc::deriv2d<Axis>: component -> slot Axis (src/numerics_pc.hpp:121-168)."""
        self._deriv(axis, infield, outfield, nstart, nend, dcomp, variable_id, component_id, axis,
                    stream, halo)

    def _deriv(self, axis, infield, outfield, nstart, nend, dcomp, var, comp, slot, stream, halo):
        import torch
        d = dcomp if isinstance(dcomp, Dcomp) else Dcomp.of(*dcomp)
        if infield.dtype != outfield.dtype:
            raise TypeError("input and output dtypes differ")
        fn = lib().cs_deriv if infield.dtype == torch.float64 else lib().cs_deriv_f32
        if infield.dtype not in (torch.float64, torch.float32):
            raise TypeError("float64 or float32 fields only")
        check(fn(self._h, axis, ptr(infield), ptr(outfield), int(nstart), int(nend), d, var, comp,
                 slot, halo, stream_ptr(stream)))

    def fill_buffers(self, infield, m_lo, m_hi, nrt, dcomp, stream=None):
        """numerics_pc::fill_buffers<m_lo,m_hi> (src/numerics_pc.hpp:231-287)."""
        d = dcomp if isinstance(dcomp, Dcomp) else Dcomp.of(*dcomp)
        check(lib().cs_fill_buffers(self._h, ptr(infield), m_lo, m_hi, nrt, d, stream_ptr(stream)))

    def mpigo(self, dcomp, mcd, itag, variable_id, stream=None, sync=None):
        """Single-rank numerics_base::mpigo (src/numerics_base.hpp:119-180).

        The block is its own neighbour on every interface axis, so the exchange
        is a device copy: face 0 receives face 1's sums and vice versa.  `mcd`
        and `itag` are accepted for signature parity and ignored.
        """
        check(lib().cs_halo_exchange_self(self._h, variable_id, stream_ptr(stream)))

    def filter(self, axis, infield, outfield, alpha_f, dcomp, stream=None):
        d = dcomp if isinstance(dcomp, Dcomp) else Dcomp.of(*dcomp)
        check(lib().cs_filter(self._h, axis, ptr(infield), ptr(outfield), float(alpha_f), d,
                              stream_ptr(stream)))


class numerics_rtc(numerics_pc):  # noqa: N801
    """numerics_rtc<double> (src/numerics_rtc.hpp:42-423).

    The NVRTC ``*_compile`` steps are no-ops: kernels are compiled ahead of
    time for sm_100a.  deriv1d/deriv2d take the face flags from ndf as the
    compiled NSTART/NEND macros did.
    """

    def deriv1d_compile(self, axis, dcomp, nstart, nend):
        self._flags = getattr(self, "_flags", {})
        self._flags[axis] = (nstart, nend)

    deriv2d_compile = deriv1d_compile

    def fill_buffer_compile(self, axis, face):
        pass

    def deriv1d(self, axis, infield, outfield, dcomp, variable_id, stream=None, halo=HALO_RECV):
        ns, ne = getattr(self, "_flags", {}).get(axis, (self.ndf[0][axis], self.ndf[1][axis]))
        super().deriv1d(axis, infield, outfield, ns, ne, dcomp, variable_id, stream, halo)

    def deriv2d(self, axis, infield, outfield, dcomp, variable_id, component_id, stream=None,
                halo=HALO_RECV):
        ns, ne = getattr(self, "_flags", {}).get(axis, (self.ndf[0][axis], self.ndf[1][axis]))
        super().deriv2d(axis, infield, outfield, ns, ne, dcomp, variable_id, component_id, stream,
                        halo)


def line_tables(n, scheme=0, nstart=0, nend=0, alpha_f=0.0):
    """Host copy of the line-solver tables (introspection for tests / autotuning)."""
    import numpy as np
    meta = (ctypes.c_int * 7)()
    check(lib().cs_line_tables(n, scheme, nstart, nend, alpha_f, meta, None, 0))
    lt = meta[1]
    size = 7 * lt * 32 + 832 + 2
    buf = np.zeros(size)
    check(lib().cs_line_tables(n, scheme, nstart, nend, alpha_f, meta,
                               buf.ctypes.data_as(ctypes.c_void_p), size))
    tl = lt * 32
    names = ["fwd1", "fwd2", "bwd1", "bwd2", "rca", "rcc"]
    out = {k: buf[i * tl:(i + 1) * tl].reshape(lt, 32) for i, k in enumerate(names)}
    o = 6 * tl
    out["k1"] = buf[o:o + 384].reshape(6, 2, 32)
    out["k2"] = buf[o + 384:o + 768].reshape(6, 2, 32)
    out["invb"] = buf[o + 768:o + 832].reshape(2, 32)
    out["cycz"] = buf[o + 832:o + 832 + tl].reshape(lt, 32)
    out["s1"], out["s2"] = buf[-2], buf[-1]
    out.update(n=meta[0], lt=lt, p=meta[2], last_len=meta[3], cyclic=bool(meta[4]), pcr64=meta[5], pcr32=meta[6])
    return out
