"""compact_schemes_b200 -- B200 (sm_100a) compact-scheme hot path of EnricoDeg/compact_schemes.

Host-side mirror of the reference's C++ operator interface for the path
(``numerics_pc`` / ``numerics_rtc``, ``physics``, ``gcbc_go``) over the C ABI of
``libcompact_b200.so`` (declared in ``include/compact_b200.h``).  Device memory
and streams come from PyTorch; all numerics run in the library's CUDA kernels.
There is no CPU fallback: if the library or a GPU is missing, calls raise.

Arrays are torch CUDA tensors in the reference's SoA layout
``q[v*lmx + i + lxi*(j + let*k)]``.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libcompact_b200.so")

BC_NON_REFLECTIVE = 10
BC_WALL_INVISCID = 20
BC_WALL_VISCOUS = 25
BC_INTER_CURV = 30
BC_INTER_STRAIGHT = 35
BC_INTER_SUBDOMAINS = 40
BC_PERIODIC = 45

HALO_RECV = 0
HALO_SELF = 1

_lib = None


class CSError(RuntimeError):
    """Non-zero status from the C ABI (reference: print + exit, src/cuda/check.hpp:36-41)."""


class Dcomp(ctypes.Structure):
    """t_dcomp (src/common/data_types.hpp:33-39)."""
    _fields_ = [("lmx", ctypes.c_int), ("lxi", ctypes.c_int), ("let", ctypes.c_int),
                ("lze", ctypes.c_int)]

    @classmethod
    def of(cls, lxi, let, lze):
        return cls(lxi * let * lze, lxi, let, lze)


def lib():
    """Load libcompact_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise CSError("libcompact_b200.so not built: run `python -m compact_schemes_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        from . import _abi
        _abi.declare(L)
        _lib = L
    return _lib


def check(rc):
    if rc != 0:
        msg = lib().cs_last_error().decode(errors="replace")
        raise CSError("compact_b200 error %d: %s" % (rc, msg))
    return rc


def ptr(t):
    """Device pointer of a torch tensor (None -> NULL)."""
    if t is None:
        return None
    return ctypes.c_void_p(t.data_ptr())


def stream_ptr(stream=None):
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def nbc_array(nbc):
    arr = (ctypes.c_int * 3 * 2)()
    for f in range(2):
        for a in range(3):
            arr[f][a] = int(nbc[f][a])
    return arr


from .numerics import numerics_pc, numerics_rtc  # noqa: E402,F401
from .solver import Solver, SolverConfig, tgv_config, tgv_init  # noqa: E402,F401
from .physics import physics, physics_rtc, gcbc_go, thermo, rk_update, wall_condition_update  # noqa: E402,F401
from .ensemble import Ensemble, draw_boxes, ensemble_tgv  # noqa: E402,F401
from .adjoint import Adjoint  # noqa: E402,F401
from . import grid  # noqa: E402,F401
from .domdcomp import domdcomp, mpigo as mpigo_dist, mpigo_local  # noqa: E402,F401
