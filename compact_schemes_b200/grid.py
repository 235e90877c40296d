"""Grid coordinates and metrics.

``generate`` mirrors grid::generate (src/grid.hpp:89-213) for one block held
by one rank: the Cartesian block of the reference's grid section (doml0,
doml1, domh, span), point (i, j, k) at x = -doml0 + i (doml0 + doml1) / (lxi - 1),
y = -domh + j 2 domh / (let - 1), z = span ((lze - 1 - k) / (lze - 1) - 0.5).

``metrics`` fills the arrays the flux kernels read (xim, etm, zem =
J^-1 grad(xi_a), yaco = J), which the reference does not generate, with the
library's compact derivative (``cs_grid_metrics``).
"""
from __future__ import annotations

import ctypes

from . import check, lib, ptr, stream_ptr


def generate(dims, doml0, doml1, domh, span, device="cuda"):
    """Coordinates [3*lmx] (float64, SoA x, y, z) of the reference's block grid."""
    import torch
    lxi, let, lze = dims
    dt = torch.float64
    i = torch.arange(lxi, dtype=dt, device=device)
    j = torch.arange(let, dtype=dt, device=device)
    k = torch.arange(lze, dtype=dt, device=device)
    ra0 = (doml1 + doml0) / (lxi - 1)
    ra1 = 2.0 * domh / (let - 1)
    x = (-doml0 + i * ra0).view(1, 1, lxi).expand(lze, let, lxi)
    y = (-domh + j * ra1).view(1, let, 1).expand(lze, let, lxi)
    z = (span * ((lze - 1 - k) / (lze - 1) - 0.5)).view(lze, 1, 1).expand(lze, let, lxi)
    return torch.stack([x.reshape(-1), y.reshape(-1), z.reshape(-1)]).reshape(-1).contiguous()


def metrics(numerics, xyz, period=None, stream=None):
    """(xim, etm, zem, yaco) of the grid xyz [3*lmx] (torch CUDA float64).

    numerics: a set-up ``numerics_pc`` of the block (its closures are used).
    period[a][c]: the jump of coordinate c across axis a, used on axes with
    interface (periodic) closures, e.g. diag(Lx, Ly, Lz) for a periodic box.
    """
    import torch
    lmx = numerics.dcomp.lmx
    if xyz.numel() != 3 * lmx or xyz.dtype != torch.float64:
        raise ValueError("xyz must be float64 with 3*lmx elements")
    xim = torch.empty(3 * lmx, dtype=torch.float64, device=xyz.device)
    etm = torch.empty_like(xim)
    zem = torch.empty_like(xim)
    yaco = torch.empty(lmx, dtype=torch.float64, device=xyz.device)
    per = None
    if period is not None:
        per = (ctypes.c_double * 3 * 3)()
        for a in range(3):
            for c in range(3):
                per[a][c] = float(period[a][c])
    check(lib().cs_grid_metrics(numerics.handle, ptr(xyz), per if per is None else ctypes.byref(per),
                                ptr(xim), ptr(etm), ptr(zem), ptr(yaco), stream_ptr(stream)))
    return xim, etm, zem, yaco


def fourier_modes(seed=0, nmodes=8):
    """Modes [(A, kx, ky, kz, phi)] of the derivative-and-filter test field,
    drawn from MT19937-64 seeded `seed`, per mode in the order A, kx, ky, kz,
    phi, each from u = (top 53 bits of one draw) * 2^-53: A = 0.1 + 0.9 u,
    k = 1 + floor(8 u), phi = 2 pi u."""
    import math as _m
    from .ensemble import MT19937_64
    g = MT19937_64(seed)
    out = []
    for _ in range(nmodes):
        a = 0.1 + 0.9 * g.uniform()
        k = [1.0 + _m.floor(8.0 * g.uniform()) for _ in range(3)]
        out.append((a, k[0], k[1], k[2], 2.0 * _m.pi * g.uniform()))
    return out


def fourier_field(dims, seed=0, nmodes=8, device="cuda"):
    """f = sum_m A_m sin(2 pi (kx x + ky y + kz z) + phi_m) on the non-periodic
    unit cube, x = i / (lxi - 1) (and y, z alike), as a float64 tensor [lmx]
    in the reference's layout (x fastest)."""
    import math as _m
    import torch
    lxi, let, lze = dims
    dt = torch.float64
    x = (torch.arange(lxi, dtype=dt, device=device) * (1.0 / (lxi - 1))).view(1, 1, lxi)
    y = (torch.arange(let, dtype=dt, device=device) * (1.0 / (let - 1))).view(1, let, 1)
    z = (torch.arange(lze, dtype=dt, device=device) * (1.0 / (lze - 1))).view(lze, 1, 1)
    f = torch.zeros((lze, let, lxi), dtype=dt, device=device)
    for a, kx, ky, kz, ph in fourier_modes(seed, nmodes):
        f += a * torch.sin(2.0 * _m.pi * (kx * x + ky * y + kz * z) + ph)
    return f.reshape(-1)
