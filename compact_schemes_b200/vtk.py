"""Headless VTK output of a state (cs_vtk_write, the layout of io::go_vtk,
src/IO.hpp:108-159)."""
from __future__ import annotations

import ctypes

import numpy as np

from . import check, lib

GAMMA = 1.4


def write_state(path, q, dims, spacing=None, origin=(0.0, 0.0, 0.0)):
    """Write rho, u, v, w, p of the state q ([5 * lmx], numpy or torch) on a
    uniform grid as a legacy binary VTK structured grid."""
    if hasattr(q, "detach"):
        q = q.detach().cpu().numpy()
    lxi, let, lze = dims
    n = lxi * let * lze
    q = np.asarray(q, dtype=np.float64).reshape(5, n)
    h = spacing if spacing is not None else tuple(2 * np.pi / d for d in dims)
    k, j, i = np.meshgrid(np.arange(lze), np.arange(let), np.arange(lxi), indexing="ij")
    rho = q[0]
    u = q[1:4] / rho
    p = (GAMMA - 1.0) * (q[4] - 0.5 * rho * (u * u).sum(0))
    data = np.stack([origin[0] + h[0] * i.ravel(), origin[1] + h[1] * j.ravel(), origin[2] + h[2] * k.ravel(),
                     rho, u[0], u[1], u[2], p]).astype(np.float32)
    names = (ctypes.c_char_p * 5)(b"rho", b"u", b"v", b"w", b"p")
    check(lib().cs_vtk_write(str(path).encode(), lxi, let, lze, data.ctypes.data_as(ctypes.c_void_p), 8, names))


def read(path):
    """Minimal reader of the files write_state produces (tests)."""
    raw = open(path, "rb").read()
    out, pos = {}, 0

    def line():
        nonlocal pos
        e = raw.index(b"\n", pos)
        s = raw[pos:e].decode()
        pos = e + 1
        return s

    for _ in range(4):
        line()
    dims = tuple(int(x) for x in line().split()[1:])
    npts = int(line().split()[1])
    out["points"] = np.frombuffer(raw, ">f4", 3 * npts, pos).reshape(npts, 3)
    pos += 12 * npts
    while pos < len(raw):
        s = line()
        if not s or s.startswith("POINT_DATA"):
            continue
        name = s.split()[1]
        line()
        out[name] = np.frombuffer(raw, ">f4", npts, pos)
        pos += 4 * npts
    out["dims"] = dims
    return out
