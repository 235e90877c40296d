"""Seeded smooth curvilinear test grids (numpy, SoA x, y, z of [3*lmx])."""
import math

import numpy as np


def axis_coords(n, periodic, length=2 * math.pi):
    """Index coordinate of one axis: n points over a period, or n points
    spanning [0, length] on a non-periodic axis."""
    h = length / n if periodic else length / (n - 1)
    return np.arange(n) * h, h


def wavy_grid(dims, amp=0.1, periodic=(True, True, True), length=2 * math.pi):
    """x = xi + A sin(eta) sin(zeta), y = eta + A sin(zeta) sin(xi),
    z = zeta + A sin(xi) sin(eta).  Returns (xyz, period, analytic index
    derivatives r[a][c] = d c / d i_a as arrays of lmx)."""
    lxi, let, lze = dims
    (xs, hx), (ys, hy), (zs, hz) = (axis_coords(n, p, length) for n, p in zip(dims, periodic))
    Z, Y, X = np.meshgrid(zs, ys, xs, indexing="ij")
    X, Y, Z = X.ravel(), Y.ravel(), Z.ravel()
    x = X + amp * np.sin(Y) * np.sin(Z)
    y = Y + amp * np.sin(Z) * np.sin(X)
    z = Z + amp * np.sin(X) * np.sin(Y)
    xyz = np.concatenate([x, y, z])
    period = np.diag([length if p else 0.0 for p in periodic])
    one = np.ones_like(X)
    d = [[one, amp * np.sin(Z) * np.cos(X), amp * np.cos(X) * np.sin(Y)],
         [amp * np.cos(Y) * np.sin(Z), one, amp * np.sin(X) * np.cos(Y)],
         [amp * np.sin(Y) * np.cos(Z), amp * np.cos(Z) * np.sin(X), one]]
    h = (hx, hy, hz)
    r = [[d[a][c] * h[a] for c in range(3)] for a in range(3)]
    return xyz, period, r


def analytic_metrics(r):
    """Cross-product metrics and Jacobian from index derivatives r[a][c]."""
    def cross(p, q):
        return [p[1] * q[2] - p[2] * q[1], p[2] * q[0] - p[0] * q[2], p[0] * q[1] - p[1] * q[0]]
    xim, etm, zem = cross(r[1], r[2]), cross(r[2], r[0]), cross(r[0], r[1])
    vol = r[0][0] * xim[0] + r[0][1] * xim[1] + r[0][2] * xim[2]
    return np.concatenate(xim), np.concatenate(etm), np.concatenate(zem), 1.0 / vol


def block_grid(dims, doml0, doml1, domh, span):
    """The Cartesian block of grid::generate (src/grid.hpp:89-213) for one rank."""
    lxi, let, lze = dims
    i, j, k = np.arange(lxi), np.arange(let), np.arange(lze)
    x = -doml0 + i * ((doml1 + doml0) / (lxi - 1))
    y = -domh + j * (2.0 * domh / (let - 1))
    z = span * ((lze - 1 - k) / (lze - 1) - 0.5)
    K, J, I = np.meshgrid(k, j, i, indexing="ij")
    return np.concatenate([x[I].ravel(), y[J].ravel(), z[K].ravel()])
