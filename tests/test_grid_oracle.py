"""Oracle grid metrics (cross-product form with compact derivatives), CPU.

The reference generates coordinates only (grid::generate,
src/grid.hpp:89-213), so the metrics are pinned to exact answers instead:
a uniform grid gives the constant metrics exactly, a smooth wavy grid
converges to the analytic metrics at the scheme's sixth order, and on a grid
extruded along z the discrete metric identities hold to rounding."""
import math

import numpy as np

import oracle as O
from grid_util import analytic_metrics, block_grid, wavy_grid

PER = [[O.BC_PERIODIC] * 3, [O.BC_PERIODIC] * 3]


def test_uniform_periodic_grid_is_exact():
    dims = (24, 20, 16)
    xyz, period, _ = wavy_grid(dims, amp=0.0)
    m = O.grid_metrics(xyz, dims, PER, period)
    u = O.uniform_metrics(*dims)
    xim, etm, zem, yaco = m._keep
    n = np.prod(dims)
    # the ramp removes the coordinate's jump exactly; the constant coordinates
    # of the cross axes differentiate to rounding-level values
    s = u.c_xim[0]
    assert np.abs(xim[:n] - s).max() < 1e-15 * s and np.abs(xim[n:]).max() < 1e-14 * s
    assert np.abs(etm[n:2 * n] - u.c_etm[1]).max() < 1e-15 * s
    assert np.abs(zem[2 * n:] - u.c_zem[2]).max() < 1e-15 * s
    assert np.abs(yaco / u.c_yaco - 1).max() < 1e-14


def test_reference_block_grid():
    dims = (20, 12, 10)
    xyz = block_grid(dims, 1.0, 3.0, 0.5, 0.4)
    nbc = [[O.BC_NON_REFLECTIVE] * 3, [O.BC_NON_REFLECTIVE] * 3]
    xim, etm, zem, yaco = O.grid_metrics(xyz, dims, nbc)._keep
    hx, hy, hz = 4.0 / 19, 1.0 / 11, -0.4 / 9
    n = np.prod(dims)
    assert np.allclose(xim[:n], hy * hz, rtol=1e-13, atol=0) and np.abs(xim[n:]).max() < 1e-15
    assert np.allclose(etm[n:2 * n], hx * hz, rtol=1e-13, atol=0)
    assert np.allclose(zem[2 * n:], hx * hy, rtol=1e-13, atol=0)
    assert np.allclose(yaco, 1.0 / (hx * hy * hz), rtol=1e-13, atol=0)
    assert (yaco < 0).all()  # z decreases with k in the reference's block


def _err_vs_analytic(n, periodic, trim=0):
    dims = (n, n, n)
    xyz, period, r = wavy_grid(dims, amp=0.1, periodic=periodic)
    nbc = [[O.BC_PERIODIC if p else O.BC_NON_REFLECTIVE for p in periodic]] * 2
    got = O.grid_metrics(xyz, dims, nbc, period)._keep
    ref = analytic_metrics(r)
    sl = slice(trim, n - trim)

    def inner(a):
        return a.reshape(-1, n, n, n)[:, sl, sl, sl]
    return max(np.abs(inner(g) - inner(e)).max() / np.abs(e).max() for g, e in zip(got, ref))


def test_wavy_grid_converges_at_the_scheme_order():
    # physical closures on every axis: sixth order inside, the boundary
    # closures' lower order at the faces
    phys = (False, False, False)
    e1, e2 = _err_vs_analytic(24, phys, trim=4), _err_vs_analytic(48, phys, trim=8)
    assert e1 / e2 > 2 ** 5.5, (e1, e2)
    f1, f2 = _err_vs_analytic(24, phys), _err_vs_analytic(48, phys)
    assert f1 / f2 > 2 ** 3.5, (f1, f2)


def test_periodic_wavy_grid():
    # periodic axes: the ramp is removed before differentiating; the
    # reference's interface closure at the line ends bounds the accuracy
    # there (a ~1e-3 derivative error that does not shrink with n)
    e = _err_vs_analytic(32, (True, True, True))
    assert e < 1e-2, e
    e1, e2 = _err_vs_analytic(32, (True, True, True), trim=12), _err_vs_analytic(64, (True, True, True), trim=24)
    assert e2 < e1 / 2 ** 5, (e1, e2)


def test_metric_identities_on_extruded_grid():
    # x, y depend on (xi, eta) only and z = zeta: the cross-product metrics
    # satisfy sum_a D_a(metric_a) = 0 discretely, since the compact
    # derivatives along different axes commute
    dims = (24, 20, 12)
    lxi, let, lze = dims
    h = [2 * math.pi / n for n in dims]
    Z, Y, X = np.meshgrid(*(np.arange(n) * hh for n, hh in zip(dims[::-1], h[::-1])), indexing="ij")
    x = X + 0.15 * np.sin(Y) * np.cos(X)
    y = Y + 0.1 * np.sin(X + Y)
    xyz = np.concatenate([x.ravel(), y.ravel(), Z.ravel()])
    xim, etm, zem, _ = O.grid_metrics(xyz, dims, PER, np.diag([2 * math.pi] * 3))._keep
    n = lxi * let * lze
    for c in range(3):
        div = (O.deriv(np.ascontiguousarray(xim[c * n:(c + 1) * n]), dims, 0, 1, 1) +
               O.deriv(np.ascontiguousarray(etm[c * n:(c + 1) * n]), dims, 1, 1, 1) +
               O.deriv(np.ascontiguousarray(zem[c * n:(c + 1) * n]), dims, 2, 1, 1))
        scale = max(np.abs(xim).max(), np.abs(etm).max())
        assert np.abs(div).max() < 1e-14 * scale * 10, (c, np.abs(div).max())


def test_zero_volume_is_rejected():
    dims = (12, 10, 8)
    xyz = np.zeros(3 * np.prod(dims))
    try:
        O.grid_metrics(xyz, dims, [[O.BC_NON_REFLECTIVE] * 3] * 2)
    except ValueError:
        return
    raise AssertionError("a degenerate grid must be rejected")
