"""Pointwise linearizations of the flux and the primitives (host side, no
GPU): tangents against central finite differences of the forward pointwise
functions, adjoints against the tangents by the dot-product identity."""
import numpy as np
import pytest

from compact_schemes_b200 import adjoint as A


def _case(seed):
    r = np.random.default_rng(seed)
    rho = 1.0 + 0.1 * r.uniform(-1, 1)
    u = 0.2 * r.uniform(-1, 1, 3)
    p = 1.0 / 1.4 * (1.0 + 0.1 * r.uniform(-1, 1))
    q = np.array([rho, *(rho * u), p / 0.4 + 0.5 * rho * u @ u])
    G = 0.3 * r.standard_normal(12)
    M = 0.02 * r.standard_normal(9) + np.diag([0.03, 0.025, 0.035]).ravel()  # non-diagonal metrics
    umf = 0.05 * r.standard_normal(3)
    return r, q, G, M, 2.5e4, 6.25e-5, umf


@pytest.mark.parametrize("viscous", [True, False])
@pytest.mark.parametrize("axis", [0, 1, 2])
@pytest.mark.parametrize("seed", [0, 1, 2])
def test_flux_tangent_matches_central_differences(viscous, axis, seed):
    r, q, G, M, J, mu, umf = _case(seed)
    dq = r.standard_normal(5) * np.array([0.1, 0.1, 0.1, 0.1, 0.3])
    dG = r.standard_normal(12)
    eps = 1e-6
    fp = np.array(A.point_flux(axis, viscous, q + eps * dq, G + eps * dG, M, J, mu, umf))
    fm = np.array(A.point_flux(axis, viscous, q - eps * dq, G - eps * dG, M, J, mu, umf))
    fd = (fp - fm) / (2 * eps)
    t = np.array(A.point_flux_jvp(axis, viscous, q, G, dq, dG, M, J, mu, umf))
    assert np.abs(t - fd).max() <= 1e-7 * max(np.abs(fd).max(), 1e-30)


@pytest.mark.parametrize("viscous", [True, False])
@pytest.mark.parametrize("axis", [0, 1, 2])
@pytest.mark.parametrize("seed", [3, 4])
def test_flux_adjoint_is_transpose_of_tangent(viscous, axis, seed):
    r, q, G, M, J, mu, umf = _case(seed)
    dq, dG, fb = r.standard_normal(5), r.standard_normal(12), r.standard_normal(5)
    t = np.array(A.point_flux_jvp(axis, viscous, q, G, dq, dG, M, J, mu, umf))
    qb, gb = A.point_flux_vjp(axis, viscous, q, G, fb, M, J, mu, umf)
    lhs = fb @ t
    rhs = np.array(qb) @ dq + np.array(gb) @ dG
    assert abs(lhs - rhs) <= 1e-13 * (abs(fb) @ abs(t) + 1e-300)
    if not viscous:
        assert np.all(np.array(gb) == 0.0)


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_primitive_linearizations(seed):
    r, q, *_ = _case(seed)
    dq = r.standard_normal(5)
    eps = 1e-6
    fd = (np.array(A.point_prim(q + eps * dq)) - np.array(A.point_prim(q - eps * dq))) / (2 * eps)
    t = np.array(A.point_prim_jvp(q, dq))
    assert np.abs(t - fd).max() <= 1e-7 * np.abs(fd).max()
    pb = r.standard_normal(4)
    qb = np.array(A.point_prim_vjp(q, pb))
    assert abs(pb @ t - qb @ dq) <= 1e-13 * (abs(pb) @ abs(t))
