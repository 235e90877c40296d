"""Adjoint of the RHS and of the RK step on the GPU: transposed line solves
by the dot-product identity, tangents against finite differences of the
forward RHS, adjoints against tangents, and the checkpointed gradient of the
kinetic energy against central finite differences."""
import numpy as np
import pytest
import torch

import oracle as O

pytestmark = pytest.mark.gpu

MACH, RE = 0.1, 1600.0


def _setup(dims, nbc=None, viscous=True, seed=0):
    import compact_schemes_b200 as cs
    cfg = cs.tgv_config(None, dims=dims, mach=MACH, re=RE, nbc=nbc, viscous=viscous, use_graph=False)
    s = cs.Solver(cfg)
    a = cs.Adjoint(cfg)
    q = torch.from_numpy(O.tgv_init(dims, MACH, 1e-4, seed)).to("cuda:0")
    return cs, s, a, q


def _dot(x, y):
    return float((x * y).sum())


@pytest.mark.parametrize("nbc_code", ["periodic", "physical"])
@pytest.mark.parametrize("dims", [(24, 40, 20), (64, 16, 48)])
def test_transposed_derivative_dot_product(cuda, dims, nbc_code):
    import compact_schemes_b200 as cs
    b = cs.BC_PERIODIC if nbc_code == "periodic" else cs.BC_NON_REFLECTIVE
    _, _, a, _ = _setup(dims, nbc=[[b] * 3] * 2)
    g = torch.Generator(device="cuda:0").manual_seed(1)
    n = int(np.prod(dims))
    x = torch.randn(2 * n, dtype=torch.float64, device="cuda:0", generator=g)
    y = torch.randn(2 * n, dtype=torch.float64, device="cuda:0", generator=g)
    for axis in range(3):
        Dx, DTy = torch.empty_like(x), torch.empty_like(y)
        a.deriv(axis, x, Dx, nfields=2)
        a.deriv(axis, y, DTy, nfields=2, transpose=True)
        lhs, rhs = _dot(y, Dx), _dot(DTy, x)
        assert abs(lhs - rhs) <= 1e-12 * float((y.abs() * Dx.abs()).sum()), (axis, lhs, rhs)


@pytest.mark.parametrize("nbc_code", ["periodic", "physical"])
@pytest.mark.parametrize("af", [0.0, 0.45, -0.3])
def test_transposed_filter_dot_product_and_forward(cuda, nbc_code, af):
    import compact_schemes_b200 as cs
    b = cs.BC_PERIODIC if nbc_code == "periodic" else cs.BC_NON_REFLECTIVE
    dims = (24, 40, 20)
    _, _, a, _ = _setup(dims, nbc=[[b] * 3] * 2)
    g = torch.Generator(device="cuda:0").manual_seed(8)
    n = int(np.prod(dims))
    x = torch.randn(n, dtype=torch.float64, device="cuda:0", generator=g)
    y = torch.randn(n, dtype=torch.float64, device="cuda:0", generator=g)
    nd = 1 if nbc_code == "periodic" else 0
    for axis in range(3):
        Fx, FTy = torch.empty_like(x), torch.empty_like(y)
        a.filter(axis, af, x, Fx)
        a.filter(axis, af, y, FTy, transpose=True)
        assert abs(_dot(y, Fx) - _dot(FTy, x)) <= 1e-12 * float((y.abs() * Fx.abs()).sum()), axis
        ref = O.filt(x.cpu().numpy(), dims, axis, nd, nd, alpha_f=af)
        assert np.abs(Fx.cpu().numpy() - ref).max() <= 1e-12 * np.abs(ref).max()


def test_tangent_derivative_matches_oracle(cuda):
    dims = (24, 40, 20)
    _, _, a, _ = _setup(dims)
    r = np.random.default_rng(2)
    f = r.standard_normal(int(np.prod(dims)))
    out = torch.empty(f.size, dtype=torch.float64, device="cuda:0")
    for axis in range(3):
        a.deriv(axis, torch.from_numpy(f).to("cuda:0"), out)
        ref = O.deriv(f, dims, axis, 1, 1)
        assert np.abs(out.cpu().numpy() - ref).max() <= 1e-12 * np.abs(ref).max()


@pytest.mark.parametrize("viscous", [True, False])
def test_rhs_tangent_matches_finite_differences(cuda, viscous):
    dims = (24, 20, 28)
    _, s, a, q = _setup(dims, viscous=viscous)
    g = torch.Generator(device="cuda:0").manual_seed(3)
    dq = torch.randn(q.shape, dtype=torch.float64, device="cuda:0", generator=g) * 1e-2
    eps = 1e-5
    rp, rm, t = torch.empty_like(q), torch.empty_like(q), torch.empty_like(q)
    s.rhs(q + eps * dq, rp)
    s.rhs(q - eps * dq, rm)
    a.rhs_jvp(q, dq, t)
    fd = (rp - rm) / (2 * eps)
    for m in range(5):
        e = (t.view(5, -1)[m] - fd.view(5, -1)[m]).abs().max() / fd.view(5, -1)[m].abs().max()
        assert e < 1e-6, (m, float(e))


@pytest.mark.parametrize("viscous", [True, False])
@pytest.mark.parametrize("nbc_code", ["periodic", "physical"])
def test_rhs_adjoint_dot_product(cuda, viscous, nbc_code):
    import compact_schemes_b200 as cs
    b = cs.BC_PERIODIC if nbc_code == "periodic" else cs.BC_NON_REFLECTIVE
    dims = (32, 24, 40)
    _, _, a, q = _setup(dims, nbc=[[b] * 3] * 2, viscous=viscous)
    g = torch.Generator(device="cuda:0").manual_seed(4)
    dq = torch.randn(q.shape, dtype=torch.float64, device="cuda:0", generator=g)
    lam = torch.randn(q.shape, dtype=torch.float64, device="cuda:0", generator=g)
    t, v = torch.empty_like(q), torch.empty_like(q)
    a.rhs_jvp(q, dq, t)
    a.rhs_vjp(q, lam, v)
    lhs, rhs = _dot(lam, t), _dot(v, dq)
    assert abs(lhs - rhs) <= 1e-12 * float((lam.abs() * t.abs()).sum())


def test_step_adjoint_dot_product_and_tangent(cuda):
    dims = (24, 32, 20)
    cs, s, a, q = _setup(dims)
    dt = 0.02
    st = [torch.empty_like(q) for _ in range(4)]
    a.stages(q, dt, st)
    g = torch.Generator(device="cuda:0").manual_seed(5)
    dq = torch.randn(q.shape, dtype=torch.float64, device="cuda:0", generator=g) * 1e-3
    lam = torch.randn(q.shape, dtype=torch.float64, device="cuda:0", generator=g)
    t, v = torch.empty_like(q), torch.empty_like(q)
    a.step_jvp(st, dt, dq, t)
    a.step_vjp(st, dt, lam, v)
    assert abs(_dot(lam, t) - _dot(v, dq)) <= 1e-12 * float((lam.abs() * t.abs()).sum())
    # tangent of the step against central differences of the forward step
    eps = 1e-5
    qp, qm = q + eps * dq, q - eps * dq
    s.step(qp, dt)
    s.step(qm, dt)
    fd = (qp - qm) / (2 * eps)
    assert float((t - fd).abs().max() / fd.abs().max()) < 1e-6


def _rho_grad(q0, lam):
    rho, u = q0.view(5, -1)[0], q0.view(5, -1)[1:4] / q0.view(5, -1)[0]
    lam = lam.view(5, -1)
    return lam[0] + (lam[1:4] * u).sum(0) + 0.5 * lam[4] * (u * u).sum(0)


def test_gradient_matches_central_differences_and_autograd(cuda):
    from adjoint_harness import KineticEnergyAfterSteps, primitives
    dims = (24, 24, 24)
    cs, s, a, q0 = _setup(dims)
    nsteps, every = 12, 5
    # frozen time steps: those of the CFL-stepped reference trajectory
    qr, dts = q0.clone(), []
    for _ in range(nsteps):
        s.step(qr, 0.0)
        dts.append(s.last_dt())
    rho0, u, p = primitives(q0)
    rho = rho0.clone().requires_grad_(True)
    J = KineticEnergyAfterSteps.apply(rho, u, p, s, a, dts, every)
    J.backward()
    grad = rho.grad
    g = torch.Generator(device="cuda:0").manual_seed(6)
    eps = 1e-6
    for _ in range(3):
        v = torch.randn(rho0.shape, dtype=torch.float64, device="cuda:0", generator=g)
        with torch.no_grad():
            jp = KineticEnergyAfterSteps.apply(rho0 + eps * v, u, p, s, a, dts, every)
            jm = KineticEnergyAfterSteps.apply(rho0 - eps * v, u, p, s, a, dts, every)
        fd = float(jp - jm) / (2 * eps)
        ad = float((grad * v).sum())
        assert abs(ad - fd) <= 1e-6 * abs(fd), (ad, fd)


def test_multi_step_dot_product(cuda):
    """<A^T y, x> = <y, A x> for the tangent A of 8 steps (checkpoint every 3)."""
    dims = (24, 20, 24)
    cs, s, a, q0 = _setup(dims)
    dts = [0.02 + 0.001 * k for k in range(8)]
    g = torch.Generator(device="cuda:0").manual_seed(7)
    x = torch.randn(q0.shape, dtype=torch.float64, device="cuda:0", generator=g)
    y = torch.randn(q0.shape, dtype=torch.float64, device="cuda:0", generator=g)
    st = [torch.empty_like(q0) for _ in range(4)]
    # tangent through all steps
    q, dx = q0.clone(), x.clone()
    for dt in dts:
        a.stages(q, dt, st)
        out = torch.empty_like(dx)
        a.step_jvp(st, dt, dx, out)
        dx = out
        s.step(q, dt)
    # adjoint backwards, recomputing the stage states
    traj, q = [], q0.clone()
    for dt in dts:
        traj.append(q.clone())
        s.step(q, dt)
    lam = y.clone()
    for k in reversed(range(len(dts))):
        a.stages(traj[k], dts[k], st)
        out = torch.empty_like(lam)
        a.step_vjp(st, dts[k], lam, out)
        lam = out
    lhs, rhs = _dot(y, dx), _dot(lam, x)
    assert abs(lhs - rhs) <= 1e-10 * abs(lhs)


@pytest.mark.parametrize("viscous", [True, False])
def test_gcbc_rhs_linearization(cuda, viscous):
    """Non-reflective x faces with the GCBC correction: tangent against central
    differences of the forward RHS (which applies the correction), adjoint
    against tangent."""
    import compact_schemes_b200 as cs
    nbc = [[cs.BC_NON_REFLECTIVE, cs.BC_PERIODIC, cs.BC_PERIODIC]] * 2
    dims = (32, 24, 20)
    cfg = cs.tgv_config(None, dims=dims, mach=MACH, re=RE, nbc=nbc, gcbc=True, viscous=viscous, use_graph=False)
    s, a = cs.Solver(cfg), cs.Adjoint(cfg)
    q = torch.from_numpy(O.tgv_init(dims, MACH, 1e-4, 9)).to("cuda:0")
    g = torch.Generator(device="cuda:0").manual_seed(10)
    dq = torch.randn(q.shape, dtype=torch.float64, device="cuda:0", generator=g) * 1e-2
    lam = torch.randn(q.shape, dtype=torch.float64, device="cuda:0", generator=g)
    eps = 1e-5
    rp, rm, t, v = (torch.empty_like(q) for _ in range(4))
    s.rhs(q + eps * dq, rp)
    s.rhs(q - eps * dq, rm)
    a.rhs_jvp(q, dq, t)
    fd = (rp - rm) / (2 * eps)
    for m in range(5):
        e = (t.view(5, -1)[m] - fd.view(5, -1)[m]).abs().max() / fd.view(5, -1)[m].abs().max()
        assert e < 1e-6, (m, float(e))
    a.rhs_vjp(q, lam, v)
    assert abs(_dot(lam, t) - _dot(v, dq)) <= 1e-12 * float((lam.abs() * t.abs()).sum())
