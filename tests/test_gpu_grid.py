"""GPU grid metrics (cs_grid_metrics) and the fused solver on per-point
metrics (cs_solver_set_metrics), against the FP64 oracle.

Tolerances: 1e-12 relative max-norm for the metrics and for one RK step or
RHS (RHS error relative to the size of the summed axis terms, as in the
uniform-grid tests), 1e-10 after 20 steps."""
import math

import numpy as np
import pytest

import oracle as O
from grid_util import block_grid, wavy_grid

pytestmark = pytest.mark.gpu

MACH, RE = 0.1, 1600.0
MU = MACH / RE
PER = [[O.BC_PERIODIC] * 3, [O.BC_PERIODIC] * 3]
GC = [[O.BC_NON_REFLECTIVE, O.BC_PERIODIC, O.BC_PERIODIC]] * 2


def dev(x):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x)).to("cuda:0")


def gpu_metrics(xyz, dims, nbc, period):
    import torch
    import compact_schemes_b200 as cs
    nm = cs.numerics_pc(dims, nbc)
    nm.deriv_setup()
    out = cs.grid.metrics(nm, dev(xyz), period)
    torch.cuda.synchronize()
    nm.close()
    return out


def relmax(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


@pytest.mark.parametrize("dims,nbc,periodic", [((32, 24, 20), PER, (True, True, True)),
                                               ((24, 20, 16), GC, (False, True, True)),
                                               ((40, 12, 9), [[O.BC_NON_REFLECTIVE] * 3] * 2, (False,) * 3)])
def test_grid_metrics_match_oracle(cuda, dims, nbc, periodic):
    xyz, period, _ = wavy_grid(dims, amp=0.12, periodic=periodic)
    got = gpu_metrics(xyz, dims, nbc, period)
    ref = O.grid_metrics(xyz, dims, nbc, period)._keep
    for g, r in zip(got, ref):
        assert relmax(g.cpu().numpy(), r) < 1e-12


def test_grid_generate_and_metrics_of_reference_block(cuda):
    import compact_schemes_b200 as cs
    dims = (20, 12, 10)
    xyz = cs.grid.generate(dims, 1.0, 3.0, 0.5, 0.4)
    ref = block_grid(dims, 1.0, 3.0, 0.5, 0.4)
    assert np.abs(xyz.cpu().numpy() - ref).max() < 1e-15
    nbc = [[O.BC_NON_REFLECTIVE] * 3] * 2
    got = gpu_metrics(ref, dims, nbc, None)
    want = O.grid_metrics(ref, dims, nbc)._keep
    for g, r in zip(got, want):
        assert np.abs(g.cpu().numpy() - r).max() <= 1e-12 * np.abs(r).max()


def test_grid_metrics_rejects_degenerate_grid(cuda):
    import compact_schemes_b200 as cs
    dims = (12, 10, 8)
    with pytest.raises(cs.CSError):
        gpu_metrics(np.zeros(3 * int(np.prod(dims))), dims, [[O.BC_NON_REFLECTIVE] * 3] * 2, None)


def curvilinear_solver(dims, nbc, periodic, gcbc=False, viscous=True, amp=0.12):
    import compact_schemes_b200 as cs
    xyz, period, _ = wavy_grid(dims, amp=amp, periodic=periodic)
    met = gpu_metrics(xyz, dims, nbc, period)
    s = cs.Solver(cs.tgv_config(None, dims=dims, mach=MACH, re=RE, nbc=nbc, gcbc=gcbc, viscous=viscous,
                                use_graph=False))
    s.set_metrics(*met)
    om = O.field_metrics(*(m.cpu().numpy() for m in met))
    return s, om


def ndf_of(nbc):
    return [[1 if b >= O.BC_INTER_STRAIGHT else 0 for b in f] for f in nbc]


@pytest.mark.parametrize("viscous", [True, False])
def test_curvilinear_rhs_matches_oracle(cuda, viscous):
    import torch
    dims = (32, 24, 20)
    s, om = curvilinear_solver(dims, PER, (True, True, True), viscous=viscous)
    q = O.tgv_init(dims, MACH, 1e-4, 0)
    out = torch.zeros(q.size, dtype=torch.float64, device=cuda)
    s.rhs(dev(q), out)
    torch.cuda.synchronize()
    ref, scale = O.rhs(q, MU, om, dims, ndf_of(PER), viscous=viscous, with_scale=True)
    err = max(np.abs(out.cpu().numpy().reshape(5, -1)[m] - ref.reshape(5, -1)[m]).max() / scale[m]
              for m in range(5))
    assert err < 1e-12


@pytest.mark.parametrize("nbc,periodic,gcbc", [(PER, (True, True, True), False),
                                               (GC, (False, True, True), True)])
def test_curvilinear_rk_steps_match_oracle(cuda, nbc, periodic, gcbc):
    import torch
    dims = (32, 24, 20)
    s, om = curvilinear_solver(dims, nbc, periodic, gcbc=gcbc)
    q0 = O.tgv_init(dims, 0.3 if gcbc else MACH, 1e-4, 0)
    q = dev(q0)
    ref = q0.copy()
    s.step(q)
    torch.cuda.synchronize()
    dt = O.rk_step(ref, MU, om, dims, nbc, cfl=0.5, gcbc=gcbc)
    assert abs(s.last_dt() - dt) <= 1e-14 * dt
    got = q.cpu().numpy().reshape(5, -1)
    r = ref.reshape(5, -1)
    # rho*w starts at 0 on the TGV and is excluded from the per-field norm
    assert max(relmax(got[m], r[m]) for m in (0, 1, 2, 4)) < 1e-12
    for _ in range(19):
        s.step(q, dt)
        O.rk_step(ref, MU, om, dims, nbc, dt=dt, gcbc=gcbc)
    torch.cuda.synchronize()
    got = q.cpu().numpy().reshape(5, -1)
    assert max(relmax(got[m], r[m]) for m in (0, 1, 2, 4)) < 1e-10


def test_uniform_metrics_as_arrays_match_uniform_solver(cuda):
    """Per-point arrays of a uniform grid reproduce the constant-metric path."""
    import torch
    import compact_schemes_b200 as cs
    dims = (32, 24, 20)
    s, _ = curvilinear_solver(dims, PER, (True, True, True), amp=0.0)
    u = cs.Solver(cs.tgv_config(None, dims=dims, mach=MACH, re=RE, use_graph=False))
    q0 = O.tgv_init(dims, MACH, 1e-4, 0)
    a, b = dev(q0), dev(q0)
    for _ in range(3):
        s.step(a)
        u.step(b)
    torch.cuda.synchronize()
    assert torch.equal(a, b) or relmax(a.cpu().numpy(), b.cpu().numpy()) < 1e-14


def test_set_metrics_validation(cuda):
    import torch
    import compact_schemes_b200 as cs
    dims = (16, 16, 16)
    n = 16 ** 3
    z = torch.ones(3 * n, dtype=torch.float64, device=cuda)
    y = torch.ones(n, dtype=torch.float64, device=cuda)
    s = cs.Solver(cs.tgv_config(None, dims=dims, use_graph=False))
    with pytest.raises(cs.CSError):
        s.set_metrics(z, z, None, y)
    m = cs.Solver(cs.tgv_config(None, dims=dims, use_graph=False, precision=cs.solver.PREC_MIXED))
    with pytest.raises(cs.CSError):
        m.set_metrics(z, z, z, y)
    p = cs.Solver(cs.tgv_config(None, dims=dims, use_graph=False, schedule=cs.solver.SCHED_PIPELINE))
    with pytest.raises(cs.CSError):
        p.set_metrics(z, z, z, y)
    s.set_metrics(z, z, z, y)
    s.set_metrics()
