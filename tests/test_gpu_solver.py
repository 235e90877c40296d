"""GPU parity of the fused RHS / RK pipeline against the FP64 oracle.

Tolerances: 1e-12 relative max-norm per RHS field,
1e-10 after 100 RK steps.  Relative max-norm of a field f:
max|f - f_oracle| / max|f_oracle|.
"""
import math

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

MACH, RE = 0.1, 1600.0
MU = MACH / RE


def relerr_fields(a, b, nf=5):
    a = a.reshape(nf, -1)
    b = b.reshape(nf, -1)
    return max(np.abs(a[i] - b[i]).max() / max(np.abs(b[i]).max(), 1e-300) for i in range(nf))


def rhs_err(a, b, scale):
    """RHS error per field relative to the size of the terms it sums:
    max|rhs - rhs_oracle| / max(sum_a |d_a F[m][a]|).  On a nearly
    incompressible flow the mass RHS is ~1e3 smaller than each axis term, so
    its own max-norm would measure the cancellation, not the kernels."""
    a = a.reshape(5, -1)
    b = b.reshape(5, -1)
    return max(np.abs(a[i] - b[i]).max() / scale[i] for i in range(5))


def solver(dims, **kw):
    import compact_schemes_b200 as cs
    return cs.Solver(cs.tgv_config(None, dims=dims, **kw))


def dev(x):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x)).to("cuda:0")


def test_tgv_init_matches_oracle(cuda):
    import torch
    import compact_schemes_b200 as cs
    dims = (32, 24, 20)
    q = torch.zeros(5 * int(np.prod(dims)), dtype=torch.float64, device=cuda)
    cs.tgv_init(q, dims, MACH, 1e-4, 0)
    torch.cuda.synchronize()
    ref = O.tgv_init(dims, MACH, 1e-4, 0)
    assert np.abs(q.cpu().numpy() - ref).max() < 1e-14


@pytest.mark.parametrize("dims", [(32, 24, 40), (48, 16, 20), (64, 64, 64)])
@pytest.mark.parametrize("viscous", [True, False])
def test_rhs_periodic(cuda, dims, viscous):
    import torch
    s = solver(dims, viscous=viscous)
    q = O.tgv_init(dims, MACH, 1e-4, 0)
    qd = dev(q)
    out = torch.zeros_like(qd)
    s.rhs(qd, out)
    torch.cuda.synchronize()
    ref, scale = O.rhs(q, MU, O.uniform_metrics(*dims), dims, [[1] * 3, [1] * 3],
                       viscous=viscous, with_scale=True)
    assert rhs_err(out.cpu().numpy(), ref, scale) < 1e-12


def test_rhs_random_state(cuda):
    """A non-smooth state exercises every term (all gradients, all fluxes)."""
    import torch
    dims = (24, 20, 18)
    rng = np.random.default_rng(7)
    n = int(np.prod(dims))
    rho = 1.0 + 0.1 * rng.uniform(-1, 1, n)
    u, v, w = (0.2 * rng.uniform(-1, 1, n) for _ in range(3))
    p = 1 / 1.4 + 0.05 * rng.uniform(-1, 1, n)
    q = np.concatenate([rho, rho * u, rho * v, rho * w, p / 0.4 + 0.5 * rho * (u * u + v * v + w * w)])
    s = solver(dims)
    out = torch.zeros(5 * n, dtype=torch.float64, device=cuda)
    s.rhs(dev(q), out)
    torch.cuda.synchronize()
    ref, scale = O.rhs(q, MU, O.uniform_metrics(*dims), dims, [[1] * 3, [1] * 3], with_scale=True)
    assert rhs_err(out.cpu().numpy(), ref, scale) < 1e-12
    assert relerr_fields(out.cpu().numpy(), ref) < 1e-12  # no cancellation on a random state


def test_rhs_nonreflective_x_with_gcbc(cuda):
    import torch
    dims = (40, 24, 16)
    nbc = [[10, 45, 45], [10, 45, 45]]
    s = solver(dims, nbc=nbc, gcbc=True)
    q = O.tgv_init(dims, 0.3, 1e-3, 1)
    n = int(np.prod(dims))
    out = torch.zeros(5 * n, dtype=torch.float64, device=cuda)
    s.rhs(dev(q), out)
    torch.cuda.synchronize()
    m = O.uniform_metrics(*dims)
    F = dims[1] * dims[2]
    drva = np.zeros(10 * F)
    ref, scale = O.rhs(q, MU, m, dims, [[0, 1, 1], [0, 1, 1]], drva_x=drva, with_scale=True)
    cm = np.zeros(6 * F)
    cm[:F] = 1.0
    cm[3 * F:4 * F] = 1.0
    sbcc = np.zeros(n)
    sbcc[::dims[0]] = 1.0 / m.c_yaco
    sbcc[dims[0] - 1::dims[0]] = 1.0 / m.c_yaco
    ungc = ref.copy()
    O.gcbc_x(ref, drva, cm, q, sbcc, m, dims, nbc)
    assert np.abs(ref - ungc).max() > 0  # the closure acts
    assert rhs_err(out.cpu().numpy(), ref, scale) < 1e-12


def test_rk_step_cfl_matches_oracle(cuda):
    import torch
    dims = (32, 32, 32)
    s = solver(dims, use_graph=False)
    q = O.tgv_init(dims, MACH, 1e-4, 0)
    qd = dev(q)
    s.step(qd, 0.0)
    torch.cuda.synchronize()
    dt_gpu = s.last_dt()
    qr = q.copy()
    dt = O.rk_step(qr, MU, O.uniform_metrics(*dims), dims, [[45] * 3, [45] * 3], cfl=0.5)
    assert abs(dt_gpu - dt) / dt < 1e-14
    # rho*w starts at zero, so its field-relative error is that of a tiny field
    assert relerr_fields(qd.cpu().numpy(), qr) < 1e-12


def test_graph_step_equals_eager(cuda):
    import torch
    dims = (32, 24, 20)
    q = O.tgv_init(dims, MACH, 1e-4, 3)
    a, b = dev(q), dev(q)
    s1, s2 = solver(dims, use_graph=False), solver(dims, use_graph=True)
    for _ in range(3):
        s1.step(a, 0.0)
        s2.step(b, 0.0)
    torch.cuda.synchronize()
    assert torch.equal(a, b)


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("dims,gcbc", [((64, 64, 64), False), ((96, 64, 80), False), ((64, 48, 32), True)])
def test_pipelined_schedule_bit_identical(cuda, dims, gcbc, precision):
    """The two-role (pipelined) passes do the one-phase passes' arithmetic in
    the same order: RHS and three RK steps agree bit for bit."""
    import torch
    import compact_schemes_b200 as cs
    from compact_schemes_b200.solver import SCHED_ONEPHASE, SCHED_PIPELINE
    nbc = [[cs.BC_NON_REFLECTIVE, cs.BC_PERIODIC, cs.BC_PERIODIC]] * 2 if gcbc else None
    q0 = O.tgv_init(dims, MACH, 1e-4, 5)
    outs = []
    for sched in (SCHED_ONEPHASE, SCHED_PIPELINE):
        s = solver(dims, use_graph=False, schedule=sched, precision=precision, nbc=nbc, gcbc=gcbc)
        q = dev(q0)
        r = torch.empty_like(q)
        s.rhs(q, r)
        for _ in range(3):
            s.step(q, 0.0)
        torch.cuda.synchronize()
        outs.append((r.view(torch.int64).clone(), q.view(torch.int64).clone()))
        s.close()
    assert torch.equal(outs[0][0], outs[1][0])
    assert torch.equal(outs[0][1], outs[1][1])


@pytest.mark.parametrize("dims,gcbc", [((64, 64, 64), False), ((96, 64, 80), False), ((64, 48, 32), True),
                                       ((40, 36, 300), False), ((42, 38, 21), False), ((36, 30, 18), True),
                                       ((48, 40, 1), False), ((64, 1, 1), False), ((200, 24, 20), True)])
def test_tma_schedule_bit_identical(cuda, dims, gcbc):
    """The TMA-staged gradient passes do the one-phase passes' arithmetic in
    the same order: RHS and three CFL-stepped RK steps agree bit for bit.
    The cases cover 300-point z lines (two boxes per line), y tiles that
    overhang the x extent (42 = 10 tiles of 4 + 2), x tiles that overhang the
    line count, two active axes and one, and GCBC x faces."""
    import torch
    import compact_schemes_b200 as cs
    from compact_schemes_b200.solver import SCHED_ONEPHASE, SCHED_TMA
    nbc = [[cs.BC_NON_REFLECTIVE, cs.BC_PERIODIC, cs.BC_PERIODIC]] * 2 if gcbc else None
    q0 = O.tgv_init(dims, MACH, 1e-4, 5)
    outs = []
    for sched in (SCHED_ONEPHASE, SCHED_TMA):
        s = solver(dims, use_graph=False, schedule=sched, nbc=nbc, gcbc=gcbc)
        if sched == SCHED_TMA:
            for a in range(3):
                if dims[a] > 1:
                    assert s.schedule()[(0, a)] == 1
        q = dev(q0)
        r = torch.empty_like(q)
        s.rhs(q, r)
        for _ in range(3):
            s.step(q, 0.0)
        torch.cuda.synchronize()
        s.last_dt()  # raises if a staging copy timed out
        outs.append((r.view(torch.int64).clone(), q.view(torch.int64).clone()))
        s.close()
    assert torch.equal(outs[0][0], outs[1][0])
    assert torch.equal(outs[0][1], outs[1][1])


@pytest.mark.parametrize("precision", [0, 1])
def test_autotuned_schedule_bit_identical(cuda, precision):
    """The autotuner only chooses among schedules that do the same arithmetic:
    after tuning, steps equal an untuned solver's bit for bit."""
    import torch
    dims = (96, 64, 80)
    q0 = O.tgv_init(dims, MACH, 1e-4, 12)
    a, b = dev(q0), dev(q0)
    s1, s2 = solver(dims, precision=precision), solver(dims, precision=precision)
    choice = s2.autotune(b, reps=1)
    assert set(choice.values()) <= {0, 1, 8, 16}
    assert torch.equal(b, dev(q0))  # tuning ran on a scratch copy
    for _ in range(2):
        s1.step(a)
        s2.step(b)
    torch.cuda.synchronize()
    assert torch.equal(a.view(torch.int64), b.view(torch.int64))


def test_100_steps_within_1e10(cuda):
    import torch
    dims = (32, 32, 32)
    q = O.tgv_init(dims, MACH, 1e-4, 0)
    qd = dev(q)
    s = solver(dims)
    m = O.uniform_metrics(*dims)
    nbc = [[45] * 3, [45] * 3]
    for _ in range(100):
        s.step(qd, 0.0)
        O.rk_step(q, MU, m, dims, nbc, cfl=0.5)
    torch.cuda.synchronize()
    assert relerr_fields(qd.cpu().numpy(), q) < 1e-10


def test_headline_rhs_256(cuda):
    """The 256^3 Taylor-Green configuration: RHS parity at full size.

    At this size the RHS of FP64 is limited by its own noise floor: the
    oracle against itself with every line solved bottom-up instead of
    top-down (exactly the same mathematics) already differs by ~1.7e-12 in
    the summed-term norm (rare last-bit flips of fluxes whose pressure part
    is ~1e5 larger than their variation, amplified ~N/(2 pi) by the
    derivative).  Parity means: within 1e-12, or within twice that floor.
    """
    import torch
    dims = (256, 256, 256)
    s = solver(dims)
    q = O.tgv_init(dims, MACH, 1e-4, 0)
    qd = dev(q)
    out = torch.empty_like(qd)
    s.rhs(qd, out)
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    del out, qd
    m = O.uniform_metrics(*dims)
    ref, scale = O.rhs(q, MU, m, dims, [[1] * 3, [1] * 3], with_scale=True)
    with O.reversed_solves():
        ref2 = O.rhs(q, MU, m, dims, [[1] * 3, [1] * 3])
    floor = rhs_err(ref2, ref, scale)
    err = rhs_err(got, ref, scale)
    assert err <= max(1e-12, 2.0 * floor), (err, floor)


@pytest.mark.parametrize("dims,gcbc", [((37, 29, 23), False), ((45, 19, 27), True)])
def test_odd_sizes_rk_steps_match_oracle(cuda, dims, gcbc):
    """Ragged lines: lengths that fill neither a warp's lanes nor their chunks."""
    import torch
    nbc = [[10, 45, 45], [10, 45, 45]] if gcbc else [[45] * 3, [45] * 3]
    s = solver(dims, use_graph=False, nbc=nbc, gcbc=gcbc)
    q = O.tgv_init(dims, 0.3 if gcbc else MACH, 1e-4, 2)
    qd = dev(q)
    qr = q.copy()
    dt = None
    for _ in range(3):
        s.step(qd, 0.0)
        dt = O.rk_step(qr, MU, O.uniform_metrics(*dims), dims, nbc, cfl=0.5, gcbc=gcbc)
    torch.cuda.synchronize()
    assert abs(s.last_dt() - dt) / dt < 1e-13
    got = qd.cpu().numpy().reshape(5, -1)
    ref = qr.reshape(5, -1)
    assert max(np.abs(got[m] - ref[m]).max() / np.abs(ref[m]).max() for m in (0, 1, 2, 4)) < 1e-12


def test_10_steps_128_match_oracle(cuda):
    """Ten CFL-stepped RK steps of the 128^3 Taylor-Green box (the headline
    configuration at half the resolution) against the oracle, within the
    1e-10 that the 100-step bar allows.  Every field is compared relative to
    its own maximum, except rho w, which starts at exactly 0 and is compared
    relative to the largest momentum component."""
    import torch
    dims = (128, 128, 128)
    q = O.tgv_init(dims, MACH, 1e-4, 0)
    qd = dev(q)
    s = solver(dims)
    m = O.uniform_metrics(*dims)
    nbc = [[45] * 3, [45] * 3]
    for _ in range(10):
        s.step(qd, 0.0)
        dt = O.rk_step(q, MU, m, dims, nbc, cfl=0.5)
    torch.cuda.synchronize()
    assert abs(s.last_dt() - dt) / dt < 1e-13
    got = qd.cpu().numpy().reshape(5, -1)
    ref = q.reshape(5, -1)
    err = {f: np.abs(got[f] - ref[f]).max() / np.abs(ref[f]).max() for f in (0, 1, 2, 4)}
    mmax = max(np.abs(ref[f]).max() for f in (1, 2, 3))
    err[3] = np.abs(got[3] - ref[3]).max() / mmax
    assert max(err.values()) < 1e-10, err


def _filter_state_oracle(q, dims, ndf, alpha_f):
    """The compact filter along x, then y, then z on each conserved field."""
    lmx = int(np.prod(dims))
    for m in range(5):
        f = q[m * lmx:(m + 1) * lmx]
        for a in range(3):
            f = O.filt(f, dims, a, ndf[a], ndf[a], alpha_f)
        q[m * lmx:(m + 1) * lmx] = f


@pytest.mark.parametrize("dims,gcbc", [((32, 24, 20), False), ((36, 24, 20), True)])
def test_filter_every_step_matches_oracle(cuda, dims, gcbc):
    """Filter in the time step (CS_FILTER_STEP): three CFL-stepped RK steps,
    each followed by the sixth-order filter (alpha_f 0.45) along x, y and z
    on all five conserved fields, against the oracle's RK step and filter at
    1e-12 (rho w, which starts at 0, relative to the largest momentum)."""
    import torch
    import compact_schemes_b200 as cs
    from compact_schemes_b200.solver import FILTER_STEP
    nbc = [[10, 45, 45], [10, 45, 45]] if gcbc else [[45] * 3, [45] * 3]
    ndf = [0, 1, 1] if gcbc else [1, 1, 1]
    s = solver(dims, use_graph=True, nbc=nbc, gcbc=gcbc, filter=FILTER_STEP, alpha_f=0.45)
    q = O.tgv_init(dims, 0.3 if gcbc else MACH, 1e-4, 3)
    qd = dev(q)
    for _ in range(3):
        s.step(qd, 0.0)
        dt = O.rk_step(q, MU, O.uniform_metrics(*dims), dims, nbc, cfl=0.5, gcbc=gcbc)
        _filter_state_oracle(q, dims, ndf, 0.45)
    torch.cuda.synchronize()
    assert abs(s.last_dt() - dt) / dt < 1e-13
    got = qd.cpu().numpy().reshape(5, -1)
    ref = q.reshape(5, -1)
    mmax = max(np.abs(ref[f]).max() for f in (1, 2, 3))
    err = [np.abs(got[f] - ref[f]).max() / (mmax if f == 3 else np.abs(ref[f]).max()) for f in range(5)]
    assert max(err) < 1e-12, err
    # the filter changed the state (against an unfiltered step)
    s2 = solver(dims, use_graph=False, nbc=nbc, gcbc=gcbc)
    q2 = dev(O.tgv_init(dims, 0.3 if gcbc else MACH, 1e-4, 3))
    for _ in range(3):
        s2.step(q2, 0.0)
    assert float((q2 - qd).abs().max()) > 0.0


def test_filter_every_stage_matches_oracle(cuda):
    """CS_FILTER_STAGE: the filter after each of the four RK stages, fixed dt."""
    import torch
    from compact_schemes_b200.solver import FILTER_STAGE
    dims = (32, 24, 20)
    nbc = [[45] * 3, [45] * 3]
    s = solver(dims, use_graph=False, filter=FILTER_STAGE, alpha_f=0.3)
    q = O.tgv_init(dims, MACH, 1e-4, 4)
    qd = dev(q)
    m = O.uniform_metrics(*dims)
    dt = 0.01
    for _ in range(2):
        s.step(qd, dt)
        qn = q.copy()
        qs = q.copy()
        for k in range(4):
            out = np.empty_like(q)
            O.rk_stage(qn, qs, out, k, dt, MU, m, dims, nbc)
            _filter_state_oracle(out, dims, [1, 1, 1], 0.3)
            qs = out
        q = qs
    torch.cuda.synchronize()
    got = qd.cpu().numpy().reshape(5, -1)
    ref = q.reshape(5, -1)
    mmax = max(np.abs(ref[f]).max() for f in (1, 2, 3))
    err = [np.abs(got[f] - ref[f]).max() / (mmax if f == 3 else np.abs(ref[f]).max()) for f in range(5)]
    assert max(err) < 1e-12, err


def test_filter_config_rejected_where_unsupported(cuda):
    import compact_schemes_b200 as cs
    from compact_schemes_b200.solver import FILTER_STAGE, FILTER_STEP
    with pytest.raises(cs.CSError):
        solver((32, 24, 20), filter=FILTER_STEP, alpha_f=0.7)
    with pytest.raises(cs.CSError):
        solver((32, 24, 20), filter=FILTER_STAGE, precision=1)
    with pytest.raises(cs.CSError):
        cs.Adjoint(cs.tgv_config(None, dims=(32, 24, 20), filter=FILTER_STEP))
