"""Mixed-precision form: FP32 fluxes and line solves (FP64 right-hand sides,
an optional FP64-residual refinement sweep), FP64 state, RK accumulation and
thermodynamics.  Precision 2 (CS_PREC_MIXED_F32) also evaluates the fluxes
and the interior right-hand sides in FP32 on axes whose lines have uniform
chunk factors, keeping the closure rows in FP64.

Target: relative state error <= 1e-6 per field after 100 RK steps
against the FP64 path.  Relative error of a field f: max|f - f64| / max|f64|.
rho*w starts at exactly zero in the Taylor-Green state, so its relative error
is measured against a field that is small throughout and gets a looser bound.
"""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu
MACH, RE = 0.1, 1600.0
MU = MACH / RE


def per_field(a, b, n):
    return [float((a[i * n:(i + 1) * n] - b[i * n:(i + 1) * n]).abs().max() /
                  b[i * n:(i + 1) * n].abs().max()) for i in range(5)]


def make(dims, precision, **kw):
    import compact_schemes_b200 as cs
    return cs.Solver(cs.tgv_config(None, dims=dims, precision=precision, **kw))


@pytest.mark.parametrize("prec,refine,dims,xphys", [(1, 1, (48, 40, 32), 0), (1, 0, (48, 40, 32), 0),
                                                     (1, 2, (48, 40, 32), 0), (2, 0, (48, 40, 32), 0),
                                                     (2, 0, (50, 33, 36), 0), (2, 1, (48, 40, 32), 0),
                                                     (2, 1, (50, 33, 36), 0), (2, 0, (36, 28, 20), 1),
                                                     (2, 1, (36, 28, 20), 1), (1, 0, (36, 28, 20), 1)])
def test_mixed_rhs_vs_oracle(cuda, prec, refine, dims, xphys):
    """Mixed RHS against the FP64 oracle, relative to the size of the summed terms
    (33-point lines are not a multiple of their chunk: that axis runs as precision 1).
    xphys: physical (non-reflective, no characteristic correction) closures on
    the x faces; 36-point x lines have uniform 2-row chunk factors but no
    interface closure, so they must run the table form."""
    import torch
    import compact_schemes_b200 as cs
    q = O.tgv_init(dims, MACH, 1e-4, 0)
    ndf = [[0 if xphys else 1, 1, 1]] * 2
    ref, scale = O.rhs(q, MU, O.uniform_metrics(*dims), dims, ndf, with_scale=True)
    nbc = [[cs.BC_NON_REFLECTIVE, cs.BC_PERIODIC, cs.BC_PERIODIC]] * 2 if xphys else None
    s = make(dims, prec, refine=refine, nbc=nbc)
    out = torch.zeros(q.size, dtype=torch.float64, device="cuda")
    s.rhs(torch.from_numpy(q).cuda(), out)
    torch.cuda.synchronize()
    got = out.cpu().numpy().reshape(5, -1)
    err = max(np.abs(got[i] - ref.reshape(5, -1)[i]).max() / scale[i] for i in range(5))
    assert err < 2e-6, err


@pytest.mark.parametrize("prec,refine", [(1, 0), (1, 1), (1, 2), (2, 0), (2, 1)])
def test_mixed_100_steps_within_1e6(cuda, prec, refine):
    import torch
    import compact_schemes_b200 as cs
    dims = (64, 64, 64)
    n = 64 ** 3
    q0 = torch.empty(5 * n, dtype=torch.float64, device="cuda")
    cs.tgv_init(q0, dims, MACH, 1e-4, 0)
    qp, qm = q0.clone(), q0.clone()
    sp, sm = make(dims, 0), make(dims, prec, refine=refine)
    for _ in range(100):
        sp.step(qp, 0.0)
        sm.step(qm, 0.0)
    torch.cuda.synchronize()
    errs = per_field(qm, qp, n)
    print("mixed %d (refine %d) vs FP64 after 100 steps at 64^3, per field:" % (prec, refine), errs)
    assert max(errs[:3] + errs[4:]) <= 1e-6, errs
    assert errs[3] <= 1e-5, errs


@pytest.mark.parametrize("prec", [1, 2])
def test_mixed_512_gcbc_100_steps(cuda, prec):
    """512^3 mixed form with non-reflective GCBC on the x faces, periodic y/z,
    100 RK steps; per-field error against the FP64 path (itself checked against
    the CPU oracle at <= 256^3)."""
    import torch
    import compact_schemes_b200 as cs
    dims = (512, 512, 512)
    n = 512 ** 3
    nbc = [[cs.BC_NON_REFLECTIVE, cs.BC_PERIODIC, cs.BC_PERIODIC]] * 2
    q0 = torch.empty(5 * n, dtype=torch.float64, device="cuda")
    cs.tgv_init(q0, dims, MACH, 1e-4, 0)
    qp = q0.clone()
    sp = make(dims, 0, nbc=nbc, gcbc=True)
    for _ in range(100):
        sp.step(qp, 0.0)
    sp.close()
    qm = q0
    sm = make(dims, prec, nbc=nbc, gcbc=True)
    for _ in range(100):
        sm.step(qm, 0.0)
    torch.cuda.synchronize()
    errs = per_field(qm, qp, n)
    print("512^3 GCBC mixed vs FP64 after 100 steps, per field:", errs)
    assert all(np.isfinite(errs))
    assert max(errs[:3] + errs[4:]) <= 1e-6, errs
    assert errs[3] <= 1e-4, errs


@pytest.mark.parametrize("prec,refine", [(1, 0), (1, 1), (2, 0), (2, 1)])
@pytest.mark.parametrize("dims,gcbc", [((64, 64, 64), False), ((40, 36, 300), False), ((36, 28, 20), True),
                                       ((48, 40, 1), False)])
def test_mixed_tma_schedule_bit_identical(cuda, prec, refine, dims, gcbc):
    """The TMA-staged gradient passes of the mixed form (every gradient pass
    but a step's first) do the one-phase passes' arithmetic: RHS and three
    CFL-stepped RK steps agree bit for bit, for the table solve with and
    without the refinement sweep and for the ChunkFactors solve with and
    without it.  The cases
    cover 300-point z lines (two boxes per line, 4-line tiles), y tiles that
    overhang the x extent (36 = 4 tiles of 8 + 4), two active axes and GCBC
    x faces (table solve along x, ChunkFactors along y and z)."""
    import torch
    import compact_schemes_b200 as cs
    from compact_schemes_b200.solver import SCHED_ONEPHASE, SCHED_TMA
    nbc = [[cs.BC_NON_REFLECTIVE, cs.BC_PERIODIC, cs.BC_PERIODIC]] * 2 if gcbc else None
    q0 = O.tgv_init(dims, MACH, 1e-4, 5)
    outs = []
    for sched in (SCHED_ONEPHASE, SCHED_TMA):
        s = make(dims, prec, refine=refine, use_graph=False, schedule=sched, nbc=nbc, gcbc=gcbc)
        if sched == SCHED_TMA:
            for a in range(3):
                if dims[a] > 1:
                    assert s.schedule()[(0, a)] == 1
        q = torch.from_numpy(q0.copy()).cuda()
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
