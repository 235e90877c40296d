"""Batched ensemble on the GPU: every box against its own per-box solver
(which the solver tests pin to the FP64 oracle) -- bit-identical where every
axis has more than 64 points, within rounding where an axis has 64 or fewer
(the ensemble solves those lines in 4-point chunks, the per-box solver in
2-point chunks) -- every tuning bit-identical to the default tuning, plus one
box against the oracle directly."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

BOXES = [((32, 48, 40), 0.1, 1600.0), ((64, 32, 32), 0.25, 500.0), ((48, 48, 48), 0.05, 3000.0),
         ((96, 32, 40), 0.2, 800.0), ((40, 128, 24), 0.15, 1200.0), ((96, 72, 80), 0.12, 1000.0)]
TOL = 1e-12  # per field; momenta relative to the largest momentum component


def _rel_errs(got, ref):
    g, r = got.view(5, -1), ref.view(5, -1)
    mom = max(r[m].abs().max().item() for m in (1, 2, 3))
    return [((g[m] - r[m]).abs().max().item() / (mom if m in (1, 2, 3) else r[m].abs().max().item()))
            for m in range(5)]


def _agrees(got, ref, dims):
    """Bit-identical when every axis has more than 64 points, else within TOL."""
    if min(dims) > 64:
        assert bool((got == ref).all()), (dims, _rel_errs(got, ref))
        return True
    errs = _rel_errs(got, ref)
    assert max(errs) < TOL, (dims, errs)
    return True


def _state(ens, boxes, seed0=0):
    import torch
    import compact_schemes_b200 as cs
    q = torch.zeros(ens.state_size(), dtype=torch.float64, device="cuda:0")
    for b, (dims, mach, _) in enumerate(boxes):
        cs.tgv_init(ens.box_view(q, b), dims, mach, 1e-4, seed0 + b)
    return q


def _per_box(boxes, q0, ens, steps, viscous=True, nbc=None):
    import torch
    import compact_schemes_b200 as cs
    outs, dts = [], []
    for b, (dims, mach, re) in enumerate(boxes):
        s = cs.Solver(cs.tgv_config(None, mach=mach, re=re, dims=dims, viscous=viscous, nbc=nbc))
        qb = ens.box_view(q0, b).clone()
        for _ in range(steps):
            s.step(qb)
        torch.cuda.synchronize()
        outs.append(qb)
        dts.append(s.last_dt())
        s.close()
    return outs, dts


@pytest.mark.parametrize("viscous", [True, False])
def test_ensemble_matches_per_box_solvers(cuda, viscous):
    import torch
    import compact_schemes_b200 as cs
    cfgs = cs.ensemble_tgv(BOXES, viscous=viscous)
    ens = cs.Ensemble(cfgs)
    q = _state(ens, BOXES)
    ref, dts = _per_box(BOXES, q, ens, 3, viscous=viscous)
    for _ in range(3):
        ens.step(q)
    edt = ens.last_dt()
    for b, (dims, _, _) in enumerate(BOXES):
        assert _agrees(ens.box_view(q, b), ref[b], dims), b
        assert edt[b] == dts[b] if min(dims) > 64 else abs(edt[b] - dts[b]) <= 1e-13 * dts[b]
    ens.close()


@pytest.mark.parametrize("tuning", [dict(window=0, tile=8, chunk=1), dict(window=2, tile=8, chunk=16),
                                    dict(window=1, tile=4, chunk=3), dict(window=3, tile=4, ctas_per_sm=1),
                                    dict(window=0, tile=8, chunk=16)])
def test_ensemble_tunings_bit_identical(cuda, tuning):
    import torch
    import compact_schemes_b200 as cs
    ens = cs.Ensemble(cs.ensemble_tgv(BOXES))
    q = _state(ens, BOXES, 7)
    q_default = q.clone()
    ref, _ = _per_box(BOXES, q, ens, 2)
    for _ in range(2):
        ens.step(q_default)
    ens.set_tuning(**tuning)
    for _ in range(2):
        ens.step(q)
    ens.last_dt()
    assert torch.equal(q, q_default)
    for b, (dims, _, _) in enumerate(BOXES):
        assert _agrees(ens.box_view(q, b), ref[b], dims), b
    ens.close()


def test_ensemble_physical_closures(cuda):
    import torch
    import compact_schemes_b200 as cs
    nbc = [[cs.BC_NON_REFLECTIVE] * 3] * 2
    boxes = BOXES[:3]
    cfgs = [cs.tgv_config(None, mach=m, re=r, dims=d, nbc=nbc) for d, m, r in boxes]
    ens = cs.Ensemble(cfgs)
    q = _state(ens, boxes, 3)
    ref, _ = _per_box(boxes, q, ens, 2, nbc=nbc)
    for _ in range(2):
        ens.step(q)
    ens.last_dt()
    for b, (dims, _, _) in enumerate(boxes):
        assert _agrees(ens.box_view(q, b), ref[b], dims), b


def test_ensemble_box_against_oracle(cuda):
    import compact_schemes_b200 as cs
    ens = cs.Ensemble(cs.ensemble_tgv(BOXES))
    q = _state(ens, BOXES, 11)
    b = 3
    dims, mach, re = BOXES[b]
    qo = ens.box_view(q, b).cpu().numpy().copy()
    ens.step(q)
    ens.last_dt()
    O.rk_step(qo, mach / re, O.uniform_metrics(*dims), dims, [[45] * 3, [45] * 3], cfl=0.5)
    got = ens.box_view(q, b).cpu().numpy().reshape(5, -1)
    ref = qo.reshape(5, -1)
    err = max(np.abs(got[i] - ref[i]).max() / np.abs(ref[i]).max() for i in range(5))
    assert err < 1e-12


@pytest.mark.parametrize("nbc_code", [45, 10])
def test_ensemble_ragged_short_lines_against_oracle(cuda, nbc_code):
    """Axes of up to 64 points that are not multiples of the 4-point chunk
    (last chunk of 2 or 3 points, 7 to 13 chunks): the half-warp solves of the
    ensemble against the FP64 oracle, periodic (45) and physical (10) closures."""
    import compact_schemes_b200 as cs
    boxes = [((50, 36, 27), 0.1, 1200.0), ((27, 62, 44), 0.2, 900.0)]
    nbc = [[nbc_code] * 3] * 2
    ens = cs.Ensemble([cs.tgv_config(None, mach=m, re=r, dims=d, nbc=nbc) for d, m, r in boxes])
    q = _state(ens, boxes, 13)
    qo = [ens.box_view(q, b).cpu().numpy().copy() for b in range(len(boxes))]
    ens.step(q)
    ens.last_dt()
    for b, (dims, mach, re) in enumerate(boxes):
        O.rk_step(qo[b], mach / re, O.uniform_metrics(*dims), dims, nbc, cfl=0.5)
        got = ens.box_view(q, b).cpu().numpy().reshape(5, -1)
        ref = qo[b].reshape(5, -1)
        mom = max(np.abs(ref[m]).max() for m in (1, 2, 3))
        err = max(np.abs(got[m] - ref[m]).max() / (mom if m in (1, 2, 3) else np.abs(ref[m]).max())
                  for m in range(5))
        assert err < 1e-12, (dims, err)
    ens.close()


def test_ensemble_autotune_keeps_state(cuda):
    import torch
    import compact_schemes_b200 as cs
    ens = cs.Ensemble(cs.ensemble_tgv(BOXES))
    q = _state(ens, BOXES)
    q0 = q.clone()
    best, ms = ens.autotune(q, reps=2)
    torch.cuda.synchronize()
    assert torch.equal(q, q0)
    assert ms > 0 and best["tile"] in (4, 8) and ens.tuning() == best
    ref, _ = _per_box(BOXES, q, ens, 1)
    ens.step(q)
    ens.last_dt()
    for b, (dims, _, _) in enumerate(BOXES):
        assert _agrees(ens.box_view(q, b), ref[b], dims), b


def test_ensemble_rejects_unsupported(cuda):
    import compact_schemes_b200 as cs
    with pytest.raises(cs.CSError, match="8..256"):
        cs.Ensemble(cs.ensemble_tgv([((4, 32, 32), 0.1, 1000.0)]))
    with pytest.raises(cs.CSError, match="FP64"):
        cs.Ensemble([cs.tgv_config(None, dims=(32, 32, 32), precision=1)])


def test_dependency_wait_timeout_returns_error_and_recovers(cuda):
    """Failure detection without a fault: every dependency wait is made
    unsatisfiable (it needs more finished items than the queue produces) and
    limited to 64 polls.  The stage kernels give up, record the item, skip
    the dependent items and return; the host sees CS_ERR_TIMEOUT.  With the
    default restored the same ensemble steps correctly again."""
    import torch
    import compact_schemes_b200 as cs
    boxes = BOXES[:2]
    ens = cs.Ensemble(cs.ensemble_tgv(boxes))
    q = _state(ens, boxes, 5)
    ens.set_wait(64, 1 << 20)
    ens.step(q)
    with pytest.raises(cs.CSError, match="ran out") as ei:
        ens.last_dt()
    assert "-6" in str(ei.value)
    ens.set_wait()
    q = _state(ens, boxes, 5)
    ref, dts = _per_box(boxes, q, ens, 2)
    for _ in range(2):
        ens.step(q)
    edt = ens.last_dt()
    for b, (dims, _, _) in enumerate(boxes):
        assert abs(edt[b] - dts[b]) <= 1e-13 * dts[b]
        assert _agrees(ens.box_view(q, b), ref[b], dims), b
    ens.close()
