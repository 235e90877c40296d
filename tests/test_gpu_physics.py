"""GPU parity of the reference-shaped physics path (drop-in API) against the oracle
and the reference's own CPU twins (tests/golden/reference_pins.npz)."""
import os
import subprocess

import numpy as np
import pytest

import oracle as O
from gpu_util import device_view

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
MU = 0.1 / 1600


def dev(x):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x, dtype=np.float64)).to("cuda:0")


def rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


@pytest.fixture(scope="module")
def gold():
    return np.load(os.path.join(ROOT, "tests", "golden", "reference_pins.npz"))


def test_fluxes_pre_against_reference_twin(cuda, gold):
    """tests/test_physics_serial.cu restated: the flux pre-compute on the reference's
    seeded inputs, vs its CPU twin (float) and vs the oracle (FP64, same operation order)."""
    import compact_schemes_b200 as cs
    g = {k: gold[k].astype(np.float64) for k in gold.files if k.startswith("flux_")}
    n = g["flux_p"].size
    ph = cs.physics((n, 1, 1), True)
    ph.umf = g["flux_umf"]
    _, _, tau, heat = ph.buffers()
    import torch
    device_view(tau, 6 * n).copy_(dev(g["flux_tau"]))
    device_view(heat, 3 * n).copy_(dev(g["flux_heat"]))
    de = dev(g["flux_de"])
    ph.calc_fluxes_pre(dev(g["flux_qa"]), dev(g["flux_p"]), de, dev(g["flux_xim"]), dev(g["flux_etm"]),
                       dev(g["flux_zem"]))
    torch.cuda.synchronize()
    b0, _, _, _ = ph.buffers()
    got = device_view(b0, 15 * n).cpu().numpy()
    assert rel(got, g["flux_buffer"]) < 1e-6          # reference twin is float32
    ref, de_ref = O.fluxes_pre(g["flux_qa"], g["flux_p"], g["flux_de"], g["flux_xim"], g["flux_etm"],
                               g["flux_zem"], g["flux_tau"], g["flux_heat"], g["flux_umf"])
    assert np.array_equal(got, ref)                   # same operations, same order
    assert np.array_equal(de.cpu().numpy(), de_ref)


def test_time_step_against_reference_twin(cuda, gold):
    """tests/test_physics.cu restated (single rank: the Allreduce is the identity)."""
    import compact_schemes_b200 as cs
    g = {k: gold[k].astype(np.float64) for k in gold.files if k.startswith("dt_")}
    n = g["dt_yaco"].size
    ph = cs.physics((n, 1, 1), False)
    ph.umf = g["dt_umf"]
    dte = ph.calc_time_step(dev(g["dt_xim"]), dev(g["dt_etm"]), dev(g["dt_zem"]), dev(g["dt_de"]),
                            dev(g["dt_yaco"]), dev(g["dt_ssk"]), float(gold["dt_cfl"]), n)
    assert abs(dte - float(gold["dt_result"])) / dte < 1e-6
    ref = O.time_step(g["dt_xim"], g["dt_etm"], g["dt_zem"], g["dt_de"], g["dt_yaco"], g["dt_ssk"],
                      g["dt_umf"], float(gold["dt_cfl"]))
    assert dte == ref


def metric_fields(dims, seed=3):
    """Smooth, non-constant metric arrays (xim, etm, zem [3][n], yaco [n])."""
    lxi, let, lze = dims
    n = lxi * let * lze
    i, j, k = np.meshgrid(np.arange(lxi), np.arange(let), np.arange(lze), indexing="ij")
    ph = (2 * np.pi * (i / lxi + 2 * j / let + k / lze)).transpose(2, 1, 0).ravel()
    h = 2 * np.pi / np.array(dims)
    xim = np.zeros(3 * n); etm = np.zeros(3 * n); zem = np.zeros(3 * n)
    xim[:n] = h[1] * h[2] * (1 + 0.05 * np.sin(ph)); xim[n:2 * n] = 0.01 * h[1] * h[2] * np.cos(ph)
    etm[n:2 * n] = h[0] * h[2] * (1 + 0.05 * np.cos(ph)); etm[2 * n:] = 0.01 * h[0] * h[2] * np.sin(ph)
    zem[2 * n:] = h[0] * h[1] * (1 - 0.05 * np.sin(ph)); zem[:n] = 0.01 * h[0] * h[1] * np.cos(2 * ph)
    yaco = 1.0 / (h[0] * h[1] * h[2]) * (1 + 0.03 * np.cos(ph))
    return xim, etm, zem, yaco


@pytest.mark.parametrize("dims,periodic", [((32, 24, 20), True), ((24, 20, 16), False)])
def test_viscous_and_fluxes_with_metric_arrays(cuda, dims, periodic):
    """physics::calc_viscous_shear_stress + calc_fluxes with per-point metrics vs the oracle RHS."""
    import torch
    import compact_schemes_b200 as cs
    b = cs.BC_PERIODIC if periodic else cs.BC_NON_REFLECTIVE
    nbc = [[b] * 3, [b] * 3]
    ndf = [[int(periodic)] * 3] * 2
    n = int(np.prod(dims))
    q = O.tgv_init(dims, 0.2, 1e-3, 5)
    xim, etm, zem, yaco = metric_fields(dims)
    m = O.field_metrics(xim, etm, zem, yaco)
    ref, scale = O.rhs(q, MU, m, dims, ndf, with_scale=True)

    nm = cs.numerics_pc(dims, nbc)
    nm.deriv_setup()
    ph = cs.physics(dims, True)
    qd, X, E, Z, Y = dev(q), dev(xim), dev(etm), dev(zem), dev(yaco)
    de = torch.zeros(5 * n, dtype=torch.float64, device="cuda")
    p = torch.zeros(n, dtype=torch.float64, device="cuda")
    ssk = torch.full((n,), MU, dtype=torch.float64, device="cuda")
    cs.thermo(qd, de, p)
    ph.calc_viscous_shear_stress(de, ssk, X, E, Z, Y, dims, None, nm)
    cs.thermo(qd, de, p)   # the viscous call leaves de0 = ssk, de4 = 2/3 div (as the reference)
    ph.calc_fluxes(qd, p, de, X, E, Z, dims, None, nm)
    torch.cuda.synchronize()
    got = de.cpu().numpy().reshape(5, n)
    err = max(np.abs(got[i] - ref.reshape(5, n)[i]).max() / scale[i] for i in range(5))
    assert err < 1e-12


def test_gcbc_go_x_faces(cuda):
    import torch
    import compact_schemes_b200 as cs
    dims = (40, 24, 16)
    n = int(np.prod(dims))
    nbc = [[10, 45, 45], [10, 45, 45]]
    q = O.tgv_init(dims, 0.3, 1e-3, 1)
    mm = O.uniform_metrics(*dims)
    F = dims[1] * dims[2]
    drva = np.zeros(10 * F)
    ref = O.rhs(q, MU, mm, dims, [[0, 1, 1], [0, 1, 1]], drva_x=drva)
    cm = np.zeros(6 * F); cm[:F] = 1.0; cm[3 * F:4 * F] = 1.0
    sbcc = np.zeros(n); sbcc[::dims[0]] = 1.0 / mm.c_yaco; sbcc[dims[0] - 1::dims[0]] = 1.0 / mm.c_yaco
    de_o, p_o = O.thermo(q)
    rhs_o = ref.copy()
    O.gcbc_x(rhs_o, drva, cm, q, sbcc, mm, dims, nbc)
    # device: same RHS and drva, then gcbc_go
    nm = cs.numerics_pc(dims, nbc)
    nm.deriv_setup()
    dp, _, _ = nm.buffers(0)
    device_view(dp, 10 * F).copy_(dev(drva))
    de = dev(ref)
    yaco = torch.full((n,), mm.c_yaco, dtype=torch.float64, device="cuda")
    cs.gcbc_go(nm, [dev(cm), None, None], dev(q), de, dev(p_o), yaco, dev(sbcc), (0.0, 0.0, 0.0), dims, nbc)
    torch.cuda.synchronize()
    got = de.cpu().numpy()
    corr_o, corr_g = rhs_o - ref, got - ref
    assert np.abs(corr_o).max() > 0
    assert np.abs(corr_g - corr_o).max() / np.abs(corr_o).max() < 1e-12


def test_dropin_cpp_demo_runs(cuda, tmp_path):
    from test_dropin_build import build_demo
    exe = build_demo(str(tmp_path / "dropin_demo"))
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and "PASS" in r.stdout, r.stdout + r.stderr


@pytest.mark.parametrize("nbc", [[[20, 45, 25], [45, 45, 20]], [[25, 20, 45], [20, 25, 25]]])
def test_wall_condition_update_matches_oracle(cuda, nbc):
    import torch
    import compact_schemes_b200 as cs
    dims = (12, 10, 9)
    n = int(np.prod(dims))
    r = np.random.default_rng(3)
    rho = 1.0 + 0.1 * r.uniform(-1, 1, n)
    m = 0.1 * r.standard_normal((3, n))
    E = 1.0 / (1.4 * 0.4) + 0.5 * (m * m).sum(0) / rho
    q = np.concatenate([rho, m.ravel(), E])
    npex = (r.uniform(size=n) > 0.4).astype(np.int32)
    umf = (0.03, -0.01, 0.02)
    ref = O.wall_update(q.copy(), npex, dims, nbc, umf)
    qd = torch.from_numpy(q).to(cuda)
    cs.wall_condition_update(qd, torch.from_numpy(npex).to(cuda), dims, nbc, umf)
    torch.cuda.synchronize()
    got = qd.cpu().numpy()
    assert np.abs(got - ref).max() <= 1e-14 * np.abs(ref).max()
    assert not np.array_equal(ref, q)  # some wall points changed


REF_GPU = os.path.join(ROOT, "oracle", "_ref", "libref_gpu.so")


@pytest.mark.skipif(not os.path.exists(REF_GPU), reason="reference kernels not built (make -C oracle ref)")
def test_fluxes_pre_against_reference_fp64_kernel(cuda):
    """The reference's own calc_fluxes_pre_compute_kernel<true,double>
    (src/cuda/kernels/physics.hpp:42-193), compiled for sm_100a from its
    sources, against cs_calc_fluxes_pre on the same FP64 inputs: a 64^3
    state, per-point metrics, stress tensor and heat flux, moving frame.
    1e-12 relative max-norm per flux component; the reference lets the
    compiler contract products into FMAs, so last bits differ."""
    import ctypes
    import torch
    import compact_schemes_b200 as cs
    R = ctypes.CDLL(REF_GPU)
    vp = ctypes.c_void_p
    R.ref_gpu_fluxes_pre.argtypes = [vp] * 9 + [ctypes.c_double] * 3 + [ctypes.c_uint, vp, vp]
    dims = (64, 64, 64)
    n = int(np.prod(dims))
    rng = np.random.default_rng(7)
    xim, etm, zem, _ = metric_fields(dims)
    rho = 1.0 + 0.1 * rng.random(n)
    vel = 0.3 * rng.standard_normal((3, n))
    p = 1 / 1.4 + 0.05 * rng.random(n)
    qa = np.concatenate([rho, rho * vel[0], rho * vel[1], rho * vel[2], p / 0.4 + 0.5 * rho * (vel ** 2).sum(0)])
    de = np.concatenate([1 / rho, vel[0], vel[1], vel[2], 1.4 * p / rho])
    tau = 1e-3 * rng.standard_normal(6 * n)
    heat = 1e-3 * rng.standard_normal(3 * n)
    umf = (0.05, -0.02, 0.01)
    ph = cs.physics(dims, True)
    ph.umf = umf
    b0, _, dtau, dheat = ph.buffers()
    device_view(dtau, 6 * n).copy_(dev(tau))
    device_view(dheat, 3 * n).copy_(dev(heat))
    d_de = dev(de)
    args = [dev(a) for a in (qa, p, xim, etm, zem)]
    ph.calc_fluxes_pre(args[0], args[1], d_de, args[2], args[3], args[4])
    torch.cuda.synchronize()
    ours = device_view(b0, 15 * n).cpu().numpy().reshape(15, n)
    ours_de4 = d_de.cpu().numpy()[4 * n:]
    theirs = torch.zeros(15 * n, dtype=torch.float64, device=cuda)
    r_de = dev(de)
    structs = torch.zeros(16, dtype=torch.float64, device=cuda)
    rc = R.ref_gpu_fluxes_pre(vp(theirs.data_ptr()), vp(args[0].data_ptr()), vp(args[1].data_ptr()),
                              vp(r_de.data_ptr()), vp(args[2].data_ptr()), vp(args[3].data_ptr()),
                              vp(args[4].data_ptr()), vp(dev(tau).data_ptr()), vp(dev(heat).data_ptr()),
                              *umf, n, vp(structs.data_ptr()), vp(torch.cuda.current_stream().cuda_stream))
    assert rc == 0
    torch.cuda.synchronize()
    th = theirs.cpu().numpy().reshape(15, n)
    for c in range(15):
        assert rel(ours[c], th[c]) < 1e-12, c
    assert rel(ours_de4, r_de.cpu().numpy()[4 * n:]) < 1e-12


def test_reference_driver_sequence_runs(cuda, tmp_path):
    """The reference driver's loop through the drop-in headers (non-reflective
    x faces, viscous y walls, periodic z; gcbc_go with the reference's
    parameter list), three RK steps on the B200."""
    from test_dropin_build import build_demo
    exe = build_demo(str(tmp_path / "driver_sequence"), "driver_sequence.cpp")
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and "PASS" in r.stdout, r.stdout + r.stderr


def _gcbc_case(dims, seed):
    """A smooth compressible state, its pressure, a right-hand side, line-end
    derivatives, unit face normals (tilted), Jacobian and boundary weights."""
    r = np.random.default_rng(seed)
    n = int(np.prod(dims))
    q = O.tgv_init(dims, 0.3, 1e-3, seed)
    q[3 * n:4 * n] = 0.05 * q[:n] * np.sin(np.arange(n) * 0.01)  # nonzero w
    de_t, p = O.thermo(q)
    de = 0.1 * r.standard_normal(5 * n)
    yaco = 1.0 + 0.2 * r.random(n)
    sbcc = r.random(n)
    F = (dims[1] * dims[2], dims[0] * dims[2], dims[0] * dims[1])
    drva, cm = [], []
    for a in range(3):
        drva.append(r.standard_normal(10 * F[a]))
        c = np.zeros((2, 3, F[a]))
        c[:, a, :] = 1.0
        c += 0.2 * r.standard_normal((2, 3, F[a]))
        c /= np.linalg.norm(c, axis=1, keepdims=True)
        cm.append(c.ravel().copy())
    return q, p, de, yaco, sbcc, drva, cm, F


@pytest.mark.parametrize("nbc", [[[10, 20, 30], [25, 10, 30]], [[30, 25, 10], [30, 20, 10]],
                                 [[20, 45, 25], [10, 45, 20]]])
def test_gcbc_apply_all_face_codes_match_oracle(cuda, nbc):
    """cs_gcbc_apply (gcbc_go with the reference's parameters) on every face
    code: non-reflective (10), inviscid / viscous wall (20 / 25), curvilinear
    interface (30) with the single-rank GCIC exchange, on all three axes,
    tilted face normals, frame velocity and acceleration: de, the
    characteristic drva and drvb against the oracle at 1e-12."""
    import torch
    import compact_schemes_b200 as cs
    dims = (20, 16, 12)
    q, p, de, yaco, sbcc, drva, cm, F = _gcbc_case(dims, 4)
    umf, dudtmf, dtwi = (0.02, -0.01, 0.015), (0.3, -0.2, 0.1), 25.0
    drvb = [np.zeros(10 * f) for f in F]
    de_o, drva_o, drvb_o = de.copy(), [x.copy() for x in drva], [x.copy() for x in drvb]
    O.gcbc_go(drva_o, cm, drvb_o, q, de_o, p, yaco, sbcc, umf, dudtmf, dims, dtwi, nbc)
    d_drva = [dev(x) for x in drva]
    d_drvb = [dev(x) for x in drvb]
    d_cm = [dev(x) for x in cm]
    d_de = dev(de)
    cs.gcbc_go(d_drva, d_cm, d_drvb, dev(q), d_de, dev(p), dev(yaco), dev(sbcc), umf, dudtmf, dims, dtwi, nbc,
               [[0] * 3, [0] * 3])
    torch.cuda.synchronize()
    corr_o = de_o - de
    corr_g = d_de.cpu().numpy() - de
    assert np.abs(corr_o).max() > 0
    assert np.abs(corr_g - corr_o).max() / np.abs(corr_o).max() < 1e-12
    for a in range(3):
        assert rel(d_drva[a].cpu().numpy(), drva_o[a]) < 1e-12, a
        if np.abs(drvb_o[a]).max() > 0:
            assert rel(d_drvb[a].cpu().numpy(), drvb_o[a]) < 1e-12, a


def test_gcbc_apply_non_reflective_equals_numerics_path(cuda):
    """On non-reflective faces the reference-signature path equals the
    numerics-object path (fused setup + update) to rounding."""
    import torch
    import compact_schemes_b200 as cs
    dims = (20, 16, 12)
    q, p, de, yaco, sbcc, drva, cm, F = _gcbc_case(dims, 5)
    nbc = [[10, 10, 10], [10, 10, 10]]
    nm = cs.numerics_pc(dims, nbc)
    nm.deriv_setup()
    for a in range(3):
        dp, _, _ = nm.buffers(a)
        device_view(dp, 10 * F[a]).copy_(dev(drva[a]))
    d1 = dev(de)
    cs.gcbc_go(nm, [dev(c) for c in cm], dev(q), d1, dev(p), dev(yaco), dev(sbcc), (0.01, 0.0, 0.0), dims, nbc)
    d2 = dev(de)
    cs.gcbc_go([dev(x) for x in drva], [dev(c) for c in cm], [None] * 3, dev(q), d2, dev(p), dev(yaco),
               dev(sbcc), (0.01, 0.0, 0.0), (0.0, 0.0, 0.0), dims, 10.0, nbc)
    torch.cuda.synchronize()
    c1, c2 = (d1 - dev(de)).cpu().numpy(), (d2 - dev(de)).cpu().numpy()
    assert np.abs(c1).max() > 0
    assert np.abs(c1 - c2).max() / np.abs(c1).max() < 1e-13
