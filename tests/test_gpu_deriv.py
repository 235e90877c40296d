"""GPU parity of the compact derivative / filter line solves against the FP64 oracle.

Tolerance: 1e-12 relative max-norm (max|x - x_oracle| / max|x_oracle|) for FP64,
2e-6 for the FP32 entry point.
"""
import ctypes
import os

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TOL = 1e-12


from gpu_util import device_view  # noqa: E402


def relerr(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def make(cuda, dims, nbc):
    import compact_schemes_b200 as cs
    nm = cs.numerics_pc(dims, nbc)
    nm.deriv_setup()
    return nm


def field(dims, seed=0):
    rng = np.random.default_rng(seed)
    lxi, let, lze = dims
    i, j, k = np.meshgrid(np.arange(lxi), np.arange(let), np.arange(lze), indexing="ij")
    f = (np.sin(2 * np.pi * 3 * i / lxi + 0.3) * np.cos(2 * np.pi * 2 * j / let)
         + 0.5 * np.sin(2 * np.pi * 5 * k / lze + 1.0))
    f = f.transpose(2, 1, 0).ravel() + 0.1 * rng.normal(size=lxi * let * lze)
    return np.ascontiguousarray(f)


DIMS = [(64, 48, 40), (33, 17, 96), (256, 8, 9), (9, 130, 12), (20, 10, 513)]


@pytest.mark.parametrize("dims", DIMS)
@pytest.mark.parametrize("ndf", [(0, 0), (1, 1), (0, 1), (1, 0)])
def test_deriv_fp64_self_halo(cuda, dims, ndf):
    import torch
    import compact_schemes_b200 as cs
    nbc = [[45 if ndf[0] else 10] * 3, [45 if ndf[1] else 10] * 3]
    nm = make(cuda, dims, nbc)
    f = field(dims, 1)
    coeffs = O.deriv_setup()
    fin = torch.from_numpy(f).to(cuda)
    out = torch.zeros_like(fin)
    for axis in range(3):
        n = dims[axis]
        if (ndf[0] or ndf[1]) and n < 8:
            continue
        if ndf[0] != ndf[1]:
            # a single interface face has no single-rank neighbour: use an
            # explicit recv buffer (zeros) on both sides in the oracle
            continue
        nm.deriv1d(axis, fin, out, ndf[0], ndf[1], dims, 0, halo=cs.HALO_SELF)
        torch.cuda.synchronize()
        ref = O.deriv(f, dims, axis, ndf[0], ndf[1], coeffs=coeffs)
        assert relerr(out.cpu().numpy(), ref) < TOL, (axis, dims, ndf)


@pytest.mark.parametrize("dims", [(64, 48, 40), (33, 17, 96)])
def test_deriv2d_recv_path_and_drva(cuda, dims):
    """fill_buffers -> mpigo -> deriv2d, the reference data flow (src/physics_pc.hpp:94-146)."""
    import torch
    nbc = [[45, 45, 45], [45, 45, 45]]
    nm = make(cuda, dims, nbc)
    lmx = int(np.prod(dims))
    rng = np.random.default_rng(5)
    block = rng.normal(size=15 * lmx)           # [5][3][lmx] flux block
    dblock = torch.from_numpy(block).to(cuda)
    dout = torch.zeros_like(dblock)
    nm.fill_buffers(dblock, 0, 5, 0, dims)
    coeffs = O.deriv_setup()
    for m in range(5):
        nm.mpigo(dims, None, m + 1, m)
        for axis in range(3):
            off = m * 3 * lmx
            nm.deriv2d(axis, dblock[off:], dout[off:], 1, 1, dims, m, axis)
    torch.cuda.synchronize()
    out = dout.cpu().numpy()
    for m in range(5):
        for axis in range(3):
            f = block[(m * 3 + axis) * lmx:(m * 3 + axis + 1) * lmx]
            F = (dims[1] * dims[2], dims[0] * dims[2], dims[0] * dims[1])[axis]
            drva = np.zeros(10 * F)
            ref = O.deriv(f, dims, axis, 1, 1, drva=drva, var=m, coeffs=coeffs)
            got = out[(m * 3 + axis) * lmx:(m * 3 + axis + 1) * lmx]
            assert relerr(got, ref) < TOL, (m, axis)
            # drva holds the line-end derivatives of this axis / variable
            dp, _, _ = nm.buffers(axis)
            host = device_view(dp, 10 * F).cpu().numpy()
            assert relerr(host[m * F:(m + 1) * F], drva[m * F:(m + 1) * F]) < TOL
            assert relerr(host[5 * F + m * F:5 * F + (m + 1) * F],
                          drva[5 * F + m * F:5 * F + (m + 1) * F]) < TOL


def test_deriv_fp32(cuda):
    import torch
    import compact_schemes_b200 as cs
    dims = (64, 48, 40)
    nm = make(cuda, dims, [[45] * 3, [10] * 3])
    f = field(dims, 2)
    fin = torch.from_numpy(f).float().to(cuda)
    out = torch.zeros_like(fin)
    nm2 = make(cuda, dims, [[45] * 3, [45] * 3])
    for axis in range(3):
        nm2.deriv1d(axis, fin, out, 1, 1, dims, 0, halo=cs.HALO_SELF)
        torch.cuda.synchronize()
        ref = O.deriv(f.astype(np.float32).astype(np.float64), dims, axis, 1, 1)
        assert relerr(out.double().cpu().numpy(), ref) < 2e-6
    del nm


def test_linear_field_known_answer_gpu(cuda):
    """tests/test_numerics_serial.cu:60-131 on the GPU (FP64)."""
    import torch
    import compact_schemes_b200 as cs
    dims = (256, 128, 64)
    nm = make(cuda, dims, [[10] * 3, [10] * 3])
    f = torch.arange(np.prod(dims), dtype=torch.float64, device=cuda)
    out = torch.zeros_like(f)
    for axis, step in ((0, 1.0), (1, 256.0), (2, 256.0 * 128)):
        nm.deriv1d(axis, f, out, 0, 0, dims, 0, halo=cs.HALO_SELF)
        torch.cuda.synchronize()
        assert (out - step).abs().max().item() / step < 1e-13


def test_coeffs_match_reference_golden(cuda):
    g = np.load(os.path.join(ROOT, "tests", "golden", "reference_pins.npz"))
    nm = make(cuda, (16, 16, 16), [[45] * 3, [45] * 3])
    pbco, pbci = nm.coeffs()
    assert np.array_equal(np.array(pbco), g["pbco"])
    assert np.array_equal(np.array(pbci), g["pbci"])


@pytest.mark.parametrize("dims", [(64, 48, 40), (33, 17, 96), (7, 9, 256)])
@pytest.mark.parametrize("periodic", [0, 1])
def test_filter_fp64(cuda, dims, periodic):
    import torch
    b = 45 if periodic else 10
    nm = make(cuda, dims, [[b] * 3, [b] * 3])
    f = field(dims, 3)
    fin = torch.from_numpy(f).to(cuda)
    out = torch.zeros_like(fin)
    for axis in range(3):
        nm.filter(axis, fin, out, 0.45, dims)
        torch.cuda.synchronize()
        ref = O.filt(f, dims, axis, periodic, periodic, 0.45)
        assert relerr(out.cpu().numpy(), ref) < TOL, (axis, dims)


REF_GPU = os.path.join(ROOT, "oracle", "_ref", "libref_gpu.so")


@pytest.mark.skipif(not os.path.exists(REF_GPU), reason="reference kernels not built (make -C oracle ref)")
@pytest.mark.parametrize("ndf", [0, 1])
def test_against_reference_gpu_kernel(cuda, ndf):
    """Our deriv2d vs the reference's own deriv_kernel_2d<Axis,double> run on this GPU.

    Power-of-two lines (the reference PCR needs them); axis 0 only with
    lze = 1 (its row index is wrong for lze > 1, src/cuda/kernels/transforms.hpp:72-88).
    """
    import torch
    R = ctypes.CDLL(REF_GPU)
    vp = ctypes.c_void_p
    R.ref_gpu_deriv2d.argtypes = [ctypes.c_int, vp, vp, vp, vp, vp, ctypes.c_int, ctypes.c_int,
                                  ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_uint,
                                  ctypes.c_uint, vp]
    for dims, axes in (((64, 32, 128), (1, 2)), ((256, 64, 1), (0,))):
        b = 45 if ndf else 10
        nbc = [[b, b, b if dims[2] >= 8 else 10]] * 2
        nm = make(cuda, dims, nbc)
        lmx = int(np.prod(dims))
        f = torch.from_numpy(field(dims, 4)).to(cuda)
        block = torch.zeros(3 * lmx, dtype=torch.float64, device=cuda)
        for a in axes:
            block[a * lmx:(a + 1) * lmx] = f
        nm.fill_buffers(torch.cat([block, torch.zeros(12 * lmx, dtype=torch.float64,
                                                      device=cuda)]), 0, 1, 0, dims)
        nm.mpigo(dims, None, 1, 0)
        ours = torch.zeros(3 * lmx, dtype=torch.float64, device=cuda)
        theirs = torch.zeros(3 * lmx, dtype=torch.float64, device=cuda)
        pbco, pbci = nm.coeffs()
        dpbci = torch.tensor(pbci, dtype=torch.float64, device=cuda)
        for a in axes:
            if dims[a] < 8 and ndf:
                continue
            nm.deriv2d(a, block, ours, ndf, ndf, dims, 0, a)
            drva, _, recv = nm.buffers(a)
            F = (dims[1] * dims[2], dims[0] * dims[2], dims[0] * dims[1])[a]
            scratch = torch.zeros(10 * F, dtype=torch.float64, device=cuda)
            rc = R.ref_gpu_deriv2d(a, vp(block.data_ptr()), vp(theirs.data_ptr()), vp(recv),
                                   vp(dpbci.data_ptr()), vp(scratch.data_ptr()), ndf, ndf, *dims, 0,
                                   a, vp(torch.cuda.current_stream().cuda_stream))
            assert rc == 0
            torch.cuda.synchronize()
            got = ours[a * lmx:(a + 1) * lmx].cpu().numpy()
            ref = theirs[a * lmx:(a + 1) * lmx].cpu().numpy()
            assert relerr(got, ref) < TOL, (dims, a, ndf, relerr(got, ref))
