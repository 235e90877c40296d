"""The derivative-and-filter workload on the GPU: the 64^3 non-periodic
[0,1]^3 field of 8 Fourier modes drawn from MT19937-64 seed 0 (physical
closures on all six faces); index-space compact derivatives along x, y and z
and the compact filter applied along x, then y, then z, each against the
FP64 oracle at 1e-12 relative max-norm.  The y and z derivatives are also
compared with the reference's own deriv_kernel_2d<Axis,double> run on this
GPU (its x kernel is valid only for lze = 1)."""
import ctypes
import os

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_GPU = os.path.join(ROOT, "oracle", "_ref", "libref_gpu.so")
DIMS = (64, 64, 64)
TOL = 1e-12
ALPHA_F = 0.45


def relerr(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


def _setup(cuda):
    import torch
    import compact_schemes_b200 as cs
    nm = cs.numerics_pc(DIMS, [[cs.BC_NON_REFLECTIVE] * 3] * 2)
    nm.deriv_setup()
    _, f = O.fourier_field(DIMS, 0, 8)
    return nm, f, torch.from_numpy(f).to(cuda)


def test_device_field_matches_oracle_field(cuda):
    import compact_schemes_b200 as cs
    _, f = O.fourier_field(DIMS, 0, 8)
    g = cs.grid.fourier_field(DIMS, 0, 8).cpu().numpy()
    assert np.abs(g - f).max() <= 1e-14 * np.abs(f).max()


def test_derivatives_xyz(cuda):
    import torch
    import compact_schemes_b200 as cs
    nm, f, fin = _setup(cuda)
    out = torch.zeros_like(fin)
    for axis in range(3):
        nm.deriv1d(axis, fin, out, 0, 0, DIMS, 0, halo=cs.HALO_SELF)
        torch.cuda.synchronize()
        ref = O.deriv(f, DIMS, axis, 0, 0)
        assert relerr(out.cpu().numpy(), ref) < TOL, axis
    nm.close()


def test_filter_x_then_y_then_z(cuda):
    import torch
    nm, f, fin = _setup(cuda)
    a, b = fin.clone(), torch.zeros_like(fin)
    ref = f.copy()
    for axis in range(3):
        nm.filter(axis, a, b, ALPHA_F, DIMS)
        a, b = b, a
        ref = O.filt(ref, DIMS, axis, 0, 0, ALPHA_F)
    torch.cuda.synchronize()
    assert relerr(a.cpu().numpy(), ref) < TOL
    # the filter damps the field (every mode resolved by at least 7 points)
    assert np.abs(ref).max() < np.abs(f).max()
    nm.close()


@pytest.mark.skipif(not os.path.exists(REF_GPU), reason="reference kernels not built (make -C oracle ref)")
def test_derivatives_yz_against_reference_kernel(cuda):
    import torch
    R = ctypes.CDLL(REF_GPU)
    vp = ctypes.c_void_p
    R.ref_gpu_deriv2d.argtypes = [ctypes.c_int, vp, vp, vp, vp, vp, ctypes.c_int, ctypes.c_int,
                                  ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_uint,
                                  ctypes.c_uint, vp]
    nm, f, fin = _setup(cuda)
    lmx = fin.numel()
    block = torch.zeros(3 * lmx, dtype=torch.float64, device=cuda)
    ours = torch.zeros_like(block)
    theirs = torch.zeros_like(block)
    _, pbci = nm.coeffs()
    dpbci = torch.tensor(pbci, dtype=torch.float64, device=cuda)
    for a in (1, 2):
        block[a * lmx:(a + 1) * lmx] = fin
        nm.deriv2d(a, block, ours, 0, 0, DIMS, 0, a)
        drva, _, recv = nm.buffers(a)
        scratch = torch.zeros(10 * 64 * 64, dtype=torch.float64, device=cuda)
        rc = R.ref_gpu_deriv2d(a, vp(block.data_ptr()), vp(theirs.data_ptr()), vp(recv), vp(dpbci.data_ptr()),
                               vp(scratch.data_ptr()), 0, 0, *DIMS, 0, a,
                               vp(torch.cuda.current_stream().cuda_stream))
        assert rc == 0
        torch.cuda.synchronize()
        got = ours[a * lmx:(a + 1) * lmx].cpu().numpy()
        ref = theirs[a * lmx:(a + 1) * lmx].cpu().numpy()
        assert relerr(got, ref) < TOL, a
        assert relerr(got, O.deriv(f, DIMS, a, 0, 0)) < TOL, a
    nm.close()
