"""cs_deriv_noalloc: the compact derivative for callers that cannot let the
library allocate device memory (its solver tables sit in a preallocated
device array).  Checked through the C ABI against cs_deriv with the
single-rank periodic halo, on two calls in a row with different lines, so the
second call must fully replace the first call's tables.  Collected last on
purpose: the file name sorts after every other test module."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _field(dims, seed):
    rng = np.random.default_rng(seed)
    return rng.normal(size=int(np.prod(dims)))


def _reference(cs, torch, dims, axis, ndf, f):
    nm = cs.numerics_pc(dims, [[45 if ndf else 10] * 3, [45 if ndf else 10] * 3])
    nm.deriv_setup()
    fin = torch.from_numpy(f).cuda()
    out = torch.zeros_like(fin)
    nm.deriv1d(axis, fin, out, ndf, ndf, dims, 0, halo=cs.HALO_SELF)
    torch.cuda.synchronize()
    return out.cpu().numpy()


def test_noalloc_matches_deriv_two_calls(cuda):
    import torch
    import compact_schemes_b200 as cs
    L = cs.lib()
    cases = [((64, 48, 40), 1, 1, 11), ((33, 17, 96), 2, 0, 12)]  # different line lengths / closures
    outs = []
    for dims, axis, ndf, seed in cases:
        f = _field(dims, seed)
        fin = torch.from_numpy(f).cuda()
        out = torch.zeros_like(fin)
        rc = L.cs_deriv_noalloc(axis, ctypes.c_void_p(fin.data_ptr()), ctypes.c_void_p(out.data_ptr()), ndf, ndf,
                                cs.Dcomp.of(*dims), cs.stream_ptr())
        assert rc == 0, L.cs_last_error()
        torch.cuda.synchronize()
        outs.append((out.cpu().numpy(), f, dims, axis, ndf))
    for got, f, dims, axis, ndf in outs:
        ref = _reference(cs, torch, dims, axis, ndf, f)
        assert np.abs(got - ref).max() / np.abs(ref).max() < TOL


def test_noalloc_rejects_lines_beyond_capacity(cuda):
    import torch
    import compact_schemes_b200 as cs
    L = cs.lib()
    dims = (1025, 2, 2)
    x = torch.zeros(int(np.prod(dims)), dtype=torch.float64, device="cuda")
    rc = L.cs_deriv_noalloc(0, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(x.data_ptr()), 0, 0,
                            cs.Dcomp.of(*dims), cs.stream_ptr())
    assert rc == -3 and b"1024" in L.cs_last_error()
