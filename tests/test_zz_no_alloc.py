"""cs_deriv_noalloc: the compact derivative for callers that cannot let the
library allocate device memory (its solver tables sit in a preallocated
device array).  Checked through the C ABI against the FP64 oracle and
against cs_deriv with the single-rank periodic halo.  The calls of each case
list go back to back on one stream with no synchronization between them, so
a later call's table upload must wait for the earlier kernels (stream order)
and must fully replace their tables.  Collected last on purpose: the file
name sorts after every other test module."""
import ctypes

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu
TOL = 1e-12

# (dims, axis, ndf, seed): different axes, line lengths and closures; the
# 700-point line takes the longest chunk (32 rows per lane)
CASES = [((64, 48, 40), 1, 1, 11), ((33, 17, 96), 2, 0, 12), ((40, 24, 20), 0, 1, 13), ((700, 6, 5), 0, 0, 14)]


def _field(dims, seed):
    rng = np.random.default_rng(seed)
    return rng.normal(size=int(np.prod(dims)))


def _cs_deriv(cs, torch, dims, axis, ndf, f):
    nm = cs.numerics_pc(dims, [[45 if ndf else 10] * 3, [45 if ndf else 10] * 3])
    nm.deriv_setup()
    fin = torch.from_numpy(f).cuda()
    out = torch.zeros_like(fin)
    nm.deriv1d(axis, fin, out, ndf, ndf, dims, 0, halo=cs.HALO_SELF)
    torch.cuda.synchronize()
    nm.close()
    return out.cpu().numpy()


def _run_back_to_back(cs, torch, cases):
    L = cs.lib()
    ins, outs = [], []
    for dims, axis, ndf, seed in cases:
        ins.append(torch.from_numpy(_field(dims, seed)).cuda())
        outs.append(torch.zeros_like(ins[-1]))
    torch.cuda.synchronize()
    for (dims, axis, ndf, _), fin, out in zip(cases, ins, outs):
        rc = L.cs_deriv_noalloc(axis, ctypes.c_void_p(fin.data_ptr()), ctypes.c_void_p(out.data_ptr()), ndf, ndf,
                                cs.Dcomp.of(*dims), cs.stream_ptr())
        assert rc == 0, L.cs_last_error()
    torch.cuda.synchronize()
    return [o.cpu().numpy() for o in outs]


@pytest.mark.parametrize("order", [1, -1])
def test_noalloc_matches_oracle_and_deriv_back_to_back(cuda, order):
    import torch
    import compact_schemes_b200 as cs
    cases = CASES[::order]
    got = _run_back_to_back(cs, torch, cases)
    for g, (dims, axis, ndf, seed) in zip(got, cases):
        f = _field(dims, seed)
        ref = O.deriv(f, dims, axis, ndf, ndf)
        assert np.abs(g - ref).max() / np.abs(ref).max() < TOL, (dims, axis, ndf)
        ref2 = _cs_deriv(cs, torch, dims, axis, ndf, f)
        assert np.abs(g - ref2).max() / np.abs(ref2).max() < TOL, (dims, axis, ndf)


def test_noalloc_rejects_lines_beyond_capacity(cuda):
    import torch
    import compact_schemes_b200 as cs
    L = cs.lib()
    dims = (1025, 2, 2)
    x = torch.zeros(int(np.prod(dims)), dtype=torch.float64, device="cuda")
    rc = L.cs_deriv_noalloc(0, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(x.data_ptr()), 0, 0,
                            cs.Dcomp.of(*dims), cs.stream_ptr())
    assert rc == -3 and b"1024" in L.cs_last_error()
