"""Multi-block compact derivative on one GPU: the blocks of a decomposition
are held by one process (one numerics object each), their interface sums are
filled on the device (cs_fill_buffers), exchanged by mpigo_local and read by
cs_deriv with CS_HALO_RECV.  Checked against the serial oracle emulation at
the derivative tolerance (1e-12 relative max-norm)."""
import numpy as np
import pytest

import oracle as O
from domdcomp_util import serial_multiblock_deriv

pytestmark = pytest.mark.gpu
P, NR = O.BC_PERIODIC, O.BC_NON_REFLECTIVE


@pytest.mark.parametrize("gdims,nbpc,nbc", [((48, 40, 24), (2, 2, 1), [[NR, P, P], [NR, P, P]]),
                                            ((40, 24, 36), (1, 2, 3), [[P] * 3, [P] * 3])])
def test_multiblock_deriv_matches_serial_emulation(cuda, gdims, nbpc, nbc):
    import torch
    import compact_schemes_b200 as cs
    from compact_schemes_b200.domdcomp import domdcomp, mpigo_local
    world = nbpc[0] * nbpc[1] * nbpc[2]
    dds = [domdcomp(gdims, nbpc, nbc, r) for r in range(world)]
    field = np.random.default_rng(9).normal(size=int(np.prod(gdims)))
    nms, fs = [], []
    for dd in dds:
        nm = cs.numerics_pc(dd.dims, dd.nbc)
        nm.deriv_setup()
        f = torch.from_numpy(dd.block(field)).to(cuda)
        nm.fill_buffers(f, 0, 1, 1, dd.dims)  # nrt = 1: the same field for every axis
        nms.append(nm)
        fs.append(f)
    mpigo_local(nms, dds, 0)
    for axis in range(3):
        ref = serial_multiblock_deriv(field, dds, axis)
        for nm, dd, f, r in zip(nms, dds, fs, ref):
            out = torch.zeros(3 * dd.lmx, dtype=torch.float64, device=cuda)
            nstart, nend = int(dd.interface(0, axis)), int(dd.interface(1, axis))
            nm.deriv2d(axis, f, out, nstart, nend, dd.dims, 0, 0)
            torch.cuda.synchronize()
            got = out[axis * dd.lmx:(axis + 1) * dd.lmx].cpu().numpy()
            assert np.abs(got - r).max() / np.abs(r).max() < 1e-12, (axis, dd.rank)
    for nm in nms:
        nm.close()


def test_mpigo_on_a_one_rank_nccl_group_equals_self_exchange(cuda):
    """mpigo over torch.distributed (here one NCCL rank, periodic on every
    axis: the rank is its own neighbour) fills the recv buffers exactly as
    the single-rank self exchange does."""
    import datetime
    import os
    import socket
    import torch
    import torch.distributed as dist
    import compact_schemes_b200 as cs
    from compact_schemes_b200.domdcomp import _buffers, domdcomp, mpigo
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60))
    try:
        gdims = (32, 24, 16)
        dd = domdcomp(gdims, (1, 1, 1), [[P] * 3, [P] * 3], 0)
        f = torch.from_numpy(np.random.default_rng(3).normal(size=int(np.prod(gdims)))).to(cuda)
        a, b = cs.numerics_pc(gdims, dd.nbc), cs.numerics_pc(gdims, dd.nbc)
        for nm in (a, b):
            nm.deriv_setup()
            nm.fill_buffers(f, 0, 1, 1, gdims)
        mpigo(a, dd, 0)
        b.mpigo(gdims, None, 1, 0)
        torch.cuda.synchronize()
        for nn in range(3):
            assert torch.equal(_buffers(a, dd, nn, 0)[1], _buffers(b, dd, nn, 0)[1])
        a.close()
        b.close()
    finally:
        dist.destroy_process_group()
