"""Block decomposition (domdcomp) and the interface-sum exchange (mpigo) on
CPU: the layout of blocks, neighbours and boundary codes, and a derivative on
2 and 4 gloo ranks whose interface sums travel through
compact_schemes_b200.domdcomp.exchange, checked against a serial emulation
in which the oracle copies the sums between blocks directly."""
import datetime
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

import oracle as O
from domdcomp_util import block_sends, serial_multiblock_deriv

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
P, NR = O.BC_PERIODIC, O.BC_NON_REFLECTIVE


def _dd(*a):
    from compact_schemes_b200.domdcomp import domdcomp
    return domdcomp(*a)


def test_split_puts_the_remainder_first():
    from compact_schemes_b200.domdcomp import split
    assert split(10, 3) == [4, 3, 3]
    assert split(64, 4) == [16, 16, 16, 16]
    with pytest.raises(ValueError):
        split(2, 3)


@pytest.mark.parametrize("nbpc", [(2, 1, 1), (2, 2, 1), (3, 2, 2), (1, 1, 1)])
def test_layout_is_consistent(nbpc):
    gdims = (40, 30, 20)
    nbc = [[NR, P, P], [NR, P, P]]
    dds = [_dd(gdims, nbpc, nbc, r) for r in range(nbpc[0] * nbpc[1] * nbpc[2])]
    for nn in range(3):
        covered = sorted({(dd.offset[nn], dd.dims[nn]) for dd in dds})
        assert covered[0][0] == 0 and sum(d for _, d in covered) == gdims[nn]
    for dd in dds:
        for nn in range(3):
            for ip in range(2):
                peer = dd.mcd[ip][nn]
                if nn == 0 and dd.ijkp[0] == (0 if ip == 0 else nbpc[0] - 1):
                    assert peer == -1 and dd.nbc[ip][nn] == NR  # global physical face
                    continue
                assert peer >= 0 and dd.interface(ip, nn)
                other = dds[peer]
                assert other.mcd[1 - ip][nn] == dd.rank  # the neighbour points back
                assert other.face_size(nn) == dd.face_size(nn)
                if peer == dd.rank:
                    assert dd.nbc[ip][nn] == P and nbpc[nn] == 1
                else:
                    assert dd.nbc[ip][nn] == O.BC_INTER_SUBDOMAINS


def test_serial_emulation_of_one_block_is_the_periodic_derivative():
    gdims = (24, 12, 10)
    dd = _dd(gdims, (1, 1, 1), [[P] * 3, [P] * 3], 0)
    f = np.random.default_rng(0).normal(size=int(np.prod(gdims)))
    for axis in range(3):
        got = serial_multiblock_deriv(f, [dd], axis)[0]
        assert np.array_equal(got, O.deriv(f, gdims, axis, 1, 1))


def test_linear_field_across_blocks():
    # the interface closure is the reference's quasi-disjoint one: on a
    # linear field it is off by ~1.7e-3 next to an interface (a wrong pairing
    # of faces is off by O(10))
    gdims = (40, 6, 5)
    nbc = [[NR] * 3, [NR] * 3]
    dds = [_dd(gdims, (2, 1, 1), nbc, r) for r in range(2)]
    i = np.arange(gdims[0], dtype=float)
    f = np.tile(i, gdims[1] * gdims[2])
    for d in serial_multiblock_deriv(f, dds, 0):
        assert np.abs(d - 1.0).max() < 2e-3


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, gdims, nbpc, nbc, out):
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from compact_schemes_b200.domdcomp import domdcomp, exchange
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        dd = domdcomp(gdims, nbpc, nbc, rank)
        field = np.random.default_rng(5).normal(size=int(np.prod(gdims)))
        f = dd.block(field)
        pbco, pbci = O.deriv_setup()
        res = {}
        for axis in range(3):
            F = dd.face_size(axis)
            send = torch.from_numpy(block_sends(f, dd.dims, axis, pbco))
            recv = torch.zeros(4 * F, dtype=torch.float64)
            exchange(send, recv, dd, axis)
            nstart, nend = int(dd.interface(0, axis)), int(dd.interface(1, axis))
            res[axis] = O.deriv(f, dd.dims, axis, nstart, nend, recv=recv.numpy(), coeffs=(pbco, pbci))
        out.put((rank, res))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("nbpc,nbc", [((2, 1, 1), [[P] * 3, [P] * 3]),
                                      ((2, 2, 1), [[NR, P, P], [NR, P, P]])])
def test_exchange_on_gloo_ranks_matches_serial_emulation(nbpc, nbc):
    gdims = (32, 20, 12)
    world = nbpc[0] * nbpc[1] * nbpc[2]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, gdims, nbpc, nbc, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
    assert all(p.exitcode == 0 for p in procs)
    dds = [_dd(gdims, nbpc, nbc, r) for r in range(world)]
    field = np.random.default_rng(5).normal(size=int(np.prod(gdims)))
    for axis in range(3):
        ref = serial_multiblock_deriv(field, dds, axis)
        for r in range(world):
            assert np.array_equal(res[r][axis], ref[r]), (axis, r)
