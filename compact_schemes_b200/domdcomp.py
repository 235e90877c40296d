"""Block decomposition of one box over a process grid, and the interface-sum
exchange between neighbouring blocks.

``domdcomp`` plays the role of the reference's domdcomp::go
(src/domdcomp.hpp:109-286) for a single block ("nblocks = 0") split over
nbpc[0] x nbpc[1] x nbpc[2] ranks, rank = px + nbpc[0] (py + nbpc[1] pz):
the first block along an axis takes the remainder points, interior faces get
BC_INTER_SUBDOMAINS and the neighbour's rank in ``mcd``, global faces keep
their code, and a periodic global axis wraps its neighbours (a single rank
along it is its own neighbour).

``mpigo`` is numerics_base::mpigo (src/numerics_base.hpp:119-180) over
torch.distributed: after ``fill_buffers``, every interface face sends its two
pbco sums per line to the neighbour across it and receives the neighbour's
into the recv buffers that ``deriv1d``/``deriv2d`` read with HALO_RECV.
``mpigo_local`` does the same between blocks held by one process (one
numerics object per block), which is how the multi-block path is checked on
a single GPU.
"""
from __future__ import annotations

import weakref

from . import BC_INTER_SUBDOMAINS, BC_PERIODIC


def split(n, parts):
    """Points per block along one axis: the first block takes the remainder
    (src/domdcomp.hpp:171-197, in point counts)."""
    if parts < 1 or n < parts:
        raise ValueError("cannot split %d points over %d blocks" % (n, parts))
    rest = n // parts
    return [n - rest * (parts - 1)] + [rest] * (parts - 1)


class domdcomp:  # noqa: N801 - reference class name
    """Decomposition of a global box of ``global_dims`` points over ``nbpc``
    ranks per axis, seen from ``rank``.

    nbc_global[face][axis]: boundary codes of the global box (BC_PERIODIC for a
    periodic axis).  Attributes: ``ijkp`` (block coordinates), ``dims`` (block
    points per axis), ``offset`` (global index of the block's first point),
    ``nbc`` (the block's codes), ``mcd`` (neighbour rank per face, -1 none).
    """

    def __init__(self, global_dims, nbpc, nbc_global, rank):
        self.global_dims = tuple(int(x) for x in global_dims)
        self.nbpc = tuple(int(x) for x in nbpc)
        self.mpro = self.nbpc[0] * self.nbpc[1] * self.nbpc[2]
        if not 0 <= rank < self.mpro:
            raise ValueError("rank %d outside the process grid %s" % (rank, self.nbpc))
        self.rank = rank
        self.ijkp = (rank % self.nbpc[0], (rank // self.nbpc[0]) % self.nbpc[1],
                     rank // (self.nbpc[0] * self.nbpc[1]))
        mp = (1, self.nbpc[0], self.nbpc[0] * self.nbpc[1])
        self.dims, self.offset = [], []
        self.nbc = [[0] * 3, [0] * 3]
        self.mcd = [[-1] * 3, [-1] * 3]
        for nn in range(3):
            parts = split(self.global_dims[nn], self.nbpc[nn])
            lp, ma = self.ijkp[nn], self.nbpc[nn]
            self.dims.append(parts[lp])
            self.offset.append(sum(parts[:lp]))
            periodic = nbc_global[0][nn] == BC_PERIODIC and nbc_global[1][nn] == BC_PERIODIC
            for ip in range(2):
                at_edge = lp == (0 if ip == 0 else ma - 1)
                step = -1 if ip == 0 else 1
                if not at_edge:
                    self.nbc[ip][nn] = BC_INTER_SUBDOMAINS
                    self.mcd[ip][nn] = rank + step * mp[nn]
                elif periodic and ma > 1:
                    # wrap: the block at the other end of the axis
                    self.nbc[ip][nn] = BC_INTER_SUBDOMAINS
                    self.mcd[ip][nn] = rank - step * (ma - 1) * mp[nn]
                else:
                    self.nbc[ip][nn] = nbc_global[ip][nn]
                    self.mcd[ip][nn] = rank if periodic else -1
        self.dims = tuple(self.dims)
        self.offset = tuple(self.offset)

    @property
    def lmx(self):
        return self.dims[0] * self.dims[1] * self.dims[2]

    def face_size(self, axis):
        lxi, let, lze = self.dims
        return (let * lze, lxi * lze, lxi * let)[axis]

    def interface(self, ip, nn):
        """True when face ip of axis nn exchanges interface sums."""
        return self.mcd[ip][nn] >= 0 and (self.nbc[ip][nn] == BC_INTER_SUBDOMAINS or
                                           self.nbc[ip][nn] == BC_PERIODIC)

    def block(self, field):
        """This rank's block of a global field (numpy or torch, SoA [lmx] flat
        in x-fastest order) as a contiguous flat array."""
        gx, gy, gz = self.global_dims
        (ox, oy, oz), (lx, ly, lz) = self.offset, self.dims
        v = field.reshape(gz, gy, gx)[oz:oz + lz, oy:oy + ly, ox:ox + lx]
        return v.reshape(-1).copy() if hasattr(v, "copy") else v.reshape(-1).clone()


class _DeviceArray:
    """A device pointer seen as a float64 vector (CUDA array interface)."""

    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (int(n),), "typestr": "<f8", "data": (int(ptr), False),
                                         "version": 2, "strides": None}


def _view(ptr, n):
    import torch
    return torch.as_tensor(_DeviceArray(ptr, n), device="cuda")


def _buffers(numerics, dd, nn, variable_id):
    """(send, recv) of one variable along axis nn: [2 faces][2 sums][F]."""
    F = dd.face_size(nn)
    _, s, r = numerics.buffers(nn)
    off = variable_id * 4 * F * 8
    return _view(s + off, 4 * F), _view(r + off, 4 * F)


def exchange(send, recv, dd, nn, group=None):
    """Move the interface sums of one variable along axis nn between ranks.

    send/recv: [4F] tensors (face 0: [0, 2F), face 1: [2F, 4F)), on the device
    the process group's backend uses.  Face ip's recv part receives the
    neighbour's face (1 - ip) sums (the tag pairing of
    src/numerics_base.hpp:161-176).  Messages go in two rounds, upward (face 1
    sums to the upper neighbour) then downward, so that two ranks that are
    neighbours across both faces match their messages in order.
    """
    import torch.distributed as dist
    F2 = send.numel() // 2
    part = lambda t, ip: t[ip * F2:(ip + 1) * F2]
    for ip_send in (1, 0):
        ip_recv = 1 - ip_send
        ops, landing = [], None
        if dd.interface(ip_send, nn):
            peer = dd.mcd[ip_send][nn]
            if peer == dd.rank:  # a single rank along a periodic axis
                part(recv, ip_recv).copy_(part(send, ip_send))
            else:
                ops.append(dist.P2POp(dist.isend, part(send, ip_send).contiguous(), peer, group=group))
        if dd.interface(ip_recv, nn) and dd.mcd[ip_recv][nn] != dd.rank:
            landing = recv.new_empty(F2)
            ops.append(dist.P2POp(dist.irecv, landing, dd.mcd[ip_recv][nn], group=group))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()
        if landing is not None:
            part(recv, ip_recv).copy_(landing)


# process groups whose first point-to-point batch has been preceded by a
# barrier; weak references, so a destroyed group (and a new one created in
# its place, possibly at the same address) is never mistaken for a ready one
_P2P_READY = weakref.WeakSet()


def mpigo(numerics, dd, variable_id, group=None):
    """numerics_base::mpigo over torch.distributed for one variable: every
    interface axis of the block exchanges the send buffers that
    ``numerics.fill_buffers`` wrote (src/numerics_base.hpp:119-180).  Every
    rank of the group calls it, in the same order of variables."""
    import torch
    import torch.distributed as dist
    key = group if group is not None else dist.group.WORLD
    if key not in _P2P_READY:
        # the first point-to-point batch of an NCCL group must involve every
        # rank; a barrier on the group first makes any later subset valid
        dist.barrier(group=group)
        _P2P_READY.add(key)
    torch.cuda.synchronize()  # the sums of fill_buffers are complete on every stream
    for nn in range(3):
        if dd.interface(0, nn) or dd.interface(1, nn):
            s, r = _buffers(numerics, dd, nn, variable_id)
            exchange(s, r, dd, nn, group)
    torch.cuda.synchronize()


def mpigo_local(numerics_list, dds, variable_id):
    """The same exchange between blocks held by one process (one numerics
    object per block, dds[i].rank == i): device copies instead of messages."""
    import torch
    for nn in range(3):
        bufs = [_buffers(nm, dd, nn, variable_id) if (dd.interface(0, nn) or dd.interface(1, nn)) else None
                for nm, dd in zip(numerics_list, dds)]
        for i, dd in enumerate(dds):
            if bufs[i] is None:
                continue
            _, recv = bufs[i]
            F2 = recv.numel() // 2
            for ip in range(2):
                if not dd.interface(ip, nn):
                    continue
                peer = dd.mcd[ip][nn]
                psend, _ = bufs[peer]
                iq = 1 - ip
                recv[ip * F2:(ip + 1) * F2].copy_(psend[iq * F2:(iq + 1) * F2])
    torch.cuda.synchronize()
