"""Serial oracle emulation of a multi-block compact derivative (test helper):
every block's interface sums (oracle fill_buffer) are copied into its
neighbours' receive buffers directly, then each block is differentiated by
the oracle with those buffers."""
import numpy as np

import oracle as O


def block_sends(f, dims, axis, pbco):
    """[4F]: face 0 sums then face 1 sums of a block field along axis."""
    return np.concatenate([O.fill_buffer(f, dims, axis, face, pbco) for face in (0, 1)])


def serial_multiblock_deriv(field, dds, axis):
    """Derivative of every block of the global field along axis (list by rank)."""
    pbco, pbci = O.deriv_setup()
    blocks = [dd.block(field) for dd in dds]
    sends = [block_sends(b, dd.dims, axis, pbco) if dd.dims[axis] >= 8 else None for b, dd in zip(blocks, dds)]
    out = []
    for b, dd in zip(blocks, dds):
        F = dd.face_size(axis)
        recv = np.zeros(4 * F)
        for ip in range(2):
            if dd.interface(ip, axis):
                peer = dd.mcd[ip][axis]
                iq = 1 - ip
                recv[2 * F * ip:2 * F * (ip + 1)] = sends[peer][2 * F * iq:2 * F * (iq + 1)]
        nstart, nend = (1 if dd.interface(0, axis) else 0), (1 if dd.interface(1, axis) else 0)
        out.append(O.deriv(b, dd.dims, axis, nstart, nend, recv=recv, coeffs=(pbco, pbci)))
    return out
