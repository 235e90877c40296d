"""The oracle's wall boundary state update (or_wall_update) against the
formulas of wall_inviscid_kernel / wall_viscous_kernel
(src/cuda/kernels/gcbc.hpp:160-249), written out here in numpy."""
import numpy as np

import oracle as O

GAM = 1.4
HAMHAMM1 = (1.0 / GAM) / (GAM - 1.0)


def _state(dims, seed):
    r = np.random.default_rng(seed)
    n = int(np.prod(dims))
    rho = 1.0 + 0.1 * r.uniform(-1, 1, n)
    m = 0.1 * r.standard_normal((3, n))
    E = 1.0 / (GAM * (GAM - 1.0)) + 0.5 * (m * m).sum(0) / rho + 0.01 * r.uniform(-1, 1, n)
    return np.concatenate([rho, m.ravel(), E]), r


def test_inviscid_and_viscous_walls():
    dims = (6, 5, 7)
    n = int(np.prod(dims))
    q, r = _state(dims, 0)
    npex = (r.uniform(size=n) > 0.3).astype(np.int32)  # 0 = wall point
    umf = (0.05, -0.02, 0.01)
    nbc = [[20, 45, 25], [45, 45, 20]]  # x lo inviscid, z lo viscous, z hi inviscid
    out = O.wall_update(q.copy(), npex, dims, nbc, umf)
    Q, O5 = q.reshape(5, *dims[::-1]), out.reshape(5, *dims[::-1])  # [v][k][j][i]
    mask = npex.reshape(dims[::-1]) == 0
    exp = Q.copy()

    def inviscid(sl):
        sel = mask[sl]
        rho = Q[0][sl]
        m2 = (Q[1][sl] ** 2 + Q[2][sl] ** 2 + Q[3][sl] ** 2)
        e = HAMHAMM1 * rho ** GAM + 0.5 * m2 / rho
        exp[4][sl] = np.where(sel, e, exp[4][sl])

    def viscous(sl):
        sel = mask[sl]
        rho = Q[0][sl]
        for d in range(3):
            exp[1 + d][sl] = np.where(sel, -rho * umf[d], exp[1 + d][sl])
        m2 = exp[1][sl] ** 2 + exp[2][sl] ** 2 + exp[3][sl] ** 2
        exp[4][sl] = np.where(sel, HAMHAMM1 * rho + 0.5 * m2 / rho, exp[4][sl])

    inviscid((slice(None), slice(None), 0))          # x = 0
    viscous((0, slice(None), slice(None)))          # z = 0
    inviscid((dims[2] - 1, slice(None), slice(None)))  # z = lze - 1
    assert np.allclose(O5, exp, rtol=1e-14, atol=0)
    # interior points untouched
    assert np.array_equal(O5[:, 1:-1, :, 1:-1], Q[:, 1:-1, :, 1:-1])
