"""Headless VTK writer (host only): round trip through the minimal reader."""
import numpy as np

import oracle as O
from compact_schemes_b200 import vtk


def test_vtk_round_trip(tmp_path):
    dims = (6, 5, 4)
    q = O.tgv_init(dims, 0.1, 1e-4, 0)
    path = tmp_path / "state.vtk"
    vtk.write_state(path, q, dims)
    d = vtk.read(path)
    assert d["dims"] == dims
    n = int(np.prod(dims))
    rho = q[:n]
    assert np.allclose(d["rho"], rho, rtol=1e-6)
    assert np.allclose(d["u"], q[n:2 * n] / rho, rtol=1e-5, atol=1e-7)
    h = 2 * np.pi / dims[0]
    assert np.allclose(d["points"][1], [h, 0.0, 0.0], atol=1e-6)
    assert np.allclose(d["points"][dims[0]], [0.0, 2 * np.pi / dims[1], 0.0], atol=1e-6)
    p = 0.4 * (q[4 * n:] - 0.5 * (q[n:2 * n] ** 2 + q[2 * n:3 * n] ** 2 + q[3 * n:4 * n] ** 2) / rho)
    assert np.allclose(d["p"], p, rtol=1e-5)
