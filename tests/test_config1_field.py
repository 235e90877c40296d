"""The derivative-and-filter workload's input field (64^3 non-periodic unit
cube, 8 Fourier modes from MT19937-64 seed 0): the package's generator
against the oracle's std::mt19937_64 one, and the oracle's derivative of the
field against the analytic derivative (CPU)."""
import numpy as np

import oracle as O

DIMS = (64, 64, 64)


def test_modes_match_std_mt19937_64():
    import compact_schemes_b200 as cs
    mine = np.array(cs.grid.fourier_modes(0, 8))
    modes, _ = O.fourier_field(DIMS, 0, 8)
    assert np.array_equal(mine, modes)
    assert ((modes[:, 1:4] >= 1) & (modes[:, 1:4] <= 8)).all()
    assert ((modes[:, 0] >= 0.1) & (modes[:, 0] < 1.0)).all()
    assert ((modes[:, 4] >= 0) & (modes[:, 4] < 2 * np.pi)).all()


def test_field_values_match():
    import compact_schemes_b200 as cs
    _, f = O.fourier_field(DIMS, 0, 8)
    mine = cs.grid.fourier_field(DIMS, 0, 8, device="cpu").numpy()
    assert np.abs(mine - f).max() <= 1e-14 * np.abs(f).max()


def test_oracle_derivative_against_analytic():
    """Index-space derivative x (n - 1) against d f / d x: the sixth-order
    interior and the third-order closures resolve the <= 8 wavelengths over
    63 intervals to a few percent at most, and the error falls with h."""
    modes, f = O.fourier_field(DIMS, 0, 8)
    errs = []
    for n in (64, 128):
        dims = (n, n, n)
        _, f = O.fourier_field(dims, 0, 8)
        i = np.arange(n) / (n - 1)
        z, y, x = np.meshgrid(i, i, i, indexing="ij")
        exact = [np.zeros(n ** 3) for _ in range(3)]
        for a, kx, ky, kz, ph in modes:
            c = (a * 2 * np.pi * np.cos(2 * np.pi * (kx * x + ky * y + kz * z) + ph)).ravel()
            for ax, k in enumerate((kx, ky, kz)):
                exact[ax] += k * c
        e = []
        for ax in range(3):
            d = O.deriv(f, dims, ax, 0, 0) * (n - 1)
            e.append(np.abs(d - exact[ax]).max() / np.abs(exact[ax]).max())
        errs.append(max(e))
    assert errs[0] < 0.1 and errs[1] < errs[0] / 4, errs
