"""Numpy emulation of the warp line solver (compact_schemes_b200/csrc/line_solver.cuh).

Runs the exact sequence of operations one warp performs -- per-lane forward /
backward elimination, the PCR steps over "shuffles" (numpy rolls with
the shuffle's own-value behaviour at the warp edges), back substitution and
the cyclic correction -- from the tables the library exports, so that the
tables can be validated on a machine without a GPU.
"""
import numpy as np


def emulate(tab, r):
    n, lt, p, last = tab["n"], tab["lt"], tab["p"], tab["last_len"]
    d = np.zeros((32, lt))
    for lane in range(p):
        ln = lt if lane < p - 1 else last
        d[lane, :ln] = r[lane * lt:lane * lt + ln]
    lens = np.array([lt if c < p - 1 else (last if c == p - 1 else 0) for c in range(32)])
    f1, f2, b1, b2 = (tab[k].T for k in ("fwd1", "fwd2", "bwd1", "bwd2"))
    for t in range(lt):
        d[:, t] = f1[:, t] * d[:, t] + (f2[:, t] * d[:, t - 1] if t > 0 else 0.0)
    for t in range(lt - 2, -1, -1):
        d[:, t] = b1[:, t] * d[:, t] + b2[:, t] * d[:, t + 1]
    y0 = d[:, 0].copy()
    y1 = np.array([d[c, lens[c] - 1] if lens[c] >= 2 else 0.0 for c in range(32)])

    def up(x, k):      # __shfl_up_sync: lanes < k keep their own value
        o = x.copy(); o[k:] = x[:-k]; return o

    def down(x, k):    # __shfl_down_sync: lanes >= 32-k keep their own value
        o = x.copy(); o[:-k] = x[k:]; return o

    k1, k2 = tab["k1"], tab["k2"]
    n0 = y0 - k1[0, 0] * up(y1, 1) - k2[0, 0] * y1
    n1 = y1 - k1[0, 1] * y0 - k2[0, 1] * down(y0, 1)
    y0, y1 = n0, n1
    for s in range(1, tab.get("pcr64", 6)):
        dl = 1 << (s - 1)
        n0 = y0 - k1[s, 0] * up(y0, dl) - k2[s, 0] * down(y0, dl)
        n1 = y1 - k1[s, 1] * up(y1, dl) - k2[s, 1] * down(y1, dl)
        y0, y1 = n0, n1
    X0, X1 = y0 * tab["invb"][0], y1 * tab["invb"][1]
    rca, rcc = tab["rca"].T, tab["rcc"].T
    x = d - rca * X0[:, None] - rcc * X1[:, None]
    x[:, 0] = X0
    for c in range(32):
        if lens[c] >= 2:
            x[c, lens[c] - 1] = X1[c]
    if tab["cyclic"]:
        lastv = X1[p - 1] if lens[p - 1] >= 2 else X0[p - 1]
        beta = (X0[0] + tab["s2"] * lastv) * tab["s1"]
        x = x - beta * tab["cycz"].T
    out = np.zeros(n)
    for lane in range(p):
        ln = lt if lane < p - 1 else last
        out[lane * lt:lane * lt + ln] = x[lane, :ln]
    return out
