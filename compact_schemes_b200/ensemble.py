"""Batched ensemble of independent boxes (cs_ensemble_* of include/compact_b200.h).

Each box is a SolverConfig (FP64, uniform grid, no GCBC); all boxes share one
packed device state in which box b's q [5][lmx_b] starts at box_offset(b).  A
step advances every box by one RK step with its own CFL time step, in one
persistent launch per RK stage replayed as a captured CUDA graph.  Per box
the arithmetic is that of Solver.step: boxes whose axes all exceed 64 points
match a per-box Solver bit for bit, shorter axes (solved in 4-point chunks)
agree with it to rounding.
"""
from __future__ import annotations

import ctypes
import math

from . import check, lib, ptr, stream_ptr
from .solver import SolverConfig, tgv_config

SIZES = (32, 48, 64, 96, 128)


class EnsembleTuning(ctypes.Structure):
    _fields_ = [("window", ctypes.c_int), ("tile", ctypes.c_int), ("ctas_per_sm", ctypes.c_int),
                ("chunk", ctypes.c_int)]

    def as_dict(self):
        return {"window": self.window, "tile": self.tile, "ctas_per_sm": self.ctas_per_sm, "chunk": self.chunk}


class Ensemble:
    def __init__(self, cfgs):
        self.cfgs = list(cfgs)
        arr = (SolverConfig * len(self.cfgs))(*self.cfgs)
        self._h = ctypes.c_void_p()
        check(lib().cs_ensemble_create(ctypes.byref(self._h), len(self.cfgs), arr))

    @property
    def nbox(self):
        return len(self.cfgs)

    def close(self):
        if self._h:
            lib().cs_ensemble_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def state_size(self):
        n = ctypes.c_int64()
        check(lib().cs_ensemble_state_size(self._h, ctypes.byref(n)))
        return n.value

    def box_offset(self, b):
        n = ctypes.c_int64()
        check(lib().cs_ensemble_box_offset(self._h, int(b), ctypes.byref(n)))
        return n.value

    def box_view(self, q, b):
        """The [5 * lmx_b] slice of the packed state q (a torch tensor) for box b."""
        c = self.cfgs[b]
        o = self.box_offset(b)
        return q[o:o + 5 * c.lxi * c.let * c.lze]

    def step(self, q, stream=None):
        check(lib().cs_ensemble_step(self._h, ptr(q), stream_ptr(stream)))

    def last_dt(self):
        out = (ctypes.c_double * self.nbox)()
        check(lib().cs_ensemble_last_dt(self._h, out))
        return list(out)

    def set_wait(self, poll_limit=20000000, extra=0):
        """Dependency-wait limit and, for tests of the timeout path, `extra`
        finished items every wait needs beyond what the queue produces."""
        check(lib().cs_ensemble_set_wait(self._h, int(poll_limit), int(extra)))

    def tuning(self):
        t = EnsembleTuning()
        check(lib().cs_ensemble_get_tuning(self._h, ctypes.byref(t)))
        return t.as_dict()

    def set_tuning(self, window=0, tile=8, ctas_per_sm=0, chunk=4):
        t = EnsembleTuning(int(window), int(tile), int(ctas_per_sm), int(chunk))
        check(lib().cs_ensemble_set_tuning(self._h, ctypes.byref(t)))

    def autotune(self, q, reps=3, stream=None):
        """Time every candidate tuning on a scratch copy of q; keep the fastest.
        Returns (tuning dict, ms per step)."""
        t = EnsembleTuning()
        ms = ctypes.c_double()
        check(lib().cs_ensemble_autotune(self._h, ptr(q), int(reps), ctypes.byref(t), ctypes.byref(ms),
                                         stream_ptr(stream)))
        return t.as_dict(), ms.value


class MT19937_64:
    """64-bit Mersenne Twister (Matsumoto & Nishimura), the published
    MT19937-64 parameters; the same sequence as std::mt19937_64."""
    _N, _M = 312, 156
    _MATRIX_A = 0xB5026F5AA96619E9
    _UPPER, _LOWER = 0xFFFFFFFF80000000, 0x7FFFFFFF
    _MASK = (1 << 64) - 1

    def __init__(self, seed=0):
        self.mt = [0] * self._N
        self.mt[0] = seed & self._MASK
        for i in range(1, self._N):
            prev = self.mt[i - 1]
            self.mt[i] = (6364136223846793005 * (prev ^ (prev >> 62)) + i) & self._MASK
        self.idx = self._N

    def _twist(self):
        mt = self.mt
        for i in range(self._N):
            x = (mt[i] & self._UPPER) | (mt[(i + 1) % self._N] & self._LOWER)
            xa = x >> 1
            if x & 1:
                xa ^= self._MATRIX_A
            mt[i] = mt[(i + self._M) % self._N] ^ xa
        self.idx = 0

    def next_u64(self):
        if self.idx >= self._N:
            self._twist()
        x = self.mt[self.idx]
        self.idx += 1
        x ^= (x >> 29) & 0x5555555555555555
        x ^= (x << 17) & 0x71D67FFFEDA60000
        x ^= (x << 37) & 0xFFF7EEE000000000
        x ^= x >> 43
        return x & self._MASK

    def uniform(self):
        """Uniform in [0, 1) from the top 53 bits."""
        return (self.next_u64() >> 11) * (1.0 / 9007199254740992.0)


def draw_boxes(nbox=64, seed=0, sizes=SIZES, mach=(0.05, 0.3), re=(400.0, 3200.0)):
    """Seeded box set: per box, in this order, lxi, let, lze uniform in `sizes`
    (index floor(u * len(sizes))), Mach uniform in [mach), Re uniform in [re)
    with u from MT19937-64 seeded `seed`.  Returns [(dims, mach, re)]."""
    g = MT19937_64(seed)
    out = []
    for _ in range(nbox):
        dims = tuple(sizes[min(int(g.uniform() * len(sizes)), len(sizes) - 1)] for _ in range(3))
        m = mach[0] + (mach[1] - mach[0]) * g.uniform()
        r = re[0] + (re[1] - re[0]) * g.uniform()
        out.append((dims, m, r))
    return out


def ensemble_tgv(boxes, cfl=0.5, viscous=True):
    """SolverConfigs of periodic Taylor-Green boxes [(dims, mach, re)]."""
    return [tgv_config(None, mach=m, re=r, cfl=cfl, viscous=viscous, use_graph=True, dims=d) for d, m, r in boxes]


def ensemble_points(boxes):
    return sum(math.prod(d) for d, _, _ in boxes)


def _main(argv=None):
    """python -m compact_schemes_b200.ensemble [--boxes B] [--steps K]: the
    first B boxes of the seeded 64-box set, K ensemble steps (profiling driver)."""
    import argparse
    import torch
    from .solver import tgv_init
    p = argparse.ArgumentParser()
    p.add_argument("--boxes", type=int, default=64)
    p.add_argument("--steps", type=int, default=2)
    a = p.parse_args(argv)
    from compact_schemes_b200 import ensemble as E  # the package's classes, not __main__'s
    boxes = E.draw_boxes(64, 0)[:a.boxes]
    ens = E.Ensemble(E.ensemble_tgv(boxes))
    q = torch.zeros(ens.state_size(), dtype=torch.float64, device="cuda")
    for b, (d, m, _) in enumerate(boxes):
        tgv_init(ens.box_view(q, b), d, m, 1e-4, b)
    for _ in range(a.steps):
        ens.step(q)
    print("boxes", a.boxes, "points", ensemble_points(boxes), "dt[0]", ens.last_dt()[0])


if __name__ == "__main__":
    _main()
