"""Generate tests/golden/reference_pins.npz from the reference's own code.

Runs only where the reference sources are present: `make -C oracle ref`
compiles, from the reference files where they lie,
  * numerics_base<double>::deriv_setup   (src/numerics_base.hpp:182-297)
  * calc_fluxes_pre_compute_cpu           (tests/test_physics_serial.cu:41-163, float)
  * calc_time_step_cpu                    (tests/test_physics.cu:57-117, float)
into oracle/_ref/.  This script feeds them seeded inputs and stores inputs and
outputs as the committed fixture that pins the oracle (tests/test_oracle_pins.py).

    python tests/golden/make_golden.py
"""
import ctypes
import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
REF = os.path.join(ROOT, "oracle", "_ref")


def main():
    subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref"])
    vp = ctypes.c_void_p
    P = lambda a: a.ctypes.data_as(vp)  # noqa: E731
    out = {}

    coeffs = ctypes.CDLL(os.path.join(REF, "libref_coeffs.so"))
    pbco, pbci = np.zeros(16), np.zeros(16)
    coeffs.ref_deriv_setup(P(pbco), P(pbci))
    out["pbco"], out["pbci"] = pbco, pbci

    # calc_fluxes_pre_compute_cpu on the input distribution of the reference
    # test (tests/test_physics_serial.cu:190-214), lmx = 1024, seeded here.
    rng = np.random.default_rng(20240601)
    n = 1024
    f = lambda k, lo=0.0, hi=1.0: rng.uniform(lo, hi, k).astype(np.float32)  # noqa: E731
    qa, p, xim, etm, zem, de = f(5 * n), f(n), f(3 * n), f(3 * n), f(3 * n), f(5 * n)
    tau, heat = f(6 * n, 0.1, 1.0), f(3 * n, 0.1, 1.0)
    umf = np.array([0.3, 0.1, 0.1], dtype=np.float32)
    buf = np.zeros(15 * n, dtype=np.float32)
    de_out = de.copy()
    flux = ctypes.CDLL(os.path.join(REF, "libref_flux_twin.so"))
    flux.ref_fluxes_pre_cpu.argtypes = [vp] * 10 + [ctypes.c_uint]
    flux.ref_fluxes_pre_cpu(P(buf), P(qa), P(p), P(de_out), P(xim), P(etm), P(zem), P(tau),
                            P(heat), P(umf), n)
    for k, v in dict(flux_qa=qa, flux_p=p, flux_xim=xim, flux_etm=etm, flux_zem=zem, flux_de=de,
                     flux_tau=tau, flux_heat=heat, flux_umf=umf, flux_buffer=buf,
                     flux_de_out=de_out).items():
        out[k] = v

    # calc_time_step_cpu (tests/test_physics.cu:133-142 distribution), cfl 0.95.
    n = 4096
    xim, etm, zem, de, yaco, ssk = f(3 * n), f(3 * n), f(3 * n), f(5 * n), f(n), f(n)
    dt = ctypes.CDLL(os.path.join(REF, "libref_dt_twin.so"))
    dt.ref_time_step_cpu.argtypes = [vp] * 7 + [ctypes.c_float, ctypes.c_uint]
    dt.ref_time_step_cpu.restype = ctypes.c_float
    res = dt.ref_time_step_cpu(P(xim), P(etm), P(zem), P(de), P(yaco), P(ssk), P(umf),
                               ctypes.c_float(0.95), n)
    for k, v in dict(dt_xim=xim, dt_etm=etm, dt_zem=zem, dt_de=de, dt_yaco=yaco, dt_ssk=ssk,
                     dt_umf=umf).items():
        out[k] = v
    out["dt_cfl"] = np.float32(0.95)
    out["dt_result"] = np.float32(res)

    path = os.path.join(ROOT, "tests", "golden", "reference_pins.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, "dt =", res)


if __name__ == "__main__":
    sys.exit(main())
