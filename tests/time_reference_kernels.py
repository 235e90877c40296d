"""Time the reference's own compact-derivative kernel against this library's.

deriv_kernel_2d<Axis, double> of the reference (src/cuda/kernels/numerics_pc.hpp,
launched as numerics_pc::deriv2d does, src/numerics_pc.hpp:121-168) is
compiled for sm_100a from the reference sources into oracle/_ref/libref_gpu.so
by `make -C oracle ref`.  Both kernels differentiate the same 16.8 M-point
field (134 MB in, 134 MB out: larger than the 126 MB L2) along one axis, with
the interface sums of the periodic (ndf = 1) case precomputed in the recv
buffers, and are timed with CUDA events on one stream after warm-up.

Axes 1 and 2 only: the reference's axis-0 kernel indexes rows correctly only
for lze = 1 (src/cuda/kernels/transforms.hpp:72-88), and a block with lze = 1
that is larger than L2 has a second axis longer than either library's lines.

Run on a B200:  python tests/time_reference_kernels.py   (prints one JSON line)
"""
import ctypes
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
REF_GPU = os.path.join(ROOT, "oracle", "_ref", "libref_gpu.so")


def main():
    import torch
    import compact_schemes_b200 as cs
    R = ctypes.CDLL(REF_GPU)
    vp = ctypes.c_void_p
    R.ref_gpu_deriv2d.argtypes = [ctypes.c_int, vp, vp, vp, vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                  ctypes.c_int, ctypes.c_int, ctypes.c_uint, ctypes.c_uint, vp]
    dev = torch.device("cuda:0")
    stream = torch.cuda.current_stream()
    sp = vp(stream.cuda_stream)
    reps, warm = 20, 3
    rows = []
    for dims, axis in (((256, 256, 256), 1), ((256, 256, 256), 2)):
        lmx = int(np.prod(dims))
        for ndf in (0, 1):
            b = cs.BC_PERIODIC if ndf else cs.BC_NON_REFLECTIVE
            nbc = [[b] * 3] * 2
            nm = cs.numerics_pc(dims, nbc)
            nm.deriv_setup()
            g = torch.Generator(device=dev).manual_seed(1)
            f = torch.randn(lmx, dtype=torch.float64, device=dev, generator=g)
            if ndf:
                # interface sums of this field on every axis, exchanged with itself
                blk = torch.zeros(15 * lmx, dtype=torch.float64, device=dev)
                blk[axis * lmx:(axis + 1) * lmx] = f
                nm.fill_buffers(blk, 0, 1, 0, dims)
                nm.mpigo(dims, None, 1, 0)
                del blk
            ours = torch.empty(3 * lmx, dtype=torch.float64, device=dev)
            theirs = torch.empty(3 * lmx, dtype=torch.float64, device=dev)
            drva, _, recv = nm.buffers(axis)
            F = (dims[1] * dims[2], dims[0] * dims[2], dims[0] * dims[1])[axis]
            scratch = torch.zeros(10 * F, dtype=torch.float64, device=dev)
            _, pbci = nm.coeffs()
            dpbci = torch.tensor(pbci, dtype=torch.float64, device=dev)

            def run_ours():
                nm.deriv2d(axis, f, ours, ndf, ndf, dims, 0, 0, stream=stream)

            def run_ref():
                rc = R.ref_gpu_deriv2d(axis, vp(f.data_ptr()), vp(theirs.data_ptr()), vp(recv),
                                       vp(dpbci.data_ptr()), vp(scratch.data_ptr()), ndf, ndf, *dims, 0, 0, sp)
                assert rc == 0, rc

            res = {}
            for name, fn in (("ours", run_ours), ("reference", run_ref)):
                for _ in range(warm):
                    fn()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                torch.cuda.synchronize()
                e0.record(stream)
                for _ in range(reps):
                    fn()
                e1.record(stream)
                torch.cuda.synchronize()
                ms = e0.elapsed_time(e1) / reps
                res[name] = {"ms": ms, "gbs": 16.0 * lmx / (ms * 1e-3) / 1e9}
            a = ours[axis * lmx:(axis + 1) * lmx]
            t = theirs[axis * lmx:(axis + 1) * lmx]
            err = float((a - t).abs().max() / t.abs().max())
            rows.append({"dims": dims, "axis": axis, "ndf": ndf, "ours_ms": res["ours"]["ms"],
                         "ours_gbs": res["ours"]["gbs"], "reference_ms": res["reference"]["ms"],
                         "reference_gbs": res["reference"]["gbs"],
                         "speedup": res["reference"]["ms"] / res["ours"]["ms"], "max_rel_diff": err})
            nm.close()
            del f, ours, theirs, scratch
            torch.cuda.empty_cache()
    print(json.dumps({"kernel": "compact first derivative, FP64, one field", "bytes_per_point": 16,
                      "reps": reps, "rows": rows}))


if __name__ == "__main__":
    main()
