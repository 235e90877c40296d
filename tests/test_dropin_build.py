"""The drop-in C++ headers (include/compact_schemes/*.hpp) compile against the C ABI."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NVCC = "/usr/local/cuda/bin/nvcc"


def build_demo(out, src="dropin_demo.cpp"):
    cmd = [NVCC, "-std=c++17", "-O2", "-gencode", "arch=compute_100a,code=sm_100a",
           "-I" + os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "cpp", src),
           "-o", out, "-L" + os.path.join(ROOT, "compact_schemes_b200"), "-lcompact_b200",
           "-Xlinker", "-rpath", "-Xlinker", os.path.join(ROOT, "compact_schemes_b200")]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return out


@pytest.mark.skipif(not os.path.exists(NVCC) and shutil.which("nvcc") is None, reason="no nvcc")
def test_dropin_headers_compile(tmp_path):
    build_demo(str(tmp_path / "dropin_demo"))


@pytest.mark.skipif(not os.path.exists(NVCC) and shutil.which("nvcc") is None, reason="no nvcc")
def test_reference_driver_sequence_compiles(tmp_path):
    """The reference driver's loop (driver/canard.cu:97-224) call for call,
    gcbc_go with the reference's parameter list included."""
    build_demo(str(tmp_path / "driver_sequence"), "driver_sequence.cpp")
