"""The C-ABI library loads and exports every symbol include/compact_b200.h declares."""
import os
import re

import compact_schemes_b200 as cs

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "compact_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(cs_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_declared_symbols():
    L = cs.lib()
    names = declared_symbols()
    assert len(names) >= 10
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_errors_are_status_codes_not_exits():
    import ctypes
    L = cs.lib()
    h = ctypes.c_void_p()
    bad = cs.nbc_array([[11, 45, 45], [45, 45, 45]])
    rc = L.cs_numerics_create(ctypes.byref(h), cs.Dcomp.of(8, 8, 8), bad)
    assert rc == -1 and b"boundary" in L.cs_last_error()
    rc = L.cs_numerics_create(ctypes.byref(h), cs.Dcomp(7, 8, 8, 8), cs.nbc_array([[45] * 3] * 2))
    assert rc == -1
    assert L.cs_deriv_setup(None) == -1


def test_interface_coeffs_bit_identical_to_reference():
    """The library's host-side deriv_setup reproduces the reference's weights exactly."""
    import ctypes
    import numpy as np
    g = np.load(os.path.join(ROOT, "tests", "golden", "reference_pins.npz"))
    a, b = (ctypes.c_double * 16)(), (ctypes.c_double * 16)()
    assert cs.lib().cs_interface_coeffs(a, b) == 0
    assert np.array_equal(np.array(a), g["pbco"])
    assert np.array_equal(np.array(b), g["pbci"])
