"""The C-ABI library loads and exports every entry point include/babelsim_b200.h declares (no GPU calls)."""
import os
import re
import subprocess

from helpers import ROOT


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "babelsim_b200.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(bsg_\w+)\s*\(", text, re.M)))


def test_header_matches_binding_table():
    from babelsim_b200._lib import EXPORTS
    assert sorted(EXPORTS) == declared_symbols()


def test_library_exports_every_declared_symbol():
    from babelsim_b200 import _lib
    L = _lib.lib()  # loads the .so; raises if it is missing
    for name in declared_symbols():
        assert hasattr(L, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (bsg_\w+)", out))
    assert set(declared_symbols()) <= exported


def test_errors_are_reported_without_a_device():
    """A context on a missing device fails with a status code and a message, never a crash."""
    import ctypes as C
    from babelsim_b200 import _lib
    h = C.c_void_p()
    code = _lib.lib().bsg_context_create(10_000, C.byref(h))
    assert code != 0
    assert _lib.lib().bsg_global_error()


def test_static_pcg_rejects_oversized_systems_without_a_device():
    """The allocation-free PCG checks its size limit before touching the device."""
    import ctypes as C
    from babelsim_b200 import _lib
    res = _lib.SolveResult()
    L = _lib.lib()
    code = L.bsg_pcg_jacobi_static(131073, None, None, None, None, None, None, 1e-30, 1e-12, 10, C.byref(res))
    assert code == 1   # BSG_ERR_ARGUMENT
    assert b"131072" in L.bsg_global_error()
    code = L.bsg_pcg_jacobi_static(0, None, None, None, None, None, None, 1e-30, 1e-12, 10, C.byref(res))
    assert code == 1
