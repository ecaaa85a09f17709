"""The C-ABI library loads on a CPU-only host and exports every entry point
declared in include/pt_b200.h (no compute calls without a GPU)."""
import ctypes
import os
import re

from conftest import REPO


def declared_symbols():
    txt = open(os.path.join(REPO, "include", "pt_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(pt_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_declared_symbols():
    from pt_b200 import _capi
    lib = _capi.load()
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing
    assert set(declared_symbols()) <= set(_capi.SIGNATURES)


def test_version_and_error_string():
    from pt_b200 import _capi
    lib = _capi.load()
    assert b"sm_100a" in lib.pt_version()
    assert isinstance(lib.pt_last_error(), bytes)


def test_bad_args_rejected_without_device():
    """Argument validation happens before any CUDA call."""
    from pt_b200 import _capi
    lib = _capi.load()
    h = ctypes.c_void_p()
    st = lib.pt_op_create(ctypes.byref(_capi.MeshDesc(0, 4, 4)), ctypes.byref(h))
    assert st == 1 and b"element counts" in lib.pt_last_error()
    assert lib.pt_op_create(None, ctypes.byref(h)) == 1
    assert lib.pt_a11_apply_d(None, None, None) == 1
