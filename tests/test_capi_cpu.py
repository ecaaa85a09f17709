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


def test_struct_layouts_match_the_header(tmp_path):
    """The ctypes mirrors have the C structs' sizes and field offsets
    (checked against gcc on include/pt_b200.h)."""
    import subprocess

    from pt_b200 import _capi
    structs = {"pt_mesh_desc": _capi.MeshDesc, "pt_solve_opts": _capi.SolveOpts,
               "pt_solve_stats": _capi.SolveStats, "pt_server_opts": _capi.ServerOpts,
               "pt_server_result": _capi.ServerResult}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "pt_b200.h"', "int main(void) {"]
    for cname, cls in structs.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for f, _ in cls._fields_:
            if f == "reserved":
                continue
            lines.append(f'printf("{cname} {f} %zu\\n", offsetof({cname}, {f}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(REPO, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    for line in filter(None, out):
        cname, field, val = line.split()
        cls = structs[cname]
        got = ctypes.sizeof(cls) if field == "size" else getattr(cls, field).offset
        assert got == int(val), (cname, field, got, val)


def test_server_option_validation_without_device():
    from pt_b200 import _capi
    lib = _capi.load()
    o = _capi.ServerOpts()
    lib.pt_server_opts_default(ctypes.byref(o))
    assert o.max_active == 256 and o.memory_budget_bytes == 120 << 30 and o.rtol == 1e-8
    o.max_active = 0
    h = ctypes.c_void_p()
    assert lib.pt_server_create(ctypes.byref(o), ctypes.byref(h)) == 1
    assert b"max_active" in lib.pt_last_error()


def test_solver_defaults_without_device():
    """pt_solve_opts_default: FGMRES(30), rtol 1e-8, Chebyshev(3)-Jacobi in FP32
    over [0.2, 1.1] lambda_max (the reference's esteig window), Galerkin
    coarse levels."""
    from pt_b200 import _capi
    from pt_b200.solver import KSP, PC
    lib = _capi.load()
    o = _capi.SolveOpts()
    lib.pt_solve_opts_default(ctypes.byref(o))
    assert o.ksp == KSP["fgmres"] and o.restart == 30 and o.rtol == 1e-8
    assert o.cheby_degree == 3 and o.cheby_fp32 == 1
    assert (o.cheby_emin, o.cheby_emax) == (0.2, 1.1)
    assert o.mg_assembled == 2 and o.pc_graph == 1 and o.mg_fine_degree == 0 and o.mg_coarse_half == 1
    assert PC["mg"] == 3
