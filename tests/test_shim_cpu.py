"""The pTatin3D plug-in (ptatin-gene_b200/shim/stokes_operators_b200.c)
compiles against the reference's own headers (with the PETSc stand-in)."""
import os
import subprocess

import pytest

from conftest import REPO


def test_shim_compiles_against_reference_headers():
    import oracle
    ref = oracle.reference_tree()
    cmd = ["make", "-s", "-C", os.path.join(REPO, "oracle"), "shim-check"] + ([f"REF={ref}"] if ref else [])
    out = subprocess.run(cmd, capture_output=True, text=True)
    if "skipped" in out.stdout:
        pytest.skip(out.stdout.strip())
    assert out.returncode == 0, out.stdout + out.stderr
    assert "shim ok" in out.stdout
