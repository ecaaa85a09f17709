"""pt_b200 -- B200-native matrix-free Q2-P1disc Stokes operator (pTatin3D hot path).

The compute path is libpt_b200.so (hand-written sm_100a CUDA behind the C ABI
of include/pt_b200.h); this package is its host-side mirror of the
reference's operator interface plus mesh/input helpers.
"""
from . import mesh
from ._capi import PtError, load
from .operator import A11_OPS, MatStokesMF

__all__ = ["MatStokesMF", "A11_OPS", "PtError", "load", "mesh"]
