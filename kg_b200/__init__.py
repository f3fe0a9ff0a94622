"""kg_b200 -- B200 (sm_100a) method-of-lines solver for the Klein-Gordon field
on a Kerr-Schild / Schwarzschild background, a drop-in for the hot path of the
FlavioRosales/KG Fortran code.

The solver lives in libkg_b200.so behind the C ABI of include/kg_capi.h;
`LinesMethod` / `ScalarField` mirror the reference's Fortran objects on top of
it.  The library is mapped on first use (`capi.load()`, called by every solver
constructor), so host-only modules of the package (request drawing, replica
plumbing, initial data) import without it; any solver operation fails loudly
with an ImportError if it has not been built.
"""
from . import capi
from .capi import KgError, KgParams
from .lines_method import LinesMethod, ScalarField

__all__ = ["capi", "KgError", "KgParams", "LinesMethod", "ScalarField"]
