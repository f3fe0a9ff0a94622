"""kg_b200 -- B200 (sm_100a) method-of-lines solver for the Klein-Gordon field
on a Kerr-Schild / Schwarzschild background, a drop-in for the hot path of the
FlavioRosales/KG Fortran code.

The solver lives in libkg_b200.so behind the C ABI of include/kg_capi.h;
`LinesMethod` / `ScalarField` mirror the reference's Fortran objects on top of
it.  Importing the package loads the library and fails loudly if it has not
been built.
"""
from . import capi
from .capi import KgError, KgParams
from .lines_method import LinesMethod, ScalarField

capi.load()

__all__ = ["capi", "KgError", "KgParams", "LinesMethod", "ScalarField"]
