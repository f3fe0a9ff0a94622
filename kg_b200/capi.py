"""ctypes binding of libkg_b200.so (the C ABI declared in include/kg_capi.h).

The library is built in-tree (kg_b200/libkg_b200.so) by kg_b200/csrc/Makefile.
Loading fails with an ImportError when it is missing: there is no host
fallback for any solver operation.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libkg_b200.so")

KG_OK, KG_EINVAL, KG_ENOMEM, KG_ECUDA, KG_ESTATE, KG_ETIMEOUT, KG_ENODEV = range(7)
KG_KERR_SCHILD, KG_SCHW_EF = 0, 1
KG_OUTFLOW, KG_INFLOW = 0, 1

STATUS_NAMES = {0: "KG_OK", 1: "KG_EINVAL", 2: "KG_ENOMEM", 3: "KG_ECUDA", 4: "KG_ESTATE",
                5: "KG_ETIMEOUT", 6: "KG_ENODEV"}


class KgParams(C.Structure):
    """struct kg_params (include/kg_capi.h)."""
    _fields_ = [("Nx", C.c_int), ("Ny", C.c_int), ("Nz", C.c_int), ("g_pts", C.c_int),
                ("xmin", C.c_double), ("xmax", C.c_double), ("tmin", C.c_double), ("tmax", C.c_double),
                ("CFL", C.c_double), ("a", C.c_double), ("M_bh", C.c_double), ("m", C.c_double),
                ("metric", C.c_int), ("bc_rmax", C.c_int), ("n_det", C.c_int), ("l_max", C.c_int),
                ("dt_override", C.c_double), ("save_", C.c_double)]


class KgError(RuntimeError):
    def __init__(self, code, msg=""):
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


_P = C.c_void_p
_D = C.POINTER(C.c_double)
_I = C.c_int
_PP = C.POINTER(C.c_void_p)

# (name, restype, argtypes) of every entry point in include/kg_capi.h
SIGNATURES = [
    ("kg_create", _I, [C.POINTER(KgParams), _I, _PP]),
    ("kg_destroy", _I, [_P]),
    ("kg_last_error", C.c_char_p, [_P]),
    ("kg_get_scalars", _I, [_P, _D]),
    ("kg_set_time", _I, [_P, C.c_double]),
    ("kg_set_dt", _I, [_P, C.c_double]),
    ("kg_get_stream", C.c_void_p, [_P]),
    ("kg_device_bytes", C.c_size_t, [_P]),
    ("kg_synchronize", _I, [_P]),
    ("kg_set_state", _I, [_P, _I, _D]),
    ("kg_get_state", _I, [_P, _I, _D]),
    ("kg_set_state_device", _I, [_P, _I, C.c_void_p]),
    ("kg_get_state_device", _I, [_P, _I, C.c_void_p]),
    ("kg_pirk2", _I, [_P, _I]),
    ("kg_pirk3", _I, [_P, _I]),
    ("kg_rk3", _I, [_P, _I]),
    ("kg_rk4", _I, [_P, _I]),
    ("kg_set_precision", _I, [_P, _I]),
    ("kg_get_precision", _I, [_P]),
    ("kg_set_scheme", _I, [_P, _I, C.c_double]),
    ("kg_get_scheme", _I, [_P]),
    ("kg_fill_ghosts_cfg", _I, [_P]),
    ("kg_set_graphs", _I, [_P, _I]),
    ("kg_rhs", _I, [_P, _D, _D, C.c_uint]),
    ("kg_boundary", _I, [_P, C.c_uint]),
    ("kg_send_recv", _I, [_P]),
    ("kg_get_metric", _I, [_P, _D]),
    ("kg_set_metric", _I, [_P, _D]),
    ("kg_validate_inverse_metric", _I, [_P, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    ("kg_density", _I, [_P]),
    ("kg_get_density", _I, [_P, _D]),
    ("kg_mass_scalar", _I, [_P, _D]),
    ("kg_currents_detectors", _I, [_P, _D]),
    ("kg_proyector_detectors", _I, [_P, _D]),
    ("kg_diagnostic", _I, [_P, _I, _D]),
    ("kg_get_detectors", _I, [_P, _D, C.POINTER(C.c_int)]),
    ("kg_set_detectors", _I, [_P, _I, _D]),
    ("kg_sph_harmonics", _I, [_P, _I, _D]),
    ("kg_project_all_shells", _I, [_P, _I, _I, _D]),
    ("kg_bessel_basis", _I, [_P, _I, _I, _D, _D]),
    ("kg_sph_ft_radial", _I, [_P, _I, _I, _I, _D]),
    ("kg_profile_enable", _I, [_P, _I]),
    ("kg_profile_read", _I, [_P, _D, C.POINTER(C.c_longlong)]),
    ("kg_profile_kinds", _I, []),
    ("kg_profile_kind_name", C.c_char_p, [_I]),
    ("kg_launch_count", C.c_longlong, [_P]),
    ("kg_set_kernel_variant", _I, [_P, _I]),
    ("kg_set_tile_rows", _I, [_P, _I]),
    ("kg_check_wait_timeout", _I, [_P, C.c_longlong]),
    ("kg_get_tile_rows", _I, [_P]),
    ("kg_batch_create", _I, [_I, _PP]),
    ("kg_batch_destroy", _I, [_P]),
    ("kg_batch_last_error", C.c_char_p, [_P]),
    ("kg_batch_add", _I, [_P, _P]),
    ("kg_batch_remove", _I, [_P, _P]),
    ("kg_batch_size", _I, [_P]),
    ("kg_batch_rk4", _I, [_P, _I]),
    ("kg_batch_synchronize", _I, [_P]),
    ("kg_batch_set_tuning", _I, [_P, _I, _I]),
    ("kg_batch_set_precision", _I, [_P, _I]),
    ("kg_batch_proyector_detectors", _I, [_P, _D]),
    ("kg_batch_alm_count", C.c_longlong, [_P]),
    ("kg_save_checkpoint", _I, [_P, C.c_char_p]),
    ("kg_load_checkpoint", _I, [_P, C.c_char_p]),
    ("kg_hier_create", _I, [C.POINTER(KgParams), _I, _D, _I, _PP]),
    ("kg_hier_destroy", _I, [_P]),
    ("kg_hier_last_error", C.c_char_p, [_P]),
    ("kg_hier_levels", _I, [_P]),
    ("kg_hier_level", _P, [_P, _I]),
    ("kg_hier_rk4", _I, [_P, _I]),
    ("kg_hier_rk3", _I, [_P, _I]),
    ("kg_hier_pirk2", _I, [_P, _I]),
    ("kg_hier_pirk3", _I, [_P, _I]),
    ("kg_hier_synchronize", _I, [_P]),
    ("kg_batch_get_tuning", _I, [_P, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    ("kg_batch_set_dispatch", _I, [_P, _I, _I]),
    ("kg_batch_get_dispatch", _I, [_P, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    ("kg_batch_set_tile_rows", _I, [_P, _I]),
    ("kg_batch_get_tile_rows", _I, [_P, C.POINTER(C.c_int)]),
    ("kg_batch_launch_count", C.c_longlong, [_P]),
    ("kg_batch_get_stream", C.c_void_p, [_P]),
    ("kg_integrate_mass_noalloc", _I, [C.c_void_p, C.c_void_p, _I, _I, _I, C.c_double, C.c_double,
                                       C.c_double, C.c_void_p, C.c_void_p]),
]

_lib = None


def load():
    """Load libkg_b200.so and declare every entry point; raises ImportError if absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is not built; run `make -C kg_b200/csrc` (or __graft_entry__.build())")
    lib = C.CDLL(LIB_PATH)
    for name, res, args in SIGNATURES:
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def check(h, code):
    if code != KG_OK:
        msg = load().kg_last_error(h) if h else b""
        raise KgError(code, msg.decode() if msg else "")
