"""CPU checks of the C ABI library: it loads without a GPU, exports every
symbol include/kg_capi.h declares, the ctypes binding covers them all, and
handle creation fails cleanly (no host fallback) when no device is present."""
import ctypes as C
import os
import re

import pytest

from conftest import ROOT, have_gpu


def _declared():
    src = open(os.path.join(ROOT, "include", "kg_capi.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(kg_\w+)\s*\(", src)))


def test_header_declares_entry_points():
    names = _declared()
    for must in ("kg_create", "kg_destroy", "kg_pirk2", "kg_pirk3", "kg_rk3", "kg_rk4", "kg_rhs", "kg_boundary",
                 "kg_set_state", "kg_get_state", "kg_proyector_detectors", "kg_mass_scalar"):
        assert must in names


def test_library_exports_every_declared_symbol():
    from kg_b200 import capi
    lib = C.CDLL(capi.LIB_PATH)
    missing = [n for n in _declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_ctypes_binding_covers_header():
    from kg_b200 import capi
    bound = {n for n, _, _ in capi.SIGNATURES}
    assert set(_declared()) <= bound


@pytest.mark.skipif(have_gpu(), reason="checks the no-device path")
def test_create_without_device_fails_loudly():
    from kg_b200 import LinesMethod, KgError
    with pytest.raises(KgError):
        LinesMethod(16, 9, 17, 1.8, 12.0, 0.25)


def test_invalid_params_rejected():
    from kg_b200 import capi
    lib = capi.load()
    p = capi.KgParams(16, 9, 17, 3, 1.8, 12.0, 0.0, 1.0, 0.25, 0.0, 1.0, 0.0, 0, 0, 5, 10, 0.0, 0.0)
    h = C.c_void_p()
    assert lib.kg_create(C.byref(p), -1, C.byref(h)) == capi.KG_EINVAL  # g_pts must be 2
    assert lib.kg_destroy(None) == capi.KG_EINVAL
    assert lib.kg_profile_kinds() >= 13
    assert lib.kg_profile_kind_name(2) == b"stage_pirk2_s2"


def test_integration_guide_names_every_entry_point():
    """every function the header declares appears in the integration guide"""
    import re
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    header = open(os.path.join(root, "include", "kg_capi.h")).read()
    guide = open(os.path.join(root, "INTEGRATION.md")).read()
    names = set(re.findall(r"\b(kg_[a-z0-9_]+)\s*\(", header))
    assert names and not sorted(n for n in names if n not in guide)
