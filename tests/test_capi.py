"""The C-ABI library builds, loads and exports every declared entry point (no GPU needed)."""
import ctypes
import os
import re

from conftest import REPO

HEADER = os.path.join(REPO, "include", "flexmm_b200.h")


def declared():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fmm_[a-z_0-9]+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared()
    for n in ["fmm_ops_create", "fmm_plan_create", "fmm_build_expansions", "fmm_evaluate",
              "fmm_plan_destroy", "fmm_last_error", "fmm_direct", "fmm_tree_export"]:
        assert n in names


def test_library_exports_every_declared_symbol(built_lib):
    lib = ctypes.CDLL(built_lib)
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header(built_lib):
    from flexmm_b200 import _lib
    bound = {s[0] for s in _lib.SIGNATURES}
    assert set(declared()) <= bound
    lib = _lib.load(built_lib)
    assert lib.fmm_last_error() is not None


def test_errors_without_device_are_status_codes(built_lib):
    """With no usable device the entry points return codes, never abort."""
    from flexmm_b200 import _lib
    lib = _lib.load(built_lib)
    h = ctypes.c_void_p()
    assert lib.fmm_ops_create(99, None, 16, ctypes.byref(h)) == 5          # unknown kernel
    assert b"kernel" in lib.fmm_last_error()
    assert lib.fmm_ops_create(0, None, 65, ctypes.byref(h)) == 1           # nequiv > 64
    assert lib.fmm_evaluate(None, None, None, 0, 0, None, None) == 1       # NULL plan
