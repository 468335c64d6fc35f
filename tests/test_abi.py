"""The C-ABI library loads and exports every entry point the header declares (CPU only)."""
import ctypes
import re
from pathlib import Path

import pytest

from pycusaxs_b200 import _native

HEADER = Path(__file__).resolve().parent.parent / "include" / "pycusaxs_b200.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_]*\s*\**\s*(saxs_[a-z0-9_]+)\s*\(",
                       text, flags=re.M)
    return names


def test_header_declares_the_binding_list():
    assert tuple(declared_functions()) == _native.EXPORTED


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(str(_native.LIB_PATH))
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_version_and_error_string():
    lib = _native.load()
    assert b"sm_100a" in lib.saxs_version()
    plan = ctypes.c_void_p()
    p = _native.SaxsParams()          # all zero: invalid grid
    rc = lib.saxs_plan_create(ctypes.byref(p), ctypes.byref(plan))
    assert rc == _native.SAXS_E_INVALID
    assert b"Grid dimensions must be positive" in lib.saxs_last_error()
    with pytest.raises(_native.SaxsError):
        _native.check(rc)


def test_invalid_order_is_rejected_before_any_device_work():
    lib = _native.load()
    p = _native.SaxsParams()
    p.grid[:] = (16, 16, 16)
    p.order = 9
    plan = ctypes.c_void_p()
    assert lib.saxs_plan_create(ctypes.byref(p), ctypes.byref(plan)) == _native.SAXS_E_INVALID
    assert b"Spline order must be between 1 and 8" in lib.saxs_last_error()
