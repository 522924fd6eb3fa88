"""The C-ABI library loads, exports every entry point include/zxh_b200.h
declares, and reports errors through status codes (no process abort)."""
import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "zxh_b200.h"
LIB = ROOT / "zxh_adae_b200" / "libzxhb200.so"


def declared():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\**\s*(zxh_[a-z_0-9]+)\s*\(", text, re.M)))


def test_header_declares_entry_points():
    names = declared()
    for must in ("zxh_create", "zxh_execute", "zxh_measure", "zxh_get_results", "zxh_get_state", "zxh_push_gates"):
        assert must in names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(str(LIB))
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_imports_library():
    import zxh_adae_b200 as zx

    assert Path(zx.library_path()) == LIB
    assert "sm_100a" in zx.version()


def test_create_rejects_bad_arguments_without_abort():
    lib = ctypes.CDLL(str(LIB))
    lib.zxh_last_error.restype = ctypes.c_char_p
    lib.zxh_last_error.argtypes = [ctypes.c_void_p]
    h = ctypes.c_void_p()
    assert lib.zxh_create(ctypes.byref(h), 0, 0, 0, 2, 0) == 5  # ZXH_ERR_LIMIT
    assert b"1..63" in lib.zxh_last_error(None)
    assert lib.zxh_create(ctypes.byref(h), 4, 0, 0, 7, 0) == 1  # ZXH_ERR_ARG
    assert lib.zxh_create(None, 4, 0, 0, 2, 0) == 1


def test_null_handles_are_argument_errors():
    # every handle-taking entry point answers a null handle with ZXH_ERR_ARG before
    # touching a device, so a caller's bookkeeping slip is an error code, not a crash
    lib = ctypes.CDLL(str(LIB))
    nu = ctypes.c_size_t(7)
    calls = {
        "zxh_execute": (None,),
        "zxh_apply": (None, None, ctypes.c_size_t(0)),
        "zxh_apply_async": (None, None, ctypes.c_size_t(0)),
        "zxh_sync": (None,),
        "zxh_measure": (None, ctypes.c_size_t(10)),
        "zxh_get_results": (None, None, ctypes.c_size_t(1)),
        "zxh_counts": (None, None, None, ctypes.c_size_t(0), ctypes.byref(nu)),
        "zxh_measured_count": (None, ctypes.byref(nu)),
    }
    for name, args in calls.items():
        assert getattr(lib, name)(*args) == 1, name  # ZXH_ERR_ARG
