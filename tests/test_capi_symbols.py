"""The C-ABI library loads and exports every entry point include/ag2d.h declares (no GPU needed)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "ag2d.h")
LIB = os.path.join(ROOT, "physicssimulation-agony_b200", "ag2d", "libag2d.so")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ag2d_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(LIB):
        import subprocess
        import sys
        subprocess.check_call([sys.executable, os.path.join(ROOT, "physicssimulation-agony_b200", "build.py")])
    return ctypes.CDLL(LIB)


def test_header_declares_the_boundary():
    names = declared_functions()
    for required in ("ag2d_world_create", "ag2d_world_step", "ag2d_world_add_polygon", "ag2d_world_read",
                     "ag2d_batch_step", "ag2d_last_error_string"):
        assert required in names


def test_library_exports_every_declared_symbol(lib):
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_errors_without_a_device_are_reported_not_fatal(lib):
    lib.ag2d_device_count.argtypes = [ctypes.POINTER(ctypes.c_int32)]
    n = ctypes.c_int32(-1)
    assert lib.ag2d_device_count(ctypes.byref(n)) == 0
    lib.ag2d_version.restype = ctypes.c_int32
    assert lib.ag2d_version() >= 1
    # Null arguments come back as AG2D_ERR_INVALID_ARG with a message, never a crash.
    lib.ag2d_world_create.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    assert lib.ag2d_world_create(None, None) == -1
    lib.ag2d_last_error_string.restype = ctypes.c_char_p
    assert lib.ag2d_last_error_string()
