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


def test_server_errors_are_reported_not_fatal(lib):
    vp = ctypes.c_void_p
    lib.ag2d_server_create.argtypes = [vp, vp]
    assert lib.ag2d_server_create(None, None) == -1
    for name, args in (("ag2d_server_wait_all", (None, ctypes.c_double(0.0))),
                       ("ag2d_server_poll", (None, ctypes.c_uint64(1), None, None)),
                       ("ag2d_server_release", (None, ctypes.c_uint64(1))),
                       ("ag2d_server_stats_get", (None, None))):
        assert getattr(lib, name)(*args) == -1, name
    assert lib.ag2d_server_destroy(None) == 0   # destroying nothing is a no-op, as free(NULL)


def test_server_without_a_device_fails_cleanly(lib):
    import sys
    sys.path.insert(0, os.path.join(ROOT, "physicssimulation-agony_b200"))
    import ag2d
    if ag2d.device_count() > 0:
        pytest.skip("a device is present: the server starts")
    with pytest.raises(ag2d.Ag2dError) as err:
        ag2d.Server(memory_budget_bytes=1 << 20)
    assert err.value.code == ag2d.ERR_NO_DEVICE
