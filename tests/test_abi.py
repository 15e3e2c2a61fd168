"""The C-ABI library builds, loads without a GPU, and exports exactly what
include/claw2.h declares; the Python binding declares the same set."""
import ctypes
import os
import re

import pytest

from conftest import ROOT


def header_functions():
    src = open(os.path.join(ROOT, "include", "claw2.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(claw2_\w+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib():
    from pyclaw_b200 import build
    path = build.build()
    return ctypes.CDLL(path)


def test_header_declares_entry_points():
    names = header_functions()
    assert "claw2_step2" in names and "claw2_step2ds" in names and "claw2_patch_step" in names


def test_library_exports_every_declared_symbol(lib):
    missing = [n for n in header_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_matches_header():
    from pyclaw_b200 import _lib
    assert sorted(_lib._SIGNATURES) == header_functions()


def test_version_and_error_strings(lib):
    lib.claw2_version.restype = ctypes.c_char_p
    lib.claw2_last_error.restype = ctypes.c_char_p
    assert b"sm_100a" in lib.claw2_version()
    assert lib.claw2_last_error()


def test_bad_arguments_rejected_without_gpu(lib):
    # argument checks run before any CUDA call
    from pyclaw_b200 import _lib
    L = _lib.load()
    rc = L.claw2_step2(10, 4, 4, 0, 3, 10, 10, None, None, None, 0.1, 0.1, 0.01, None, None, None, 0, 3,
                       None, 0)
    assert rc == _lib.EINVAL
    assert b"null" in L.claw2_last_error()
    rc = L.claw2_selftest_rcp(0, 100, 1, None)
    assert rc == _lib.EINVAL
    import ctypes
    bad = ctypes.c_int(-1)
    assert L.claw2_selftest_lpt(0, 10, 1, None) == _lib.EINVAL
    assert L.claw2_selftest_lpt(0, 0, 1, ctypes.byref(bad)) == _lib.EINVAL
    assert L.claw2_selftest_lpt(0, 8193, 1, ctypes.byref(bad)) == _lib.EINVAL
