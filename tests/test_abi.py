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
    assert L.claw2_selftest_sqrt(0, 100, 1, None) == _lib.EINVAL
    assert L.claw2_selftest_rsqrt(0, 100, 1, None) == _lib.EINVAL
    import ctypes
    bad = ctypes.c_int(-1)
    assert L.claw2_selftest_lpt(0, 10, 1, None) == _lib.EINVAL
    assert L.claw2_selftest_lpt(0, 0, 1, ctypes.byref(bad)) == _lib.EINVAL
    assert L.claw2_selftest_lpt(0, 8193, 1, ctypes.byref(bad)) == _lib.EINVAL


def _valid_desc():
    from pyclaw_b200 import _lib
    d = _lib.Claw2Desc()
    d.mx, d.my = 40, 30
    d.num_eqn, d.num_waves, d.num_aux, d.num_ghost = 4, 4, 0, 2
    d.riemann, d.order, d.transverse, d.dimensional_split, d.fwave = _lib.RP_EULER_ROE, 2, 2, 0, 0
    for k in range(4):
        d.mthlim[k] = 4
    for s in range(2):
        d.bc_lower[s] = d.bc_upper[s] = 1
    d.dx = d.dy = 0.025
    d.cparam[0], d.cparam[1], d.ncparam = 1.4, 1.0, 2
    return d


def _set(**kw):
    def f(d):
        for k, v in kw.items():
            if isinstance(v, tuple):
                getattr(d, k)[v[0]] = v[1]
            else:
                setattr(d, k, v)
    return f


@pytest.mark.parametrize("name,mutate,code", [
    ("empty grid", _set(mx=0), "EINVAL"),
    ("negative rows", _set(my=-3), "EINVAL"),
    ("unknown solver", _set(riemann=99), "EINVAL"),
    ("num_eqn mismatch", _set(num_eqn=3), "EINVAL"),
    ("num_waves mismatch", _set(num_waves=3), "EINVAL"),
    ("three ghost cells", _set(num_ghost=3), "EINVAL"),
    ("capacity index beyond aux", _set(mcapa=1), "EINVAL"),
    ("non-positive dx", _set(dx=0.0), "EINVAL"),
    ("order 3", _set(order=3), "EINVAL"),
    ("transverse 3", _set(transverse=3), "EINVAL"),
    ("limiter 6", _set(mthlim=(2, 6)), "EINVAL"),
    ("use_fwave 2", _set(fwave=2), "EINVAL"),
    ("BC code 7", _set(bc_upper=(0, 7)), "EINVAL"),
    ("periodic on one side", _set(bc_lower=(1, 2)), "EINVAL"),
    ("wall with one cell", lambda d: (_set(mx=1)(d), _set(bc_lower=(0, 3))(d)), "EINVAL"),
    ("caller-filled x ghosts", _set(bc_lower=(0, -1)), "EINVAL"),
    ("custom BC code", _set(bc_upper=(1, 0)), "EUNSUPPORTED"),
])
def test_patch_descriptor_rejected_without_gpu(name, mutate, code):
    # the reference raises for bad solver settings before stepping
    # (solver.py:262-287, classic/solver.py:162-171); the library checks a
    # descriptor completely before its first CUDA call
    import ctypes
    from pyclaw_b200 import _lib
    L = _lib.load()
    d = _valid_desc()
    mutate(d)
    h = ctypes.c_void_p()
    rc = L.claw2_patch_create(ctypes.byref(d), ctypes.byref(h))
    assert rc == getattr(_lib, code), (name, rc, L.claw2_last_error())
    assert not h.value


def test_transverse_solve_rejected_for_solvers_without_one():
    import ctypes
    from pyclaw_b200 import _lib
    L = _lib.load()
    d = _valid_desc()
    d.riemann, d.num_eqn, d.num_waves = _lib.RP_SHALLOW_HLLE, 3, 2
    h = ctypes.c_void_p()
    assert L.claw2_patch_create(ctypes.byref(d), ctypes.byref(h)) == _lib.EINVAL
    assert b"transverse" in L.claw2_last_error()


@pytest.mark.parametrize("name,mx,my,pitch,plane", [
    # a plane so large that num_eqn * plane overflows 64 bits if multiplied first
    ("huge plane", 40, 30, 48, 1 << 61),
    # my near INT_MAX: my + 4 overflows int if computed without the bound
    ("huge my", 40, 2**31 - 2, 48, 1 << 40),
    ("huge mx", 2**31 - 3, 30, 1 << 30, 1 << 40),
    ("one cell over the scratch", 1020, 1020, 1024, 1024 * 1024),
])
def test_noalloc_sizes_rejected_without_gpu(name, mx, my, pitch, plane):
    # claw2_step2ds_noalloc checks every size against its fixed scratch array
    # before its first CUDA call, without integer overflow
    import ctypes
    from pyclaw_b200 import _lib
    L = _lib.load()
    d = _valid_desc()
    d.mx, d.my, d.transverse, d.dimensional_split = mx, my, 0, 1
    cfl = ctypes.c_double(0.0)
    fake = ctypes.c_void_p(1 << 20)  # never dereferenced: rejected first
    rc = L.claw2_step2ds_noalloc(ctypes.byref(d), fake, fake, pitch, plane, 1e-4, ctypes.byref(cfl), None)
    assert rc == _lib.EINVAL, (name, rc, L.claw2_last_error())
