"""ctypes binding of ``lib/libclaw2.so`` (C ABI declared in ``include/claw2.h``).

The library is the only compute path of this package: if it is missing or
cannot be loaded, every solver call raises; there is no CPU fallback.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libclaw2.so")

CLAW2_MAX_PARAMS = 8
CLAW2_MAX_WAVES = 8
CLAW2_NOALLOC_SCRATCH_BYTES = 32 << 20

RP_ADVECTION, RP_ACOUSTICS, RP_EULER_ROE, RP_SHALLOW_ROE, RP_EULER_EXACT = 1, 2, 3, 4, 5
RP_VC_ACOUSTICS = 6
RP_VC_ADVECTION = 7
RP_PSYSTEM = 8
RP_VC_ADVECTION_VEC = 9
RP_EULER_5WAVE = 10
RP_SHALLOW_HLLE = 12

OK, EINVAL, ECUDA, ENONFINITE, ETIMEOUT, ENOMEM, EUNSUPPORTED = 0, 1, 2, 3, 4, 5, 6

_c_int_p = ctypes.POINTER(ctypes.c_int)
_c_double_p = ctypes.POINTER(ctypes.c_double)


class Claw2Desc(ctypes.Structure):
    """Mirror of ``claw2_desc``."""
    _fields_ = [
        ("mx", ctypes.c_int), ("my", ctypes.c_int),
        ("num_eqn", ctypes.c_int), ("num_waves", ctypes.c_int),
        ("num_aux", ctypes.c_int), ("num_ghost", ctypes.c_int),
        ("riemann", ctypes.c_int), ("order", ctypes.c_int),
        ("transverse", ctypes.c_int), ("dimensional_split", ctypes.c_int),
        ("fwave", ctypes.c_int),
        ("mthlim", ctypes.c_int * CLAW2_MAX_WAVES),
        ("bc_lower", ctypes.c_int * 2), ("bc_upper", ctypes.c_int * 2),
        ("dx", ctypes.c_double), ("dy", ctypes.c_double),
        ("cparam", ctypes.c_double * CLAW2_MAX_PARAMS),
        ("ncparam", ctypes.c_int),
        ("device", ctypes.c_int),
        ("mcapa", ctypes.c_int),
    ]


class Claw2EvolveState(ctypes.Structure):
    """Mirror of ``claw2_evolve_state``."""
    _fields_ = [(n, ctypes.c_double) for n in ("t", "tstart", "tend", "dt", "cfl", "cfl_desired", "cfl_max",
                                               "dt_max", "dtmin", "dtmax", "cflmax")] + \
               [(n, ctypes.c_int) for n in ("dt_variable", "dt_old_set", "max_steps", "num_steps", "attempts",
                                            "cfl_error")]


class Claw2Error(RuntimeError):
    """A status code other than CLAW2_OK, with the library's message."""

    def __init__(self, code, msg):
        super().__init__("claw2 error %d: %s" % (code, msg))
        self.code = code


class NonFiniteError(Claw2Error):
    pass


# name -> (restype, argtypes); exactly the declarations of include/claw2.h
_SIGNATURES = {
    "claw2_step2": (ctypes.c_int, [ctypes.c_int] * 7 + [_c_double_p, _c_double_p, _c_double_p,
                                                        ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                                        _c_int_p, _c_int_p, _c_double_p, ctypes.c_int,
                                                        ctypes.c_int, _c_double_p, ctypes.c_int]),
    "claw2_step2ds": (ctypes.c_int, [ctypes.c_int] * 7 + [_c_double_p, _c_double_p, _c_double_p,
                                                          ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                                          _c_int_p, _c_int_p, _c_double_p, ctypes.c_int,
                                                          ctypes.c_int, ctypes.c_int, _c_double_p,
                                                          ctypes.c_int]),
    "claw2_bc_fill": (ctypes.c_int, [ctypes.c_int] * 4 + [_c_double_p, _c_int_p, _c_int_p]),
    "claw2_patch_create": (ctypes.c_int, [ctypes.POINTER(Claw2Desc), ctypes.POINTER(ctypes.c_void_p)]),
    "claw2_patch_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "claw2_patch_set_cparam": (ctypes.c_int, [ctypes.c_void_p, _c_double_p, ctypes.c_int]),
    "claw2_patch_upload_q": (ctypes.c_int, [ctypes.c_void_p, _c_double_p]),
    "claw2_patch_download_q": (ctypes.c_int, [ctypes.c_void_p, _c_double_p]),
    "claw2_patch_upload_aux": (ctypes.c_int, [ctypes.c_void_p, _c_double_p, _c_int_p, _c_int_p]),
    "claw2_patch_upload_auxbc": (ctypes.c_int, [ctypes.c_void_p, _c_double_p]),
    "claw2_patch_upload_qbc": (ctypes.c_int, [ctypes.c_void_p, _c_double_p]),
    "claw2_write_ascii": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, ctypes.c_char_p, _c_double_p, ctypes.c_int,
                                         ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "claw2_patch_write_ascii_async": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_char_p,
                                                     ctypes.c_int]),
    "claw2_patch_wait_output": (ctypes.c_int, [ctypes.c_void_p]),
    "claw2_patch_gather_q": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _c_int_p, _c_double_p]),
    "claw2_patch_linear_source": (ctypes.c_int, [ctypes.c_void_p, _c_double_p, ctypes.c_int, ctypes.c_double]),
    "claw2_patch_euler_axisymmetric_source": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, ctypes.c_int,
                                                            ctypes.c_double]),
    "claw2_patch_step": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, _c_double_p]),
    "claw2_patch_step_part": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, ctypes.c_int, _c_double_p]),
    "claw2_patch_evolve": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Claw2EvolveState)]),
    "claw2_patch_run_host": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p),
                                            ctypes.POINTER(ctypes.c_void_p), _c_double_p, _c_double_p]),
    "claw2_patch_accept": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "claw2_patch_cfl": (ctypes.c_int, [ctypes.c_void_p, _c_double_p]),
    "claw2_patch_sync": (ctypes.c_int, [ctypes.c_void_p]),
    "claw2_patch_device_q": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(_c_double_p),
                                            ctypes.POINTER(ctypes.c_longlong)]),
    "claw2_patch_set_stream": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "claw2_patch_set_timing": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "claw2_patch_kernel_ms": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_float)]),
    "claw2_probe_fp64": (ctypes.c_int, [ctypes.c_int, _c_double_p]),
    "claw2_selftest_rcp": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_ulonglong, _c_double_p]),
    "claw2_selftest_sqrt": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_ulonglong, _c_double_p]),
    "claw2_selftest_rsqrt": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_ulonglong, _c_double_p]),
    "claw2_patch_launch_count": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_longlong)]),
    "claw2_selftest_lpt": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_ulonglong,
                                          ctypes.POINTER(ctypes.c_int)]),
    "claw2_tune_set": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "claw2_tune_get": (ctypes.c_int, [ctypes.c_int, _c_int_p, _c_int_p]),
    "claw2_step2ds_noalloc": (ctypes.c_int, [ctypes.POINTER(Claw2Desc), ctypes.c_void_p, ctypes.c_void_p,
                                             ctypes.c_longlong, ctypes.c_longlong, ctypes.c_double, _c_double_p,
                                             ctypes.c_void_p]),
    "claw2_batch_create": (ctypes.c_int, [ctypes.POINTER(Claw2Desc), ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]),
    "claw2_batch_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "claw2_batch_set_rows": (ctypes.c_int, [ctypes.c_void_p, _c_int_p]),
    "claw2_batch_upload_q": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _c_double_p]),
    "claw2_batch_download_q": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _c_double_p]),
    "claw2_batch_set_time": (ctypes.c_int, [ctypes.c_void_p, _c_double_p] + [ctypes.c_double] * 5),
    "claw2_batch_run": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_float)]),
    "claw2_batch_get_state": (ctypes.c_int, [ctypes.c_void_p, _c_double_p, _c_double_p, _c_int_p, _c_int_p,
                                             _c_double_p, _c_int_p]),
    "claw2_batch_tiles": (ctypes.c_int, [ctypes.c_void_p, _c_int_p, _c_int_p]),
    "claw2_mlp_create": (ctypes.c_int, [ctypes.c_int, ctypes.c_ulonglong, ctypes.POINTER(ctypes.c_void_p)]),
    "claw2_mlp_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "claw2_mlp_set_params": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_float), ctypes.c_int]),
    "claw2_mlp_get_params": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_float), ctypes.c_int]),
    "claw2_mlp_generate": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_ulonglong, ctypes.c_longlong, ctypes.c_double,
                                          ctypes.c_double, ctypes.POINTER(ctypes.c_longlong)]),
    "claw2_mlp_samples": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_longlong, ctypes.c_int,
                                         ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float), _c_int_p]),
    "claw2_mlp_gradient": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_longlong, ctypes.c_int,
                                          ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float)]),
    "claw2_mlp_train": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                       ctypes.POINTER(ctypes.c_float)]),
    "claw2_mlp_infer": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_float), ctypes.c_int,
                                       ctypes.POINTER(ctypes.c_float)]),
    "claw2_mlp_set_engine": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "claw2_patch_set_mlp": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "claw2_patch_counters": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_ulonglong), ctypes.c_int]),
    "claw2_patch_newton_counts": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_ulonglong), ctypes.c_int]),
    "claw2_patch_set_exact_guess": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "claw2_patch_set_exact_guess_error": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double]),
    "claw2_last_error": (ctypes.c_char_p, []),
    "claw2_version": (ctypes.c_char_p, []),
}

_lib = None


def load():
    """Load the CUDA library once; raise with a clear message if it is absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError("pyclaw_b200: CUDA extension %s is missing; build it with "
                          "`python -m pyclaw_b200.build` (no CPU fallback exists)" % LIB_PATH)
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(rc):
    if rc != OK:
        msg = load().claw2_last_error().decode()
        if rc == ENONFINITE:
            raise NonFiniteError(rc, msg)
        raise Claw2Error(rc, msg)


def dptr(a):
    """double* of a C- or F-contiguous float64 array."""
    assert a.dtype == np.float64 and (a.flags.c_contiguous or a.flags.f_contiguous)
    return a.ctypes.data_as(_c_double_p)


def iptr(a):
    assert a.dtype == np.intc and a.flags.c_contiguous
    return a.ctypes.data_as(_c_int_p)
