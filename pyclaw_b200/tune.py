"""Autotuner for the launch shape of the unsplit step kernel.

For one device patch (a problem size and Riemann solver) it times the step
kernel -- CUDA events recorded by the library on the patch's stream -- for
each compiled register budget and a set of row-block heights, rejecting every
trial step so the state does not change, and installs the fastest shape with
claw2_tune_set.  Results are cached per (solver id, mx, my) for the process.
"""
import ctypes
import statistics

from . import _lib

ROWS = (2, 4, 8, 12, 14, 16, 18, 20, 24, 28, 32, 48, 64)
VARIANTS = (0, 1, 2, 3, 4, 8)
_cache = {}


def set_shape(rp_id, variant, rows):
    _lib.check(_lib.load().claw2_tune_set(int(rp_id), int(variant), int(rows)))


def get_shape(rp_id):
    v, r = ctypes.c_int(0), ctypes.c_int(0)
    _lib.check(_lib.load().claw2_tune_get(int(rp_id), ctypes.byref(v), ctypes.byref(r)))
    return v.value, r.value


def autotune(patch, dt, reps=5, rows=ROWS, variants=VARIANTS, before_step=None):
    """Pick the fastest (variant, rows) for ``patch`` (a pyclaw_b200.device.DevicePatch)
    at time step ``dt``; returns (best, {shape: median ms}).  ``before_step``, if
    given, is called before every trial step (e.g. a write that evicts the
    state from L2, so the trials see the memory system the real steps see;
    it must run on the patch's stream)."""
    d = patch.desc
    key = (d.riemann, d.mx, d.my)
    if key in _cache:
        set_shape(d.riemann, *_cache[key][0])
        return _cache[key]
    patch.set_timing(True)
    results = {}
    for v in variants:
        for r in rows:
            set_shape(d.riemann, v, r)
            times = []
            for _ in range(reps + 1):
                if before_step is not None:
                    before_step()
                patch.step(dt, want_cfl=False)
                patch.accept(False)
                times.append(patch.kernel_ms())
            results[(v, r)] = statistics.median(times[1:])
    best = min(results, key=results.get)
    set_shape(d.riemann, *best)
    _cache[key] = (best, results)
    return best, results
