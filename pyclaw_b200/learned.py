"""The exact Euler solver's learned Newton guess.

``Network`` owns the 6-32-32-1 tanh network on the device (claw2_mlp_* in
include/claw2.h): it draws seeded training problems (rho, p log-uniform in
[1e-2, 1e2], normal velocity uniform in [-3, 3]) and solves each to the FP64
Newton tolerance, trains with the library's own forward/backward kernels and
Adam, and evaluates itself in BF16 on the tensor cores.  Attached to a
ClawSolver2D using ``riemann.euler_exact_2D`` (``attach``), every step first
predicts a starting pressure for every interface; the Newton iteration then
converges to the same p* as from the adaptive PVRS guess, which stays the
fallback for an invalid prediction.

Feature and target definition (also in csrc/exact_euler.h, features()):
x = (log rho_L/rb, log rho_R/rb, u_L/cb, u_R/cb, log p_L/pb, log p_R/pb),
rb = sqrt(rho_L rho_R), pb = sqrt(p_L p_R), cb = sqrt(gamma pb / rb);
target y = log(p*/p_pvrs) / w with w = J^2/(1 + J^2), J^2 the squared
normalised jump; guess = p_pvrs * exp(w y).  The PVRS guess decides:
interfaces with w < 0.05 (weak jumps, where PVRS is accurate and the training
distribution has no samples) keep it.
"""
import ctypes

import numpy as np

from . import _lib

NPARAM = 1313
MLP_TCGEN05, MLP_MMA_SYNC = 0, 1  # claw2_mlp_set_engine
_fp = ctypes.POINTER(ctypes.c_float)


def _f(a):
    return a.ctypes.data_as(_fp)


class Network(object):
    def __init__(self, device=0, seed=1234):
        self._lib = _lib.load()
        h = ctypes.c_void_p()
        _lib.check(self._lib.claw2_mlp_create(int(device), ctypes.c_ulonglong(seed), ctypes.byref(h)))
        self.h = h
        self.nsamples = 0

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self._lib.claw2_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def params(self):
        p = np.zeros(NPARAM, dtype=np.float32)
        _lib.check(self._lib.claw2_mlp_get_params(self.h, _f(p), NPARAM))
        return p

    @params.setter
    def params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        _lib.check(self._lib.claw2_mlp_set_params(self.h, _f(p), NPARAM))

    def generate(self, n, seed=7, gamma=1.4, tol=1e-12):
        nv = ctypes.c_longlong(0)
        _lib.check(self._lib.claw2_mlp_generate(self.h, ctypes.c_ulonglong(seed), int(n), gamma, tol,
                                                ctypes.byref(nv)))
        self.nsamples = int(n)
        return nv.value

    def samples(self, first, count):
        x = np.zeros((count, 8), dtype=np.float32)
        y = np.zeros(count, dtype=np.float32)
        ok = np.zeros(count, dtype=np.intc)
        _lib.check(self._lib.claw2_mlp_samples(self.h, int(first), int(count), _f(x), _f(y), _lib.iptr(ok)))
        return x, y, ok

    def gradient(self, first, count):
        g = np.zeros(NPARAM, dtype=np.float32)
        loss = ctypes.c_float(0.0)
        _lib.check(self._lib.claw2_mlp_gradient(self.h, int(first), int(count), _f(g), ctypes.byref(loss)))
        return g, loss.value

    def train(self, epochs, batch=8192, lr=3e-3):
        loss = ctypes.c_float(0.0)
        _lib.check(self._lib.claw2_mlp_train(self.h, int(epochs), int(batch), float(lr), ctypes.byref(loss)))
        return loss.value

    def infer(self, x8):
        x8 = np.ascontiguousarray(x8, dtype=np.float32)
        y = np.zeros(x8.shape[0], dtype=np.float32)
        _lib.check(self._lib.claw2_mlp_infer(self.h, _f(x8), x8.shape[0], _f(y)))
        return y

    def set_engine(self, engine):
        """Tensor-core path of the inference and the guess pass: "tcgen05"
        (tcgen05.mma with TMEM accumulators, the default) or "mma.sync"."""
        code = {"tcgen05": MLP_TCGEN05, "mma.sync": MLP_MMA_SYNC}[engine]
        _lib.check(self._lib.claw2_mlp_set_engine(self.h, code))


def attach(solver, net):
    """Start the exact solver's Newton iterations from ``net``'s guesses
    (``net=None``: the adaptive PVRS guess).  Call after solver.setup()."""
    dev = solver._dev
    _lib.check(dev._lib.claw2_patch_set_mlp(dev.h, net.h if net is not None else None))
    dev.mlp = net  # keep it alive as long as the patch uses it


def counters(solver, reset=True):
    """(Newton updates, Riemann solves) since the last reset."""
    dev = solver._dev
    out = (ctypes.c_ulonglong * 2)()
    _lib.check(dev._lib.claw2_patch_counters(dev.h, out, 1 if reset else 0))
    return int(out[0]), int(out[1])


def newton_counts(solver, reset=True):
    """(Newton steps needed, Newton steps applied, Riemann solves) since the
    last reset: "applied" also counts the final step below the tolerance,
    which every interface with two different states takes."""
    dev = solver._dev
    out = (ctypes.c_ulonglong * 3)()
    _lib.check(dev._lib.claw2_patch_newton_counts(dev.h, out, 1 if reset else 0))
    return int(out[0]), int(out[1]), int(out[2])


def converged_guess(solver, on=True, rel_error=0.0):
    """Measurement aid: every step of the exact solver starts Newton from the
    converged pressures (a pre-pass outside the kernel timing), so the step
    kernel's time is the floor for any guess, learned or not.  With
    rel_error > 0 the interfaces where the adaptive guess needs Newton steps
    start from the converged pressure off by a fixed relative error of at
    most that size, the others from the adaptive guess: the step time of a
    guess of that precision with the adaptive guess as fallback."""
    dev = solver._dev
    _lib.check(dev._lib.claw2_patch_set_exact_guess_error(dev.h, float(rel_error)))
    _lib.check(dev._lib.claw2_patch_set_exact_guess(dev.h, 1 if on else 0))
