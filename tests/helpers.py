"""Shared helpers for the parity tests: seeded physical states and the
max-norm comparison used as the parity bar."""
import numpy as np

from pyclaw_b200 import _lib

RP_INFO = {  # id -> (name, meqn, mwaves, cparam vector)
    _lib.RP_ADVECTION: ("advection", 1, 1, [0.5, -1.0]),
    _lib.RP_ACOUSTICS: ("acoustics", 3, 2, [1.0, 4.0, 2.0, 2.0]),
    _lib.RP_EULER_ROE: ("euler_roe", 4, 4, [1.4, 1.0]),
    _lib.RP_SHALLOW_ROE: ("shallow_roe", 3, 3, [1.0, 1.0]),
}

# the same parameters as problem_data entries (what state.set_cparam would
# assign to the f2py module's cparam block)
PROBLEM_DATA = {
    _lib.RP_ADVECTION: {"u": 0.5, "v": -1.0},
    _lib.RP_ACOUSTICS: {"rho": 1.0, "bulk": 4.0, "cc": 2.0, "zz": 2.0},
    _lib.RP_EULER_ROE: {"gamma": 1.4, "efix": True},
    _lib.RP_SHALLOW_ROE: {"grav": 1.0, "efix": True},
}


def set_cparam(module, rp):
    """state.set_cparam(module) for the test parameters (state.py:206-231)."""
    for k, v in PROBLEM_DATA[rp].items():
        setattr(module.cparam, k, v)

PARITY_RTOL = 1e-12  # relative, max norm over the interior cells


def random_qbc(rp, mx, my, seed, smooth_frac=0.5):
    """Seeded qbc (meqn, mx+4, my+4), F-order: piecewise-constant quadrants
    (exact zero jumps, exercising the zero-wave paths) with noise added on a
    fraction of the cells (rough data, exercising every limiter branch)."""
    rng = np.random.default_rng(seed)
    nx, ny = mx + 4, my + 4
    X, Y = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    quad = (X > nx // 2).astype(int) + 2 * (Y > ny // 3).astype(int)
    noise = rng.random((nx, ny)) < smooth_frac

    def field(lo, hi):
        base = rng.uniform(lo, hi, size=4)[quad]
        return np.where(noise, rng.uniform(lo, hi, size=(nx, ny)), base)

    if rp == _lib.RP_ADVECTION:
        q = field(0.0, 1.0)[None]
    elif rp == _lib.RP_ACOUSTICS:
        q = np.stack([field(-1.0, 1.0), field(-1.0, 1.0), field(-1.0, 1.0)])
    elif rp == _lib.RP_EULER_ROE:
        g = 1.4
        rho, u, v, p = field(0.2, 2.0), field(-1.0, 1.0), field(-1.0, 1.0), field(0.2, 2.0)
        q = np.stack([rho, rho * u, rho * v, p / (g - 1.0) + 0.5 * rho * (u * u + v * v)])
    elif rp == _lib.RP_SHALLOW_ROE:
        h, u, v = field(0.5, 2.0), field(-0.8, 0.8), field(-0.8, 0.8)
        q = np.stack([h, h * u, h * v])
    else:
        raise ValueError(rp)
    return np.asfortranarray(q)


def max_rel(a, b):
    """||a - b||_inf / ||b||_inf."""
    scale = max(np.max(np.abs(b)), 1e-300)
    return float(np.max(np.abs(a - b)) / scale)


def method_vector(order, transverse, split=False):
    m = np.zeros(7, dtype=np.intc)
    m[0] = 1
    m[1] = order
    m[2] = -1 if split else transverse
    m[5] = 0
    m[6] = 0
    return m
