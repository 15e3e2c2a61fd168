"""The exact Euler solver of the oracle (no reference counterpart; restated
from Toro 2009, ch. 4) and the CPU reference of the learned-guess network."""
import ctypes

import numpy as np
import pytest

from oracle import mlp_ref


def _star(oracle, gamma, rl, ul, pl, rr, ur, pr, tol=1e-12):
    lib = oracle.load()
    p, u, it = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
    rc = lib.oracle_exact_star(gamma, rl, ul, pl, rr, ur, pr, tol, 0, ctypes.byref(p), ctypes.byref(u),
                               ctypes.byref(it))
    assert rc == 0
    return p.value, u.value, it.value


def test_sod_star_state(oracle):
    # Sod's shock tube: the classic star values p* = 0.30313, u* = 0.92745
    p, u, it = _star(oracle, 1.4, 1.0, 0.0, 1.0, 0.125, 0.0, 0.1)
    assert abs(p - 0.30313) < 5e-5 and abs(u - 0.92745) < 5e-5 and it >= 1


def test_mirror_symmetry_and_trivial_problem(oracle):
    rng = np.random.default_rng(3)
    for _ in range(50):
        rl, rr, pl, pr = np.exp(rng.uniform(-2, 2, 4))
        ul, ur = rng.uniform(-1, 1, 2)
        p1, u1, _ = _star(oracle, 1.4, rl, ul, pl, rr, ur, pr)
        p2, u2, _ = _star(oracle, 1.4, rr, -ur, pr, rl, -ul, pl)
        assert abs(p1 - p2) <= 1e-12 * p1 and abs(u1 + u2) <= 1e-12 * (1 + abs(u1))
    p, u, it = _star(oracle, 1.4, 0.7, 0.3, 2.0, 0.7, 0.3, 2.0)
    assert (p, u, it) == (2.0, 0.3, 0)


def test_exact_rpn2_waves_and_fluxes_are_consistent(oracle):
    lib = oracle.load()
    g = 1.4
    rng = np.random.default_rng(5)
    mx, mbc = 40, 2
    n = mx + 2 * mbc
    rho = np.exp(rng.uniform(-1, 1, n))
    u, v = rng.uniform(-0.5, 0.5, n), rng.uniform(-0.5, 0.5, n)
    p = np.exp(rng.uniform(-1, 1, n))
    q = np.stack([rho, rho * u, rho * v, p / (g - 1) + 0.5 * rho * (u * u + v * v)], axis=1).copy()
    wave = np.zeros((n, 3, 4))
    s = np.zeros((n, 3))
    am, ap = np.zeros((n, 4)), np.zeros((n, 4))
    cp = np.array([g, 1e-12] + [0.0] * 6)
    P = ctypes.POINTER(ctypes.c_double)
    d = lambda a: a.ctypes.data_as(P)
    rc = lib.oracle_rpn2(5, 1, mx, 4, 3, mbc, mx, d(q), d(q), d(wave), d(s), d(am), d(ap), d(cp))
    assert rc == 0

    def flux(qq):
        r, mu, mv, E = qq
        uu = mu / r
        pp = (g - 1) * (E - 0.5 * (mu * mu + mv * mv) / r)
        return np.array([mu, mu * uu + pp, mv * uu, uu * (E + pp)])

    for i in range(1, n):  # interface i between cells i-1 and i
        assert np.allclose(wave[i].sum(0), q[i] - q[i - 1], rtol=1e-12, atol=1e-13)
        assert np.allclose(am[i] + ap[i], flux(q[i]) - flux(q[i - 1]), rtol=1e-11, atol=1e-12)
        assert s[i, 0] < s[i, 1] < s[i, 2]


def test_network_reference_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    P = rng.normal(0, 0.3, mlp_ref.NPARAM)
    x, y = rng.normal(0, 1, (20, 6)), rng.normal(0, 1, 20)
    g, _ = mlp_ref.gradient(P, x, y)
    eps = 1e-6
    for k in rng.choice(mlp_ref.NPARAM, 60, replace=False):
        Pp, Pm = P.copy(), P.copy()
        Pp[k] += eps
        Pm[k] -= eps
        num = (mlp_ref.gradient(Pp, x, y)[1] - mlp_ref.gradient(Pm, x, y)[1]) / (2 * eps)
        assert abs(num - g[k]) < 1e-7 * max(1.0, abs(g[k]))
