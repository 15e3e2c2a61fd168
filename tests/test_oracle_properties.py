"""Property tests that pin the oracle's Riemann solvers and full step where no
reference golden reaches them.

The transverse solvers (rpt2) of acoustics, Euler and shallow water run only in
the unsplit step, and none of the reference's regression goldens runs that
step for those equations (the goldens are split runs, step2ds.f90, which never
calls rpt2).  The tests below pin them through their mathematical definition
instead:

* rpn2: the waves sum to the jump and the fluctuations sum to the flux
  difference (the Roe property; Harten-Hyman's entropy fix keeps the sum,
  LeVeque 2002 sec. 15.3.5);
* rpt2: bmasdq = B^- asdq and bpasdq = B^+ asdq with B the transverse flux
  Jacobian at the Roe average of the two cells (rpt2's contract,
  flux2.f90:181-203), B^+- built here from numpy's eigendecomposition;
* a whole step2 is symmetric under a 90 degree rotation (x <-> y, u <-> v);
* step2 conserves every component on a periodic domain;
* step2 with transverse corrections is second-order accurate on an oblique
  acoustic plane wave, whose exact solution is known.
"""
import ctypes

import numpy as np
import pytest

from tests.helpers import RP_INFO, method_vector, random_qbc, max_rel
from pyclaw_b200 import _lib

P = ctypes.POINTER(ctypes.c_double)


def _d(a):
    return a.ctypes.data_as(P)


def _cparam(rp):
    return np.asarray(RP_INFO[rp][3] + [0.0] * 8, dtype=np.float64)


def _slice(rp, n, seed):
    """n cells of a 1D slice, array (n, meqn) = the Fortran (meqn, n) layout."""
    q = random_qbc(rp, n - 4, 1, seed, smooth_frac=1.0)[:, :, 2]
    return np.ascontiguousarray(q.T)


def _flux(rp, q, ixy):
    """Physical flux in direction ixy (1 = x, 2 = y) of states q (..., meqn)."""
    if rp == _lib.RP_ADVECTION:
        u, v = RP_INFO[rp][3][:2]
        return q * (u if ixy == 1 else v)
    mu, mv = (1, 2) if ixy == 1 else (2, 1)
    f = np.zeros_like(q)
    if rp == _lib.RP_ACOUSTICS:
        rho, bulk = RP_INFO[rp][3][:2]
        f[..., 0] = bulk * q[..., mu]
        f[..., mu] = q[..., 0] / rho
        return f
    if rp == _lib.RP_EULER_ROE:
        g = RP_INFO[rp][3][0]
        r = q[..., 0]
        un = q[..., mu] / r
        p = (g - 1) * (q[..., 3] - 0.5 * (q[..., 1] ** 2 + q[..., 2] ** 2) / r)
        f[..., 0] = q[..., mu]
        f[..., mu] = q[..., mu] * un + p
        f[..., mv] = q[..., mv] * un
        f[..., 3] = un * (q[..., 3] + p)
        return f
    if rp == _lib.RP_SHALLOW_ROE:
        grav = RP_INFO[rp][3][0]
        h = q[..., 0]
        un = q[..., mu] / h
        f[..., 0] = q[..., mu]
        f[..., mu] = q[..., mu] * un + 0.5 * grav * h * h
        f[..., mv] = q[..., mv] * un
        return f
    raise ValueError(rp)


def _roe_jacobian(rp, ql, qr, tdir):
    """Flux Jacobian in direction tdir (1 = x, 2 = y) at the Roe average of the
    states ql, qr; for the linear systems the constant Jacobian."""
    meqn = RP_INFO[rp][1]
    B = np.zeros((meqn, meqn))
    mt, mo = (1, 2) if tdir == 1 else (2, 1)  # component along tdir, the other one
    if rp == _lib.RP_ADVECTION:
        B[0, 0] = RP_INFO[rp][3][tdir - 1]
        return B
    if rp == _lib.RP_ACOUSTICS:
        rho, bulk = RP_INFO[rp][3][:2]
        B[0, mt] = bulk
        B[mt, 0] = 1.0 / rho
        return B
    sl, sr = np.sqrt(ql[0]), np.sqrt(qr[0])
    vt = (ql[mt] / sl + qr[mt] / sr) / (sl + sr)
    uo = (ql[mo] / sl + qr[mo] / sr) / (sl + sr)
    if rp == _lib.RP_EULER_ROE:
        g = RP_INFO[rp][3][0]

        def enth(q):
            p = (g - 1) * (q[3] - 0.5 * (q[1] ** 2 + q[2] ** 2) / q[0])
            return q[3] + p

        H = (enth(ql) / sl + enth(qr) / sr) / (sl + sr)
        k2 = 0.5 * (g - 1) * (vt * vt + uo * uo)
        B[0, mt] = 1.0
        B[mo, 0], B[mo, mo], B[mo, mt] = -uo * vt, vt, uo
        B[mt, 0], B[mt, mo], B[mt, mt], B[mt, 3] = k2 - vt * vt, -(g - 1) * uo, (3 - g) * vt, g - 1
        B[3, 0], B[3, mo], B[3, mt], B[3, 3] = vt * (k2 - H), -(g - 1) * uo * vt, H - (g - 1) * vt * vt, g * vt
        return B
    if rp == _lib.RP_SHALLOW_ROE:
        c2 = RP_INFO[rp][3][0] * 0.5 * (ql[0] + qr[0])
        B[0, mt] = 1.0
        B[mo, 0], B[mo, mo], B[mo, mt] = -uo * vt, vt, uo
        B[mt, 0], B[mt, mt] = c2 - vt * vt, 2 * vt
        return B
    raise ValueError(rp)


def _split(B):
    """(B^-, B^+) of a diagonalisable B with real eigenvalues, from the spectral
    projectors P_k = prod_{j != k} (B - l_j I) / (l_k - l_j) over its distinct
    eigenvalues l_k (Sylvester's formula), which stays well defined where an
    eigenvalue repeats (the Euler contact and shear speeds coincide)."""
    lam = np.sort(np.linalg.eigvals(B).real)
    distinct = [lam[0]]
    for x in lam[1:]:
        if abs(x - distinct[-1]) > 1e-7 * (1.0 + abs(x)):
            distinct.append(x)
    n = B.shape[0]
    Bm, Bp = np.zeros_like(B), np.zeros_like(B)
    for k, lk in enumerate(distinct):
        Pk = np.eye(n)
        for j, lj in enumerate(distinct):
            if j != k:
                Pk = Pk @ (B - lj * np.eye(n)) / (lk - lj)
        Bm += min(lk, 0.0) * Pk
        Bp += max(lk, 0.0) * Pk
    return Bm, Bp


ALL_RP = [_lib.RP_ADVECTION, _lib.RP_ACOUSTICS, _lib.RP_EULER_ROE, _lib.RP_SHALLOW_ROE]


@pytest.mark.parametrize("rp", ALL_RP)
@pytest.mark.parametrize("ixy", [1, 2])
def test_rpn2_waves_sum_to_jump_and_fluctuations_to_flux_difference(oracle, rp, ixy):
    lib = oracle.load()
    _, meqn, mwaves, _ = RP_INFO[rp]
    mx, mbc = 60, 2
    n = mx + 2 * mbc
    q = _slice(rp, n, 11 + ixy)
    wave = np.zeros((n, mwaves, meqn))
    s = np.zeros((n, mwaves))
    am, ap = np.zeros((n, meqn)), np.zeros((n, meqn))
    assert lib.oracle_rpn2(rp, ixy, mx, meqn, mwaves, mbc, mx, _d(q), _d(q), _d(wave), _d(s), _d(am), _d(ap),
                           _d(_cparam(rp))) == 0
    F = _flux(rp, q, ixy)
    # acoustics carries no zero-speed shear wave: the tangential velocity jump is not a wave
    comp = [0, 1 if ixy == 1 else 2] if rp == _lib.RP_ACOUSTICS else list(range(meqn))
    for i in range(1, n):  # interface between cells i-1 and i
        scale = 1.0 + np.max(np.abs(q[i])) + np.max(np.abs(F[i]))
        assert np.max(np.abs(wave[i].sum(0) - (q[i] - q[i - 1]))[comp]) <= 1e-13 * scale
        assert np.max(np.abs(am[i] + ap[i] - (F[i] - F[i - 1]))) <= 1e-12 * scale
        assert np.all(np.diff(s[i]) >= 0)


@pytest.mark.parametrize("rp", ALL_RP)
@pytest.mark.parametrize("ixy", [1, 2])
def test_rpt2_splits_the_transverse_roe_jacobian(oracle, rp, ixy):
    lib = oracle.load()
    _, meqn, mwaves, _ = RP_INFO[rp]
    mx, mbc = 60, 2
    n = mx + 2 * mbc
    q = _slice(rp, n, 21 + ixy)
    rng = np.random.default_rng(5 + ixy)
    asdq = rng.uniform(-1, 1, (n, meqn))
    bm, bp = np.zeros((n, meqn)), np.zeros((n, meqn))
    assert lib.oracle_rpt2(rp, ixy, 1, mx, meqn, mwaves, mbc, mx, _d(q), _d(q), _d(asdq), _d(bm), _d(bp),
                           _d(_cparam(rp))) == 0
    tdir = 2 if ixy == 1 else 1
    for i in range(1, n):
        B = _roe_jacobian(rp, q[i - 1], q[i], tdir)
        # the Roe property of B itself, which pins the averaged state
        G = _flux(rp, q[[i - 1, i]], tdir)
        assert np.allclose(B @ (q[i] - q[i - 1]), G[1] - G[0], rtol=1e-11, atol=1e-12)
        Bm, Bp = _split(B)
        scale = 1.0 + np.max(np.abs(B)) * np.max(np.abs(asdq[i]))
        assert np.max(np.abs(bm[i] - Bm @ asdq[i])) <= 1e-12 * scale
        assert np.max(np.abs(bp[i] - Bp @ asdq[i])) <= 1e-12 * scale


def _rotate(q):
    """90 degree rotation of a qbc array: x <-> y and the two velocity components."""
    r = np.transpose(q, (0, 2, 1)).copy()
    if q.shape[0] >= 3:
        r[[1, 2]] = r[[2, 1]]
    return np.asfortranarray(r)


@pytest.mark.parametrize("rp", [_lib.RP_ACOUSTICS, _lib.RP_EULER_ROE, _lib.RP_SHALLOW_ROE])
@pytest.mark.parametrize("transverse", [1, 2])
def test_full_step_is_symmetric_under_rotation(oracle, rp, transverse):
    _, meqn, mwaves, cp = RP_INFO[rp]
    mx, my = 23, 17
    q0 = random_qbc(rp, mx, my, seed=31 + transverse)
    method = method_vector(2, transverse)
    mthlim = [4] * mwaves
    dt = 0.3 * 0.05 / 2.5
    qa = q0.copy(order="F")
    cfl_a = oracle.step2(q0, qa, 0.05, 0.05, dt, method, mthlim, rp, cp)
    r0 = _rotate(q0)
    qb = r0.copy(order="F")
    cfl_b = oracle.step2(r0, qb, 0.05, 0.05, dt, method, mthlim, rp, cp)
    assert max_rel(_rotate(qb)[:, 2:-2, 2:-2], qa[:, 2:-2, 2:-2]) <= 1e-13
    assert abs(cfl_a - cfl_b) <= 1e-14 * cfl_a


@pytest.mark.parametrize("rp", ALL_RP)
def test_step_conserves_every_component_on_a_periodic_domain(oracle, rp):
    _, meqn, mwaves, cp = RP_INFO[rp]
    mx, my = 40, 30
    q = random_qbc(rp, mx, my, seed=41)
    method = method_vector(2, 2)
    mthlim = [4] * mwaves
    dx = dy = 0.02
    total0 = q[:, 2:-2, 2:-2].sum(axis=(1, 2))
    scale = np.abs(q[:, 2:-2, 2:-2]).sum(axis=(1, 2))
    for _ in range(10):
        oracle.bc_fill(q, [2, 2], [2, 2])
        qn = q.copy(order="F")
        cfl = oracle.step2(q, qn, dx, dy, 0.004, method, mthlim, rp, cp)
        assert 0 < cfl < 1
        q = qn
    total = q[:, 2:-2, 2:-2].sum(axis=(1, 2))
    assert np.all(np.abs(total - total0) <= 1e-13 * scale)


def _plane_wave(n, t):
    """Acoustics (rho = 1, K = 4, c = 2, Z = 2) oblique plane wave on the
    periodic unit square: p = sin(2 pi (x + y - sqrt(2) c t)), (u, v) = p/(Z sqrt 2)."""
    xc = (np.arange(n) + 0.5) / n
    X, Y = np.meshgrid(xc, xc, indexing="ij")
    p = np.sin(2 * np.pi * (X + Y - np.sqrt(2.0) * 2.0 * t))
    un = p / (2.0 * np.sqrt(2.0))
    return np.stack([p, un, un])


@pytest.mark.parametrize("transverse", [0, 1, 2])
def test_unsplit_step_is_second_order_on_an_oblique_plane_wave(oracle, transverse):
    """L1 error of p at t = 0.1 on 32^2, 64^2, 128^2 (no limiter): the rate is
    2.0 with either transverse mode, i.e. rpt2 supplies exactly the cross
    derivative terms, and 1.0 without them (measured 2.02/2.01 and 0.97/0.99)."""
    rp = _lib.RP_ACOUSTICS
    cp = RP_INFO[rp][3]
    tend = 0.1
    errs = []
    for n in (32, 64, 128):
        dx = 1.0 / n
        nsteps = int(np.ceil(tend * 2.0 / (0.8 * dx)))
        dt = tend / nsteps
        q = np.zeros((3, n + 4, n + 4), order="F")
        q[:, 2:-2, 2:-2] = _plane_wave(n, 0.0)
        for _ in range(nsteps):
            oracle.bc_fill(q, [2, 2], [2, 2])
            qn = q.copy(order="F")
            oracle.step2(q, qn, dx, dx, dt, method_vector(2, transverse), [0, 0], rp, cp)
            q = qn
        errs.append(np.abs(q[0, 2:-2, 2:-2] - _plane_wave(n, tend)[0]).mean())
    rates = np.log2(np.array(errs[:-1]) / np.array(errs[1:]))
    if transverse:
        assert np.all(rates > 1.9), (errs, rates)
    else:
        assert np.all(rates < 1.2), (errs, rates)
