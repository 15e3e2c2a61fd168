"""Parity of the CUDA step against the CPU oracle (the reference's step2 /
step2ds / flux2 / limiter / philim restated), called through the C ABI.

Bar: interior cells within 1e-12 relative in the max norm, CFL within 1e-12
relative, on identical inputs (FP64; the only differences are the order of
the per-cell increment sums and fused multiply-adds).
"""
import numpy as np
import pytest

from helpers import PARITY_RTOL, RP_INFO, max_rel, method_vector, random_qbc, set_cparam
from pyclaw_b200 import _lib, classic2

pytestmark = pytest.mark.gpu

SIZES = [(1, 1), (3, 5), (37, 23), (130, 70), (257, 9), (9, 300)]


def _dt_for(oracle, qbc, rp, cp, method, mthlim, dx, dy, target=0.8, split=False):
    q2 = qbc.copy(order="F")
    if split:
        c = oracle.step2ds(qbc, q2, dx, dy, 1e-3, method, mthlim, 1, rp, cp)
    else:
        c = oracle.step2(qbc, q2, dx, dy, 1e-3, method, mthlim, rp, cp)
    return 1e-3 * target / max(c, 1e-12)


@pytest.mark.parametrize("rp", sorted(RP_INFO))
@pytest.mark.parametrize("transverse", [0, 1, 2])
@pytest.mark.parametrize("mx,my", SIZES)
def test_step2_unsplit(oracle, rp, transverse, mx, my):
    name, meqn, mwaves, cp = RP_INFO[rp]
    qbc = random_qbc(rp, mx, my, seed=mx * 1000 + my + transverse)
    method = method_vector(2, transverse)
    mthlim = np.full(mwaves, 4, dtype=np.intc)
    dx, dy = 1.0 / mx, 1.3 / my
    dt = _dt_for(oracle, qbc, rp, cp, method, mthlim, dx, dy)
    q_o = qbc.copy(order="F")
    cfl_o = oracle.step2(qbc, q_o, dx, dy, dt, method, mthlim, rp, cp)
    set_cparam(classic2, rp)
    q_g, cfl_g = classic2.step2(max(mx, my), 2, mx, my, qbc, qbc.copy(order="F"), None, dx, dy, dt, method,
                                mthlim, rpn2=rp)
    assert abs(cfl_g - cfl_o) <= PARITY_RTOL * cfl_o
    assert max_rel(q_g[:, 2:-2, 2:-2], q_o[:, 2:-2, 2:-2]) <= PARITY_RTOL
    # ghost cells are returned as they were on entry
    assert np.array_equal(q_g[:, :2, :], qbc[:, :2, :])


@pytest.mark.parametrize("rp", sorted(RP_INFO))
@pytest.mark.parametrize("lim", [0, 1, 2, 3, 4, 5])
@pytest.mark.parametrize("order", [1, 2])
def test_step2_limiters_and_order(oracle, rp, lim, order):
    name, meqn, mwaves, cp = RP_INFO[rp]
    mx, my = 61, 47
    qbc = random_qbc(rp, mx, my, seed=7 + lim)
    method = method_vector(order, 2)
    mthlim = np.array([(lim + k) % 6 if lim else 0 for k in range(mwaves)], dtype=np.intc)
    dx, dy = 0.02, 0.015
    dt = _dt_for(oracle, qbc, rp, cp, method, mthlim, dx, dy)
    q_o = qbc.copy(order="F")
    cfl_o = oracle.step2(qbc, q_o, dx, dy, dt, method, mthlim, rp, cp)
    set_cparam(classic2, rp)
    q_g, cfl_g = classic2.step2(max(mx, my), 2, mx, my, qbc, qbc.copy(order="F"), None, dx, dy, dt, method,
                                mthlim, rpn2=rp)
    assert abs(cfl_g - cfl_o) <= PARITY_RTOL * cfl_o
    assert max_rel(q_g[:, 2:-2, 2:-2], q_o[:, 2:-2, 2:-2]) <= PARITY_RTOL


@pytest.mark.parametrize("rp", sorted(RP_INFO))
@pytest.mark.parametrize("ids", [1, 2])
@pytest.mark.parametrize("mx,my", [(1, 1), (37, 23), (130, 70), (250, 260)])
def test_step2ds_sweeps(oracle, rp, ids, mx, my):
    name, meqn, mwaves, cp = RP_INFO[rp]
    qbc = random_qbc(rp, mx, my, seed=31 * mx + my + ids)
    method = method_vector(2, 0, split=True)
    mthlim = np.full(mwaves, 4, dtype=np.intc)
    dx, dy = 1.0 / mx, 1.0 / my
    dt = _dt_for(oracle, qbc, rp, cp, method, mthlim, dx, dy, split=True)
    q_o = qbc.copy(order="F")
    cfl_o = oracle.step2ds(qbc, q_o, dx, dy, dt, method, mthlim, ids, rp, cp)
    set_cparam(classic2, rp)
    q_g, cfl_g = classic2.step2ds(max(mx, my), 2, mx, my, qbc, qbc.copy(order="F"), None, dx, dy, dt, method,
                                  mthlim, ids=ids, rpn2=rp)
    assert abs(cfl_g - cfl_o) <= PARITY_RTOL * cfl_o
    if ids == 1:
        # the x-sweep result covers every row, ghost rows included
        assert max_rel(q_g[:, 2:-2, :], q_o[:, 2:-2, :]) <= PARITY_RTOL
        assert np.array_equal(q_g[:, :2, :], q_o[:, :2, :])
    else:
        assert max_rel(q_g[:, 2:-2, 2:-2], q_o[:, 2:-2, 2:-2]) <= PARITY_RTOL


@pytest.mark.parametrize("rp", sorted(RP_INFO))
@pytest.mark.parametrize("ids", [1, 2])
@pytest.mark.parametrize("order,mthlim_kind", [(2, "mc"), (2, "mixed"), (1, "mc")])
def test_step2ds_sweeps_zero_jump_shortcut(oracle, rp, ids, order, mthlim_kind):
    # data with long constant runs (1% noisy cells): whole warps of a sweep
    # have equal cells on both sides and take the zero-jump shortcut; the
    # generic and the method-specialised sweep kernels both
    name, meqn, mwaves, cp = RP_INFO[rp]
    mx, my = 300, 150
    qbc = random_qbc(rp, mx, my, seed=7 * rp + ids + order, smooth_frac=0.01)
    method = method_vector(order, 0, split=True)
    mthlim = np.full(mwaves, 4, dtype=np.intc) if mthlim_kind == "mc" else \
        np.array([4, 1, 2, 3, 5][:mwaves], dtype=np.intc)
    dx, dy = 1.0 / mx, 1.0 / my
    dt = _dt_for(oracle, qbc, rp, cp, method, mthlim, dx, dy, split=True)
    q_o = qbc.copy(order="F")
    cfl_o = oracle.step2ds(qbc, q_o, dx, dy, dt, method, mthlim, ids, rp, cp)
    set_cparam(classic2, rp)
    q_g, cfl_g = classic2.step2ds(max(mx, my), 2, mx, my, qbc, qbc.copy(order="F"), None, dx, dy, dt, method,
                                  mthlim, ids=ids, rpn2=rp)
    assert abs(cfl_g - cfl_o) <= PARITY_RTOL * cfl_o
    rows = slice(None) if ids == 1 else slice(2, -2)
    assert max_rel(q_g[:, 2:-2, rows], q_o[:, 2:-2, rows]) <= PARITY_RTOL


@pytest.mark.parametrize("rp", sorted(RP_INFO))
@pytest.mark.parametrize("variant,rows", [(0, 2), (0, 16), (1, 7), (2, 16), (3, 16), (3, 40), (4, 8)])
def test_step2_piecewise_constant_tiles(oracle, rp, variant, rows):
    # piecewise-constant quadrants with one noisy patch: most tiles read one
    # state only (every warp of them takes the zero-jump shortcut), some
    # straddle a quadrant edge or the patch; every launch shape, ragged last
    # strip and row block
    from pyclaw_b200 import tune
    name, meqn, mwaves, cp = RP_INFO[rp]
    mx, my = 300, 170
    qbc = random_qbc(rp, mx, my, seed=11 * rp + variant, smooth_frac=0.0)
    noisy = random_qbc(rp, mx, my, seed=5 * rp + 1, smooth_frac=1.0)
    qbc[:, 40:60, 100:130] = noisy[:, 40:60, 100:130]
    method = method_vector(2, 2)
    mthlim = np.full(mwaves, 4, dtype=np.intc)
    dx, dy = 1.0 / mx, 1.0 / my
    dt = _dt_for(oracle, qbc, rp, cp, method, mthlim, dx, dy)
    q_o = qbc.copy(order="F")
    cfl_o = oracle.step2(qbc, q_o, dx, dy, dt, method, mthlim, rp, cp)
    set_cparam(classic2, rp)
    tune.set_shape(rp, variant, rows)
    try:
        q_g, cfl_g = classic2.step2(max(mx, my), 2, mx, my, qbc, qbc.copy(order="F"), None, dx, dy, dt, method,
                                    mthlim, rpn2=rp)
    finally:
        tune.set_shape(rp, 0, 0)
    assert abs(cfl_g - cfl_o) <= PARITY_RTOL * cfl_o
    assert max_rel(q_g[:, 2:-2, 2:-2], q_o[:, 2:-2, 2:-2]) <= PARITY_RTOL


@pytest.mark.parametrize("rp", sorted(RP_INFO))
def test_step2_all_uniform_grid(oracle, rp):
    # one state everywhere: every interface joins equal cells; the cells come
    # back unchanged and the Courant number is the oracle's
    from pyclaw_b200 import tune
    name, meqn, mwaves, cp = RP_INFO[rp]
    mx, my = 260, 90
    base = random_qbc(rp, 4, 4, seed=rp, smooth_frac=0.0)
    qbc = np.asfortranarray(np.broadcast_to(base[:, :1, :1], (meqn, mx + 4, my + 4)).copy())
    method = method_vector(2, 2)
    mthlim = np.full(mwaves, 4, dtype=np.intc)
    dx, dy = 1.0 / mx, 1.0 / my
    dt = 1e-4
    q_o = qbc.copy(order="F")
    cfl_o = oracle.step2(qbc, q_o, dx, dy, dt, method, mthlim, rp, cp)
    set_cparam(classic2, rp)
    for variant in (0, 3):
        tune.set_shape(rp, variant, 16)
        try:
            q_g, cfl_g = classic2.step2(max(mx, my), 2, mx, my, qbc, qbc.copy(order="F"), None, dx, dy, dt,
                                        method, mthlim, rpn2=rp)
        finally:
            tune.set_shape(rp, 0, 0)
        assert abs(cfl_g - cfl_o) <= PARITY_RTOL * cfl_o
        assert np.array_equal(q_g[:, 2:-2, 2:-2], qbc[:, 2:-2, 2:-2])
        assert np.array_equal(q_o[:, 2:-2, 2:-2], qbc[:, 2:-2, 2:-2])


@pytest.mark.parametrize("bcl,bcu", [((1, 1), (1, 1)), ((2, 2), (2, 2)), ((3, 3), (3, 3)), ((1, 3), (3, 1)),
                                     ((2, 1), (2, 3)), ((3, 2), (1, 2))])
@pytest.mark.parametrize("mx,my", [(2, 2), (2, 3), (17, 29)])
def test_bc_fill(oracle, bcl, bcu, mx, my):
    qbc = random_qbc(_lib.RP_EULER_ROE, mx, my, seed=mx + 100 * my)
    q_o = qbc.copy(order="F")
    oracle.bc_fill(q_o, bcl, bcu)
    q_g = classic2.bc_fill(qbc.copy(order="F"), bcl, bcu)
    assert np.array_equal(q_g, q_o)


def test_bc_fill_single_cell_extrap(oracle):
    qbc = random_qbc(_lib.RP_SHALLOW_ROE, 1, 1, seed=5)
    q_o = qbc.copy(order="F")
    oracle.bc_fill(q_o, (1, 1), (1, 1))
    assert np.array_equal(classic2.bc_fill(qbc.copy(order="F"), (1, 1), (1, 1)), q_o)


def test_bc_fill_rejects_wall_on_single_cell():
    qbc = random_qbc(_lib.RP_SHALLOW_ROE, 1, 4, seed=5)
    with pytest.raises(_lib.Claw2Error):
        classic2.bc_fill(qbc, (3, 1), (3, 1))


@pytest.mark.parametrize("name,bound", [("claw2_selftest_rcp", 1.0), ("claw2_selftest_sqrt", 1.0),
                                        ("claw2_selftest_rsqrt", 2.0)])
def test_kernel_reciprocal_and_roots_close_to_ieee(name, bound):
    # the limiter ratio and the Roe solvers' reciprocal densities use a
    # Newton-Raphson reciprocal, their square roots a Goldschmidt iteration,
    # the Roe averages' 1/c Newton steps on the reciprocal root; over 2^22
    # values spanning 2^-1000..2^1000 each stays within 1 ulp of CUDA's IEEE
    # quotient / square root (2 ulps of 1.0 / sqrt(x), itself rounded twice),
    # and the special values (zeros, infinities, NaN, subnormals) give the
    # documented results
    import ctypes
    L = _lib.load()
    for seed in (1, 2024):
        ulp = ctypes.c_double(-1.0)
        _lib.check(getattr(L, name)(0, 1 << 22, seed, ctypes.byref(ulp)))
        assert 0.0 <= ulp.value <= bound, ulp.value


@pytest.mark.parametrize("n", [1, 5, 31, 32, 33, 576, 1000, 1024, 1025, 3000, 8192])
def test_schedule_sort_matches_stable_host_sort(n):
    # the longest-first schedule's sort (shuffle stages up to 1024 tiles, the
    # shared-memory network beyond) against a stable descending host sort,
    # on costs with many ties
    import ctypes
    L = _lib.load()
    for seed in (1, 77):
        bad = ctypes.c_int(-1)
        _lib.check(L.claw2_selftest_lpt(0, n, seed, ctypes.byref(bad)))
        assert bad.value == 0


@pytest.mark.parametrize("split,per_step", [(False, 2), (True, 3)])
def test_step_launch_count(split, per_step):
    # the counter bench.py reports as gpu_launches: ghost fill + the step
    # kernel (two sweeps when split); a grid this small runs no schedule sort
    import ctypes
    from pyclaw_b200 import workloads
    claw = workloads.euler_quadrants_unsplit(n=64, tfinal=0.01)
    claw.solver.dimensional_split = split
    claw.solver.setup(claw.solution)
    p = claw.solver._dev
    L = _lib.load()
    n0, n1 = ctypes.c_longlong(-1), ctypes.c_longlong(-1)
    _lib.check(L.claw2_patch_launch_count(p.h, ctypes.byref(n0)))
    for _ in range(3):
        p.step(1e-4, want_cfl=False)
        p.accept(True)
    _lib.check(L.claw2_patch_launch_count(p.h, ctypes.byref(n1)))
    assert n1.value - n0.value == 3 * per_step
