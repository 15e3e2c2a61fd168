"""The Euler solver with a tracer (euler_5wave_2D) and the shallow-water HLLE
solver (shallow_hlle_2D) on the GPU, held to the oracle at 1e-12 step by step
and to the reference's radial dam-break golden."""
import numpy as np
import pytest

from helpers import PARITY_RTOL, max_rel, method_vector, random_qbc
from pyclaw_b200 import _lib, classic2, workloads

pytestmark = pytest.mark.gpu

E5 = _lib.RP_EULER_5WAVE
SH = _lib.RP_SHALLOW_HLLE


def _euler5(mx, my, seed):
    q4 = random_qbc(_lib.RP_EULER_ROE, mx, my, seed)
    rng = np.random.default_rng(seed + 1)
    tracer = np.where(rng.random((mx + 4, my + 4)) < 0.5, rng.random((mx + 4, my + 4)), 0.0)
    return np.asfortranarray(np.concatenate([q4, tracer[None]]))


@pytest.mark.parametrize("efix", [1.0, 0.0])
@pytest.mark.parametrize("transverse", [0, 1, 2])
@pytest.mark.parametrize("mx,my", [(3, 5), (130, 70), (9, 300)])
def test_euler5_step2(oracle, efix, transverse, mx, my):
    qbc = _euler5(mx, my, mx + my + transverse)
    method = method_vector(2, transverse)
    # a different limiter on every family: the families must line up with the
    # reference's order (acoustic, shear, entropy, acoustic, tracer)
    mthlim = np.array([4, 1, 2, 3, 5], dtype=np.intc)
    cp = [1.4, efix]
    dx, dy = 1.0 / mx, 1.0 / my
    dt = 0.12 * min(dx, dy)
    q_o = qbc.copy(order="F")
    cfl_o = oracle.step2(qbc, q_o, dx, dy, dt, method, mthlim, E5, cp)
    classic2.cparam.gamma = 1.4
    classic2.cparam.efix = bool(efix)
    q_g, cfl_g = classic2.step2(max(mx, my), 2, mx, my, qbc, qbc.copy(order="F"), None, dx, dy, dt, method,
                                mthlim, rpn2=E5)
    assert abs(cfl_g - cfl_o) <= PARITY_RTOL * cfl_o
    assert max_rel(q_g[:, 2:-2, 2:-2], q_o[:, 2:-2, 2:-2]) <= PARITY_RTOL


@pytest.mark.parametrize("ids", [1, 2])
def test_euler5_step2ds(oracle, ids):
    mx, my = 130, 70
    qbc = _euler5(mx, my, 3 + ids)
    method = method_vector(2, 0, split=True)
    mthlim = np.array([4, 4, 4, 4, 2], dtype=np.intc)
    dx, dy = 1.0 / mx, 1.0 / my
    dt = 0.12 * min(dx, dy)
    q_o = qbc.copy(order="F")
    cfl_o = oracle.step2ds(qbc, q_o, dx, dy, dt, method, mthlim, ids, E5, [1.4, 1.0])
    classic2.cparam.gamma = 1.4
    classic2.cparam.efix = True
    q_g, cfl_g = classic2.step2ds(max(mx, my), 2, mx, my, qbc, qbc.copy(order="F"), None, dx, dy, dt, method,
                                  mthlim, ids=ids, rpn2=E5)
    assert abs(cfl_g - cfl_o) <= PARITY_RTOL * cfl_o
    sl = (slice(None), slice(2, -2), slice(None)) if ids == 1 else (slice(None), slice(2, -2), slice(2, -2))
    assert max_rel(q_g[sl], q_o[sl]) <= PARITY_RTOL


@pytest.mark.parametrize("ids", [1, 2])
@pytest.mark.parametrize("mx,my", [(1, 1), (37, 23), (257, 70)])
def test_shallow_hlle_step2ds(oracle, ids, mx, my):
    qbc = random_qbc(_lib.RP_SHALLOW_ROE, mx, my, seed=mx + 3 * my + ids)
    method = method_vector(2, 0, split=True)
    mthlim = np.array([4, 1], dtype=np.intc)
    dx, dy = 1.0 / mx, 1.0 / my
    dt = 0.3 * min(dx, dy)
    q_o = qbc.copy(order="F")
    cfl_o = oracle.step2ds(qbc, q_o, dx, dy, dt, method, mthlim, ids, SH, [1.0])
    classic2.cparam.grav = 1.0
    q_g, cfl_g = classic2.step2ds(max(mx, my), 2, mx, my, qbc, qbc.copy(order="F"), None, dx, dy, dt, method,
                                  mthlim, ids=ids, rpn2=SH)
    assert abs(cfl_g - cfl_o) <= PARITY_RTOL * cfl_o
    sl = (slice(None), slice(2, -2), slice(None)) if ids == 1 else (slice(None), slice(2, -2), slice(2, -2))
    assert max_rel(q_g[sl], q_o[sl]) <= PARITY_RTOL


def test_shallow_hlle_unsplit_without_transverse(oracle):
    mx, my = 130, 70
    qbc = random_qbc(_lib.RP_SHALLOW_ROE, mx, my, seed=11)
    method = method_vector(2, 0)
    mthlim = np.array([4, 4], dtype=np.intc)
    dx, dy = 1.0 / mx, 1.0 / my
    dt = 0.2 * min(dx, dy)
    q_o = qbc.copy(order="F")
    cfl_o = oracle.step2(qbc, q_o, dx, dy, dt, method, mthlim, SH, [1.0])
    classic2.cparam.grav = 1.0
    q_g, cfl_g = classic2.step2(max(mx, my), 2, mx, my, qbc, qbc.copy(order="F"), None, dx, dy, dt, method,
                                mthlim, rpn2=SH)
    assert abs(cfl_g - cfl_o) <= PARITY_RTOL * cfl_o
    assert max_rel(q_g[:, 2:-2, 2:-2], q_o[:, 2:-2, 2:-2]) <= PARITY_RTOL
    with pytest.raises(_lib.Claw2Error):
        classic2.step2(max(mx, my), 2, mx, my, qbc, qbc.copy(order="F"), None, dx, dy, dt, method_vector(2, 1),
                       mthlim, rpn2=SH)


def test_shallow_hlle_device_run_matches_golden(goldens):
    claw = workloads.radial_dam_break(riemann_solver='hlle')
    claw.run()
    q = claw.frames[claw.num_output_times].state.get_q_global()[0].reshape([-1])
    dx, dy = claw.solution.domain.grid.delta
    err = dx * dy * np.sum(np.abs(q - goldens["shallow_radialdambreak_classic_hlle"]))
    assert err < 1e-5  # the reference test's bound
    assert err < 1e-11
