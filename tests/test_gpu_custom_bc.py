"""Custom boundary conditions (BC.custom with user functions) and the
5-wave Euler solver with a geometric source on the GPU.

A custom BC is a Python function of the host's qbc / auxbc, so with one the
host fills every ghost cell each step in the reference's order (dimension by
dimension, lower then upper, aux before q; solver.py:351-437) and uploads the
arrays; the device step then keeps those ghost cells.  Held to the oracle
(which applies the same functions to its host arrays) at 1e-12 and to the
reference's shock-bubble golden.
"""
import numpy as np
import pytest

from helpers import max_rel
from pyclaw_b200 import workloads
from pyclaw_b200.solver import BC

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("device_source", [False, True])
def test_shock_bubble_device_run(goldens, device_source):
    claw = workloads.shock_bubble(mx=160, my=40, tfinal=0.2, num_output_times=1, device_source=device_source)
    claw.run()
    d = claw.frames[claw.num_output_times].state.get_q_global()[0].reshape([-1])
    dx, dy = claw.solution.domain.grid.delta
    diff = dx * dy * np.sum(np.abs(d - goldens["euler_shock_bubble"]))
    assert diff < 1e-6  # the reference test's bound
    assert diff < 1e-12


def test_device_source_equals_host_function():
    # the device's axisymmetric source step rounds like the host function
    a = workloads.shock_bubble(mx=96, my=24, tfinal=0.05, num_output_times=1, device_source=False)
    b = workloads.shock_bubble(mx=96, my=24, tfinal=0.05, num_output_times=1, device_source=True)
    a.run()
    b.run()
    assert a.solver.status['numsteps'] == b.solver.status['numsteps']
    assert np.array_equal(a.solution.state.get_q_global(), b.solution.state.get_q_global())


def test_shock_bubble_frames_match_oracle(oracle):
    kw = dict(mx=320, my=80, tfinal=0.1, num_output_times=4)
    g = workloads.shock_bubble(device_source=True, **kw)
    o = workloads.shock_bubble(oracle.make_solver_class(), **kw)
    g.run()
    o.run()
    assert g.solver.status['numsteps'] == o.solver.status['numsteps']
    for a, b in zip(g.frames, o.frames):
        assert max_rel(a.q, b.q) <= 1e-12


def _time_inflow_lower_y(state, dim, t, qbc, auxbc, num_ghost):
    # a time-dependent inflow through the bottom (close to the quadrant state
    # there), written over every column
    for j in range(num_ghost):
        qbc[0, :, j] = 0.15 + 0.01 * np.sin(5 * t)
        qbc[1, :, j] = 1.2 * qbc[0, :, j]
        qbc[2, :, j] = 1.3 * qbc[0, :, j]
        qbc[3, :, j] = 0.03 / 0.4 + 0.5 * qbc[0, :, j] * (1.2 ** 2 + 1.3 ** 2)


def _damped_extrap_upper_x(state, dim, t, qbc, auxbc, num_ghost):
    # reads the interior next to the boundary: extrapolation with damped momentum
    for i in range(num_ghost):
        qbc[:, -i - 1, :] = qbc[:, -num_ghost - 1, :]
        qbc[1, -i - 1, :] *= 0.5


@pytest.mark.parametrize("custom_x", [True, False])
def test_custom_bcs_match_oracle(oracle, custom_x):
    # custom functions on a y side (applied after x: they own the corners) and
    # optionally on an x side (applied first: the y rule fills its corners)
    runs = []
    for cls in (None, oracle.make_solver_class()):
        claw = workloads.euler_quadrants_unsplit(cls, n=140, tfinal=0.05)
        claw.num_output_times = 3
        s = claw.solver
        s.user_bc_lower = _time_inflow_lower_y
        s.user_bc_upper = _damped_extrap_upper_x
        s.bc_lower[1] = BC.custom
        s.bc_lower[0] = BC.extrap
        s.bc_upper[1] = BC.extrap
        s.bc_upper[0] = BC.custom if custom_x else BC.extrap
        claw.run()
        runs.append(claw)
    g, o = runs
    assert g.solver.status['numsteps'] == o.solver.status['numsteps']
    for a, b in zip(g.frames, o.frames):
        assert max_rel(a.q, b.q) <= 1e-12
