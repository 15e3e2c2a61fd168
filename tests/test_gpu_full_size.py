"""Size-independent properties at the benchmark's own sizes, where the oracle
would take minutes per step: the Euler quadrant problem at 1024^2 (the
headline workload) and the shallow-water dam break at 4096^2, run through the
Controller on the device time loop.

* mirror symmetry: both problems are symmetric about the diagonal x = y with
  the two momenta exchanged, and so must the computed states be (the fused
  kernel treats x and y interfaces in different orders, so this holds to
  rounding, not bit for bit);
* conservation: with periodic boundaries (Euler) or a front that has not
  reached the boundary (dam break) the sums of the conserved quantities stay
  at their initial values to rounding.
"""
import math

import numpy as np
import pytest

from helpers import max_rel
from pyclaw_b200 import BC, workloads

pytestmark = pytest.mark.gpu


def _sums(q):
    # correctly rounded sums (a plain float sum over 10^6 cells drifts by 1e-11 relative)
    return np.array([math.fsum(q[m].ravel()) for m in range(q.shape[0])])


def _mirror(q):
    qt = np.transpose(q, (0, 2, 1)).copy()
    qt[[1, 2]] = qt[[2, 1]]
    return qt


def _run(claw):
    claw.num_output_times = 1
    claw.keep_copy = True
    claw.run()
    return claw


def test_euler_1024_diagonal_symmetry():
    claw = _run(workloads.euler_quadrants_unsplit(n=1024, tfinal=0.05))
    assert claw.solver.status['numsteps'] > 100
    q = claw.frames[-1].q
    assert np.all(np.isfinite(q))
    assert max_rel(_mirror(q), q) <= 1e-11


def test_euler_1024_periodic_conservation():
    claw = workloads.euler_quadrants_unsplit(n=1024, tfinal=0.03)
    for d in (0, 1):
        claw.solver.bc_lower[d] = BC.periodic
        claw.solver.bc_upper[d] = BC.periodic
    q0 = claw.solution.state.get_q_global()
    s0, scale = _sums(q0), _sums(np.abs(q0))
    _run(claw)
    assert claw.solver.status['numsteps'] > 50
    s1 = _sums(claw.frames[-1].q)
    assert np.all(np.abs(s1 - s0) <= 1e-14 * scale)


def test_shallow_4096_mass_and_symmetry():
    # the C3 configuration for 0.15 time units (about 200 steps at CFL 0.9):
    # the front moves about 0.2 and stays far from the boundary
    claw = workloads.shallow_dam_break_unsplit(n=4096, tfinal=0.15)
    q0 = claw.solution.state.get_q_global()
    m0, scale = _sums(q0[:1])[0], _sums(np.abs(q0[:1]))[0]
    _run(claw)
    assert claw.solver.status['numsteps'] > 150
    q = claw.frames[-1].q
    assert abs(_sums(q[:1])[0] - m0) <= 1e-14 * scale
    assert max_rel(_mirror(q), q) <= 1e-11
