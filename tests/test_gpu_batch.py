"""Batched form: many independent problems of uneven size stepped by one
persistent kernel per step with device-side accept/reject and dt, the steps
captured in a CUDA graph.

Every problem's result must equal the single-problem CUDA path (which is
itself parity-checked against the oracle): a cell's increments are summed in
the same order whatever the tile shape, but the batched kernel is its own
instantiation of the tile code and the compiler may fuse a multiply-add
differently there, so to a few units in the last place (1e-13 relative) with
the same step counts; and the graph run must equal the plain
one-launch-sequence-per-problem loop bit for bit (the same kernel)."""
import numpy as np
import pytest

from helpers import max_rel
from pyclaw_b200 import workloads
from pyclaw_b200.batch import Batch, autotune_rows

pytestmark = pytest.mark.gpu

SIDES = (16, 32, 48, 80, 130, 260)


def _dt0(claws):
    return [c.solver.dt_initial for c in claws]


def test_batch_graph_equals_plain_loop_and_single_problems():
    claws, sides = workloads.batched_quadrants(12, seed=5, sides=SIDES)
    bat = Batch(claws)
    nsteps = 6
    bat.run(nsteps, mode=0)
    st_graph = bat.state()
    q_graph = [bat.q(i) for i in range(bat.n)]
    assert np.all(st_graph["nsteps"] + st_graph["nreject"] == nsteps)

    bat.upload()
    bat.set_time(_dt0(claws), 0.0, 1e99)
    bat.run(nsteps, mode=2)
    st_plain = bat.state()
    for k in ("t", "dt", "nsteps", "nreject"):
        assert np.array_equal(st_graph[k], st_plain[k]), k
    for i in range(bat.n):
        assert np.array_equal(q_graph[i], bat.q(i))

    # the single-problem path: ClawSolver2D.evolve_to_time one step at a time
    for i in (0, 3, 7):
        claw, _ = workloads.batched_quadrants(12, seed=5, sides=SIDES)
        c = claw[i]
        s, sol = c.solver, c.solution
        s.setup(sol)
        s.dt = s.dt_initial
        for _ in range(nsteps):
            s.evolve_to_time(sol)
        assert abs(sol.t - st_graph["t"][i]) <= 1e-13 * sol.t
        assert max_rel(sol.state.get_q_global(), q_graph[i]) <= 1e-13


def test_batch_rejects_and_retakes_per_problem():
    claws, sides = workloads.batched_quadrants(4, seed=9, sides=(32, 64))
    bat = Batch(claws)
    bat.run(3, mode=0)
    base = bat.state()
    bat.upload()
    dt0 = _dt0(claws)
    dt0[2] *= 10.0  # far above the CFL limit on the first step: rejected, then retaken
    bat.set_time(dt0, 0.0, 1e99)
    bat.run(3, mode=0)
    st = bat.state()
    assert st["nreject"][2] == base["nreject"][2] + 1 and st["nsteps"][2] == base["nsteps"][2] - 1
    for i in (0, 1, 3):
        assert st["nreject"][i] == base["nreject"][i] and st["nsteps"][i] == base["nsteps"][i]


def test_batch_stops_at_tend_and_retires_failures():
    claws, sides = workloads.batched_quadrants(6, seed=2, sides=(32,))
    bat = Batch(claws)
    tend = 3.5 * max(_dt0(claws))
    bat.set_time(_dt0(claws), 0.0, tend)
    bat.run(40, mode=0)
    st = bat.state()
    ok = ~st["failed"]
    assert np.all(st["t"][ok] == tend)
    for i in np.nonzero(st["failed"])[0]:  # retired at its last good (finite) state
        assert np.all(np.isfinite(bat.q(i))) and st["t"][i] < tend


def test_batch_failure_is_isolated():
    # one problem given a negative density fails on its first step; the
    # others must step exactly as in a batch without it
    claws, sides = workloads.batched_quadrants(4, seed=11, sides=(48, 64))
    good = Batch(claws)
    good.run(5, mode=0)
    ref = good.state()
    qref = [good.q(i) for i in range(4)]
    claws[1].solution.state.q[0, 3, 3] = -1.0
    bat = Batch(claws)
    bat.run(5, mode=0)
    st = bat.state()
    assert st["failed"][1] and st["nsteps"][1] == 0
    for i in (0, 2, 3):
        assert not st["failed"][i] and st["nsteps"][i] == ref["nsteps"][i]
        assert np.array_equal(bat.q(i), qref[i])


def test_batch_autotune_keeps_results():
    claws, sides = workloads.batched_quadrants(8, seed=3, sides=(64, 144, 272))
    bat = Batch(claws)
    bat.run(2, mode=1)
    ref = [bat.q(i) for i in range(bat.n)]
    rows, trials, choice = autotune_rows(bat, sides, candidates=(8, 32), steps=1)
    bat.upload()
    bat.set_time(_dt0(claws), 0.0, 1e99)
    bat.run(2, mode=0)
    for i in range(bat.n):
        assert np.array_equal(bat.q(i), ref[i])
