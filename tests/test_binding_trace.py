"""The binding trace (tests/golden/binding_trace.npz, recorded from the
reference's own ClawSolver2D driving a step module with f2py's signature) is
self-consistent with the oracle: every kept call, replayed through the oracle,
gives the recorded result bit for bit, and the recorded runs reproduced the
reference's goldens.  The same calls go through the CUDA path in
tests/test_gpu_binding.py."""
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def trace():
    return dict(np.load(os.path.join(HERE, "golden", "binding_trace.npz")))


def test_recorded_runs_reproduced_the_goldens(trace):
    for key in ("advection", "quadrants"):
        assert float(trace[key + "_l1_oracle_vs_golden"]) < 1e-12
        n = int(trace[key + "_n"])
        assert len(trace[key + "_dt"]) == n and np.all(np.isfinite(trace[key + "_cfl"]))  # rejected attempts included
    # quadrants runs split: x then y sweep every step
    ids = trace["quadrants_ids"]
    assert np.array_equal(ids, np.tile([1, 2], len(ids) // 2))


@pytest.mark.parametrize("key,k", [("advection", 0), ("advection", 1), ("advection", 2), ("quadrants", 0),
                                   ("quadrants", 1)])
def test_kept_calls_match_the_oracle(oracle, trace, key, k):
    from pyclaw_b200 import riemann
    p = "%s_call%d_" % (key, k)
    rp = getattr(riemann, str(trace[p + "rp"]))
    cp = rp.cparam({str(a): float(b) for a, b in zip(trace[p + "cparam_keys"], trace[p + "cparam_vals"])})
    qold = np.asfortranarray(trace[p + "qold"])
    q = qold.copy(order="F")
    dx, dy, dt = float(trace[p + "dx"]), float(trace[p + "dy"]), float(trace[p + "dt"])
    if str(trace[p + "name"]) == "step2":
        cfl = oracle.step2(qold, q, dx, dy, dt, trace[p + "method"], trace[p + "mthlim"], rp.rp_id, cp)
    else:
        cfl = oracle.step2ds(qold, q, dx, dy, dt, trace[p + "method"], trace[p + "mthlim"], int(trace[p + "ids"]),
                             rp.rp_id, cp)
    assert cfl == float(trace[p + "cfl"])
    assert np.array_equal(q, trace[p + "qout"])


def test_binding_preconditions_without_gpu():
    # what the reference's unmodified ClawSolver2D does with the step module
    # and the Riemann solver object before its first step
    # (classic/solver.py:208-232, state.py:206-231, solver.py:230-238)
    import importlib
    import pyclaw_b200.classic2 as fmod
    from pyclaw_b200 import riemann
    importlib.reload(fmod)  # setup() reloads the module to flush its cparam block
    assert vars(fmod.cparam) == {}
    for name in ("advection_2D", "acoustics_2D", "euler_4wave_2D", "shallow_roe_with_efix_2D"):
        rp = getattr(riemann, name)
        assert rp.__name__.split('.')[-1] == name
        assert rp.rpn2._cpointer is rp and rp.rpt2._cpointer is rp
        assert name in riemann.static.num_eqn and name in riemann.static.num_waves
        # state.set_cparam(rp): lists the block's parameters (none demanded), then assigns
        assert [p for p in rp.cparam.__dir__() if '__' not in p] == []
        setattr(rp.cparam, "gamma", 1.4)
