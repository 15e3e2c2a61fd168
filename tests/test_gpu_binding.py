"""The reference-side binding: the reference's own ClawSolver2D with
``solver.fmod = pyclaw_b200.classic2`` and this package's Riemann solvers as
its ``rp`` modules.

The reference's step_hyperbolic (src/pyclaw/classic/solver.py:498-549) calls
``fmod.step2(maxm, num_ghost, mx, my, qold, qbc, auxbc, dx, dy, dt, method,
mthlim, aux1, aux2, aux3, work, fwave, rpn2, rpt2)`` (and ``step2ds`` with
``ids`` before ``fwave``), with cparam set by ``state.set_cparam(fmod)``.
tests/golden/make_binding_trace.py ran the reference's unmodified host layer
-- its advection_2d (unsplit trans_cor) and euler_2d quadrants (split Roe)
examples, reproducing their goldens -- and recorded those calls.  Here each
recorded call goes through pyclaw_b200.classic2 with exactly the recorded
positional arguments and cparam block, and must give the recorded result:
interior cells and Courant number within 1e-12 relative.  (The reference
reads back only the interior of qbc, state.py:239-253.)"""
import types

import numpy as np
import pytest

from helpers import PARITY_RTOL, max_rel
from pyclaw_b200 import classic2, riemann

pytestmark = pytest.mark.gpu

CASES = [("advection", k) for k in range(3)] + [("quadrants", k) for k in range(2)]


def _call(trace, key, k):
    p = "%s_call%d_" % (key, k)
    g = {f: trace[p + f] for f in ("name", "rp", "ids", "maxm", "num_ghost", "mx", "my", "dx", "dy", "dt", "cfl",
                                    "method", "mthlim", "cparam_keys", "cparam_vals", "qold", "qout")}
    return g


@pytest.fixture(scope="module")
def trace():
    import os
    here = os.path.dirname(os.path.abspath(__file__))
    return dict(np.load(os.path.join(here, "golden", "binding_trace.npz")))


@pytest.mark.parametrize("key,k", CASES)
def test_reference_calls_replayed_through_classic2(trace, key, k):
    c = _call(trace, key, k)
    # state.set_cparam(fmod): problem_data entries as attributes of fmod.cparam
    classic2.cparam = types.SimpleNamespace()
    for name, val in zip(c["cparam_keys"], c["cparam_vals"]):
        setattr(classic2.cparam, str(name), float(val))
    rp = getattr(riemann, str(c["rp"]))
    qold = np.asfortranarray(c["qold"])
    qbc = qold.copy(order="F")
    args = (int(c["maxm"]), int(c["num_ghost"]), int(c["mx"]), int(c["my"]), qold, qbc, None,
            float(c["dx"]), float(c["dy"]), float(c["dt"]), c["method"], c["mthlim"], None, None, None, None)
    if str(c["name"]) == "step2":
        q, cfl = classic2.step2(*args, 0, rp, rp)
    else:
        q, cfl = classic2.step2ds(*args, int(c["ids"]), 0, rp, rp)
    ref_q, ref_cfl = c["qout"], float(c["cfl"])
    assert abs(cfl - ref_cfl) <= PARITY_RTOL * ref_cfl
    assert max_rel(q[:, 2:-2, 2:-2], ref_q[:, 2:-2, 2:-2]) <= PARITY_RTOL
