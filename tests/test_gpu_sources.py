"""Source steps (step_source, Godunov and Strang splitting) and the
advection-reaction example's vector advection solver on the GPU.

With a source step the hyperbolic result is committed on the device first and
the source acts on it: a host function through state.q (downloaded, edited,
uploaded before the next step), a LinearSource on the device without leaving
it; a rejected step restores q from before the step's hooks, as the
reference's q_backup does.  Held to the oracle at 1e-12 and to the reference's
advection-reaction golden.
"""
import numpy as np
import pytest

from helpers import PARITY_RTOL, max_rel, method_vector
from pyclaw_b200 import _lib, classic2, workloads
from pyclaw_b200.sources import LinearSource

pytestmark = pytest.mark.gpu

VEC = _lib.RP_VC_ADVECTION_VEC


def _vec_data(mx, my, seed):
    rng = np.random.default_rng(seed)
    nx, ny = mx + 4, my + 4
    q = np.asfortranarray(rng.uniform(0.0, 1.0, (2, nx, ny)))
    aux = np.asfortranarray(rng.uniform(-1.2, 1.2, (2, nx, ny)))
    return q, aux


@pytest.mark.parametrize("mx,my", [(1, 1), (37, 23), (257, 70)])
def test_vector_advection_step2_no_transverse(oracle, mx, my):
    qbc, aux = _vec_data(mx, my, mx + my)
    method = method_vector(2, 0)
    mthlim = np.full(1, 1, dtype=np.intc)
    dx, dy = 1.0 / mx, 1.0 / my
    dt = 0.4 * min(dx, dy)
    q_o = qbc.copy(order="F")
    cfl_o = oracle.step2(qbc, q_o, dx, dy, dt, method, mthlim, VEC, [], aux=aux)
    q_g, cfl_g = classic2.step2(max(mx, my), 2, mx, my, qbc, qbc.copy(order="F"), aux, dx, dy, dt, method,
                                mthlim, rpn2=VEC)
    assert abs(cfl_g - cfl_o) <= PARITY_RTOL * cfl_o
    assert max_rel(q_g[:, 2:-2, 2:-2], q_o[:, 2:-2, 2:-2]) <= PARITY_RTOL


@pytest.mark.parametrize("ids", [1, 2])
def test_vector_advection_step2ds(oracle, ids):
    mx, my = 130, 70
    qbc, aux = _vec_data(mx, my, 5 + ids)
    method = method_vector(2, 0, split=True)
    mthlim = np.full(1, 4, dtype=np.intc)
    dx, dy = 1.0 / mx, 1.0 / my
    dt = 0.8 * min(dx, dy) / 1.2
    q_o = qbc.copy(order="F")
    cfl_o = oracle.step2ds(qbc, q_o, dx, dy, dt, method, mthlim, ids, VEC, [], aux=aux)
    q_g, cfl_g = classic2.step2ds(max(mx, my), 2, mx, my, qbc, qbc.copy(order="F"), aux, dx, dy, dt, method,
                                  mthlim, ids=ids, rpn2=VEC)
    assert abs(cfl_g - cfl_o) <= PARITY_RTOL * cfl_o
    sl = (slice(None), slice(2, -2), slice(None)) if ids == 1 else (slice(None), slice(2, -2), slice(2, -2))
    assert max_rel(q_g[sl], q_o[sl]) <= PARITY_RTOL


def test_vector_advection_rejects_transverse():
    qbc, aux = _vec_data(8, 8, 1)
    with pytest.raises(_lib.Claw2Error):
        classic2.step2(8, 2, 8, 8, qbc, qbc.copy(order="F"), aux, 0.1, 0.1, 0.01, method_vector(2, 1),
                       np.full(1, 1, dtype=np.intc), rpn2=VEC)


@pytest.mark.parametrize("device_source", [False, True])
def test_advection_reaction_device_run(oracle, goldens, device_source):
    # the reference's example on the device: before-step velocities (aux
    # re-uploaded every step), source as the host function or on the device
    claw = workloads.advection_reaction(device_source=device_source)
    claw.run()
    q = claw.solution.state.get_q_global()
    exp = goldens["advection_reaction_density"]
    assert np.linalg.norm(exp - q[0]) / np.linalg.norm(exp) < 1e-12
    ref = workloads.advection_reaction(oracle.make_solver_class(), tfinal=1.0, num_output_times=4)
    dev = workloads.advection_reaction(device_source=device_source, tfinal=1.0, num_output_times=4)
    ref.run()
    dev.run()
    for a, b in zip(dev.frames, ref.frames):
        assert max_rel(a.q, b.q) <= 1e-12


def test_host_and_device_source_agree_bitwise():
    a = workloads.advection_reaction(device_source=False, n=64, tfinal=0.5, num_output_times=2)
    b = workloads.advection_reaction(device_source=True, n=64, tfinal=0.5, num_output_times=2)
    a.run()
    b.run()
    assert np.array_equal(a.solution.state.get_q_global(), b.solution.state.get_q_global())


def test_linear_source_kernel_matches_numpy():
    claw = workloads.euler_quadrants_unsplit(n=96, tfinal=0.01)
    solver, sol = claw.solver, claw.solution
    solver.setup(sol)
    st = sol.state
    q0 = st.get_q_global()
    M = np.array([[0.0, 0.3, 0.0, -0.1], [0.2, 0.0, 0.0, 0.0], [0.0, 0.0, -1.5, 0.0], [0.1, 0.0, 0.4, 0.0]])
    LinearSource(M)(solver, st, 0.05)   # on the device (the device copy is current)
    got = st.get_q_global()
    exp = q0.copy()
    for i in range(4):
        for k in range(4):
            if M[i, k] != 0.0:
                exp[i] = exp[i] + (M[i, k] * 0.05) * q0[k]
    assert np.array_equal(got, exp)


@pytest.mark.parametrize("split", [1, 2])
def test_source_step_reject_and_retake(oracle, split):
    # a first dt far above the CFL limit: the step is rejected, q restored
    # from before the hooks, and retaken; Godunov and Strang splitting
    runs = []
    for cls in (None, oracle.make_solver_class()):
        claw = workloads.advection_reaction(cls, n=80, tfinal=0.3, num_output_times=1,
                                            device_source=cls is None)
        claw.solver.source_split = split
        claw.solver.dt_initial = 0.5
        claw.run()
        runs.append(claw)
    g, o = runs
    assert g.solver.status['numsteps'] == o.solver.status['numsteps']
    assert max_rel(g.solution.state.get_q_global(), o.solution.state.get_q_global()) <= 1e-12
