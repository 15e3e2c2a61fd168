"""The variable-coefficient acoustics solver (vc_acoustics_2D, aux = density
and sound speed per cell) on the GPU.

Its transverse solve uses the impedance and sound speed of the cells beside
the cell a fluctuation enters, so the fused step runs the x-interface's
transverse solve one row late (when the row above is on chip); these tests
hold every path to the oracle (itself pinned to the reference's goldens at
3e-16) at 1e-12 relative and run the reference's own example on the device.
"""
import numpy as np
import pytest

from helpers import PARITY_RTOL, max_rel, method_vector, random_qbc
from pyclaw_b200 import _lib, classic2, workloads

pytestmark = pytest.mark.gpu

RP = _lib.RP_VC_ACOUSTICS


def _random_aux(mx, my, seed):
    """auxbc (2, mx+4, my+4): density in [0.5, 4] and sound speed in [0.5, 2.5],
    piecewise constant in four blocks with noise on half the cells (ghost
    cells included: the stateless step uses the caller's ghost values)."""
    rng = np.random.default_rng(seed)
    nx, ny = mx + 4, my + 4
    X, Y = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    block = (X > nx // 3).astype(int) + 2 * (Y > ny // 2).astype(int)
    noise = rng.random((nx, ny)) < 0.5
    rho = np.where(noise, rng.uniform(0.5, 4.0, (nx, ny)), rng.uniform(0.5, 4.0, 4)[block])
    c = np.where(noise, rng.uniform(0.5, 2.5, (nx, ny)), rng.uniform(0.5, 2.5, 4)[block])
    return np.asfortranarray(np.stack([rho, c]))


def _dt(aux, dx, dy, target=0.8):
    return target * min(dx, dy) / np.max(aux[1])


@pytest.mark.parametrize("transverse", [0, 1, 2])
@pytest.mark.parametrize("mx,my", [(1, 1), (3, 5), (37, 23), (130, 70), (257, 9), (9, 300)])
def test_vc_step2_matches_oracle(oracle, transverse, mx, my):
    qbc = random_qbc(_lib.RP_ACOUSTICS, mx, my, seed=mx * 100 + my + transverse)
    aux = _random_aux(mx, my, seed=mx + 7 * my)
    method = method_vector(2, transverse)
    mthlim = np.full(2, 4, dtype=np.intc)
    dx, dy = 1.0 / mx, 1.3 / my
    dt = _dt(aux, dx, dy)
    q_o = qbc.copy(order="F")
    cfl_o = oracle.step2(qbc, q_o, dx, dy, dt, method, mthlim, RP, [], aux=aux)
    q_g, cfl_g = classic2.step2(max(mx, my), 2, mx, my, qbc, qbc.copy(order="F"), aux, dx, dy, dt, method,
                                mthlim, rpn2=RP)
    assert abs(cfl_g - cfl_o) <= PARITY_RTOL * cfl_o
    assert max_rel(q_g[:, 2:-2, 2:-2], q_o[:, 2:-2, 2:-2]) <= PARITY_RTOL


@pytest.mark.parametrize("lim", [0, 1, 3, 5])
@pytest.mark.parametrize("order", [1, 2])
def test_vc_step2_limiters_and_order(oracle, lim, order):
    mx, my = 61, 47
    qbc = random_qbc(_lib.RP_ACOUSTICS, mx, my, seed=17 + lim)
    aux = _random_aux(mx, my, seed=3 + lim)
    method = method_vector(order, 2)
    mthlim = np.array([lim, (lim + 1) % 6], dtype=np.intc)
    dx, dy = 0.02, 0.015
    dt = _dt(aux, dx, dy)
    q_o = qbc.copy(order="F")
    cfl_o = oracle.step2(qbc, q_o, dx, dy, dt, method, mthlim, RP, [], aux=aux)
    q_g, cfl_g = classic2.step2(max(mx, my), 2, mx, my, qbc, qbc.copy(order="F"), aux, dx, dy, dt, method,
                                mthlim, rpn2=RP)
    assert abs(cfl_g - cfl_o) <= PARITY_RTOL * cfl_o
    assert max_rel(q_g[:, 2:-2, 2:-2], q_o[:, 2:-2, 2:-2]) <= PARITY_RTOL


@pytest.mark.parametrize("ids", [1, 2])
def test_vc_step2ds_sweeps_match_oracle(oracle, ids):
    mx, my = 130, 70
    qbc = random_qbc(_lib.RP_ACOUSTICS, mx, my, seed=5 + ids)
    aux = _random_aux(mx, my, seed=9 + ids)
    method = method_vector(2, 0, split=True)
    mthlim = np.full(2, 4, dtype=np.intc)
    dx, dy = 1.0 / mx, 1.0 / my
    dt = _dt(aux, dx, dy)
    q_o = qbc.copy(order="F")
    cfl_o = oracle.step2ds(qbc, q_o, dx, dy, dt, method, mthlim, ids, RP, [], aux=aux)
    q_g, cfl_g = classic2.step2ds(max(mx, my), 2, mx, my, qbc, qbc.copy(order="F"), aux, dx, dy, dt, method,
                                  mthlim, ids=ids, rpn2=RP)
    assert abs(cfl_g - cfl_o) <= PARITY_RTOL * cfl_o
    sl = (slice(None), slice(2, -2), slice(None)) if ids == 1 else (slice(None), slice(2, -2), slice(2, -2))
    assert max_rel(q_g[sl], q_o[sl]) <= PARITY_RTOL


def test_vc_device_run_matches_reference_goldens(goldens):
    # the reference's examples/acoustics_2d_variable on the device-resident path
    claw = workloads.acoustics_variable(n=50)
    claw.run()
    q = claw.frames[20].q
    exp = goldens["acoustics_variable_io_q20"]
    assert np.linalg.norm(exp - q) / np.linalg.norm(exp) < 1e-8  # 8 significant digits in the file
    assert np.max(np.abs(goldens["acoustics_variable_pressure_classic"] - q[0])) < 1e-12


@pytest.mark.parametrize("transverse,variant", [(1, 0), (2, 0), (2, 1), (2, 2), (1, 4), (2, 4)])
def test_vc_device_steps_match_oracle(oracle, transverse, variant):
    # several strips and row blocks; each step of the device patch (aux ghost
    # cells filled on the device from the aux BCs) against the oracle from the
    # same state; variant 2 would stage rows by TMA for other solvers
    from pyclaw_b200 import tune
    claw = workloads.acoustics_variable(n=130, tfinal=1.0)
    claw.solver.transverse_waves = transverse
    tune.set_shape(RP, variant, 12)
    try:
        solver, sol = claw.solver, claw.solution
        solver.setup(sol)
        solver.dt = 0.9 * sol.state.grid.delta[0] / 2.0
        st = sol.state
        dx, dy = st.grid.delta
        mx, my = st.grid.num_cells
        auxbc = np.zeros((2, mx + 4, my + 4), order="F")
        auxbc[:, 2:-2, 2:-2] = st.aux
        oracle.bc_fill_aux(auxbc, solver.aux_bc_lower, solver.aux_bc_upper)
        for _ in range(8):
            q0 = st.get_q_global()
            qbc = np.zeros((3, mx + 4, my + 4), order="F")
            qbc[:, 2:-2, 2:-2] = q0
            oracle.bc_fill(qbc, solver.bc_lower, solver.bc_upper)
            qold = qbc.copy(order="F")
            solver.evolve_to_time(sol)
            cfl_o = oracle.step2(qold, qbc, dx, dy, solver.dt, solver._method, solver._mthlim, RP, [], aux=auxbc)
            if not solver.accept_step:
                continue
            assert max_rel(st.get_q_global(), qbc[:, 2:-2, 2:-2]) <= PARITY_RTOL
            assert abs(solver.cfl.get_cached_max() - cfl_o) <= PARITY_RTOL * cfl_o
    finally:
        tune.set_shape(RP, 0, 0)
