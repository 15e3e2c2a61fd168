"""Host-side logic of the drop-in, on CPU: geometry and State layout, the
solver's attribute rules and method vectors, the dt/accept/reject loop (driven
with the oracle as the step), and the loud failure of the CUDA path without a
GPU (there is no CPU fallback)."""
import numpy as np
import pytest

import pyclaw_b200 as pyclaw
from conftest import cuda_available
from pyclaw_b200 import riemann, workloads


def test_dimension_matches_reference_docstring():
    # geometry.py:497-516
    x = pyclaw.Dimension(0., 1., 100, name='x')
    assert x.num_cells == 100 and x.delta == 0.01
    assert x.nodes[0] == 0.0 and x.nodes[1] == 0.01 and x.nodes[-1] == 1.0
    assert x.centers[-1] == 0.995 and len(x.centers) == 100 and len(x.nodes) == 101


def test_domain_and_state_layout():
    domain = pyclaw.Domain((0., 0.), (1., 1.), (100, 100))
    assert domain.num_dim == 2 and domain.grid.num_cells == [100, 100]
    st = pyclaw.State(pyclaw.Domain([pyclaw.Dimension(0, 1, 4), pyclaw.Dimension(0, 1, 4)]), 3)
    assert st.q.shape == (3, 4, 4) and st.q.flags['F_CONTIGUOUS']
    X, Y = st.grid.p_centers
    assert X.shape == (4, 4) and X[1, 0] > X[0, 0] and Y[0, 1] > Y[0, 0]


def test_solver_defaults_and_attribute_guard():
    s = pyclaw.ClawSolver2D(riemann.euler_4wave_2D)
    assert s.dimensional_split is True and s.transverse_waves == 1 and s.limiters == 1
    assert s.cfl_max == 1.0 and s.cfl_desired == 0.9 and s.num_ghost == 2 and s.dt_initial == 0.1
    assert s.num_eqn == 4 and s.num_waves == 4 and s.fwave is False
    assert s.kernel_language == 'CUDA'
    with pytest.raises(TypeError):
        s.no_such_option = 1


def test_mthlim_and_method_vectors():
    s = pyclaw.ClawSolver2D(riemann.euler_4wave_2D)
    s.limiters = pyclaw.limiters.tvd.MC
    s._set_mthlim()
    assert s._mthlim == [4, 4, 4, 4]
    s.limiters = [1, 2]
    with pytest.raises(Exception):
        s._set_mthlim()
    st = pyclaw.State(pyclaw.Domain((0, 0), (1, 1), (4, 4)), 4)
    s.dimensional_split = False
    s.transverse_waves = 2
    s._set_method(st)
    assert list(s._method) == [1, 2, 2, 0, 0, 0, 0]
    s.dimensional_split = True
    s._set_method(st)
    assert s._method[2] == -1


def test_get_dt_rules():
    s = pyclaw.ClawSolver2D(riemann.acoustics_2D)
    s.dt = 0.1
    s.cfl.set_global_max(0.45)
    s.get_dt(0.0, 0.0, 1.0, False)   # first call only records dt_old
    assert s.dt == 0.1
    s.get_dt(0.0, 0.0, 1.0, False)   # dt <- dt * cfl_desired / cfl
    assert s.dt == pytest.approx(0.1 * 0.9 / 0.45)
    s.cfl.set_global_max(0.9)
    s.get_dt(0.95, 0.0, 1.0, False)  # clipped to tend
    assert s.dt == pytest.approx(0.05)


def test_riemann_cparam_requires_problem_data():
    with pytest.raises(Exception):
        riemann.acoustics_2D.cparam({'rho': 1.0})
    assert riemann.euler_4wave_2D.cparam({'gamma': 1.4}) == [1.4, 1.0]
    assert riemann.euler_4wave_2D.cparam({'gamma': 1.4, 'efix': False}) == [1.4, 0.0]


def test_reject_and_retake_with_oracle(oracle):
    claw = workloads.acoustics_wall(oracle.make_solver_class(), n=32, tfinal=0.05)
    s, sol = claw.solver, claw.solution
    s.dt_initial = 1.0
    q0 = sol.state.get_q_global()
    s.setup(sol)
    s.dt = s.dt_initial
    s.evolve_to_time(sol)
    assert not s.accept_step and sol.t == 0.0
    assert np.array_equal(sol.state.get_q_global(), q0)
    s.evolve_to_time(sol)
    assert s.accept_step and sol.t > 0.0


def test_fixed_dt_must_divide_interval(oracle):
    claw = workloads.acoustics_wall(oracle.make_solver_class(), n=16, tfinal=0.05)
    s, sol = claw.solver, claw.solution
    s.dt_variable = False
    s.setup(sol)
    s.dt = 0.003
    with pytest.raises(Exception, match="divide"):
        s.evolve_to_time(sol, 0.01)


def test_fixed_dt_cfl_violation_raises(oracle):
    claw = workloads.acoustics_wall(oracle.make_solver_class(), n=16, tfinal=0.05)
    s, sol = claw.solver, claw.solution
    s.dt_variable = False
    s.setup(sol)
    s.dt = 0.1  # CFL = 0.1 * 2 / 0.125 = 1.6
    with pytest.raises(pyclaw.CFLError):
        s.evolve_to_time(sol, 0.1)


def test_controller_frames_and_times(oracle):
    claw = workloads.acoustics_wall(oracle.make_solver_class(), n=24, tfinal=0.1)
    claw.num_output_times = 4
    claw.run()
    assert len(claw.frames) == 5
    assert [f.t for f in claw.frames] == pytest.approx(list(np.linspace(0, 0.1, 5)))


@pytest.mark.skipif(cuda_available(), reason="checks the behaviour without a GPU")
def test_cuda_path_fails_loudly_without_gpu():
    from pyclaw_b200 import _lib
    claw = workloads.acoustics_wall(n=16, tfinal=0.01)
    with pytest.raises(_lib.Claw2Error):
        claw.run()


def test_host_auxbc_fill_matches_oracle(oracle):
    # the product's host fill of auxbc for custom aux BCs (dimension by
    # dimension, user function or built-in rule) against the oracle's
    # restatement of Solver._apply_bcs, on the annulus (custom in r, periodic in
    # theta) and on every built-in pair with a custom lower side in y
    import numpy as np
    from pyclaw_b200 import hostbc as auxbc, workloads
    from pyclaw_b200.solver import BC
    claw = workloads.advection_annulus(m_r=12, m_theta=20)
    solver, state = claw.solver, claw.solution.state
    a = auxbc.fill_auxbc(solver, state, np.zeros((3, 16, 24), order='F'))
    b = oracle.apply_aux_bcs(solver, state, np.zeros((3, 16, 24), order='F'))
    assert np.array_equal(a, b)
    # the ghost cells in r are the geometric values of the cells beyond the annulus
    dx, dy = state.grid.delta
    xn, yn = state.grid.p_nodes_with_ghost(2)
    full = workloads.annulus_edge_aux(xn, yn, dx, dy)
    assert np.allclose(a[:, :2, 2:-2], full[:, :2, 2:-2], rtol=0, atol=1e-14)

    def lower_y(st, dim, t, qbc, aux, ng):
        aux[:, :, :ng] = 7.0 + t

    rng = np.random.default_rng(3)
    state.aux = np.asfortranarray(rng.random((3, 12, 20)))
    solver.user_aux_bc_lower = lower_y
    solver.aux_bc_lower[1] = BC.custom
    for kind in (BC.extrap, BC.wall):
        solver.aux_bc_upper[1] = kind
        solver.aux_bc_lower[0] = kind
        solver.aux_bc_upper[0] = BC.periodic if kind == BC.extrap else BC.wall
        a = auxbc.fill_auxbc(solver, state, np.zeros((3, 16, 24), order='F'))
        b = oracle.apply_aux_bcs(solver, state, np.zeros((3, 16, 24), order='F'))
        assert np.array_equal(a, b)
        assert np.all(a[:, :, :2] == 7.0)


def test_gauges_and_functional_files(oracle, tmp_path):
    # the host loop's gauges (Grid.add_gauges / setup_gauge_files,
    # Solver.write_gauge_values) and the F functional file on the oracle's
    # p-system run: one row per accepted step plus the initial one, files equal
    # to the in-memory data, gauges outside the grid dropped
    import numpy as np
    from pyclaw_b200 import workloads
    claw = workloads.psystem(oracle.make_solver_class(), outdir=str(tmp_path))
    grid = claw.solution.state.grid
    assert grid.gauges == [[0, 0], [105, 6], [18, 111], [69, 69]]
    grid2 = workloads.psystem(oracle.make_solver_class(), outdir=str(tmp_path / "x")).solution.state.grid
    grid2.add_gauges([[30.0, 1.0], [0.0, 1.0]])
    assert len(grid2.gauges) == 4
    claw.run()
    st = claw.solution.state
    n = claw.solver.status['numsteps'] + 1
    for k, f in enumerate(grid.gauge_files):
        assert f.closed
        data = np.loadtxt(f.name)
        assert data.shape == (n, 3) and np.array_equal(data, st.gauge_data[k])
    assert np.allclose(st.gauge_data[0][:, 2], 10 * st.gauge_data[0][:, 1])
    F = np.loadtxt(str(tmp_path / "F.txt"))
    assert F.shape == (11, 2) and np.all(F[:, 1] > 0)


def test_device_time_loop_only_without_host_callbacks():
    # evolve_to_time runs on the GPU only when nothing needs the host between
    # steps; each host callback of the reference's loop sends it back to the
    # host loop (the predicate needs no GPU)
    from pyclaw_b200 import BC, workloads
    from pyclaw_b200.classic import ClawSolver2D

    def fresh():
        claw = workloads.euler_quadrants_unsplit(n=16, tfinal=0.1)
        return claw.solver, claw.solution

    s, sol = fresh()
    assert s._device_loop_ok(sol, 0.1)
    assert not s._device_loop_ok(sol, None)          # take_one_step form
    s.device_time_loop = False
    assert not s._device_loop_ok(sol, 0.1)

    s, sol = fresh()
    s.before_step = lambda solver, state: None
    assert not s._device_loop_ok(sol, 0.1)
    s, sol = fresh()
    s.step_source = lambda solver, state, dt: None
    assert not s._device_loop_ok(sol, 0.1)
    s, sol = fresh()
    sol.state.grid.add_gauges([(0.5, 0.5)])
    assert not s._device_loop_ok(sol, 0.1)
    s, sol = fresh()
    s.bc_lower[1] = BC.custom
    s.user_bc_lower = lambda *a: None
    assert not s._device_loop_ok(sol, 0.1)

    # a subclass that replaces a stepping method keeps the host loop
    class Sub(ClawSolver2D):
        def step_hyperbolic(self, solution):
            return super().step_hyperbolic(solution)
    s, sol = fresh()
    sub = Sub(s.rp)
    assert sub.rp is s.rp
    assert not sub._device_loop_ok(sol, 0.1)
    assert ClawSolver2D(s.rp)._device_loop_ok(sol, 0.1)
