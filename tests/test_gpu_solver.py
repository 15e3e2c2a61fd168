"""The device-resident path (ghost fill, fused step and CFL on the GPU, q kept
on the device) driven by the package's Controller/Solver loop.

* whole runs of the reference's regression examples against the reference's
  own goldens (the same checks tests/test_oracle_golden.py makes of the oracle);
* step-by-step parity with the oracle on the benchmark problems: from the same
  state, one GPU step (ghost fill + step2 + CFL on the device) and one oracle
  step (ghost fill + step2 on the host) must agree to 1e-12 relative;
* conservation on closed (wall) domains.
"""
import numpy as np
import pytest

from helpers import PARITY_RTOL, max_rel
from pyclaw_b200 import _lib, workloads

pytestmark = pytest.mark.gpu


def _l1(claw, expected, comp=None):
    q = claw.frames[claw.num_output_times].state.get_q_global()
    if comp is not None:
        q = q[comp]
    dx, dy = claw.solution.domain.grid.delta
    return dx * dy * np.sum(np.abs(q.reshape([-1]) - expected))


@pytest.mark.parametrize("key,kw", [
    ("advection_classic_dim_split", dict(dimensional_split=True)),
    ("advection_classic_unsplit_no_trans", dict(dimensional_split=False, transverse_waves=0)),
    ("advection_classic_unsplit_trans_inc", dict(dimensional_split=False, transverse_waves=1)),
    ("advection_classic_unsplit_trans_cor", dict(dimensional_split=False, transverse_waves=2)),
])
def test_cuda_advection_goldens(goldens, key, kw):
    claw = workloads.advection_2d(**kw)
    claw.run()
    err = _l1(claw, goldens[key])
    assert err < 1e-6
    assert err < 1e-12


def test_cuda_acoustics_goldens(goldens):
    claw = workloads.acoustics_2d_homogeneous()
    claw.run()
    exp = goldens["acoustics_verify_classic"]
    rel = np.linalg.norm(exp - claw.frames[-1].q[0]) / np.linalg.norm(exp)
    assert rel < 1e-3


def test_cuda_euler_goldens(goldens):
    claw = workloads.quadrants()
    claw.run()
    err = _l1(claw, goldens["euler_quadrants_roe"], comp=0)
    assert err < 1e-6
    assert err < 1e-11


def test_cuda_shallow_goldens(goldens):
    claw = workloads.radial_dam_break()
    claw.run()
    err = _l1(claw, goldens["shallow_radialdambreak_classic_roe"], comp=0)
    assert err < 1e-5
    assert err < 1e-11


def _stepwise(oracle, claw, nsteps):
    """Advance the GPU solver step by step; before each step run the oracle on
    the same state and dt and compare the results."""
    solver, sol = claw.solver, claw.solution
    solver.setup(sol)
    solver.dt = solver.dt_initial
    st = sol.state
    dx, dy = st.grid.delta
    mx, my = st.grid.num_cells
    cp = solver.rp.cparam(st.problem_data)
    worst = 0.0
    for n in range(nsteps):
        q0 = st.get_q_global()
        qbc = np.zeros((q0.shape[0], mx + 4, my + 4), order="F")
        qbc[:, 2:-2, 2:-2] = q0
        oracle.bc_fill(qbc, solver.bc_lower, solver.bc_upper)
        qold = qbc.copy(order="F")
        solver.evolve_to_time(sol)  # one step (take_one_step)
        dt = solver.dt
        cfl_o = oracle.step2(qold, qbc, dx, dy, dt, solver._method, solver._mthlim, solver.rp.rp_id, cp)
        if not solver.accept_step:
            continue
        q1 = st.get_q_global()
        worst = max(worst, max_rel(q1, qbc[:, 2:-2, 2:-2]))
        assert abs(solver.cfl.get_cached_max() - cfl_o) <= PARITY_RTOL * cfl_o
        assert worst <= PARITY_RTOL, (n, worst)
    return worst


def test_stepwise_acoustics_wall_full_run(oracle):
    # acoustics, 200x200, walls, MC, trans_cor: every step to t = 0.6
    claw = workloads.acoustics_wall(n=200, tfinal=0.6)
    _stepwise(oracle, claw, nsteps=140)


def test_stepwise_euler_quadrants(oracle):
    claw = workloads.euler_quadrants_unsplit(n=160)
    _stepwise(oracle, claw, nsteps=40)


def test_stepwise_euler_on_the_longest_first_schedule(oracle):
    # 640^2 gives 6 strips x 72 row blocks = 432 tiles, more than the 296 CTA
    # slots, so the step kernel runs on the measured-cost tile schedule (sorted
    # after the first step and every fourth step); results must not depend on it
    import os
    from pyclaw_b200 import tune
    tune.set_shape(_lib.RP_EULER_ROE, 0, 0)  # the heuristic row height (9 rows here)
    oracle.set_threads(os.cpu_count() or 1)
    claw = workloads.euler_quadrants_unsplit(n=640)
    _stepwise(oracle, claw, nsteps=7)
    oracle.set_threads(1)


def test_stepwise_shallow_dam_break(oracle):
    claw = workloads.shallow_dam_break_unsplit(n=192)
    _stepwise(oracle, claw, nsteps=30)


def test_acoustics_wall_conserves_pressure_sum():
    claw = workloads.acoustics_wall(n=200, tfinal=0.6)
    p0 = claw.solution.state.get_q_global()[0].sum()
    scale = np.abs(claw.solution.state.get_q_global()[0]).sum()
    claw.run()
    p1 = claw.frames[-1].q[0].sum()
    assert abs(p1 - p0) <= 1e-13 * scale


def test_whole_run_acoustics_matches_oracle(oracle):
    claw_g = workloads.acoustics_wall(n=200, tfinal=0.6)
    claw_g.run()
    claw_o = workloads.acoustics_wall(oracle.make_solver_class(), n=200, tfinal=0.6)
    claw_o.run()
    assert claw_g.solver.status['numsteps'] == claw_o.solver.status['numsteps']
    assert max_rel(claw_g.frames[-1].q, claw_o.frames[-1].q) <= 1e-11


def test_reject_and_retake_on_device():
    # a first dt far above the CFL limit must be rejected and retaken
    claw = workloads.acoustics_wall(n=64, tfinal=0.05)
    claw.solver.dt_initial = 1.0
    q0 = claw.solution.state.get_q_global()
    claw.solver.setup(claw.solution)
    claw.solver.dt = claw.solver.dt_initial
    claw.solver.evolve_to_time(claw.solution)
    assert not claw.solver.accept_step
    assert np.array_equal(claw.solution.state.get_q_global(), q0)
    assert claw.solution.t == 0.0
    claw.solver.evolve_to_time(claw.solution)
    assert claw.solver.accept_step and claw.solution.t > 0.0


def _sums(claw):
    q = claw.solution.state.get_q_global()
    return q.sum(axis=(1, 2)), np.abs(q).sum(axis=(1, 2))


def test_euler_periodic_run_conserves_every_component():
    # the quadrant problem on a periodic domain: mass, both momenta and energy
    # stay at their initial sums to roundoff over a whole run
    from pyclaw_b200 import BC
    claw = workloads.euler_quadrants_unsplit(n=256, tfinal=0.3)
    for d in (0, 1):
        claw.solver.bc_lower[d] = BC.periodic
        claw.solver.bc_upper[d] = BC.periodic
    s0, scale = _sums(claw)
    claw.run()
    assert claw.solver.status['numsteps'] > 50
    q1 = claw.frames[-1].q
    assert np.all(np.abs(q1.sum(axis=(1, 2)) - s0) <= 1e-13 * scale)


def test_shallow_dam_break_conserves_mass():
    # the front stays inside the domain, so the extrapolation boundaries carry no flux
    claw = workloads.shallow_dam_break_unsplit(n=256, tfinal=0.5)
    s0, scale = _sums(claw)
    claw.run()
    h1 = claw.frames[-1].q[0].sum()
    assert abs(h1 - s0[0]) <= 1e-13 * scale[0]


def test_whole_run_euler_quadrants_matches_oracle(oracle):
    # the benchmark's Euler problem at 256^2 run to its final time t = 0.8
    # (543 steps) on both paths; per-step differences are ~1e-16, so the
    # whole-run difference measures their growth through a nonlinear run.
    import os
    oracle.set_threads(os.cpu_count() or 1)
    claw_g = workloads.euler_quadrants_unsplit(n=256, tfinal=0.8)
    claw_g.num_output_times = 1
    claw_g.run()
    claw_o = workloads.euler_quadrants_unsplit(oracle.make_solver_class(), n=256, tfinal=0.8)
    claw_o.num_output_times = 1
    claw_o.run()
    oracle.set_threads(1)
    assert claw_g.solver.status['numsteps'] == claw_o.solver.status['numsteps']
    qg, qo = claw_g.frames[-1].q, claw_o.frames[-1].q
    diff = max_rel(qg, qo)
    # the data are symmetric about x = y (with u <-> v); so is the result
    qt = np.transpose(qg, (0, 2, 1)).copy()
    qt[[1, 2]] = qt[[2, 1]]
    sym = max_rel(qt, qg)
    print("whole-run max rel diff %.3e, diagonal symmetry %.3e" % (diff, sym))
    assert diff <= 1e-9
    assert sym <= 1e-9


def test_run_host_equals_one_call_per_step():
    # claw2_patch_run_host (overlapped host-to-host steps) gives, step for
    # step, the same result and CFL as upload + step + accept + download
    claw = workloads.euler_quadrants_unsplit(n=96, tfinal=0.1)
    s, sol = claw.solver, claw.solution
    s.setup(sol)
    p = s._dev
    rng = np.random.default_rng(3)
    q0 = sol.state.get_q_global()
    qs = [np.asfortranarray(q0 * (1.0 + 0.01 * rng.random(q0.shape))) for _ in range(3)]
    dts = [2e-4, 3e-4, 1e-4]
    ref, cref = [], []
    for q, dt in zip(qs, dts):
        sol.state.q = q
        p.push(sol.state)
        cref.append(p.step(dt))
        p.accept(True)
        out = np.empty(q.shape, order="F")
        _lib.check(p._lib.claw2_patch_download_q(p.h, _lib.dptr(out)))
        ref.append(out)
    outs = [np.empty(q.shape, order="F") for q in qs]
    cfl = p.run_host(qs, outs, dts)
    for a, b in zip(outs, ref):
        assert np.array_equal(a, b)
    assert list(cfl) == cref
    # the patch holds the last result
    assert np.array_equal(sol.state.get_q_global(), ref[-1])


@pytest.mark.parametrize("variant", [2, 3, 4])
@pytest.mark.parametrize("name,n", [("euler", 130), ("shallow", 70), ("acoustics", 257), ("advection", 131)])
def test_tma_row_staging_matches_oracle(oracle, variant, name, n):
    # launch variants 2 and 3 stage every row of a strip by TMA (tensor map of
    # the q planes, mbarrier completion); sizes with a ragged last strip, whose
    # columns past the grid the copy fills with zeros; variant 4 is the
    # two-barrier tile (x-interfaces finished one row late)
    from pyclaw_b200 import tune
    make = {"euler": lambda: workloads.euler_quadrants_unsplit(n=n),
            "shallow": lambda: workloads.shallow_dam_break_unsplit(n=n),
            "acoustics": lambda: workloads.acoustics_wall(n=n),
            "advection": lambda: workloads.advection_2d(dimensional_split=False, transverse_waves=2, mx=n, my=n - 37)}
    claw = make[name]()
    rp = claw.solver.rp.rp_id
    tune.set_shape(rp, variant, 12)
    try:
        _stepwise(oracle, claw, nsteps=4)
    finally:
        tune.set_shape(rp, 0, 0)


def test_largest_benchmark_size_one_step_matches_oracle(oracle):
    # the shallow-water benchmark size, 4096 x 4096 (50 M unknowns): one unsplit
    # step through the stateless entry point against the oracle on all cores
    import os
    from helpers import method_vector, random_qbc, set_cparam
    from pyclaw_b200 import classic2
    mx = my = 4096
    rp = _lib.RP_SHALLOW_ROE
    qbc = random_qbc(rp, mx, my, seed=4096)
    method = method_vector(2, 2)
    mthlim = np.full(3, 4, dtype=np.intc)
    dx = dy = 1.0 / mx
    dt = 0.2 * dx
    oracle.set_threads(os.cpu_count() or 1)
    try:
        q_o = qbc.copy(order="F")
        cfl_o = oracle.step2(qbc, q_o, dx, dy, dt, method, mthlim, rp, [1.0, 1.0])
    finally:
        oracle.set_threads(1)
    set_cparam(classic2, rp)
    q_g, cfl_g = classic2.step2(mx, 2, mx, my, qbc, qbc.copy(order="F"), None, dx, dy, dt, method, mthlim,
                                rpn2=rp)
    assert abs(cfl_g - cfl_o) <= PARITY_RTOL * cfl_o
    assert max_rel(q_g[:, 2:-2, 2:-2], q_o[:, 2:-2, 2:-2]) <= PARITY_RTOL


def test_run_host_after_the_tile_schedule_grows():
    # a step on a finer tiling (more tiles than the schedule arrays held)
    # reallocates only the schedule; the host pipeline set up by an earlier
    # claw2_patch_run_host stays valid for the next one
    from pyclaw_b200 import tune
    claw = workloads.euler_quadrants_unsplit(n=640, tfinal=0.1)
    s, sol = claw.solver, claw.solution
    s.setup(sol)
    p = s._dev
    rng = np.random.default_rng(5)
    q0 = sol.state.get_q_global()
    qs = [np.asfortranarray(q0 * (1.0 + 0.01 * rng.random(q0.shape))) for _ in range(2)]
    dts = [2e-4, 1e-4]
    tune.set_shape(_lib.RP_EULER_ROE, 0, 0)
    try:
        outs = [np.empty(q.shape, order="F") for q in qs]
        p.run_host(qs, outs, dts)           # reserves the pipeline; ~432 tiles
        tune.set_shape(_lib.RP_EULER_ROE, 0, 2)
        p.step(1e-4, want_cfl=False)        # 6 strips x 320 row blocks: the schedule grows
        p.accept(False)
        outs2 = [np.empty(q.shape, order="F") for q in qs]
        cfl2 = p.run_host(qs, outs2, dts)
        ref, cref = [], []
        for q, dt in zip(qs, dts):
            sol.state.q = q
            p.push(sol.state)
            cref.append(p.step(dt))
            p.accept(True)
            out = np.empty(q.shape, order="F")
            _lib.check(p._lib.claw2_patch_download_q(p.h, _lib.dptr(out)))
            ref.append(out)
    finally:
        tune.set_shape(_lib.RP_EULER_ROE, 0, 0)
    for a, b in zip(outs2, ref):
        assert np.array_equal(a, b)
    assert list(cfl2) == cref
