"""Oracle parity at the benchmark configurations themselves.

* Euler Roe 1024^2 (the headline workload): the quadrant problem advanced on
  the device to t = 0.4 exactly as bench.py advances it, then five steps on
  each launch shape the autotuner can pick for it -- 576 tiles at 16 rows,
  more than the CTA slots, so the longest-first tile schedule and its sort
  run -- each step compared with the oracle's step2 on the same state and dt
  (interior cells and the Courant number within 1e-12 relative); and the
  whole run from t = 0 to 0.8 on the device time loop against the oracle's
  host loop (same steps, final state within 1e-8);
* the exact Euler solver at 2048^2 on the same problem's t = 0.4 state, one
  step with the PVRS guess and one with a learned guess, against the oracle;
* the batched form at its benchmark size (512 problems, 100 steps): the
  smallest problem, the largest and one that goes non-finite, each against an
  oracle loop over the same attempts with the reference's dt rule; the failing
  problem must fail at the same attempt in the oracle.
"""
import os

import numpy as np
import pytest

from helpers import PARITY_RTOL, max_rel
from pyclaw_b200 import _lib, workloads

pytestmark = pytest.mark.gpu


def _all_cores(oracle):
    oracle.set_threads(os.cpu_count() or 1)


def _advance(patch, t_end, dt=2.5e-4):
    """bench.py's untimed advance: the reference's dt rule at cfl_desired 0.9,
    rejected attempts retaken.  Returns the last dt."""
    t, cfl = 0.0, None
    while t < t_end:
        dt = min(dt, t_end - t) if cfl is None else min(dt * 0.9 / cfl, t_end - t)
        cfl = patch.step(dt)
        ok = cfl <= 1.0
        patch.accept(ok)
        if ok:
            t += dt
    return dt


def _qbc(oracle, q, bcl, bcu):
    qbc = np.zeros((q.shape[0], q.shape[1] + 4, q.shape[2] + 4), order="F")
    qbc[:, 2:-2, 2:-2] = q
    oracle.bc_fill(qbc, bcl, bcu)
    return qbc


def _download(patch, shape):
    q = np.empty(shape, order="F")
    _lib.check(_lib.load().claw2_patch_download_q(patch.h, _lib.dptr(q)))
    return q


@pytest.fixture(scope="module")
def euler_1024_t04():
    """The headline problem's t = 0.4 state, advanced on the device."""
    claw = workloads.euler_quadrants_unsplit(n=1024)
    s, sol = claw.solver, claw.solution
    s.setup(sol)
    p = s._dev
    _advance(p, 0.4)
    q = _download(p, (4, 1024, 1024))
    p.close()
    return q


SHAPES_1024 = [(3, 16), (2, 16), (3, 18), (0, 16), (1, 16), (4, 16), (0, 8), (8, 16), (8, 12)]


@pytest.mark.parametrize("variant,rows", SHAPES_1024)
def test_headline_euler_1024_steps_match_oracle(oracle, euler_1024_t04, variant, rows):
    from pyclaw_b200 import tune
    claw = workloads.euler_quadrants_unsplit(n=1024)
    s, sol = claw.solver, claw.solution
    sol.state.q = euler_1024_t04
    s.setup(sol)
    p = s._dev
    dx, dy = sol.state.grid.delta
    cp = s.rp.cparam(sol.state.problem_data)
    # bench.py's fixed dt: Courant number 0.9 from a probe step
    dt = 2.5e-4
    c = p.step(dt)
    p.accept(False)
    dt = dt * 0.9 / c
    tune.set_shape(_lib.RP_EULER_ROE, variant, rows)
    _all_cores(oracle)
    try:
        q = euler_1024_t04
        for k in range(5):
            qbc = _qbc(oracle, q, s.bc_lower, s.bc_upper)
            qold = qbc.copy(order="F")
            cfl_o = oracle.step2(qold, qbc, dx, dy, dt, s._method, s._mthlim, _lib.RP_EULER_ROE, cp)
            cfl_g = p.step(dt)
            p.accept(True)
            q = _download(p, (4, 1024, 1024))
            assert abs(cfl_g - cfl_o) <= PARITY_RTOL * cfl_o, (k, cfl_g, cfl_o)
            err = max_rel(q, qbc[:, 2:-2, 2:-2])
            assert err <= PARITY_RTOL, (k, err)
            # continue from the oracle's state, so every step starts from identical data
            q = np.asfortranarray(qbc[:, 2:-2, 2:-2])
            _lib.check(_lib.load().claw2_patch_upload_q(p.h, _lib.dptr(q)))
    finally:
        oracle.set_threads(1)
        tune.set_shape(_lib.RP_EULER_ROE, 0, 0)
        p.close()


def test_exact_euler_2048_step_matches_oracle_with_both_guesses(oracle):
    from pyclaw_b200 import learned, riemann
    n = 2048
    claw = workloads.euler_quadrants_unsplit(n=n)
    s, sol = claw.solver, claw.solution
    s.setup(sol)
    dt = _advance(s._dev, 0.4)
    q_mid = _download(s._dev, (4, n, n))
    s._dev.close()
    net = learned.Network(seed=2024)
    net.generate(1 << 20, seed=7)
    net.train(epochs=2, batch=16384, lr=3e-3)
    dx = dy = 1.0 / n
    results = {}
    for mode in ("pvrs", "learned"):
        ce = workloads.euler_quadrants_unsplit(n=n)
        ce.solver.rp = riemann.euler_exact_2D
        ce.solver.num_waves = 3
        ce.solution.state.q = q_mid
        ce.solver.setup(ce.solution)
        pe = ce.solver._dev
        learned.attach(ce.solver, net if mode == "learned" else None)
        cfl = pe.step(dt)
        pe.accept(True)
        results[mode] = (_download(pe, (4, n, n)), cfl, ce.solver._method, ce.solver._mthlim,
                         ce.solver.bc_lower, ce.solver.bc_upper)
        pe.close()
    _, _, method, mthlim, bcl, bcu = results["pvrs"]
    qbc = _qbc(oracle, q_mid, bcl, bcu)
    q_o = qbc.copy(order="F")
    _all_cores(oracle)
    try:
        cfl_o = oracle.step2(qbc, q_o, dx, dy, dt, method, mthlim, _lib.RP_EULER_EXACT, [1.4, 1e-12])
    finally:
        oracle.set_threads(1)
    for mode, (q, cfl, *_rest) in results.items():
        assert abs(cfl - cfl_o) <= PARITY_RTOL * cfl_o, (mode, cfl, cfl_o)
        err = max_rel(q, q_o[:, 2:-2, 2:-2])
        assert err <= PARITY_RTOL, (mode, err)
    net.close()


def _oracle_batch_loop(oracle, claw, attempts, cfl_desired=0.9, cfl_max=1.0, dt_max=1e99):
    """One problem of the batch on the oracle: per attempt the step from the
    current state and dt, accepted when cfl <= cfl_max, then the reference's
    dt rule (src/pyclaw/solver.py:531-533).  Returns (q, t, accepted,
    rejected, attempt at which the result first went non-finite or None)."""
    s, sol = claw.solver, claw.solution
    s._check_cfl_settings()
    s._set_mthlim()
    s._set_method(sol.state)
    st = sol.state
    dx, dy = st.grid.delta
    cp = s.rp.cparam(st.problem_data)
    q = np.asfortranarray(st.get_q_global().copy())
    dt, t, acc, rej = s.dt_initial, 0.0, 0, 0
    for k in range(attempts):
        qbc = _qbc(oracle, q, s.bc_lower, s.bc_upper)
        qnew = qbc.copy(order="F")
        cfl = oracle.step2(qbc, qnew, dx, dy, dt, s._method, s._mthlim, _lib.RP_EULER_ROE, cp)
        if not np.all(np.isfinite(qnew[:, 2:-2, 2:-2])):
            return q, t, acc, rej, k
        if cfl <= cfl_max:
            q = np.asfortranarray(qnew[:, 2:-2, 2:-2])
            t += dt
            acc += 1
        else:
            rej += 1
        dt = min(dt_max, dt * cfl_desired / cfl) if cfl > 0.0 else dt_max
    return q, t, acc, rej, None


def test_batched_512_instances_match_oracle_runs(oracle):
    from pyclaw_b200.batch import Batch
    claws, sides = workloads.batched_quadrants(512)
    bat = Batch(claws)
    steps = 100
    bat.run(steps, mode=0)
    st = bat.state()
    failed = np.nonzero(st["failed"])[0]
    assert len(failed) > 0  # the benchmark's draw has failing problems
    picks = {"smallest": int(np.argmin(sides)), "largest": int(np.argmax(sides)), "failing": int(failed[0])}
    _all_cores(oracle)
    try:
        for what, i in picks.items():
            fresh, _ = workloads.batched_quadrants(512)
            q_o, t_o, acc, rej, bad = _oracle_batch_loop(oracle, fresh[i], steps)
            q_g = bat.q(i)
            if what == "failing":
                # the device retires the problem at the attempt whose result is
                # non-finite and keeps the state before it; the oracle goes
                # non-finite at the same attempt
                assert bad is not None, (i, acc, rej)
                assert bad == st["nsteps"][i] + st["nreject"][i], (bad, st["nsteps"][i], st["nreject"][i])
            else:
                assert bad is None
            assert acc == st["nsteps"][i] and rej == st["nreject"][i], (what, acc, rej)
            assert abs(t_o - st["t"][i]) <= 1e-12 * max(t_o, 1e-300), (what, t_o, st["t"][i])
            err = max_rel(q_g, q_o)
            assert err <= PARITY_RTOL, (what, i, err)
    finally:
        oracle.set_threads(1)
        bat.close()


def test_headline_euler_1024_whole_run_matches_oracle(oracle):
    # the benchmark problem's whole run, t = 0 to 0.8 (about 1.7k steps,
    # cfl_desired 0.9), on the device time loop against the oracle's host
    # loop over the same dt rule: the same accepted and rejected steps, the
    # same dt to the last steps, and the final state within 1e-8 relative
    # (each step's roundoff-level differences feed the next steps' dt and
    # data through the limiters; measured 3.9e-9 after 1.7k steps)
    claw_g = workloads.euler_quadrants_unsplit(n=1024)
    claw_o = workloads.euler_quadrants_unsplit(oracle.make_solver_class(), n=1024)
    for c in (claw_g, claw_o):
        c.num_output_times = 1
        c.output_format = None
    _all_cores(oracle)
    try:
        claw_o.run()
    finally:
        oracle.set_threads(1)
    claw_g.run()
    sg, so = claw_g.solver.status, claw_o.solver.status
    assert sg['numsteps'] == so['numsteps'] and sg['numsteps'] > 1000
    assert abs(sg['dtmin'] - so['dtmin']) <= 1e-9 * so['dtmin']
    assert abs(sg['cflmax'] - so['cflmax']) <= 1e-9 * so['cflmax']
    qg = claw_g.frames[-1].state.get_q_global()
    qo = claw_o.frames[-1].state.get_q_global()
    assert np.isfinite(qg).all()
    assert max_rel(qg, qo) <= 1e-8
