"""Exact Euler solver and its learned Newton guess on the GPU.

* the CUDA exact-solver step equals the oracle's (Toro restated
  independently) within 1e-12, from the PVRS guess and from a learned guess
  (Newton converges to the same p* from either start);
* the device's training-sample generator, gradient kernels and BF16 tensor-
  core inference against the FP64 CPU reference of the network;
* training lowers the loss and the trained guess needs fewer Newton updates
  than the PVRS guess on problems from the training distribution.
"""
import numpy as np
import pytest

from helpers import PARITY_RTOL, max_rel, method_vector
from oracle import mlp_ref
from pyclaw_b200 import _lib, classic2, learned, workloads
from pyclaw_b200 import riemann as rmod

pytestmark = pytest.mark.gpu
G = 1.4


def _euler_qbc(mx, my, seed, spread=0.6):
    rng = np.random.default_rng(seed)
    nx, ny = mx + 4, my + 4
    X, Y = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    quad = (X > nx // 2).astype(int) + 2 * (Y > ny // 3).astype(int)
    noise = rng.random((nx, ny)) < 0.5

    def field(lo, hi):
        return np.where(noise, rng.uniform(lo, hi, (nx, ny)), rng.uniform(lo, hi, 4)[quad])

    rho, p = np.exp(field(-spread, spread)), np.exp(field(-spread, spread))
    u, v = field(-0.5, 0.5), field(-0.5, 0.5)
    return np.asfortranarray(np.stack([rho, rho * u, rho * v, p / (G - 1) + 0.5 * rho * (u * u + v * v)]))


def test_exact_step_matches_oracle(oracle):
    for (mx, my, seed) in [(37, 23, 1), (130, 70, 2)]:
        qbc = _euler_qbc(mx, my, seed)
        method = method_vector(2, 2)
        mthlim = np.full(3, 4, dtype=np.intc)
        dx, dy, dt = 1.0 / mx, 1.0 / my, 0.1 / max(mx, my)
        q_o = qbc.copy(order="F")
        cfl_o = oracle.step2(qbc, q_o, dx, dy, dt, method, mthlim, _lib.RP_EULER_EXACT, [G, 1e-12])
        classic2.cparam.gamma = G
        q_g, cfl_g = classic2.step2(max(mx, my), 2, mx, my, qbc, qbc.copy(order="F"), None, dx, dy, dt, method,
                                    mthlim, rpn2=rmod.euler_exact_2D)
        assert abs(cfl_g - cfl_o) <= PARITY_RTOL * cfl_o
        assert max_rel(q_g[:, 2:-2, 2:-2], q_o[:, 2:-2, 2:-2]) <= PARITY_RTOL


@pytest.mark.parametrize("variant,rows", [(2, 12), (3, 32), (1, 7), (8, 16)])
def test_exact_step_matches_oracle_every_launch_shape(oracle, variant, rows):
    # the shapes the autotuner picks for the exact solver (rows staged by TMA,
    # 2 or 3 CTAs per SM) and the others, against the oracle
    from pyclaw_b200 import tune
    mx, my = 150, 97
    qbc = _euler_qbc(mx, my, seed=variant + 3)
    method = method_vector(2, 2)
    mthlim = np.full(3, 4, dtype=np.intc)
    dx, dy, dt = 1.0 / mx, 1.0 / my, 0.1 / max(mx, my)
    q_o = qbc.copy(order="F")
    cfl_o = oracle.step2(qbc, q_o, dx, dy, dt, method, mthlim, _lib.RP_EULER_EXACT, [G, 1e-12])
    classic2.cparam.gamma = G
    tune.set_shape(_lib.RP_EULER_EXACT, variant, rows)
    try:
        q_g, cfl_g = classic2.step2(max(mx, my), 2, mx, my, qbc, qbc.copy(order="F"), None, dx, dy, dt, method,
                                    mthlim, rpn2=rmod.euler_exact_2D)
    finally:
        tune.set_shape(_lib.RP_EULER_EXACT, 0, 0)
    assert abs(cfl_g - cfl_o) <= PARITY_RTOL * cfl_o
    assert max_rel(q_g[:, 2:-2, 2:-2], q_o[:, 2:-2, 2:-2]) <= PARITY_RTOL


def _exact_claw(n):
    claw = workloads.euler_quadrants_unsplit(n=n)
    claw.solver.rp = rmod.euler_exact_2D
    claw.solver.num_waves = 3
    return claw


def test_learned_guess_converges_to_the_same_step(oracle):
    net = learned.Network(seed=11)  # untrained: a poor but finite guess
    results = []
    for use_net in (False, True):
        claw = _exact_claw(96)
        s, sol = claw.solver, claw.solution
        s.setup(sol)
        s.dt = 2e-4
        if use_net:
            learned.attach(s, net)
        for _ in range(3):
            s.evolve_to_time(sol)
        it, ns = learned.counters(s)
        results.append((sol.state.get_q_global(), it, ns))
    (q0, it0, n0), (q1, it1, n1) = results
    assert n0 == n1 > 0
    assert max_rel(q1, q0) <= PARITY_RTOL


def test_sample_generator_matches_reference():
    net = learned.Network()
    net.generate(64, seed=99)
    x, y, ok = net.samples(0, 64)
    for i in range(64):
        rl, ul, pl, rr, ur, pr = mlp_ref.draw_problem(99, i)
        f, w = mlp_ref.features(G, rl, ul, pl, rr, ur, pr)
        assert np.allclose(x[i, :6], f, rtol=1e-6, atol=1e-6)
        assert abs(x[i, 6] - w) <= 1e-6


def test_gradient_kernel_matches_fp64_reference():
    net = learned.Network(seed=5)
    net.generate(4096, seed=3)
    x, y, ok = net.samples(0, 4096)
    P = net.params
    g_gpu, loss_gpu = net.gradient(0, 4096)
    sel = ok.astype(bool)
    # the device averages over all 4096 slots with zero error on invalid ones
    g_ref, _ = mlp_ref.gradient(P, x[sel, :6].astype(np.float64), y[sel].astype(np.float64))
    g_ref *= sel.sum() / 4096.0
    rel = np.linalg.norm(g_gpu - g_ref) / np.linalg.norm(g_ref)
    assert rel < 1e-4, rel


@pytest.mark.parametrize("engine", ["tcgen05", "mma.sync"])
@pytest.mark.parametrize("n", [1000, 256, 1, 70001])
def test_tensor_core_inference_matches_reference(engine, n):
    """BF16 operands, FP32 accumulation, on either tensor-core path: against
    the same rounding in numpy and against the FP64 network.  The sizes cover
    a partial tile pair, one row, and more tile pairs than resident CTAs."""
    net = learned.Network(seed=7)
    net.set_engine(engine)
    rng = np.random.default_rng(1)
    x = np.zeros((n, 8), dtype=np.float32)
    x[:, :6] = rng.normal(0, 1.0, (n, 6))
    y_gpu = net.infer(x)
    y_ref = mlp_ref.forward_bf16(net.params, x[:, :6])
    y_fp64, _, _ = mlp_ref.forward(net.params, x[:, :6].astype(np.float64))
    assert np.max(np.abs(y_gpu - y_ref)) < 2e-2
    assert np.max(np.abs(y_gpu - y_fp64)) < 5e-2


def test_tcgen05_and_mma_sync_inference_agree():
    """The two tensor-core paths round the same operands to BF16; they differ
    only in the order of the FP32 sums and where the bias is added."""
    net = learned.Network(seed=3)
    rng = np.random.default_rng(2)
    x = np.zeros((5000, 8), dtype=np.float32)
    x[:, :6] = rng.normal(0, 1.5, (5000, 6))
    ys = {}
    for engine in ("tcgen05", "mma.sync"):
        net.set_engine(engine)
        ys[engine] = net.infer(x)
        ys[engine + "2"] = net.infer(x)  # a second call on the same CTAs' barriers and TMEM
    assert np.array_equal(ys["tcgen05"], ys["tcgen052"])
    assert np.max(np.abs(ys["tcgen05"] - ys["mma.sync"])) < 5e-3


def test_training_reduces_loss_and_guess_error():
    """What the trained network gains over the method without it: on held-out
    problems of the training distribution its guess (BF16 tensor-core
    inference) is closer to the converged p* than the adaptive PVRS guess,
    above all in the tail where PVRS is poor."""
    net = learned.Network(seed=2024)
    net.generate(1 << 24, seed=7)  # the full training set (about a second with training)
    _, loss0 = net.gradient(0, 1 << 16)
    net.train(epochs=4, batch=16384, lr=3e-3)
    _, loss1 = net.gradient(0, 1 << 16)
    assert loss1 < 0.2 * loss0, (loss0, loss1)
    hold = learned.Network(seed=1)
    hold.generate(1 << 16, seed=12345)
    x, y, ok = hold.samples(0, 1 << 16)
    sel = ok.astype(bool)
    w = x[sel, 6].astype(np.float64)
    err_pvrs = np.abs(w * y[sel])                       # |log(p_pvrs / p*)|
    err_net = np.abs(w * (net.infer(x[sel]) - y[sel]))  # |log(p_net / p*)|
    print("log guess error p50/p90/p99: pvrs %s network %s" % (
        np.percentile(err_pvrs, [50, 90, 99]).round(4), np.percentile(err_net, [50, 90, 99]).round(4)))
    for pct in (90, 99):
        assert np.percentile(err_net, pct) < 0.5 * np.percentile(err_pvrs, pct), pct
    assert np.percentile(err_net, 50) < np.percentile(err_pvrs, 50)


def test_newton_updates_with_both_guesses_on_random_problems():
    """What the network gains over the method without it, in Newton steps:
    on a grid whose cells are independent draws from the training
    distribution (held out: another seed than the training set's), the
    learned start needs strictly fewer Newton steps per interface than the
    adaptive PVRS start -- counted both ways, without and with the final step
    below the tolerance that every non-trivial interface takes -- and the
    converged-pressure start (the floor) needs almost none."""
    net = learned.Network(seed=2024)
    net.generate(1 << 24, seed=7)
    net.train(epochs=4, batch=16384, lr=3e-3)
    n = 128
    claw = _exact_claw(n)
    rng = np.random.default_rng(8)
    rho = np.exp(rng.uniform(np.log(1e-2), np.log(1e2), (n, n)))
    p = np.exp(rng.uniform(np.log(1e-2), np.log(1e2), (n, n)))
    u, v = rng.uniform(-3, 3, (n, n)), rng.uniform(-3, 3, (n, n))
    st = claw.solution.state
    st.q[0], st.q[1], st.q[2] = rho, rho * u, rho * v
    st.q[3] = p / (G - 1) + 0.5 * rho * (u * u + v * v)
    s = claw.solver
    s.setup(claw.solution)
    its, app = {}, {}
    for use_net in (False, True):
        learned.attach(s, net if use_net else None)
        learned.newton_counts(s)
        s._dev.step(1e-6, want_cfl=False)
        s._dev.accept(False)
        it, ap, ns = learned.newton_counts(s)
        its[use_net], app[use_net] = it / ns, ap / ns
    learned.attach(s, None)
    learned.converged_guess(s)
    learned.newton_counts(s)
    s._dev.step(1e-6, want_cfl=False)
    s._dev.accept(False)
    it_c, ap_c, ns_c = learned.newton_counts(s)
    learned.converged_guess(s, False)
    print("Newton steps per interface (needed / applied): pvrs %.3f / %.3f, learned %.3f / %.3f, "
          "converged %.3f / %.3f" % (its[False], app[False], its[True], app[True], it_c / ns_c, ap_c / ns_c))
    assert its[True] < its[False], its
    assert app[True] < app[False], app
    # (near-vacuum draws, whose p* is at the solver's pressure floor, still take steps)
    assert it_c / ns_c < 0.05 * its[False] and ap_c <= ns_c


def test_converged_guess_gives_the_same_step(oracle):
    # the measurement aid's pre-pass: Newton from the converged p* ends where
    # it would from the PVRS guess (same step within the parity bar), with no
    # Newton step needed
    claw = _exact_claw(130)
    st = claw.solution.state
    qbc = _euler_qbc(130, 130, seed=9)
    q_init = np.asfortranarray(qbc[:, 2:-2, 2:-2])
    st.q = q_init.copy(order="F")
    s = claw.solver
    s.setup(claw.solution)
    outs = []
    for on in (False, True):
        learned.converged_guess(s, on)
        learned.newton_counts(s)
        s._dev.step(2e-4, want_cfl=False)
        s._dev.accept(False)
        outs.append(learned.newton_counts(s))
        s._dev.step(2e-4, want_cfl=False)
        s._dev.accept(True)
        outs.append(st.get_q_global())
        st.q = q_init.copy(order="F")
        s._dev.push(st)
    (c0, q0, c1, q1) = outs
    assert c0[0] > 0 and c1[0] == 0 and c1[2] == c0[2]
    assert max_rel(q1, q0) <= PARITY_RTOL


def test_converged_guess_with_error_bounds_a_guess_of_that_precision(oracle):
    # the measurement aid with a relative error on the converged p* where
    # the adaptive guess needs Newton steps: a coarser guess never needs fewer
    # steps than a finer one, none needs more than the adaptive guess alone
    # where that needs none, none changes the step beyond the parity bar, and
    # an error of half an FP32 ulp already needs steps where the exact
    # converged value needs none
    claw = _exact_claw(130)
    st = claw.solution.state
    qbc = _euler_qbc(130, 130, seed=11)
    q_init = np.asfortranarray(qbc[:, 2:-2, 2:-2])
    st.q = q_init.copy(order="F")
    s = claw.solver
    s.setup(claw.solution)
    counts, qs = [], []
    for rel in (None, 2.0 ** -9, 2.0 ** -12, 2.0 ** -25, 0.0):
        if rel is None:
            learned.converged_guess(s, False)
        else:
            learned.converged_guess(s, True, rel_error=rel)
        learned.newton_counts(s)
        s._dev.step(2e-4, want_cfl=False)
        s._dev.accept(True)
        counts.append(learned.newton_counts(s))
        qs.append(st.get_q_global())
        st.q = q_init.copy(order="F")
        s._dev.push(st)
    learned.converged_guess(s, False)
    needed = [c[0] for c in counts]
    assert all(c[2] == counts[0][2] for c in counts)
    assert needed[1] >= needed[2] >= needed[3] >= needed[4] == 0, needed
    assert needed[3] > 0
    for q in qs[1:]:
        assert max_rel(q, qs[0]) <= PARITY_RTOL
    with pytest.raises(_lib.Claw2Error):
        learned.converged_guess(s, True, rel_error=0.5)
