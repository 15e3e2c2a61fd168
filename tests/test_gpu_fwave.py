"""f-waves (use_fwave, flux2.f90:147-159) and the p-system solver
(psystem_2D) on the GPU, with the host loop's gauges and before-step hook.

flux2's f-wave branch weights the second-order correction by sign(s) instead
of |s|; the kernels take it from the method at run time.  These tests hold the
branch (with the f-wave p-system and with q-wave solvers run as the reference
would run them with fwave = True) and the p-system's normal and transverse
solves to the oracle at 1e-12 relative, and the p-system example's device run
(gauges gathered on the device every step, the strain copied into aux by the
before-step hook) to the oracle's run and to the reference's own gauge files.
"""
import os

import numpy as np
import pytest

from helpers import PARITY_RTOL, max_rel, method_vector, random_qbc, set_cparam
from pyclaw_b200 import _lib, classic2, workloads

pytestmark = pytest.mark.gpu

PS = _lib.RP_PSYSTEM


def _psystem_data(mx, my, seed):
    """qbc (3, mx+4, my+4) and auxbc (4, mx+4, my+4): strain in [-0.3, 0.6],
    momenta in [-1, 1]; density and bulk modulus in [1, 4] in blocks with
    noise, both stress-strain relations, the aux strain near q's."""
    rng = np.random.default_rng(seed)
    nx, ny = mx + 4, my + 4
    X, Y = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    block = (X > nx // 3).astype(int) + 2 * (Y > ny // 2).astype(int)
    noise = rng.random((nx, ny)) < 0.5

    def field(lo, hi):
        return np.where(noise, rng.uniform(lo, hi, (nx, ny)), rng.uniform(lo, hi, 4)[block])

    eps = field(-0.3, 0.6)
    q = np.asfortranarray(np.stack([eps, field(-1.0, 1.0), field(-1.0, 1.0)]))
    rel = np.where(rng.random((nx, ny)) < 0.5, 1.0, 2.0)
    aux = np.asfortranarray(np.stack([field(1.0, 4.0), field(1.0, 4.0), rel,
                                      eps + rng.uniform(-0.05, 0.05, (nx, ny))]))
    return q, aux


def _dt(aux, q, dx, dy, target=0.7):
    K, rho = aux[1], aux[0]
    sigp = np.where(aux[2] == 1.0, K, K * np.exp(K * np.maximum(q[0], aux[3])))
    return target * min(dx, dy) / np.sqrt(np.max(sigp / rho))


@pytest.mark.parametrize("transverse", [0, 1, 2])
@pytest.mark.parametrize("mx,my", [(1, 1), (3, 5), (37, 23), (130, 70), (257, 9), (9, 300)])
def test_psystem_step2_matches_oracle(oracle, transverse, mx, my):
    qbc, aux = _psystem_data(mx, my, seed=mx * 13 + my + transverse)
    method = method_vector(2, transverse)
    mthlim = np.full(2, 2, dtype=np.intc)
    dx, dy = 1.0 / mx, 1.2 / my
    dt = _dt(aux, qbc, dx, dy)
    q_o = qbc.copy(order="F")
    cfl_o = oracle.step2(qbc, q_o, dx, dy, dt, method, mthlim, PS, [], True, aux=aux)
    q_g, cfl_g = classic2.step2(max(mx, my), 2, mx, my, qbc, qbc.copy(order="F"), aux, dx, dy, dt, method,
                                mthlim, fwave=True, rpn2=PS)
    assert abs(cfl_g - cfl_o) <= PARITY_RTOL * cfl_o
    assert max_rel(q_g[:, 2:-2, 2:-2], q_o[:, 2:-2, 2:-2]) <= PARITY_RTOL


@pytest.mark.parametrize("lim", [0, 1, 2, 3, 4, 5])
@pytest.mark.parametrize("order", [1, 2])
def test_psystem_limiters_and_order(oracle, lim, order):
    mx, my = 61, 47
    qbc, aux = _psystem_data(mx, my, seed=31 + lim)
    method = method_vector(order, 2)
    mthlim = np.array([lim, (lim + 2) % 6], dtype=np.intc)
    dx, dy = 0.02, 0.015
    dt = _dt(aux, qbc, dx, dy)
    q_o = qbc.copy(order="F")
    cfl_o = oracle.step2(qbc, q_o, dx, dy, dt, method, mthlim, PS, [], True, aux=aux)
    q_g, cfl_g = classic2.step2(max(mx, my), 2, mx, my, qbc, qbc.copy(order="F"), aux, dx, dy, dt, method,
                                mthlim, fwave=True, rpn2=PS)
    assert abs(cfl_g - cfl_o) <= PARITY_RTOL * cfl_o
    assert max_rel(q_g[:, 2:-2, 2:-2], q_o[:, 2:-2, 2:-2]) <= PARITY_RTOL


@pytest.mark.parametrize("ids", [1, 2])
def test_psystem_step2ds_sweeps(oracle, ids):
    mx, my = 130, 70
    qbc, aux = _psystem_data(mx, my, seed=70 + ids)
    method = method_vector(2, 0, split=True)
    mthlim = np.full(2, 4, dtype=np.intc)
    dx, dy = 1.0 / mx, 1.0 / my
    dt = _dt(aux, qbc, dx, dy)
    q_o = qbc.copy(order="F")
    cfl_o = oracle.step2ds(qbc, q_o, dx, dy, dt, method, mthlim, ids, PS, [], True, aux=aux)
    q_g, cfl_g = classic2.step2ds(max(mx, my), 2, mx, my, qbc, qbc.copy(order="F"), aux, dx, dy, dt, method,
                                  mthlim, ids=ids, fwave=True, rpn2=PS)
    assert abs(cfl_g - cfl_o) <= PARITY_RTOL * cfl_o
    sl = (slice(None), slice(2, -2), slice(None)) if ids == 1 else (slice(None), slice(2, -2), slice(2, -2))
    assert max_rel(q_g[sl], q_o[sl]) <= PARITY_RTOL


@pytest.mark.parametrize("rp", [_lib.RP_ACOUSTICS, _lib.RP_EULER_ROE, _lib.RP_SHALLOW_ROE])
@pytest.mark.parametrize("transverse", [1, 2])
def test_fwave_branch_with_q_wave_solvers(oracle, rp, transverse):
    # flux2's f-wave branch as the reference runs it for any solver when
    # fwave = True: sign(s) in place of |s| in the correction
    from helpers import RP_INFO
    mx, my = 130, 70
    qbc = random_qbc(rp, mx, my, seed=rp * 7 + transverse)
    _, _, mw, cp = RP_INFO[rp]
    method = method_vector(2, transverse)
    mthlim = np.full(mw, 4, dtype=np.intc)
    dx, dy = 1.0 / mx, 1.0 / my
    dt = 0.15 * min(dx, dy)
    q_o = qbc.copy(order="F")
    cfl_o = oracle.step2(qbc, q_o, dx, dy, dt, method, mthlim, rp, cp, True)
    set_cparam(classic2, rp)
    q_g, cfl_g = classic2.step2(max(mx, my), 2, mx, my, qbc, qbc.copy(order="F"), None, dx, dy, dt, method,
                                mthlim, fwave=True, rpn2=rp)
    assert abs(cfl_g - cfl_o) <= PARITY_RTOL * cfl_o
    assert max_rel(q_g[:, 2:-2, 2:-2], q_o[:, 2:-2, 2:-2]) <= PARITY_RTOL


def test_psystem_device_run_matches_oracle(oracle, tmp_path):
    # the p-system example on the device path (f-waves, before-step hook
    # editing aux in place, gauges gathered on the device, F functional)
    # against the oracle's run of the same setup, on a finer grid
    claw_g = workloads.psystem(cells_per_layer=12, tfinal=2.0, outdir=str(tmp_path / "g"))
    claw_o = workloads.psystem(oracle.make_solver_class(), cells_per_layer=12, tfinal=2.0,
                               outdir=str(tmp_path / "o"))
    claw_g.run()
    claw_o.run()
    sg, so = claw_g.solution.state, claw_o.solution.state
    assert claw_g.solver.status['numsteps'] == claw_o.solver.status['numsteps']
    assert len(sg.gauge_data) == 4
    for a, b in zip(sg.gauge_data, so.gauge_data):
        assert a.shape == b.shape
        assert np.array_equal(a[:, 0], b[:, 0]) or np.max(np.abs(a[:, 0] - b[:, 0])) <= 1e-12
        assert np.max(np.abs(a[:, 1:] - b[:, 1:])) <= 1e-10 * max(1.0, np.max(np.abs(b[:, 1:])))
    for fg, fo in zip(claw_g.frames, claw_o.frames):
        assert max_rel(fg.q, fo.q) <= 1e-11
    # the gauge files hold the in-memory values
    for k, f in enumerate(sg.grid.gauge_files):
        assert np.allclose(np.loadtxt(f.name), sg.gauge_data[k], rtol=1e-12, atol=0)
    Fg = np.loadtxt(os.path.join(str(tmp_path / "g"), "F.txt"))
    Fo = np.loadtxt(os.path.join(str(tmp_path / "o"), "F.txt"))
    assert Fg.shape == (11, 2) and np.allclose(Fg, Fo, rtol=1e-11, atol=0)


def test_psystem_gauge_goldens_on_device(goldens, tmp_path):
    # examples/psystem_2d/test_2d_psystem.py:8-24 on the device path: the
    # reference's four gauges (in memory and in the files) after the run to t = 1
    claw = workloads.psystem(cells_per_layer=6, tfinal=1., outdir=str(tmp_path))
    claw.run()
    st = claw.solution.state
    for k, g in enumerate(("0.25_0.25", "17.85_1.25", "3.25_18.75", "11.75_11.75")):
        expected = goldens["psystem_gauge" + g]
        mem = np.asarray(st.gauge_data[k])
        assert mem.shape == expected.shape
        assert np.allclose(expected, mem)
        assert np.allclose(expected, np.loadtxt(st.grid.gauge_files[k].name))
        assert np.max(np.abs(mem - expected)) <= 1e-9


def test_gauge_gather_matches_download(tmp_path):
    claw = workloads.psystem(cells_per_layer=6, tfinal=0.3, outdir=str(tmp_path))
    claw.run()
    st = claw.solution.state
    dev = st._mirror
    cells = [(0, 0), (119, 119), (5, 77), (60, 3)]
    g = dev.gather(cells)
    q = st.get_q_global()
    for k, (i, j) in enumerate(cells):
        assert np.array_equal(g[k], q[:, i, j])
    with pytest.raises(_lib.Claw2Error):
        dev.gather([(120, 0)])
