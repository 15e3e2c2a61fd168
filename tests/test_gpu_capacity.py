"""Capacity functions (state.index_capa, method(6)) and the edge-velocity
advection solver (vc_advection_2D) on the GPU.

With a capacity function kappa every increment of a cell is divided by its
kappa, a transverse increment also by the kappa of the cell its fluctuation
entered, the second-order correction uses the mean of the two cells'
dt/(dx kappa) and the Courant number the larger one-sided product
(step2.f90:132-160, flux2.f90:104-203).  The fused kernel sums a cell's
increments and scales the sum once; these tests hold the unsplit kernel (both
transverse paths: the in-row one of solvers without aux data and the
one-row-late one of vc_advection / vc_acoustics), the split sweeps and the
device-resident solver to the oracle at 1e-12 relative, and run the
reference's annulus example (mapped polar grid, custom aux BCs) on the device.
"""
import numpy as np
import pytest

from helpers import PARITY_RTOL, max_rel, method_vector, random_qbc, set_cparam
from pyclaw_b200 import _lib, classic2, workloads

pytestmark = pytest.mark.gpu

VCA = _lib.RP_VC_ADVECTION


def _blocky(rng, nx, ny, lo, hi):
    X, Y = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    block = (X > nx // 3).astype(int) + 2 * (Y > ny // 2).astype(int)
    noise = rng.random((nx, ny)) < 0.5
    return np.where(noise, rng.uniform(lo, hi, (nx, ny)), rng.uniform(lo, hi, 4)[block])


def _capa(rng, nx, ny):
    return _blocky(rng, nx, ny, 0.5, 2.0)


def _vc_adv_aux(mx, my, seed):
    """auxbc (3, mx+4, my+4): edge velocities u, v in [-1.5, 1.5] (both signs,
    exercising both halves of every fluctuation) and kappa in [0.5, 2]."""
    rng = np.random.default_rng(seed)
    nx, ny = mx + 4, my + 4
    return np.asfortranarray(np.stack([_blocky(rng, nx, ny, -1.5, 1.5), _blocky(rng, nx, ny, -1.5, 1.5),
                                       _capa(rng, nx, ny)]))


def _method(order, transverse, mcapa, split=False):
    m = method_vector(order, transverse, split=split)
    m[5] = mcapa
    return m


def _dt(speed, capa, dx, dy, target=0.8):
    return target * min(dx, dy) * float(np.min(capa)) / speed


@pytest.mark.parametrize("transverse", [0, 1, 2])
@pytest.mark.parametrize("mx,my", [(1, 1), (3, 5), (37, 23), (130, 70), (257, 9), (9, 300)])
def test_vc_advection_capa_step2(oracle, transverse, mx, my):
    qbc = random_qbc(_lib.RP_ADVECTION, mx, my, seed=mx * 31 + my + transverse)
    aux = _vc_adv_aux(mx, my, seed=mx + 11 * my)
    method = _method(2, transverse, 3)
    mthlim = np.full(1, 3, dtype=np.intc)
    dx, dy = 1.0 / mx, 1.3 / my
    dt = _dt(1.5, aux[2], dx, dy)
    q_o = qbc.copy(order="F")
    cfl_o = oracle.step2(qbc, q_o, dx, dy, dt, method, mthlim, VCA, [], aux=aux)
    q_g, cfl_g = classic2.step2(max(mx, my), 2, mx, my, qbc, qbc.copy(order="F"), aux, dx, dy, dt, method,
                                mthlim, rpn2=VCA)
    assert abs(cfl_g - cfl_o) <= PARITY_RTOL * cfl_o
    assert max_rel(q_g[:, 2:-2, 2:-2], q_o[:, 2:-2, 2:-2]) <= PARITY_RTOL


@pytest.mark.parametrize("mcapa", [0, 3])
@pytest.mark.parametrize("lim", [0, 1, 2, 4, 5])
@pytest.mark.parametrize("order", [1, 2])
def test_vc_advection_limiters_and_order(oracle, mcapa, lim, order):
    mx, my = 61, 47
    qbc = random_qbc(_lib.RP_ADVECTION, mx, my, seed=5 + lim)
    aux = _vc_adv_aux(mx, my, seed=2 + lim)
    method = _method(order, 2, mcapa)
    mthlim = np.full(1, lim, dtype=np.intc)
    dx, dy = 0.02, 0.015
    dt = _dt(1.5, aux[2] if mcapa else np.ones(1), dx, dy)
    q_o = qbc.copy(order="F")
    cfl_o = oracle.step2(qbc, q_o, dx, dy, dt, method, mthlim, VCA, [], aux=aux)
    q_g, cfl_g = classic2.step2(max(mx, my), 2, mx, my, qbc, qbc.copy(order="F"), aux, dx, dy, dt, method,
                                mthlim, rpn2=VCA)
    assert abs(cfl_g - cfl_o) <= PARITY_RTOL * cfl_o
    assert max_rel(q_g[:, 2:-2, 2:-2], q_o[:, 2:-2, 2:-2]) <= PARITY_RTOL


@pytest.mark.parametrize("transverse", [0, 1, 2])
@pytest.mark.parametrize("mx,my", [(37, 23), (257, 70)])
def test_euler_capa_step2(oracle, transverse, mx, my):
    # a solver without aux data: the capacity plane is the only aux component
    rp = _lib.RP_EULER_ROE
    qbc = random_qbc(rp, mx, my, seed=mx + my + 100 * transverse)
    rng = np.random.default_rng(mx * my)
    aux = np.asfortranarray(_capa(rng, mx + 4, my + 4)[None])
    method = _method(2, transverse, 1)
    mthlim = np.full(4, 4, dtype=np.intc)
    dx, dy = 1.0 / mx, 1.0 / my
    dt = _dt(6.0, aux[0], dx, dy)
    q_o = qbc.copy(order="F")
    cfl_o = oracle.step2(qbc, q_o, dx, dy, dt, method, mthlim, rp, [1.4, 1.0], aux=aux)
    set_cparam(classic2, rp)
    q_g, cfl_g = classic2.step2(max(mx, my), 2, mx, my, qbc, qbc.copy(order="F"), aux, dx, dy, dt, method,
                                mthlim, rpn2=rp)
    assert abs(cfl_g - cfl_o) <= PARITY_RTOL * cfl_o
    assert max_rel(q_g[:, 2:-2, 2:-2], q_o[:, 2:-2, 2:-2]) <= PARITY_RTOL


@pytest.mark.parametrize("transverse", [1, 2])
def test_vc_acoustics_capa_step2(oracle, transverse):
    mx, my = 130, 70
    rp = _lib.RP_VC_ACOUSTICS
    qbc = random_qbc(_lib.RP_ACOUSTICS, mx, my, seed=41 + transverse)
    rng = np.random.default_rng(7)
    nx, ny = mx + 4, my + 4
    aux = np.asfortranarray(np.stack([_blocky(rng, nx, ny, 0.5, 4.0), _blocky(rng, nx, ny, 0.5, 2.5),
                                      _capa(rng, nx, ny)]))
    method = _method(2, transverse, 3)
    mthlim = np.full(2, 4, dtype=np.intc)
    dx, dy = 1.0 / mx, 1.0 / my
    dt = _dt(2.5, aux[2], dx, dy)
    q_o = qbc.copy(order="F")
    cfl_o = oracle.step2(qbc, q_o, dx, dy, dt, method, mthlim, rp, [], aux=aux)
    q_g, cfl_g = classic2.step2(max(mx, my), 2, mx, my, qbc, qbc.copy(order="F"), aux, dx, dy, dt, method,
                                mthlim, rpn2=rp)
    assert abs(cfl_g - cfl_o) <= PARITY_RTOL * cfl_o
    assert max_rel(q_g[:, 2:-2, 2:-2], q_o[:, 2:-2, 2:-2]) <= PARITY_RTOL


@pytest.mark.parametrize("rp", [VCA, _lib.RP_EULER_ROE])
@pytest.mark.parametrize("ids", [1, 2])
def test_capa_step2ds_sweeps(oracle, rp, ids):
    mx, my = 130, 70
    if rp == VCA:
        qbc = random_qbc(_lib.RP_ADVECTION, mx, my, seed=3 + ids)
        aux = _vc_adv_aux(mx, my, seed=13 + ids)
        mcapa, mthlim, cp, speed = 3, np.full(1, 4, dtype=np.intc), [], 1.5
    else:
        qbc = random_qbc(rp, mx, my, seed=3 + ids)
        aux = np.asfortranarray(_capa(np.random.default_rng(ids), mx + 4, my + 4)[None])
        mcapa, mthlim, cp, speed = 1, np.full(4, 4, dtype=np.intc), [1.4, 1.0], 6.0
        set_cparam(classic2, rp)
    method = _method(2, 0, mcapa, split=True)
    dx, dy = 1.0 / mx, 1.0 / my
    dt = _dt(speed, aux[mcapa - 1], dx, dy)
    q_o = qbc.copy(order="F")
    cfl_o = oracle.step2ds(qbc, q_o, dx, dy, dt, method, mthlim, ids, rp, cp, aux=aux)
    q_g, cfl_g = classic2.step2ds(max(mx, my), 2, mx, my, qbc, qbc.copy(order="F"), aux, dx, dy, dt, method,
                                  mthlim, ids=ids, rpn2=rp)
    assert abs(cfl_g - cfl_o) <= PARITY_RTOL * cfl_o
    sl = (slice(None), slice(2, -2), slice(None)) if ids == 1 else (slice(None), slice(2, -2), slice(2, -2))
    assert max_rel(q_g[sl], q_o[sl]) <= PARITY_RTOL


def test_unit_capacity_is_the_plain_step():
    # kappa = 1 everywhere: the capacity form multiplies by exact ones, so it
    # reproduces the plain step to rounding of the summation order
    mx, my = 130, 70
    rp = _lib.RP_EULER_ROE
    qbc = random_qbc(rp, mx, my, seed=77)
    aux = np.ones((1, mx + 4, my + 4), order="F")
    mthlim = np.full(4, 4, dtype=np.intc)
    set_cparam(classic2, rp)
    dx, dy, dt = 1.0 / mx, 1.0 / my, 0.1 / mx
    out = []
    for mcapa in (0, 1):
        q, c = classic2.step2(max(mx, my), 2, mx, my, qbc, qbc.copy(order="F"), aux, dx, dy, dt,
                              _method(2, 2, mcapa), mthlim, rpn2=rp)
        out.append((q, c))
    assert max_rel(out[1][0][:, 2:-2, 2:-2], out[0][0][:, 2:-2, 2:-2]) <= 1e-14
    assert out[1][1] == out[0][1]


def test_annulus_device_run_matches_reference_golden(goldens):
    # the reference's examples/advection_2d_annulus on the device-resident path
    # (capacity = cell area, edge velocities, custom aux BCs filled on the host)
    claw = workloads.advection_annulus()
    claw.run()
    q = claw.frames[claw.num_output_times].state.get_q_global().reshape([-1])
    dx, dy = claw.solution.domain.grid.delta
    area = claw.frames[0].state.aux[2].reshape([-1]) * dx * dy
    diff = np.sum(np.abs(area * (q - goldens["advection_annulus_classic"])))
    assert diff < 1e-6  # the reference test's bound
    assert diff < 1e-11


def test_annulus_device_frames_match_oracle(oracle):
    # every output frame of the device run against the oracle's, on a finer grid
    # (several strips and row blocks of the fused kernel)
    claw_g = workloads.advection_annulus(m_r=160, m_theta=300, tfinal=0.25, num_output_times=5)
    claw_o = workloads.advection_annulus(oracle.make_solver_class(), m_r=160, m_theta=300, tfinal=0.25,
                                         num_output_times=5)
    claw_g.run()
    claw_o.run()
    assert claw_g.solver.status['numsteps'] == claw_o.solver.status['numsteps']
    for fg, fo in zip(claw_g.frames, claw_o.frames):
        assert fg.t == fo.t
        assert max_rel(fg.q, fo.q) <= 1e-11


@pytest.mark.parametrize("variant", [0, 4])
def test_capacity_in_both_tiles(oracle, variant):
    # the capacity form of the one-row-late x finish (variant 4) and of the
    # original tile, through the stateless step
    from pyclaw_b200 import tune
    mx, my = 257, 70
    qbc = random_qbc(_lib.RP_ADVECTION, mx, my, seed=99)
    aux = _vc_adv_aux(mx, my, seed=98)
    method = _method(2, 2, 3)
    mthlim = np.full(1, 4, dtype=np.intc)
    dx, dy = 1.0 / mx, 1.0 / my
    dt = _dt(1.5, aux[2], dx, dy)
    q_o = qbc.copy(order="F")
    cfl_o = oracle.step2(qbc, q_o, dx, dy, dt, method, mthlim, VCA, [], aux=aux)
    tune.set_shape(VCA, variant, 12)
    try:
        q_g, cfl_g = classic2.step2(max(mx, my), 2, mx, my, qbc, qbc.copy(order="F"), aux, dx, dy, dt, method,
                                    mthlim, rpn2=VCA)
    finally:
        tune.set_shape(VCA, 0, 0)
    assert abs(cfl_g - cfl_o) <= PARITY_RTOL * cfl_o
    assert max_rel(q_g[:, 2:-2, 2:-2], q_o[:, 2:-2, 2:-2]) <= PARITY_RTOL
