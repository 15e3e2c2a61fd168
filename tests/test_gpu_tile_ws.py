"""The direction-split tile (launch variant 8: two threads per column, the
y-interfaces in one warp group and the x-interfaces in the other) against the
oracle at 1e-12 through the stateless step, for every solver it runs (no aux
data) -- all transverse modes, orders 1 and 2, the method-specialised
instantiation (order 2, trans_cor, MC everywhere) and mixed limiters, f-waves,
ragged sizes, and data with long constant runs, where whole warps take the
zero-jump shortcut.  Solvers with aux data run the one-thread tile under the
same setting (checked too)."""
import numpy as np
import pytest

from helpers import PARITY_RTOL, RP_INFO, max_rel, method_vector, random_qbc, set_cparam
from pyclaw_b200 import _lib, classic2, tune
from test_gpu_tile2 import _case

pytestmark = pytest.mark.gpu

MW = {_lib.RP_ADVECTION: 1, _lib.RP_ACOUSTICS: 2, _lib.RP_EULER_ROE: 4, _lib.RP_SHALLOW_ROE: 3,
      _lib.RP_EULER_5WAVE: 5, _lib.RP_VC_ACOUSTICS: 2, _lib.RP_VC_ADVECTION: 1, _lib.RP_PSYSTEM: 2}


def _run(oracle, rp, qbc, aux, cp, order, transverse, mthlim, rows, fw=False):
    mx, my = qbc.shape[1] - 4, qbc.shape[2] - 4
    method = method_vector(order, transverse)
    dx, dy = 1.0 / mx, 1.0 / my
    dt = 0.05 * min(dx, dy)
    q_o = qbc.copy(order="F")
    cfl_o = oracle.step2(qbc, q_o, dx, dy, dt, method, mthlim, rp, cp, fw, aux=aux)
    tune.set_shape(rp, 8, rows)
    try:
        q_g, cfl_g = classic2.step2(max(mx, my), 2, mx, my, qbc, qbc.copy(order="F"), aux, dx, dy, dt, method,
                                    mthlim, fwave=fw, rpn2=rp)
    finally:
        tune.set_shape(rp, 0, 0)
    assert abs(cfl_g - cfl_o) <= PARITY_RTOL * cfl_o
    assert max_rel(q_g[:, 2:-2, 2:-2], q_o[:, 2:-2, 2:-2]) <= PARITY_RTOL


@pytest.mark.parametrize("transverse", [0, 1, 2])
@pytest.mark.parametrize("rp", [_lib.RP_ADVECTION, _lib.RP_ACOUSTICS, _lib.RP_EULER_ROE, _lib.RP_SHALLOW_ROE,
                                _lib.RP_EULER_5WAVE, _lib.RP_VC_ACOUSTICS, _lib.RP_VC_ADVECTION])
@pytest.mark.parametrize("mx,my,rows", [(130, 70, 12), (9, 300, 40), (257, 9, 8), (1, 1, 2)])
def test_direction_split_tile_matches_oracle(oracle, rp, transverse, mx, my, rows):
    qbc, aux, cp = _case(rp, mx, my, seed=rp * 100 + mx + transverse)
    mthlim = np.array([4, 1, 2, 3, 5][:MW[rp]], dtype=np.intc)
    _run(oracle, rp, qbc, aux, cp, 2, transverse, mthlim, rows)


@pytest.mark.parametrize("rp", [_lib.RP_ACOUSTICS, _lib.RP_EULER_ROE, _lib.RP_SHALLOW_ROE])
@pytest.mark.parametrize("order", [1, 2])
@pytest.mark.parametrize("smooth_frac", [0.5, 0.01])
def test_direction_split_tile_specialised_method(oracle, rp, order, smooth_frac):
    # order 2 + trans_cor + MC on every family is the specialised kernel; few
    # noisy cells leave whole warps of equal neighbours (zero-jump shortcut)
    mx, my = 300, 150
    qbc = random_qbc(rp, mx, my, seed=31 + rp, smooth_frac=smooth_frac)
    cp = RP_INFO[rp][3]
    set_cparam(classic2, rp)
    _run(oracle, rp, qbc, None, cp, order, 2, np.full(MW[rp], 4, dtype=np.intc), 16)


@pytest.mark.parametrize("rp", [_lib.RP_ACOUSTICS, _lib.RP_EULER_ROE])
def test_direction_split_tile_fwave_branch(oracle, rp):
    # q-wave solvers with use_fwave: the f-wave correction (sign(s)), no shortcut
    mx, my = 140, 60
    qbc = random_qbc(rp, mx, my, seed=77, smooth_frac=0.05)
    cp = RP_INFO[rp][3]
    set_cparam(classic2, rp)
    _run(oracle, rp, qbc, None, cp, 2, 2, np.full(MW[rp], 4, dtype=np.intc), 8, fw=True)
