"""The two-barrier tile (launch variant 4: x-interfaces solved on their row
and finished one row later, with the y work) for every solver with a
transverse solve, against the oracle at 1e-12, through the stateless step."""
import numpy as np
import pytest

from helpers import PARITY_RTOL, max_rel, method_vector, random_qbc, set_cparam
from pyclaw_b200 import _lib, classic2, tune

pytestmark = pytest.mark.gpu


def _case(rp, mx, my, seed):
    rng = np.random.default_rng(seed)
    aux, cp = None, []
    if rp in (_lib.RP_ADVECTION, _lib.RP_ACOUSTICS, _lib.RP_EULER_ROE, _lib.RP_SHALLOW_ROE):
        qbc = random_qbc(rp, mx, my, seed)
        from helpers import RP_INFO
        cp = RP_INFO[rp][3]
        set_cparam(classic2, rp)
    elif rp == _lib.RP_EULER_5WAVE:
        q4 = random_qbc(_lib.RP_EULER_ROE, mx, my, seed)
        qbc = np.asfortranarray(np.concatenate([q4, rng.random((1, mx + 4, my + 4))]))
        cp = [1.4, 1.0]
        classic2.cparam.gamma, classic2.cparam.efix = 1.4, True
    elif rp == _lib.RP_VC_ACOUSTICS:
        qbc = random_qbc(_lib.RP_ACOUSTICS, mx, my, seed)
        aux = np.asfortranarray(np.stack([rng.uniform(0.5, 4.0, (mx + 4, my + 4)),
                                          rng.uniform(0.5, 2.5, (mx + 4, my + 4))]))
    elif rp == _lib.RP_VC_ADVECTION:
        qbc = random_qbc(_lib.RP_ADVECTION, mx, my, seed)
        aux = np.asfortranarray(rng.uniform(-1.5, 1.5, (2, mx + 4, my + 4)))
    elif rp == _lib.RP_PSYSTEM:
        eps = rng.uniform(-0.3, 0.6, (mx + 4, my + 4))
        qbc = np.asfortranarray(np.stack([eps, rng.uniform(-1, 1, eps.shape), rng.uniform(-1, 1, eps.shape)]))
        aux = np.asfortranarray(np.stack([rng.uniform(1, 4, eps.shape), rng.uniform(1, 4, eps.shape),
                                          np.where(rng.random(eps.shape) < 0.5, 1.0, 2.0), eps]))
    return qbc, aux, cp


@pytest.mark.parametrize("transverse", [1, 2])
@pytest.mark.parametrize("rp", [_lib.RP_ADVECTION, _lib.RP_ACOUSTICS, _lib.RP_EULER_ROE, _lib.RP_SHALLOW_ROE,
                                _lib.RP_EULER_5WAVE, _lib.RP_VC_ACOUSTICS, _lib.RP_VC_ADVECTION, _lib.RP_PSYSTEM])
@pytest.mark.parametrize("mx,my,rows", [(130, 70, 12), (9, 300, 40), (257, 9, 8)])
def test_two_barrier_tile_matches_oracle(oracle, rp, transverse, mx, my, rows):
    qbc, aux, cp = _case(rp, mx, my, seed=rp * 100 + mx + transverse)
    fw = rp == _lib.RP_PSYSTEM
    mw = {_lib.RP_ADVECTION: 1, _lib.RP_ACOUSTICS: 2, _lib.RP_EULER_ROE: 4, _lib.RP_SHALLOW_ROE: 3,
          _lib.RP_EULER_5WAVE: 5, _lib.RP_VC_ACOUSTICS: 2, _lib.RP_VC_ADVECTION: 1, _lib.RP_PSYSTEM: 2}[rp]
    mthlim = np.array([4, 1, 2, 3, 5][:mw], dtype=np.intc)
    method = method_vector(2, transverse)
    dx, dy = 1.0 / mx, 1.0 / my
    dt = 0.05 * min(dx, dy)
    q_o = qbc.copy(order="F")
    cfl_o = oracle.step2(qbc, q_o, dx, dy, dt, method, mthlim, rp, cp, fw, aux=aux)
    tune.set_shape(rp, 4, rows)
    try:
        q_g, cfl_g = classic2.step2(max(mx, my), 2, mx, my, qbc, qbc.copy(order="F"), aux, dx, dy, dt, method,
                                    mthlim, fwave=fw, rpn2=rp)
    finally:
        tune.set_shape(rp, 0, 0)
    assert abs(cfl_g - cfl_o) <= PARITY_RTOL * cfl_o
    assert max_rel(q_g[:, 2:-2, 2:-2], q_o[:, 2:-2, 2:-2]) <= PARITY_RTOL
