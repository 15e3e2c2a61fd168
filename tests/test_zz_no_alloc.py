"""claw2_step2ds_noalloc: the split step for callers that cannot allocate
device memory (a framework that has reserved the GPU's memory in its own pool,
or a loop that cannot take cudaMalloc's implicit synchronisation).  It keeps
its scratch -- the state after the x-sweep and the CFL/status words -- in one
fixed device array inside the library instead of allocating it.

Checked through the C ABI against the existing entry point (claw2_step2ds with
ids = 1 then ids = 2, the reference's two step2ds calls) on two calls in a row
with different inputs, so the second call finds the first call's contents in
the shared array; plus the size limit.  This file is named to run last.
"""
import ctypes

import numpy as np
import pytest

from helpers import PARITY_RTOL, RP_INFO, max_rel, method_vector, random_qbc, set_cparam
from pyclaw_b200 import _lib, classic2

pytestmark = pytest.mark.gpu


def _desc(rp, mx, my, dx, dy, mthlim, order=2):
    name, meqn, mwaves, cp = RP_INFO[rp]
    d = _lib.Claw2Desc()
    d.mx, d.my = mx, my
    d.num_eqn, d.num_waves, d.num_aux, d.num_ghost = meqn, mwaves, 0, 2
    d.riemann, d.order, d.transverse, d.dimensional_split, d.fwave = rp, order, 0, 1, 0
    for k in range(mwaves):
        d.mthlim[k] = int(mthlim[k])
    d.dx, d.dy = dx, dy
    for k, v in enumerate(cp):
        d.cparam[k] = v
    d.ncparam = len(cp)
    return d


def _reference_pair(rp, qbc, dx, dy, dt, mthlim, order=2):
    """The existing entry point: claw2_step2ds x-sweep then y-sweep."""
    mx, my = qbc.shape[1] - 4, qbc.shape[2] - 4
    method = method_vector(order, 0, split=True)
    set_cparam(classic2, rp)
    q1, c1 = classic2.step2ds(max(mx, my), 2, mx, my, qbc, qbc.copy(order="F"), None, dx, dy, dt, method,
                              mthlim, ids=1, rpn2=rp)
    q2, c2 = classic2.step2ds(max(mx, my), 2, mx, my, q1, q1, None, dx, dy, dt, method, mthlim, ids=2, rpn2=rp)
    return q2, max(c1, c2)


def _noalloc(torch, rp, qbc, dx, dy, dt, mthlim, pitch, order=2):
    """The new entry point on caller-owned device planes (the test allocates
    them; the entry point allocates nothing)."""
    meqn, nx, ny = qbc.shape
    mx, my = nx - 4, ny - 4
    planes = np.zeros((meqn, ny, pitch))
    planes[:, :, :nx] = np.transpose(qbc, (0, 2, 1))
    qold = torch.from_numpy(planes).cuda()
    qnew = qold.clone()
    cfl = ctypes.c_double(-1.0)
    d = _desc(rp, mx, my, dx, dy, mthlim, order)
    stream = torch.cuda.current_stream().cuda_stream
    lib = _lib.load()
    rc = lib.claw2_step2ds_noalloc(ctypes.byref(d), ctypes.c_void_p(qold.data_ptr()),
                                   ctypes.c_void_p(qnew.data_ptr()), pitch, ny * pitch, dt, ctypes.byref(cfl),
                                   ctypes.c_void_p(stream or None))
    _lib.check(rc)
    out = np.transpose(qnew.cpu().numpy()[:, :, :nx], (0, 2, 1))
    return out, cfl.value


def _check(torch, rp, mx, my, seed, courant, order=2, pitch=None):
    name, meqn, mwaves, cp = RP_INFO[rp]
    qbc = random_qbc(rp, mx, my, seed=seed)
    mthlim = np.full(mwaves, 4, dtype=np.intc)
    dx, dy = 1.0 / mx, 1.0 / my
    dt = courant * min(dx, dy)
    q_ref, cfl_ref = _reference_pair(rp, qbc, dx, dy, dt, mthlim, order)
    if pitch is None:
        pitch = ((mx + 4 + 7) // 8) * 8
    q_new, cfl_new = _noalloc(torch, rp, qbc, dx, dy, dt, mthlim, pitch, order)
    assert abs(cfl_new - cfl_ref) <= PARITY_RTOL * cfl_ref
    assert max_rel(q_new[:, 2:-2, 2:-2], q_ref[:, 2:-2, 2:-2]) <= PARITY_RTOL
    return cfl_new


def test_noalloc_matches_existing_entry_point_twice():
    torch = pytest.importorskip("torch")
    # two calls in a row, different shapes and solvers; the second call's
    # Courant number is far below the first's, so a Courant-number word left
    # over from the first call (not cleared) would show as a mismatch
    cfl1 = _check(torch, _lib.RP_EULER_ROE, 150, 90, 11, courant=0.2)
    cfl2 = _check(torch, _lib.RP_SHALLOW_ROE, 61, 117, 12, courant=0.02)
    assert cfl2 < 0.5 * cfl1, (cfl1, cfl2)


def test_noalloc_first_order_acoustics():
    torch = pytest.importorskip("torch")
    _check(torch, _lib.RP_ACOUSTICS, 77, 45, 13, courant=0.1, order=1)


def test_noalloc_largest_grid_that_fits():
    # Euler with a 1024-double pitch: 4 planes of 1024 x 1023 doubles plus the
    # 256-byte header fit in the 32 MiB array exactly as the limit states
    torch = pytest.importorskip("torch")
    mx, my, pitch = 1020, 1019, 1024
    assert 256 + 4 * pitch * (my + 4) * 8 <= _lib.CLAW2_NOALLOC_SCRATCH_BYTES
    _check(torch, _lib.RP_EULER_ROE, mx, my, 14, courant=0.1, pitch=pitch)


def test_noalloc_rejects_grids_beyond_its_scratch():
    torch = pytest.importorskip("torch")
    rp = _lib.RP_EULER_ROE
    mx = my = 1100  # 4 planes of 1104 x 1104 doubles > the fixed array
    d = _desc(rp, mx, my, 1.0 / mx, 1.0 / my, [4, 4, 4, 4])
    pitch = mx + 4
    cfl = ctypes.c_double(0.0)
    buf = torch.zeros(8, dtype=torch.float64, device="cuda")  # never touched: rejected first
    lib = _lib.load()
    rc = lib.claw2_step2ds_noalloc(ctypes.byref(d), ctypes.c_void_p(buf.data_ptr()),
                                   ctypes.c_void_p(buf.data_ptr()), pitch, pitch * (my + 4), 1e-4,
                                   ctypes.byref(cfl), None)
    assert rc == _lib.EINVAL
    msg = lib.claw2_last_error().decode()
    assert "too large" in msg and str(_lib.CLAW2_NOALLOC_SCRATCH_BYTES) in msg
