"""Drop-in for the reference's f2py module ``clawpack.pyclaw.classic.classic2``.

The reference's ClawSolver2D.step_hyperbolic calls (classic/solver.py:527-541)

    qbc, cfl = fmod.step2(maxm, num_ghost, mx, my, qold, qbc, auxbc, dx, dy, dt,
                          method, mthlim, aux1, aux2, aux3, work, fwave, rpn2, rpt2)
    qbc, cfl = fmod.step2ds(..., work, ids, fwave, rpn2, rpt2)

and sets Riemann parameters through ``state.set_cparam(fmod)`` (state.py:206-231),
which assigns problem_data entries as attributes of ``fmod.cparam``.  This
module accepts the same positional arguments and returns the same tuple; the
step runs on the GPU through claw2_step2 / claw2_step2ds.  ``rpn2`` names the
Riemann solver: a pyclaw_b200.riemann solver object or its integer id (a
Fortran function pointer cannot select device code).  ``auxbc`` (ghost cells
filled) feeds the solvers that read aux data and the capacity function
(method(6) > 0); ``aux1..3`` and ``work`` are
accepted and ignored (the device gathers the aux rows itself and allocates its
own workspace).
"""
import types

import numpy as np

from . import _lib
from . import riemann as _riemann

cparam = types.SimpleNamespace()

_BY_ID = {s.rp_id: s for s in _riemann._ALL}


def _solver(rpn2):
    if isinstance(rpn2, _riemann.RiemannSolver):
        return rpn2
    rp = _BY_ID.get(int(rpn2))
    if rp is None:
        raise ValueError("unknown Riemann solver id %r" % (rpn2,))
    return rp


def _cparam_vector(rp):
    vals = vars(cparam)
    return np.asarray(rp.cparam(vals) + [0.0] * (_lib.CLAW2_MAX_PARAMS - len(rp.cparam(vals))),
                      dtype=np.float64)


def _aux(aux, rp, method):
    """(num_aux, array) of an auxbc array (maux, mx+4, my+4), Fortran order,
    ghost cells filled, for solvers that read aux or a step with a capacity
    function (method(6) > 0); (0, None) otherwise."""
    if not getattr(rp, 'num_aux', 0) and int(method[5]) == 0:
        return 0, None
    if aux is None:
        raise ValueError("Riemann solver %s with method(6) = %d needs the aux array" % (rp.name, int(method[5])))
    a = np.asfortranarray(aux, dtype=np.float64)
    return a.shape[0], a


def _prep(qold, qnew, method, mthlim):
    qold = np.asfortranarray(qold, dtype=np.float64)
    if qnew is qold:
        out = qold
    else:
        out = np.array(qnew, dtype=np.float64, order='F', copy=True)
    return qold, out, np.ascontiguousarray(method, dtype=np.intc), np.ascontiguousarray(mthlim, dtype=np.intc)


def step2(maxm, num_ghost, mx, my, qold, qnew, aux, dx, dy, dt, method, mthlim, aux1=None, aux2=None,
          aux3=None, work=None, fwave=False, rpn2=None, rpt2=None):
    """Unsplit step (step2.f90); returns (qnew, cfl)."""
    rp = _solver(rpn2)
    lib = _lib.load()
    qold, out, method, mthlim = _prep(qold, qnew, method, mthlim)
    meqn = qold.shape[0]
    cfl = np.zeros(1)
    cp = _cparam_vector(rp)
    maux, auxa = _aux(aux, rp, method)
    _lib.check(lib.claw2_step2(int(maxm), meqn, len(mthlim), maux, int(num_ghost), int(mx), int(my),
                               _lib.dptr(qold), _lib.dptr(out), _lib.dptr(auxa) if maux else None,
                               float(dx), float(dy), float(dt),
                               _lib.iptr(method), _lib.iptr(mthlim), _lib.dptr(cfl), int(bool(fwave)),
                               rp.rp_id, _lib.dptr(cp), len(cp)))
    return out, float(cfl[0])


def step2ds(maxm, num_ghost, mx, my, qold, qnew, aux, dx, dy, dt, method, mthlim, aux1=None, aux2=None,
            aux3=None, work=None, ids=1, fwave=False, rpn2=None, rpt2=None):
    """One sweep of the split step (step2ds.f90); returns (qnew, cfl)."""
    rp = _solver(rpn2)
    lib = _lib.load()
    if qold is qnew:
        qold = np.array(qold, dtype=np.float64, order='F', copy=True)
    qold, out, method, mthlim = _prep(qold, qnew, method, mthlim)
    meqn = qold.shape[0]
    cfl = np.zeros(1)
    cp = _cparam_vector(rp)
    maux, auxa = _aux(aux, rp, method)
    _lib.check(lib.claw2_step2ds(int(maxm), meqn, len(mthlim), maux, int(num_ghost), int(mx), int(my),
                                 _lib.dptr(qold), _lib.dptr(out), _lib.dptr(auxa) if maux else None,
                                 float(dx), float(dy), float(dt),
                                 _lib.iptr(method), _lib.iptr(mthlim), _lib.dptr(cfl), int(ids),
                                 int(bool(fwave)), rp.rp_id, _lib.dptr(cp), len(cp)))
    return out, float(cfl[0])


def bc_fill(qbc, bc_lower, bc_upper):
    """Ghost-cell fill of a host qbc array (solver.py:351-519), in place."""
    lib = _lib.load()
    assert qbc.dtype == np.float64 and qbc.flags.f_contiguous
    meqn, nx, ny = qbc.shape
    bl = np.ascontiguousarray(bc_lower, dtype=np.intc)
    bu = np.ascontiguousarray(bc_upper, dtype=np.intc)
    _lib.check(lib.claw2_bc_fill(meqn, 2, nx - 4, ny - 4, _lib.dptr(qbc), _lib.iptr(bl), _lib.iptr(bu)))
    return qbc
