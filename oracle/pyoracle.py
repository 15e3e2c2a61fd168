"""Python access to the CPU oracle (TEST INFRASTRUCTURE ONLY).

The oracle restates the reference's classic 2D kernels in C++
(oracle/claw_oracle.cpp; see its header for the file:line map).  This module
loads it with ctypes and provides ``OracleClawSolver2D``, a ClawSolver2D whose
step_hyperbolic is the reference's host algorithm
(src/pyclaw/classic/solver.py:498-549: ghost fill, ``qold = qbc.copy('F')``,
step2 or the step2ds pair, CFL update, ``set_q_from_qbc``) on host arrays, and
whose reject path restores a host backup like src/pyclaw/solver.py:610-645.
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libclaw_oracle.so")

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        build()
    lib = ctypes.CDLL(LIB_PATH)
    i = ctypes.c_int
    d = ctypes.c_double
    lib.oracle_step2.argtypes = [i] * 7 + [_dp, _dp, _dp, d, d, d, _ip, _ip, _dp, i, i, _dp]
    lib.oracle_step2ds.argtypes = [i] * 7 + [_dp, _dp, _dp, d, d, d, _ip, _ip, _dp, i, i, i, _dp]
    lib.oracle_bc_fill.argtypes = [i, i, i, i, _dp, _ip, _ip]
    lib.oracle_bc_fill_aux.argtypes = [i, i, i, i, _dp, _ip, _ip]
    lib.oracle_rpn2_aux.argtypes = [i] * 8 + [_dp] * 7
    lib.oracle_rpt2_aux.argtypes = [i] * 9 + [_dp] * 8
    lib.oracle_rpn2.argtypes = [i] * 7 + [_dp, _dp, _dp, _dp, _dp, _dp, _dp]
    lib.oracle_rpt2.argtypes = [i] * 8 + [_dp, _dp, _dp, _dp, _dp, _dp]
    lib.oracle_exact_star.argtypes = [d] * 8 + [i, _dp, _dp, _ip]
    lib.oracle_rpn2.argtypes = [i] * 7 + [_dp] * 7
    lib.oracle_set_threads.argtypes = [i]
    lib.oracle_set_threads.restype = None
    _lib = lib
    return lib


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return np.ascontiguousarray(a, dtype=np.intc).ctypes.data_as(_ip)


def set_threads(n):
    load().oracle_set_threads(int(n))


def step2(qold, qnew, dx, dy, dt, method, mthlim, rp_id, cparam, use_fwave=False, aux=None):
    """Oracle step2 on qbc arrays (meqn, mx+4, my+4) F-order, optional auxbc
    (maux, mx+4, my+4) F-order; returns cfl."""
    lib = load()
    meqn, nxg, nyg = qold.shape
    mx, my = nxg - 4, nyg - 4
    maux, auxp = _aux(aux)
    cfl = ctypes.c_double(0.0)
    cp = np.asarray(list(cparam) + [0.0] * 8, dtype=np.float64)
    method = np.ascontiguousarray(method, dtype=np.intc)
    mthlim = np.ascontiguousarray(mthlim, dtype=np.intc)
    rc = lib.oracle_step2(max(mx, my), meqn, len(mthlim), maux, 2, mx, my, _d(qold), _d(qnew), auxp,
                          dx, dy, dt, _i(method), _i(mthlim), ctypes.byref(cfl), int(use_fwave),
                          rp_id, _d(cp))
    if rc:
        raise RuntimeError("oracle_step2 returned %d" % rc)
    return cfl.value


def step2ds(qold, qnew, dx, dy, dt, method, mthlim, ids, rp_id, cparam, use_fwave=False, aux=None):
    lib = load()
    meqn, nxg, nyg = qold.shape
    mx, my = nxg - 4, nyg - 4
    maux, auxp = _aux(aux)
    cfl = ctypes.c_double(0.0)
    cp = np.asarray(list(cparam) + [0.0] * 8, dtype=np.float64)
    method = np.ascontiguousarray(method, dtype=np.intc)
    mthlim = np.ascontiguousarray(mthlim, dtype=np.intc)
    rc = lib.oracle_step2ds(max(mx, my), meqn, len(mthlim), maux, 2, mx, my, _d(qold), _d(qnew), auxp,
                            dx, dy, dt, _i(method), _i(mthlim), ctypes.byref(cfl), ids, int(use_fwave),
                            rp_id, _d(cp))
    if rc:
        raise RuntimeError("oracle_step2ds returned %d" % rc)
    return cfl.value


def _aux(aux):
    if aux is None:
        return 0, None
    assert aux.flags.f_contiguous and aux.dtype == np.float64
    return aux.shape[0], _d(aux)


def bc_fill_aux(auxbc, bc_lower, bc_upper):
    """Ghost cells of an aux array (a wall mirrors without sign change)."""
    lib = load()
    maux, nxg, nyg = auxbc.shape
    assert auxbc.flags.f_contiguous
    rc = lib.oracle_bc_fill_aux(maux, 2, nxg - 4, nyg - 4, _d(auxbc), _i(bc_lower), _i(bc_upper))
    if rc:
        raise RuntimeError("oracle_bc_fill_aux returned %d" % rc)


def bc_fill(qbc, bc_lower, bc_upper):
    lib = load()
    meqn, nxg, nyg = qbc.shape
    assert qbc.flags.f_contiguous
    rc = lib.oracle_bc_fill(meqn, 2, nxg - 4, nyg - 4, _d(qbc), _i(bc_lower), _i(bc_upper))
    if rc:
        raise RuntimeError("oracle_bc_fill returned %d" % rc)


def _rule(kind, arr, ng, lower, reflect):
    """One built-in rule on one side (solver.py:439-519); arr has the
    dimension on axis 1; reflect = the component a wall negates, or None."""
    from pyclaw_b200.solver import BC
    if kind == BC.extrap:
        for i in range(ng):
            if lower:
                arr[:, i, ...] = arr[:, ng, ...]
            else:
                arr[:, -i - 1, ...] = arr[:, -ng - 1, ...]
    elif kind == BC.periodic:
        if lower:
            arr[:, :ng, ...] = arr[:, -2 * ng:-ng, ...]
        else:
            arr[:, -ng:, ...] = arr[:, ng:2 * ng, ...]
    elif kind == BC.wall:
        for i in range(ng):
            src = 2 * ng - 1 - i if lower else -2 * ng + i
            dst = i if lower else -i - 1
            arr[:, dst, ...] = arr[:, src, ...]
            if reflect is not None:
                arr[reflect, dst, ...] = -arr[reflect, src, ...]
    else:
        raise NotImplementedError("boundary condition %r" % (kind,))


def apply_bcs(solver, state, qbc, auxbc):
    """Solver._apply_bcs (src/pyclaw/solver.py:351-437) for q and aux:
    interiors from the state, then per dimension the lower and the upper side,
    on each side aux before q, a user function for BC.custom (called with the
    host qbc and auxbc), else the built-in rule.  qbc or auxbc may be None."""
    from pyclaw_b200.solver import BC
    ng = 2
    if qbc is not None:
        qbc[:, ng:-ng, ng:-ng] = state._q
    if auxbc is not None:
        auxbc[:, ng:-ng, ng:-ng] = state.aux
    for idim, dim in enumerate(state.grid.dimensions):
        for lower in (True, False):
            items = []
            if auxbc is not None:
                items.append((auxbc, solver.aux_bc_lower if lower else solver.aux_bc_upper,
                              solver.user_aux_bc_lower if lower else solver.user_aux_bc_upper, None))
            if qbc is not None:
                items.append((qbc, solver.bc_lower if lower else solver.bc_upper,
                              solver.user_bc_lower if lower else solver.user_bc_upper, solver.reflect_index[idim]))
            for arr, kinds, fun, reflect in items:
                if kinds[idim] == BC.custom:
                    fun(state, dim, state.t, qbc, auxbc, ng)
                else:
                    _rule(kinds[idim], np.rollaxis(arr, idim + 1, 1), ng, lower, reflect)


def apply_aux_bcs(solver, state, auxbc):
    """apply_bcs for the aux array alone (a custom function gets qbc = None)."""
    apply_bcs(solver, state, None, auxbc)
    return auxbc


def make_solver_class():
    """ClawSolver2D running the oracle on host arrays (built lazily so that
    importing this module does not import the product package)."""
    from pyclaw_b200.classic import ClawSolver, ClawSolver2D

    class OracleClawSolver2D(ClawSolver2D):
        def __init__(self, riemann_solver=None, claw_package=None):
            self._backup = None
            super().__init__(riemann_solver, claw_package)

        def step(self, solution, take_one_step, tstart, tend):
            # classic/solver.py:96-146 on host arrays: the source step acts on
            # state.q, which step_hyperbolic has already replaced
            return ClawSolver.step(self, solution, take_one_step, tstart, tend)

        def setup(self, solution):
            self._check_cfl_settings()
            self._set_mthlim()
            state = solution.states[0]
            self._set_method(state)
            mx, my = state.grid.num_cells
            self.qbc = np.zeros((state.num_eqn, mx + 4, my + 4), order='F')
            self.auxbc = np.zeros((state.num_aux, mx + 4, my + 4), order='F') if state.num_aux else None
            self._is_set_up = True

        def _begin_step(self, solution):
            self._backup = solution.state._q.copy('F')

        def _end_step(self, solution, accept):
            if not accept:
                solution.state._q = self._backup

        def step_hyperbolic(self, solution):
            state = solution.states[0]
            dx, dy = state.grid.delta
            qbc = self.qbc
            aux = self.auxbc
            custom = any(b == 0 for b in list(self.bc_lower) + list(self.bc_upper) +
                         (list(self.aux_bc_lower) + list(self.aux_bc_upper) if aux is not None else []))
            if custom:  # user functions (BC.custom): the reference's order, in numpy
                apply_bcs(self, state, qbc, aux)
            else:  # solver.py:351-437 fills qbc and auxbc every step
                qbc[:, 2:-2, 2:-2] = state._q
                bc_fill(qbc, self.bc_lower, self.bc_upper)
                if aux is not None:
                    aux[:, 2:-2, 2:-2] = state.aux
                    bc_fill_aux(aux, self.aux_bc_lower, self.aux_bc_upper)
            qold = qbc.copy('F')
            cp = self.rp.cparam(state.problem_data)
            fw = bool(self.fwave)
            if self.dimensional_split:
                c1 = step2ds(qold, qbc, dx, dy, self.dt, self._method, self._mthlim, 1, self.rp.rp_id, cp, fw,
                             aux=aux)
                c2 = step2ds(qbc, qbc, dx, dy, self.dt, self._method, self._mthlim, 2, self.rp.rp_id, cp, fw,
                             aux=aux)
                cfl = max(c1, c2)
            else:
                cfl = step2(qold, qbc, dx, dy, self.dt, self._method, self._mthlim, self.rp.rp_id, cp, fw, aux=aux)
            self.cfl.update_global_max(cfl)
            state._q = np.asfortranarray(qbc[:, 2:-2, 2:-2].copy())

    return OracleClawSolver2D
