"""Classic Clawpack solvers with a CUDA kernel language.

Host mirror of src/pyclaw/classic/solver.py: ClawSolver (:19-234) and
ClawSolver2D (:393-549).  ``kernel_language = 'CUDA'`` (the default here, and
the only language of this package) runs each hyperbolic step on the GPU
through the C ABI of include/claw2.h: ghost-cell fill, the unsplit step2 (or
the split step2ds pair) and the CFL reduction all happen on the device, and q
stays there between steps.
"""
import numpy as np

from .limiters import tvd
from .solver import BC, AttemptBudget, CFLError, Solver
from . import _lib
from . import hostbc as _hostbc


class ClawSolver(Solver):
    """Generic classic solver (classic/solver.py:19-234)."""

    def __init__(self, riemann_solver=None, claw_package=None):
        self.num_ghost = 2
        self.limiters = tvd.minmod
        self.order = 2
        self.source_split = 1
        self.fwave = False
        self.step_source = None
        self.kernel_language = 'CUDA'
        self.verbosity = 0
        self.cfl_max = 1.0
        self.cfl_desired = 0.9
        self._mthlim = self.limiters
        self._method = None
        self.dt_old = None
        super(ClawSolver, self).__init__(riemann_solver, claw_package)

    def step(self, solution, take_one_step, tstart, tend):
        """classic/solver.py:96-146."""
        self.get_dt(solution.t, tstart, tend, take_one_step)
        self.cfl.set_global_max(0.)
        if self.source_split == 2 and self.step_source is not None:
            self.step_source(self, solution.states[0], self.dt / 2.0)
        self.step_hyperbolic(solution)
        if self.cfl.get_cached_max() >= self.cfl_max:
            return False
        if self.step_source is not None:
            if self.source_split == 2:
                self.step_source(self, solution.states[0], self.dt / 2.0)
            if self.source_split == 1:
                self.step_source(self, solution.states[0], self.dt)
        return True

    def _check_cfl_settings(self):
        pass

    def _set_mthlim(self):
        """classic/solver.py:162-171."""
        self._mthlim = self.limiters
        if not isinstance(self.limiters, list):
            self._mthlim = [self._mthlim]
        if len(self._mthlim) == 1:
            self._mthlim = self._mthlim * self.num_waves
        if len(self._mthlim) != self.num_waves:
            raise Exception('Length of solver.limiters is not equal to 1 or to solver.num_waves')

    def _set_method(self, state):
        """method[7] as classic/solver.py:173-193 builds it."""
        import numpy as np
        self._method = np.empty(7, dtype=int, order='F')
        self._method[0] = self.dt_variable
        self._method[1] = self.order
        if self.num_dim == 1:
            self._method[2] = 0
        elif self.dimensional_split:
            self._method[2] = -1
        else:
            self._method[2] = self.transverse_waves
        self._method[3] = self.verbosity
        self._method[4] = 0
        self._method[5] = state.index_capa + 1
        self._method[6] = state.num_aux

    def step_hyperbolic(self, solution):
        raise Exception("Dummy routine, please override!")


class ClawSolver2D(ClawSolver):
    """2D classic solver (classic/solver.py:393-549)."""

    no_trans = 0
    trans_inc = 1
    trans_cor = 2

    def __init__(self, riemann_solver=None, claw_package=None):
        self.dimensional_split = True
        self.transverse_waves = self.trans_inc
        self.num_dim = 2
        self.reflect_index = [1, 2]
        self.aux1 = None
        self.aux2 = None
        self.aux3 = None
        self.work = None
        self.device = 0
        self._dev = None
        self._aux_pushed = None  # the State.aux array last uploaded to the device
        self._aux_copy = None    # its contents then (kept when a before-step hook may edit it)
        self.device_time_loop = True  # evolve_to_time on the GPU when no host callback needs a step
        self._q_backup = None    # q before the host hooks of a step (before_step, step_source)
        self._committed = False  # the step's result is already current (a source step followed it)
        super(ClawSolver2D, self).__init__(riemann_solver, claw_package)

    def _check_cfl_settings(self):
        if (not self.dimensional_split) and (self.transverse_waves == 0):
            cfl_recommended = 0.5
        else:
            cfl_recommended = 1.0
        if self.cfl_max > cfl_recommended:
            import warnings
            warnings.warn('cfl_max is set higher than the recommended value of %s' % cfl_recommended)
            warnings.warn(str(self.cfl_desired))

    def setup(self, solution):
        """classic/solver.py:195-219 with the device patch in place of the f2py
        module, its workspace and the qbc arrays."""
        self._check_cfl_settings()
        self._set_mthlim()
        if self.kernel_language != 'CUDA':
            raise Exception("pyclaw_b200 runs kernel_language='CUDA' only (got %r)" % self.kernel_language)
        state = solution.states[0]
        self._set_method(state)
        self._check_bc_signatures()
        self._make_device_patch(solution)
        super(ClawSolver, self).setup(solution)

    def _check_bc_signatures(self):
        """A custom BC function with 5 arguments has the old signature
        (state, dim, t, array, num_ghost) (solver.py:328-339)."""
        import inspect
        for fun in (self.user_bc_lower, self.user_bc_upper, self.user_aux_bc_lower, self.user_aux_bc_upper):
            if fun is not None and len(inspect.getfullargspec(fun)[0]) == 5:
                self.logger.warning("The custom boundary condition function signature has been changed; "
                                    "the 5-argument form is deprecated.")
                self._use_old_bc_sig = True

    def _device_desc(self, solution):
        state = solution.states[0]
        grid = state.grid
        if self.rp is None or not hasattr(self.rp, 'rp_id'):
            raise Exception("ClawSolver2D needs a pyclaw_b200.riemann solver")
        need_aux = getattr(self.rp, 'num_aux', 0)
        if need_aux and state.num_aux < need_aux:
            raise ValueError("Riemann solver %s reads %d aux components per cell; state has num_aux=%d"
                             % (self.rp.name, need_aux, state.num_aux))
        if state.index_capa >= 0 and state.index_capa >= state.num_aux:
            raise ValueError("index_capa=%d names no component of the aux array (num_aux=%d)"
                             % (state.index_capa, state.num_aux))
        if self._device_aux(state):
            for b in list(self.aux_bc_lower) + list(self.aux_bc_upper):
                if b is None:
                    raise Exception('One of the aux boundary conditions has not been set.')
        for b in list(self.bc_lower) + list(self.bc_upper):
            if b is None:
                raise Exception('One of the boundary conditions has not been set.')
        d = _lib.Claw2Desc()
        d.mx, d.my = grid.num_cells
        d.num_eqn, d.num_waves = state.num_eqn, self.num_waves
        if state.num_eqn != self.rp.num_eqn:
            raise ValueError("state has num_eqn=%d, Riemann solver %s needs %d"
                             % (state.num_eqn, self.rp.name, self.rp.num_eqn))
        d.num_aux = state.num_aux if self._device_aux(state) else 0  # else State.aux is not read
        d.mcapa = state.index_capa + 1 if state.index_capa >= 0 else 0
        d.num_ghost = self.num_ghost
        d.riemann = self.rp.rp_id
        d.order = self.order
        d.transverse = int(self.transverse_waves)
        d.dimensional_split = 1 if self.dimensional_split else 0
        d.fwave = 1 if self.fwave else 0
        for k, v in enumerate(self._mthlim):
            d.mthlim[k] = int(v)
        if _hostbc.has_custom_q(self):
            # the host supplies every ghost cell each step (claw2_patch_upload_qbc)
            d.bc_lower[0] = d.bc_lower[1] = d.bc_upper[0] = d.bc_upper[1] = int(BC.extrap)
        else:
            d.bc_lower[0], d.bc_lower[1] = self.bc_lower
            d.bc_upper[0], d.bc_upper[1] = self.bc_upper
        d.dx, d.dy = grid.delta
        vals = self.rp.cparam(state.problem_data)
        for k, v in enumerate(vals):
            d.cparam[k] = v
        d.ncparam = len(vals)
        d.device = int(self.device)
        return d

    def _device_aux(self, state):
        """True when the device holds aux data: whenever the state has some
        (the Riemann solver, the capacity function or a device source step
        reads it)."""
        return state.num_aux > 0

    def _bc_shape(self, state, ncomp):
        return (ncomp,) + tuple(n + 2 * self.num_ghost for n in state.grid.num_cells)

    def _push_aux(self, state, force, auxbc=None):
        """Aux data to the device: State.aux with ghost cells filled on the
        device, or, with a custom BC, auxbc filled on the host every step
        (solver.py:351-437; given as ``auxbc`` when q's custom BCs filled it)
        and uploaded when it changed."""
        if not self._device_aux(state):
            return
        if auxbc is not None or _hostbc.needs_host_fill(self):
            if auxbc is not None:
                new = auxbc
            else:
                shape = self._bc_shape(state, state.num_aux)
                if self.auxbc is None or self.auxbc.shape != shape:
                    self.auxbc = np.zeros(shape, order='F')
                new = _hostbc.fill_auxbc(self, state, self.auxbc.copy(order='F'))
            if force or self._aux_pushed is None or not np.array_equal(new, self._aux_pushed):
                self._dev.push_auxbc(new)
            self.auxbc = new
            self._aux_pushed = new
        elif (force or state.aux is not self._aux_pushed or
              (self.before_step is not None and not np.array_equal(state.aux, self._aux_copy))):
            # a new State.aux array, or one a before-step hook edited in place
            self._dev.push_aux(state.aux, self.aux_bc_lower, self.aux_bc_upper)
            self._aux_pushed = state.aux
            self._aux_copy = state.aux.copy(order='F') if self.before_step is not None else None

    def _make_device_patch(self, solution):
        from .device import DevicePatch
        if self._dev is not None:
            self._dev.close()
        state = solution.states[0]
        self._dev = DevicePatch(self._device_desc(solution))
        state._mirror = self._dev
        self._dev.push(state)
        self._push_aux(state, force=True)

    # ---- per-step hooks ------------------------------------------------------
    def _begin_step(self, solution):
        """The device keeps the current q untouched until accept, so a plain
        step needs no backup.  Host hooks (before_step, step_source) may change
        q before or after the hyperbolic step; for them q is kept as it was
        before them, like the reference's q_backup (solver.py:610-612)."""
        self._q_backup = None
        if self.before_step is not None or self.step_source is not None:
            self._q_backup = solution.states[0]._read_q().copy(order='F')

    def _end_step(self, solution, accept):
        if not self._committed:
            self._dev.accept(accept)
        self._committed = False
        if not accept and self._q_backup is not None:
            solution.states[0].q = self._q_backup  # uploaded before the next step

    def _device_loop_ok(self, solution, tend):
        """The whole evolve_to_time can run on the GPU: a target time, no host
        callback between steps (before_step, step_source, gauges, custom BCs)
        and none of this class's stepping methods replaced by a subclass."""
        cls = type(self)
        return (self.device_time_loop and tend is not None and self.before_step is None and
                self.step_source is None and not solution.state.grid.gauges and
                not _hostbc.has_custom_q(self) and not _hostbc.needs_host_fill(self) and
                cls.step is ClawSolver2D.step and cls.step_hyperbolic is ClawSolver2D.step_hyperbolic and
                cls._begin_step is ClawSolver2D._begin_step and cls._end_step is ClawSolver2D._end_step and
                cls.get_dt is ClawSolver2D.get_dt and cls.accept_reject_step is ClawSolver2D.accept_reject_step)

    def evolve_to_time(self, solution, tend=None):
        """solver.py:554-666.  Without host callbacks between steps the loop
        runs on the GPU (claw2_patch_evolve: the same get_dt, CFL test,
        accept/reject and dt sequence, the host waiting only every few dozen
        steps); otherwise the host loop."""
        if not self._device_loop_ok(solution, tend):
            return super(ClawSolver2D, self).evolve_to_time(solution, tend)
        if not self._is_set_up:
            self.setup(solution)
        tstart = solution.t
        budget = AttemptBudget(self, tstart, tend)
        state = solution.states[0]
        dev = self._dev
        if dev is None or state._mirror is not dev:
            self._make_device_patch(solution)
            dev = self._dev
        if dev.host_dirty:
            dev.push(state)
        self._push_aux(state, force=False)
        es = _lib.Claw2EvolveState(
            t=solution.t, tstart=tstart, tend=tend, dt=self.dt, cfl=self.cfl.get_cached_max(),
            cfl_desired=self.cfl_desired, cfl_max=self.cfl_max, dt_max=self.dt_max,
            dtmin=self.status['dtmin'], dtmax=self.status['dtmax'], cflmax=self.status['cflmax'],
            dt_variable=1 if self.dt_variable else 0, dt_old_set=0 if self.dt_old is None else 1,
            max_steps=budget.count)
        rc = dev.evolve(es)
        if es.attempts > 0:
            solution.t = es.t
            self.dt = es.dt
            self.cfl.set_global_max(es.cfl)
            if es.dt_old_set and self.dt_old is None:
                self.dt_old = self.dt
            self.status['dtmin'] = es.dtmin
            self.status['dtmax'] = es.dtmax
            self.status['cflmax'] = es.cflmax
            self.status['numsteps'] += es.num_steps
        _lib.check(rc)
        if es.cfl_error:
            self.accept_step = False
            raise CFLError("Courant number %.17g above cfl_max = %g with a fixed dt of %.17g"
                           % (float(es.cfl), self.cfl_max, float(self.dt)))
        self.accept_step = True
        budget.check_finished(self, solution.t, tend, es.num_steps)
        return self.status

    def step(self, solution, take_one_step, tstart, tend):
        """classic/solver.py:96-146.  With a source step the hyperbolic result
        is committed on the device first (the source acts on it; a rejected
        step restores the backup), and a LinearSource runs on the device."""
        self._committed = False
        if self.step_source is None:
            return super(ClawSolver2D, self).step(solution, take_one_step, tstart, tend)
        state = solution.states[0]
        self.get_dt(solution.t, tstart, tend, take_one_step)
        self.cfl.set_global_max(0.)
        if self.source_split == 2:
            self.step_source(self, state, self.dt / 2.0)
        self.step_hyperbolic(solution)
        if self.cfl.get_cached_max() >= self.cfl_max:
            return False
        self._dev.accept(True)
        self._committed = True
        if self.source_split == 2:
            self.step_source(self, state, self.dt / 2.0)
        if self.source_split == 1:
            self.step_source(self, state, self.dt)
        return True

    def step_hyperbolic(self, solution):
        """classic/solver.py:498-549 on the device: BC fill + step2 (or the
        step2ds pair) + CFL; the result is pending until accepted."""
        state = solution.states[0]
        dev = self._dev
        if dev is None or state._mirror is not dev:
            self._make_device_patch(solution)
            dev = self._dev
        if dev.host_dirty:
            dev.push(state)
        if _hostbc.has_custom_q(self):
            # custom q BCs: every ghost cell (q and aux) filled on the host
            shape = self._bc_shape(state, state.num_eqn)
            if self.qbc is None or self.qbc.shape != shape:
                self.qbc = np.zeros(shape, order='F')
            auxbc = None
            if state.num_aux > 0:
                ashape = self._bc_shape(state, state.num_aux)
                auxbc = (self.auxbc if self.auxbc is not None and self.auxbc.shape == ashape
                         else np.zeros(ashape, order='F')).copy(order='F')
            _hostbc.fill_bcs(self, state, self.qbc, auxbc)
            dev.upload_qbc(self.qbc)
            self._push_aux(state, force=False, auxbc=auxbc if self._device_aux(state) else None)
            if auxbc is not None:
                self.auxbc = auxbc
        else:
            self._push_aux(state, force=False)  # a new State.aux array, or custom aux BCs
        cfl = dev.step(self.dt)
        self.cfl.update_global_max(cfl)

    def __del__(self):
        if getattr(self, '_dev', None) is not None:
            self._dev.close()
        self._is_set_up = False
