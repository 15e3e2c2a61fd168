"""Solver base class: time-step control, accept/reject and the BC enumeration.

Host mirror of src/pyclaw/solver.py.  The dt rules (get_dt :535-552,
get_dt_new :531-533, accept_reject_step :524-529) and the evolve_to_time loop
(:554-666) follow the reference line for line.  Two hooks replace the
reference's host copies: ``_begin_step`` (its ``q_backup = state.q.copy('F')``,
:610-612) and ``_end_step(accept)`` (its ``state.q = q_backup`` on reject,
:641-645); the CUDA solver implements both as a buffer swap on the device.
"""
import logging

import numpy as np


class CFLError(Exception):
    """Raised when cfl_max is exceeded with a fixed time step (solver.py:7-11)."""

    def __init__(self, msg):
        super(CFLError, self).__init__(msg)


class BC():
    """Boundary-condition names (solver.py:13-19)."""
    custom = 0
    extrap = 1
    periodic = 2
    wall = 3


def default_compute_gauge_values(q, aux):
    return q


def before_step(solver, solution):
    pass


class Solver(object):
    """Abstract solver; see ClawSolver2D (solver.py:32-242)."""

    def __setattr__(self, key, value):
        # reject attributes that do not exist once initialised (solver.py:139-144)
        if not hasattr(self, '_isinitialized'):
            self.__dict__['_isinitialized'] = False
        if self._isinitialized and not hasattr(self, key):
            raise TypeError("%s has no attribute %s" % (self.__class__, key))
        object.__setattr__(self, key, value)

    @property
    def all_bcs(self):
        return self.bc_lower, self.bc_upper

    @all_bcs.setter
    def all_bcs(self, all_bcs):
        for i in range(self.num_dim):
            self.bc_lower[i] = all_bcs
            self.bc_upper[i] = all_bcs

    def __init__(self, riemann_solver=None, claw_package=None):
        from .cfl import CFL
        self.logger = logging.getLogger('pyclaw.solver')
        self.dt_initial = 0.1
        self.dt_max = 1e99
        self.max_steps = 10000
        self.dt_variable = True
        self.num_waves = None
        self.qbc = None
        self.auxbc = None
        self.rp = None
        self.fmod = None
        self._is_set_up = False
        self._use_old_bc_sig = False
        self.accept_step = True
        self.before_step = None
        self.dt = self.dt_initial
        self.cfl = CFL(self.cfl_desired)
        self.status = {'cflmax': -np.inf, 'dtmin': np.inf, 'dtmax': -np.inf, 'numsteps': 0}
        self.bc_lower = [None] * self.num_dim
        self.bc_upper = [None] * self.num_dim
        self.aux_bc_lower = [None] * self.num_dim
        self.aux_bc_upper = [None] * self.num_dim
        self.user_bc_lower = None
        self.user_bc_upper = None
        self.user_aux_bc_lower = None
        self.user_aux_bc_upper = None
        self.num_eqn = None
        self.num_waves = None
        self.fwave = None
        self.compute_gauge_values = default_compute_gauge_values
        if riemann_solver is not None:
            # num_eqn/num_waves/fwave from riemann.static (solver.py:230-238)
            from . import riemann
            self.rp = riemann_solver
            rp_name = riemann_solver.__name__.split('.')[-1]
            if "ptwise" in rp_name:
                rp_name = rp_name.replace("_ptwise", "")
            self.num_eqn = riemann.static.num_eqn.get(rp_name, None)
            self.num_waves = riemann.static.num_waves.get(rp_name, None)
            self.fwave = riemann.static.fwave.get(rp_name, None)
        self._isinitialized = True
        super(Solver, self).__init__()

    def is_valid(self):
        """Required-attribute checks (solver.py:262-293)."""
        valid, reason = True, None
        if any(b == BC.custom for b in self.bc_lower) and self.user_bc_lower is None:
            valid, reason = False, 'Lower custom BC function has not been set.'
        if any(b == BC.custom for b in self.bc_upper) and self.user_bc_upper is None:
            valid, reason = False, 'Upper custom BC function has not been set.'
        if self.num_waves is None:
            valid, reason = False, 'solver.num_waves has not been set.'
        if self.num_eqn is None:
            valid, reason = False, 'solver.num_eqn has not been set.'
        if self.fwave is None:
            valid, reason = False, 'solver.fwave has not been set.'
        if (None in self.bc_lower) or (None in self.bc_upper):
            valid, reason = False, 'One of the boundary conditions has not been set.'
        if reason is not None:
            self.logger.debug(reason)
        return valid, reason

    def setup(self, solution):
        self._is_set_up = True

    def __del__(self):
        self._is_set_up = False

    def __str__(self):
        out = "Solver Status:\n"
        for (k, v) in self.status.items():
            out = "\n".join((out, "%s = %s" % (k.rjust(25), v)))
        return out

    # ---- time stepping (solver.py:524-666) ---------------------------------
    def accept_reject_step(self, state):
        cfl = self.cfl.get_cached_max()
        if cfl > self.cfl_max:
            return False
        else:
            return True

    def get_dt_new(self):
        cfl = self.cfl.get_cached_max()
        self.dt = min(self.dt_max, self.dt * self.cfl_desired / cfl)

    def get_dt(self, t, tstart, tend, take_one_step):
        cfl = self.cfl.get_cached_max()
        if self.dt_variable and self.dt_old is not None:
            if cfl > 0.0:
                self.get_dt_new()
                self.status['dtmin'] = min(self.dt, self.status['dtmin'])
                self.status['dtmax'] = max(self.dt, self.status['dtmax'])
            else:
                self.dt = self.dt_max
        else:
            self.dt_old = self.dt
        if not take_one_step:
            if t + self.dt > tend and tstart < tend:
                self.dt = tend - t
            if tend - t - self.dt < 1.e-14 * t:
                self.dt = tend - t

    def _begin_step(self, solution):
        """Keep what a rejected step must restore (solver.py:610-612)."""

    def _end_step(self, solution, accept):
        """Commit or roll back the step just taken (solver.py:619-651)."""

    def evolve_to_time(self, solution, tend=None):
        if not self._is_set_up:
            self.setup(solution)
        take_one_step = tend is None
        tstart = solution.t
        num_steps = 0
        if not self.dt_variable:
            if take_one_step:
                self.max_steps = 1
            else:
                self.max_steps = int((tend - tstart + 1e-10) / self.dt)
                if abs(self.max_steps * self.dt - (tend - tstart)) > 1e-5 * (tend - tstart):
                    raise Exception('dt does not divide (tend-tstart) and dt is fixed!')
        if self.dt_variable == 1 and self.cfl_desired > self.cfl_max:
            raise Exception('Variable time-stepping and desired CFL > maximum CFL')
        if not take_one_step:
            if tend <= tstart:
                self.logger.info("Already at or beyond end time: no evolution required.")
                self.max_steps = 0

        for n in range(self.max_steps):
            state = solution.state
            if self.dt_variable:
                self._begin_step(solution)
                told = solution.t
            if self.before_step is not None:
                self.before_step(self, solution.states[0])
            self.step(solution, take_one_step, tstart, tend)
            cfl = self.cfl.get_cached_max()
            self.accept_step = self.accept_reject_step(state)
            if self.accept_step:
                self._end_step(solution, True)
                self.status['cflmax'] = max(cfl, self.status['cflmax'])
                if self.dt_variable:
                    solution.t += self.dt
                else:
                    solution.t = tstart + (n + 1) * self.dt
                self.logger.debug("Step %i  CFL = %f   dt = %f   t = %f" % (n, cfl, self.dt, solution.t))
                self.write_gauge_values(solution)
                num_steps += 1
                self.status['numsteps'] += 1
            else:
                self.logger.debug("Rejecting time step, CFL number too large")
                if self.dt_variable:
                    self._end_step(solution, False)
                    solution.t = told
                else:
                    self._end_step(solution, False)
                    self.status['cflmax'] = max(cfl, self.status['cflmax'])
                    raise CFLError('CFL too large, giving up!')
            if take_one_step:
                break
            elif solution.t >= tend:
                break

        if not take_one_step:
            if self.dt_variable and solution.t < tend and num_steps == self.max_steps:
                raise Exception("Maximum number of timesteps have been taken")
        return self.status

    def step(self, solution, take_one_step, tstart, tend):
        raise NotImplementedError("No stepping routine has been defined!")

    def write_gauge_values(self, solution):
        """Values of compute_gauge_values(q, aux) at every gauge cell, appended
        to state.gauge_data (keep_gauges) and to the gauge files
        (solver.py:680-715).  q at the gauge cells is gathered on the device."""
        state = solution.state
        gauges = state.grid.gauges
        if not gauges:
            return
        qg = state.gauge_q([tuple(g) for g in gauges])
        for i, (ix, iy) in enumerate(gauges):
            aux = state.aux[:, ix, iy] if state.num_aux > 0 else None
            p = self.compute_gauge_values(qg[i], aux)
            if not hasattr(p, '__iter__'):
                p = [p]
            t = solution.t
            if state.keep_gauges:
                gauge_data = state.gauge_data
                if len(gauge_data) == len(gauges):
                    gauge_data[i] = np.vstack((gauge_data[i], np.append(t, p)))
                else:
                    gauge_data.append(np.append(t, p))
            try:
                state.grid.gauge_files[i].write(str(t) + ' ' + ' '.join(str(j) for j in p) + '\n')
            except IOError:
                raise Exception("Gauge files are not set up correctly. You should call \nthe method "
                                "`setup_gauge_files` of the Grid class object \nbefore any call for "
                                "`write_gauge_values` from the Solver class.")
