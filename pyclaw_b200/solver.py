"""Time-step control of the CUDA solvers: the attempt loop, accept/reject, the
dt rule, gauges and the boundary-condition codes.

What a drop-in must reproduce is the sequence of attempts a run makes, since
that fixes every dt and therefore every result: the next dt follows from the
last Courant number (src/pyclaw/solver.py:531-552), it is clipped to the target
time, an attempt whose Courant number exceeds cfl_max is rejected and retaken
with the smaller dt, and a fixed dt must divide the interval (:574-594).  Those
rules are the functions `next_dt`, `clip_to_target` and the `AttemptBudget`
below.  The loop around them is this package's own: q stays on the GPU, so the
backup the reference copies before every attempt (:610-612) is a buffer the
device already keeps (`_begin_step` / `_end_step`, implemented by the CUDA
solver as accept = buffer swap), and a run with no host callback between
steps never enters this loop at all -- ClawSolver2D.evolve_to_time hands it,
with the same budget, to the device time loop (claw2_patch_evolve).
"""
import logging

import numpy as np


class CFLError(Exception):
    """A fixed-dt attempt broke cfl_max: the run cannot continue (the
    reference raises a plain Exception there, solver.py:646-650)."""


class BC():
    """Boundary-condition codes of the solver's bc_lower/bc_upper lists
    (solver.py:13-19; the numbers are the ones the C ABI takes)."""
    custom = 0
    extrap = 1
    periodic = 2
    wall = 3


def default_compute_gauge_values(q, aux):
    return q


def before_step(solver, solution):
    pass


# ---- the dt rules -----------------------------------------------------------
def next_dt(dt, cfl, cfl_desired, dt_max):
    """dt of the next attempt after one of Courant number `cfl`: scaled to
    cfl_desired (solver.py:531-533, same operation order), or dt_max when
    nothing moved (cfl == 0, :541-542)."""
    if cfl > 0.0:
        return min(dt_max, dt * cfl_desired / cfl)
    return dt_max


def clip_to_target(dt, t, tstart, tend):
    """Never step past tend, and take the remainder rather than leave a
    sliver below 1e-14 t before it (solver.py:547-551)."""
    if tstart < tend and t + dt > tend:
        dt = tend - t
    if tend - t - dt < 1.e-14 * t:
        dt = tend - t
    return dt


class AttemptBudget(object):
    """The attempts one evolve_to_time call may make, checked before the first
    one (solver.py:574-595).  A fixed dt allows exactly (tend - tstart) / dt of
    them and must divide the interval; a variable dt needs cfl_desired <=
    cfl_max (otherwise no attempt could be accepted) and may use max_steps; a
    target at or before the start allows none.  As in the reference the count
    is stored in solver.max_steps, where later calls see it."""

    def __init__(self, solver, tstart, tend):
        self.one_step = tend is None
        count = solver.max_steps
        if not solver.dt_variable:
            if self.one_step:
                count = 1
            else:
                span = tend - tstart
                count = int((span + 1e-10) / solver.dt)
                if abs(count * solver.dt - span) > 1e-5 * span:
                    raise Exception("a fixed dt of %.17g does not divide the interval %.17g -> %.17g "
                                    "(dt_variable is False)" % (float(solver.dt), float(tstart), float(tend)))
        if solver.dt_variable == 1 and solver.cfl_desired > solver.cfl_max:
            raise Exception("cfl_desired = %g is above cfl_max = %g: with a variable dt every attempt "
                            "would be rejected" % (solver.cfl_desired, solver.cfl_max))
        if not self.one_step and tend <= tstart:
            solver.logger.info("target time %r is not after the current time %r: nothing to do",
                               tend, tstart)
            count = 0
        solver.max_steps = count
        self.count = count

    def check_finished(self, solver, t, tend, accepted):
        """A variable-dt run that used its whole budget short of tend fails
        (solver.py:662-665)."""
        if not self.one_step and solver.dt_variable and t < tend and accepted == self.count:
            raise Exception("max_steps = %d steps taken, stopped at t = %.17g short of tend = %.17g"
                            % (self.count, float(t), float(tend)))


class Solver(object):
    """Solver base (the attribute surface of solver.py:32-242).

    Attributes are fixed once __init__ has run: assigning a name the solver
    does not have raises TypeError, so a misspelt option fails at once
    instead of being ignored."""

    def __setattr__(self, key, value):
        if self.__dict__.get('_frozen', False) and not hasattr(self, key):
            raise TypeError("%s has no option %r (misspelt?)" % (type(self).__name__, key))
        object.__setattr__(self, key, value)

    @property
    def all_bcs(self):
        return self.bc_lower, self.bc_upper

    @all_bcs.setter
    def all_bcs(self, code):
        for d in range(self.num_dim):
            self.bc_lower[d] = code
            self.bc_upper[d] = code

    def __init__(self, riemann_solver=None, claw_package=None):
        from .cfl import CFL
        nd = self.num_dim
        defaults = dict(
            logger=logging.getLogger('pyclaw.solver'),
            dt_initial=0.1, dt_max=1e99, max_steps=10000, dt_variable=True,
            num_eqn=None, num_waves=None, fwave=None, rp=None, fmod=None,
            qbc=None, auxbc=None, accept_step=True, before_step=None,
            user_bc_lower=None, user_bc_upper=None, user_aux_bc_lower=None, user_aux_bc_upper=None,
            compute_gauge_values=default_compute_gauge_values,
            _is_set_up=False, _use_old_bc_sig=False)
        for k, v in defaults.items():
            object.__setattr__(self, k, v)
        self.bc_lower, self.bc_upper = [None] * nd, [None] * nd
        self.aux_bc_lower, self.aux_bc_upper = [None] * nd, [None] * nd
        self.dt = self.dt_initial
        self.cfl = CFL(self.cfl_desired)
        self.status = {'cflmax': -np.inf, 'dtmin': np.inf, 'dtmax': -np.inf, 'numsteps': 0}
        if riemann_solver is not None:
            self._adopt_riemann(riemann_solver)
        self._frozen = True

    def _adopt_riemann(self, rp):
        """num_eqn, num_waves and fwave from the solver tables, keyed by the
        module's last name with any '_ptwise' dropped (solver.py:230-238)."""
        from . import riemann
        name = rp.__name__.split('.')[-1].replace("_ptwise", "")
        self.rp = rp
        self.num_eqn = riemann.static.num_eqn.get(name)
        self.num_waves = riemann.static.num_waves.get(name)
        self.fwave = riemann.static.fwave.get(name)

    def is_valid(self):
        """(valid, reason): every setting a run needs is present
        (solver.py:262-293).  The reason names the first missing one."""
        missing = []
        for side, codes, fn in (("lower", self.bc_lower, self.user_bc_lower),
                                ("upper", self.bc_upper, self.user_bc_upper)):
            if any(b == BC.custom for b in codes) and fn is None:
                missing.append("a %s boundary is BC.custom but user_bc_%s is not set" % (side, side))
        for name in ('num_waves', 'num_eqn', 'fwave'):
            if getattr(self, name) is None:
                missing.append("solver.%s is not set" % name)
        if None in self.bc_lower or None in self.bc_upper:
            missing.append("bc_lower/bc_upper has an unset entry")
        reason = missing[0] if missing else None
        if reason is not None:
            self.logger.debug(reason)
        return reason is None, reason

    def setup(self, solution):
        self._is_set_up = True

    def __del__(self):
        self._is_set_up = False

    def __str__(self):
        return "Solver Status:\n" + "\n".join("%25s = %s" % (k, v) for k, v in self.status.items())

    # ---- dt and the accept test -------------------------------------------
    def accept_reject_step(self, state):
        """Accept an attempt whose Courant number is within cfl_max."""
        return not (self.cfl.get_cached_max() > self.cfl_max)

    def get_dt_new(self):
        self.dt = next_dt(self.dt, self.cfl.get_cached_max(), self.cfl_desired, self.dt_max)

    def get_dt(self, t, tstart, tend, take_one_step):
        """dt for the coming attempt (solver.py:535-552): the first call of a
        variable-dt solver keeps dt (and records it as dt_old); later calls
        scale it by the last Courant number; a run to a target time is then
        clipped to it."""
        if self.dt_variable and self.dt_old is not None:
            cfl = self.cfl.get_cached_max()
            self.dt = next_dt(self.dt, cfl, self.cfl_desired, self.dt_max)
            if cfl > 0.0:
                self.status['dtmin'] = min(self.dt, self.status['dtmin'])
                self.status['dtmax'] = max(self.dt, self.status['dtmax'])
        else:
            self.dt_old = self.dt
        if not take_one_step:
            self.dt = clip_to_target(self.dt, t, tstart, tend)

    # ---- the attempt loop --------------------------------------------------
    def _begin_step(self, solution):
        """Keep what a rejected attempt must restore (the CUDA solver keeps
        the old q on the device; nothing to copy)."""

    def _end_step(self, solution, accept):
        """Commit or drop the attempt just taken."""

    def evolve_to_time(self, solution, tend=None):
        """Advance `solution` to `tend`, or by one accepted-or-rejected attempt
        when tend is None (solver.py:554-666).  Returns the status dict."""
        if not self._is_set_up:
            self.setup(solution)
        tstart = solution.t
        budget = AttemptBudget(self, tstart, tend)
        accepted = 0
        for n in range(budget.count):
            accepted += self._attempt(solution, n, tstart, tend, budget.one_step)
            if budget.one_step or solution.t >= tend:
                break
        budget.check_finished(self, solution.t, tend, accepted)
        return self.status

    def _attempt(self, solution, n, tstart, tend, one_step):
        """One attempt: hooks, the step (which picks dt), the Courant test,
        then commit (t advanced, gauges written) or roll back.  Returns 1 when
        accepted; a rejected fixed-dt attempt raises CFLError."""
        if self.dt_variable:
            self._begin_step(solution)
        if self.before_step is not None:
            self.before_step(self, solution.states[0])
        self.step(solution, one_step, tstart, tend)
        cfl = self.cfl.get_cached_max()
        self.accept_step = self.accept_reject_step(solution.state)
        self._end_step(solution, self.accept_step)
        if not self.accept_step:
            self.logger.debug("attempt %d rejected: Courant number %g > %g", n, cfl, self.cfl_max)
            if self.dt_variable:
                return 0
            self.status['cflmax'] = max(cfl, self.status['cflmax'])
            raise CFLError("Courant number %.17g above cfl_max = %g with a fixed dt of %.17g"
                           % (float(cfl), self.cfl_max, float(self.dt)))
        self.status['cflmax'] = max(cfl, self.status['cflmax'])
        # a fixed dt advances by whole multiples of dt from tstart (no drift)
        solution.t = solution.t + self.dt if self.dt_variable else tstart + (n + 1) * self.dt
        self.logger.debug("attempt %d accepted: Courant number %g, dt %g, t %g", n, cfl, self.dt, solution.t)
        self.write_gauge_values(solution)
        self.status['numsteps'] += 1
        return 1

    def step(self, solution, take_one_step, tstart, tend):
        raise NotImplementedError("%s defines no step()" % type(self).__name__)

    # ---- gauges -------------------------------------------------------------
    def write_gauge_values(self, solution):
        """One line per gauge and accepted step: t followed by
        compute_gauge_values(q, aux) at the gauge's cell, appended to the
        gauge's file and (keep_gauges) to state.gauge_data, in the
        reference's line format (solver.py:680-715).  The gauge cells' q is
        gathered on the device in one call."""
        state = solution.state
        cells = [tuple(g) for g in state.grid.gauges]
        if not cells:
            return
        t = solution.t
        qg = state.gauge_q(cells)
        data = state.gauge_data
        first = len(data) != len(cells)
        files = state.grid.gauge_files
        for i, (ix, iy) in enumerate(cells):
            aux = state.aux[:, ix, iy] if state.num_aux > 0 else None
            vals = self.compute_gauge_values(qg[i], aux)
            vals = list(vals) if hasattr(vals, '__iter__') else [vals]
            row = np.append(t, vals)
            if state.keep_gauges:
                if first:
                    data.append(row)
                else:
                    data[i] = np.vstack((data[i], row))
            if i >= len(files):
                raise Exception("gauge %d has no open file: call grid.setup_gauge_files(outdir) "
                                "before stepping" % i)
            files[i].write(" ".join([str(t)] + [str(v) for v in vals]) + "\n")
