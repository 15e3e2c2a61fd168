"""Source-term steps that run on the device.

The reference's ``solver.step_source`` is any Python function
``f(solver, state, dt)`` that updates ``state.q`` in place after the
hyperbolic step (Godunov splitting, ``source_split = 1``) or around it in two
half steps (Strang, ``source_split = 2``) (src/pyclaw/classic/solver.py:
126-144).  A plain function works with the CUDA solver too: ``state.q`` comes
to the host for it and goes back before the next step.  The classes here are
such functions whose work stays on the device when the state is there.

``LinearSource(M)``: q <- q + dt M q in every cell, M a (num_eqn, num_eqn)
matrix, the right-hand side evaluated with the q before the update (as a
forward-Euler source step does with ``qq = state.q.copy()``); for example the
reaction term of examples/advection_reaction_2d (advection_reaction.py:39-43)
is ``LinearSource([[0, eps], [eps, 0]])``.
"""
import numpy as np

from . import _lib


class LinearSource(object):
    def __init__(self, matrix):
        self.matrix = np.ascontiguousarray(np.atleast_2d(np.asarray(matrix, dtype=np.float64)))
        if self.matrix.shape[0] != self.matrix.shape[1]:
            raise ValueError("the source matrix must be square")

    def __call__(self, solver, state, dt):
        m = state._mirror
        M = self.matrix
        if M.shape[0] != state.num_eqn:
            raise ValueError("source matrix is %dx%d; state has num_eqn=%d" % (M.shape + (state.num_eqn,)))
        if m is not None and not m.host_dirty:
            m.linear_source(M, dt)  # on the device copy, which is the current one
            return
        q = state.q
        qq = q.copy()
        for i in range(M.shape[0]):
            for k in range(M.shape[1]):
                if M[i, k] != 0.0:
                    q[i] = q[i] + (M[i, k] * dt) * qq[k]


class EulerAxisymmetricSource(object):
    """Geometric source of the Euler equations in r-z coordinates with
    cylindrical symmetry, r = aux[radius_aux] the distance from the axis
    (the second coordinate), as in examples/euler_2d/shock_bubble_interaction.py
    :113-146: a two-stage Runge-Kutta step of
    q_t = -(rho v, rho u v, rho v^2, v (E + p)) / r, components past the
    fourth (a tracer) unchanged."""

    def __init__(self, gamma, radius_aux=0):
        self.gamma = float(gamma)
        self.radius_aux = int(radius_aux)

    def __call__(self, solver, state, dt):
        m = state._mirror
        if m is not None and not m.host_dirty:
            m.euler_axisymmetric_source(self.gamma, self.radius_aux, dt)
            return
        gamma = self.gamma
        dt2 = dt / 2.
        q = state.q
        rad = state.aux[self.radius_aux, :, :]
        rho = q[0, :, :]
        u = q[1, :, :] / rho
        v = q[2, :, :] / rho
        press = (gamma - 1.) * (q[3, :, :] - 0.5 * rho * (u ** 2 + v ** 2))
        qstar = np.empty(q.shape)
        qstar[0, :, :] = q[0, :, :] - dt2 / rad * q[2, :, :]
        qstar[1, :, :] = q[1, :, :] - dt2 / rad * rho * u * v
        qstar[2, :, :] = q[2, :, :] - dt2 / rad * rho * v * v
        qstar[3, :, :] = q[3, :, :] - dt2 / rad * v * (q[3, :, :] + press)
        rho = qstar[0, :, :]
        u = qstar[1, :, :] / rho
        v = qstar[2, :, :] / rho
        press = (gamma - 1.) * (qstar[3, :, :] - 0.5 * rho * (u ** 2 + v ** 2))
        q[0, :, :] = q[0, :, :] - dt / rad * qstar[2, :, :]
        q[1, :, :] = q[1, :, :] - dt / rad * rho * u * v
        q[2, :, :] = q[2, :, :] - dt / rad * rho * v * v
        q[3, :, :] = q[3, :, :] - dt / rad * v * (qstar[3, :, :] + press)
