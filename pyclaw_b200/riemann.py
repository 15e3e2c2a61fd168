"""Riemann solvers available to the CUDA step.

Stands in for the external ``clawpack.riemann`` package (not vendored in the
reference; used at src/pyclaw/solver.py:230-238 and
classic/solver.py:516-521).  Each solver object is what a user passes to
``ClawSolver2D(...)``: its ``__name__`` ends in the reference's module name, the
``static`` tables give num_eqn/num_waves/fwave by that name, and ``cparam``
lists the ``problem_data`` keys that become its parameter vector (the
reference's COMMON /cparam/, state.py:206-231).  The device functors live in
csrc/riemann.cuh.
"""
import types

from . import _lib


class _ParamBlock(object):
    """A solver's parameters, in both of the forms the reference uses them.

    Called with ``problem_data`` it returns the parameter vector for the C ABI
    (the device solver's cparam).  Assigned to, it behaves like an f2py
    module's ``cparam`` COMMON block: the reference's ``state.set_cparam(rp)``
    (state.py:206-231) lists its attributes and assigns every problem_data
    entry to it, which it accepts (the device takes the values from
    problem_data or the step module's cparam, not from here)."""

    def __init__(self, solver):
        object.__setattr__(self, '_owner', solver)

    def __dir__(self):
        # nothing to demand: the required keys are checked when the vector is built
        return []

    def __call__(self, problem_data):
        rp = self._owner
        missing = [k for k in rp.cparam_names if k not in problem_data]
        if missing:
            raise Exception("Riemann solver %s reads problem_data[%s], which is not set"
                            % (rp.name, ", ".join(repr(k) for k in missing)))
        vals = [float(problem_data[k]) for k in rp.cparam_names]
        if rp.efix is not None:
            vals.append(1.0 if problem_data.get('efix', rp.efix) else 0.0)
        for key, default in rp.extra:
            vals.append(float(problem_data.get(key, default)))
        return vals


class RiemannSolver(object):
    """One device Riemann solver.  Usable where the reference expects a
    clawpack.riemann module: ``__name__`` ends in the module name, ``rpn2`` /
    ``rpt2`` carry ``_cpointer`` (here the solver itself, which
    pyclaw_b200.classic2 resolves to the device code where an f2py module
    would receive a Fortran function pointer, classic/solver.py:516-521), and
    ``cparam`` takes the reference's set_cparam."""

    def __init__(self, name, rp_id, num_eqn, num_waves, cparam, fwave=False, efix=None, extra=()):
        self.__name__ = 'clawpack.riemann.' + name
        self.name = name
        self.rp_id = rp_id
        self.num_eqn = num_eqn
        self.num_waves = num_waves
        self.cparam_names = tuple(cparam)
        self.fwave = fwave
        self.efix = efix  # entropy fix switch (a compile-time constant in Fortran)
        self.extra = tuple(extra)  # (problem_data key, default) pairs appended to cparam
        self.cparam = _ParamBlock(self)
        self.rpn2 = types.SimpleNamespace(_cpointer=self)
        self.rpt2 = types.SimpleNamespace(_cpointer=self)

    def __repr__(self):
        return "<Riemann solver %s>" % self.name


advection_2D = RiemannSolver('advection_2D', _lib.RP_ADVECTION, 1, 1, ('u', 'v'))
acoustics_2D = RiemannSolver('acoustics_2D', _lib.RP_ACOUSTICS, 3, 2, ('rho', 'bulk', 'cc', 'zz'))
euler_4wave_2D = RiemannSolver('euler_4wave_2D', _lib.RP_EULER_ROE, 4, 4, ('gamma',), efix=True)
shallow_roe_with_efix_2D = RiemannSolver('shallow_roe_with_efix_2D', _lib.RP_SHALLOW_ROE, 3, 3,
                                         ('grav',), efix=True)

# Exact Euler solver (no counterpart in clawpack/riemann): Newton for p* to
# relative tolerance `exact_tol`; three waves (1-wave, contact+shear, 3-wave).
euler_exact_2D = RiemannSolver('euler_exact_2D', _lib.RP_EULER_EXACT, 4, 3, ('gamma',),
                               extra=(('exact_tol', 1e-12),))

# Acoustics with variable coefficients: no cparam; aux = (density, sound speed)
# per cell (clawpack.riemann.vc_acoustics_2D).
vc_acoustics_2D = RiemannSolver('vc_acoustics_2D', _lib.RP_VC_ACOUSTICS, 3, 2, ())
vc_acoustics_2D.num_aux = 2

# Advection with edge velocities: no cparam; aux = (u at the left edge, v at
# the bottom edge) per cell (clawpack.riemann.vc_advection_2D).
vc_advection_2D = RiemannSolver('vc_advection_2D', _lib.RP_VC_ADVECTION, 1, 1, ())
vc_advection_2D.num_aux = 2

# The p-system (nonlinear elasticity) in a heterogeneous medium, f-waves: no
# cparam; aux = (density, bulk modulus, stress-strain relation 1 linear /
# 2 exponential, strain at the start of the step) per cell, as
# clawpack.riemann.psystem_2D takes them.  Restated from the mathematics
# (linearisation at each cell's own strain); it does not reproduce the
# reference's p-system gauge files, whose solver makes another choice.
psystem_2D = RiemannSolver('psystem_2D', _lib.RP_PSYSTEM, 3, 2, (), fwave=True)
psystem_2D.num_aux = 4

# The advection-reaction example's own solver
# (examples/advection_reaction_2d/rpn2_vc_advection_vector.f90, built there as
# the module ``advection_2d``): vc_advection_2D's normal solve for two
# components; no transverse solve (split step or transverse_waves = 0).
vc_advection_vector_2D = RiemannSolver('vc_advection_vector_2D', _lib.RP_VC_ADVECTION_VEC, 2, 1, ())
vc_advection_vector_2D.num_aux = 2

# Euler with a passive tracer (fifth component), Roe solver with five waves
# (acoustic, shear, entropy, acoustic, tracer) and the entropy fix
# (clawpack.riemann.euler_5wave_2D).
euler_5wave_2D = RiemannSolver('euler_5wave_2D', _lib.RP_EULER_5WAVE, 5, 5, ('gamma',), efix=True)

# Shallow water HLLE solver (two waves through the HLL middle state, Einfeldt
# speeds); no transverse solve: split step or transverse_waves = 0
# (clawpack.riemann.shallow_hlle_2D).
shallow_hlle_2D = RiemannSolver('shallow_hlle_2D', _lib.RP_SHALLOW_HLLE, 3, 2, ('grav',))

_ALL = [advection_2D, acoustics_2D, euler_4wave_2D, shallow_roe_with_efix_2D, euler_exact_2D, vc_acoustics_2D,
        vc_advection_2D, psystem_2D, vc_advection_vector_2D, euler_5wave_2D, shallow_hlle_2D]

static = types.SimpleNamespace(
    num_eqn={s.name: s.num_eqn for s in _ALL},
    num_waves={s.name: s.num_waves for s in _ALL},
    fwave={s.name: s.fwave for s in _ALL},
)

# component-index constants modules (clawpack.riemann.<name>_constants)
euler_exact_2D_constants = types.SimpleNamespace(density=0, x_momentum=1, y_momentum=2, energy=3, num_eqn=4)
euler_4wave_2D_constants = types.SimpleNamespace(density=0, x_momentum=1, y_momentum=2, energy=3,
                                                 num_eqn=4)
euler_5wave_2D_constants = types.SimpleNamespace(density=0, x_momentum=1, y_momentum=2, energy=3, num_eqn=5)
shallow_roe_with_efix_2D_constants = types.SimpleNamespace(depth=0, x_momentum=1, y_momentum=2,
                                                           num_eqn=3)
acoustics_2D_constants = types.SimpleNamespace(pressure=0, x_velocity=1, y_velocity=2, num_eqn=3)
vc_acoustics_2D_constants = types.SimpleNamespace(pressure=0, x_velocity=1, y_velocity=2, num_eqn=3)
vc_advection_2D_constants = types.SimpleNamespace(num_eqn=1)
