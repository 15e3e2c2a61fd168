"""pyclaw_b200: PyClaw's classic 2D wave-propagation step on the B200 (sm_100a).

Drop-in for ``clawpack.pyclaw`` on the ClawSolver2D path:

    import pyclaw_b200 as pyclaw
    from pyclaw_b200 import riemann
    solver = pyclaw.ClawSolver2D(riemann.euler_4wave_2D)   # kernel_language='CUDA'

The hot path (ghost fill, fused step2/step2ds, CFL reduction) runs in the
hand-written CUDA library ``lib/libclaw2.so``; importing the package does not
load it, the first solver setup does, and fails loudly if it is missing.
"""
from .geometry import Dimension, Grid, Patch, Domain
from .state import State
from .solution import Solution
from .cfl import CFL
from .solver import BC, CFLError, Solver
from .classic import ClawSolver, ClawSolver2D
from .controller import Controller
from . import limiters, riemann

__all__ = ["Dimension", "Grid", "Patch", "Domain", "State", "Solution", "CFL", "BC", "CFLError",
           "Solver", "ClawSolver", "ClawSolver2D", "Controller", "limiters", "riemann"]
