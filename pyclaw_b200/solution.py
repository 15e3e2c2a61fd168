"""Solution: container of States on a Domain (host mirror of
src/pyclaw/solution.py:105-187)."""
import copy

from .geometry import Dimension, Domain, Patch
from .state import State


class Solution(object):
    """``Solution(state, domain)``, ``Solution(num_eqn, domain)`` or
    ``Solution([states], domain)``.  Reading frames from files (one argument)
    is not part of this package."""

    def __init__(self, *arg, **kargs):
        self.states = []
        self.domain = None
        self._start_frame = 0
        if len(arg) == 2:
            if isinstance(arg[1], Domain):
                self.domain = arg[1]
            else:
                geom = list(arg[1]) if not isinstance(arg[1], (list, tuple)) else arg[1]
                if isinstance(geom[0], Dimension):
                    self.domain = Domain(Patch(geom))
                elif isinstance(geom[0], Patch):
                    self.domain = Domain(geom)
                else:
                    raise Exception("Invalid arguments for Solution initialization.")
            if isinstance(arg[0], State):
                self.states.append(arg[0])
            elif isinstance(arg[0], (list, tuple)) and arg[0] and isinstance(arg[0][0], State):
                self.states = list(arg[0])
            elif isinstance(arg[0], (list, tuple)) and arg[0] and isinstance(arg[0][0], int):
                self.states.append(State(self.domain, arg[0][0], arg[0][1]))
            elif isinstance(arg[0], int):
                self.states.append(State(self.domain, arg[0]))
            if not self.states or self.domain is None:
                raise Exception("Invalid arguments for Solution initialization.")
        elif len(arg) == 0 and not kargs:
            pass
        else:
            raise Exception("Invalid arguments for Solution initialization "
                            "(reading frames from files is not supported).")

    state = property(lambda self: self.states[0])
    patch = property(lambda self: self.domain.patch)
    grid = property(lambda self: self.domain.grid)
    start_frame = property(lambda self: self._start_frame)

    @property
    def t(self):
        return self.state.t

    @t.setter
    def t(self, t):
        for s in self.states:
            s.t = t

    @property
    def q(self):
        return self.state.q

    @property
    def aux(self):
        return self.state.aux

    @property
    def problem_data(self):
        return self.state.problem_data

    def is_valid(self):
        return all(s.is_valid() for s in self.states)

    def __deepcopy__(self, memo={}):
        result = Solution()
        result.domain = copy.deepcopy(self.domain)
        result.states = [copy.deepcopy(s) for s in self.states]
        result._start_frame = self._start_frame
        return result
