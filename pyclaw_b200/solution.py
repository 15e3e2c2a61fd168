"""Solution: container of States on a Domain (host mirror of
src/pyclaw/solution.py:105-187)."""
import copy

from .geometry import Dimension, Domain, Patch
from .state import State


class Solution(object):
    """``Solution(state, domain)``, ``Solution(num_eqn, domain)``,
    ``Solution([states], domain)``, or ``Solution(frame, path=..., ...)`` /
    ``Solution(frame=..., ...)`` reading an ascii frame (solution.py:105-187)."""

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
        elif len(arg) == 1:
            frame = int(arg[0])
            if 'count_from_zero' in kargs:
                self._start_frame = 0 if kargs.pop('count_from_zero') else frame
            self.read(frame, **kargs)
        elif len(arg) == 0 and 'frame' in kargs:
            frame = int(kargs.pop('frame'))
            self.read(frame, **kargs)
        elif len(arg) == 0 and not kargs:
            pass
        else:
            raise Exception("Invalid arguments for Solution initialization.")

    num_eqn = property(lambda self: self.state.num_eqn)
    num_aux = property(lambda self: self.state.num_aux)
    mp = property(lambda self: self.state.mp)
    mF = property(lambda self: self.state.mF)

    def write(self, frame, path='./', file_format='ascii', file_prefix=None, write_aux=False, options={},
              write_p=False):
        """Write the frame's files (solution.py:253-303); 'ascii' only."""
        import os
        from . import fileio
        path = os.path.expandvars(os.path.expanduser(path))
        os.makedirs(path, exist_ok=True)
        for form in ([file_format] if isinstance(file_format, str) else list(file_format)):
            if form != 'ascii':
                raise NotImplementedError("output format %r: pyclaw_b200 writes 'ascii'" % (form,))
            fileio.write(self, frame, path, file_prefix=file_prefix or 'fort', write_aux=write_aux,
                         options=options, write_p=write_p)

    def read(self, frame, path='./_output', file_format=None, file_prefix='fort', read_aux=True, options={},
             **kargs):
        """Read a frame written in the ascii format (solution.py:305-364)."""
        import os
        from . import fileio
        path = os.path.expandvars(os.path.expanduser(path))
        fmt = None
        try:
            fmt = fileio.read_t(frame, path, file_prefix=file_prefix)[6]
        except (IOError, IndexError, ValueError):
            pass
        fmt = fmt if fmt is not None else (file_format or 'ascii')
        if fmt != 'ascii':
            raise NotImplementedError("input format %r: pyclaw_b200 reads 'ascii'" % (fmt,))
        fileio.read(self, frame, path, file_prefix=file_prefix, read_aux=read_aux, options=options)

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
