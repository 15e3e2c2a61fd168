"""State: the solution arrays of one patch (host mirror of src/pyclaw/state.py).

``q`` has the reference's shape (num_eqn, mx, my) in Fortran order
(state.py:330-335).  When a CUDA solver owns the patch, the authoritative copy
of q lives on the device; reading ``state.q`` downloads it on demand and
assigning or modifying it makes the next step upload it again.
"""
import copy

import numpy as np

from .geometry import Domain, Patch


class State(object):
    """``State(domain_or_patch, num_eqn, num_aux=0)`` (state.py:119-152)."""

    def __init__(self, geom, num_eqn, num_aux=0):
        if isinstance(geom, Patch):
            self.patch = geom
        elif isinstance(geom, Domain):
            self.patch = geom.patches[0]
        else:
            raise Exception("A State must be initialized with a Patch or a Domain.")
        self.p = None
        self.F = None
        self.problem_data = {}
        self.t = 0.
        self.index_capa = -1
        self.keep_gauges = False
        self.gauge_data = []
        self._mirror = None  # device copy owner (pyclaw_b200.device.DevicePatch)
        self._q = self.new_array(num_eqn)
        self.aux = self.new_array(num_aux)

    # ---- q with device residency ------------------------------------------
    @property
    def q(self):
        """Host view of q.  Pulls the device copy if it is newer and assumes the
        caller may write into the array (the next step re-uploads it)."""
        m = self._mirror
        if m is not None:
            m.pull_to_host(self)
            m.host_modified()
        return self._q

    @q.setter
    def q(self, value):
        value = np.asarray(value, dtype=np.float64)
        if value.shape != self._q.shape:
            raise ValueError("q must have shape %s (got %s)" % (self._q.shape, value.shape))
        self._q = np.asfortranarray(value)
        if self._mirror is not None:
            self._mirror.host_modified(pulled=True)

    def _read_q(self):
        """q for reading only (no re-upload is scheduled)."""
        if self._mirror is not None:
            self._mirror.pull_to_host(self)
        return self._q

    # ---- geometry shortcuts ------------------------------------------------
    grid = property(lambda self: self.patch.grid)
    num_eqn = property(lambda self: self._q.shape[0])
    num_aux = property(lambda self: self.aux.shape[0] if self.aux is not None else 0)
    p_centers = property(lambda self: self.grid.p_centers)
    c_centers = property(lambda self: self.grid.c_centers)

    @property
    def mp(self):
        return self.p.shape[0] if self.p is not None else 0

    @mp.setter
    def mp(self, mp):
        """Allocate p, the derived quantities of compute_p (state.py:90-101)."""
        if self.p is not None:
            raise Exception('Cannot change state.mp after p is initialized.')
        self.p = self.new_array(mp)

    @property
    def mF(self):
        return self.F.shape[0] if self.F is not None else 0

    @mF.setter
    def mF(self, mF):
        """Allocate F, the integrands of compute_F (state.py:103-114)."""
        if self.F is not None:
            raise Exception('Cannot change state.mF after F is initialized.')
        self.F = self.new_array(mF)

    def gauge_q(self, cells):
        """q at the interior cells [(i, j), ...]: gathered on the device when it
        holds the newer q (a few values instead of the whole array)."""
        m = self._mirror
        if m is not None and m.device_newer:
            return m.gather(cells)
        q = self._q
        return np.array([q[:, i, j] for i, j in cells]).reshape(len(cells), self.num_eqn)

    def is_valid(self):
        """F-contiguity and capacity-index checks (state.py:166-204)."""
        valid = True
        q = self._read_q()
        if not q.flags['F_CONTIGUOUS']:
            valid = False
        if self.aux is not None and not self.aux.flags['F_CONTIGUOUS']:
            valid = False
        if self.index_capa >= 0 and (self.aux is None or self.index_capa > self.num_aux - 1):
            raise ValueError("Capacity function index out of range.")
        return valid

    def new_array(self, dof):
        if dof == 0:
            return None
        shape = [dof] + list(self.grid.num_cells)
        return np.empty(shape, order='F')

    def get_q_global(self):
        """A copy of q (state.py:337-341)."""
        return self._read_q().copy()

    def get_aux_global(self):
        return None if self.aux is None else self.aux.copy()

    def get_qbc_from_q(self, num_ghost, qbc):
        qbc[:, num_ghost:-num_ghost, num_ghost:-num_ghost] = self._read_q()
        return qbc

    def set_q_from_qbc(self, num_ghost, qbc):
        self.q = qbc[:, num_ghost:-num_ghost, num_ghost:-num_ghost]

    def sum_F(self, i):
        return np.sum(np.abs(self.F[i, ...]))

    def __deepcopy__(self, memo={}):
        result = State(copy.deepcopy(self.patch), self.num_eqn, self.num_aux)
        result.t = self.t
        result._q = np.asfortranarray(self._read_q().copy())
        if self.aux is not None:
            result.aux = copy.deepcopy(self.aux)
        result.problem_data = copy.deepcopy(self.problem_data)
        result.index_capa = self.index_capa
        return result

    def __str__(self):
        return ("PyClaw State object\nPatch dimensions: %s\nTime  t=%s\n"
                "Number of conserved quantities: %s\n" % (self.patch.num_cells_global, self.t, self.num_eqn))
