"""Device-resident patch: owner of the CUDA copy of one State's q.

Wraps the ``claw2_patch_*`` entry points of include/claw2.h.  The patch holds
two q buffers on the GPU; a step writes the pending one, and accept/reject
either swaps them or drops the result, so neither the reference's
``q_backup = state.q.copy('F')`` (src/pyclaw/solver.py:611) nor its
``qold = self.qbc.copy('F')`` (classic/solver.py:514) is ever made.
"""
import ctypes

import numpy as np

from . import _lib


class DevicePatch(object):
    def __init__(self, desc):
        lib = _lib.load()
        self._lib = lib
        h = ctypes.c_void_p()
        _lib.check(lib.claw2_patch_create(ctypes.byref(desc), ctypes.byref(h)))
        self.h = h
        self.desc = desc
        self.shape = (desc.num_eqn, desc.mx, desc.my)
        self.device_newer = False   # device q is ahead of the host copy
        self.host_dirty = True      # host q must be uploaded before the next step
        self._cfl = ctypes.c_double(0.0)
        self.mlp = None

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self._lib.claw2_patch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- residency protocol used by State ----------------------------------
    def pull_to_host(self, state):
        if self.device_newer:
            q = np.empty(self.shape, order='F')
            _lib.check(self._lib.claw2_patch_download_q(self.h, _lib.dptr(q)))
            state._q = q
            self.device_newer = False

    def host_modified(self, pulled=False):
        if pulled:
            self.device_newer = False
        self.host_dirty = True

    def push(self, state):
        q = np.asfortranarray(state._q, dtype=np.float64)
        _lib.check(self._lib.claw2_patch_upload_q(self.h, _lib.dptr(q)))
        self.host_dirty = False
        self.device_newer = False

    def push_aux(self, aux, bc_lower, bc_upper):
        """Upload State.aux and fill its ghost cells from the aux BCs on the
        device (claw2_patch_upload_aux)."""
        a = np.asfortranarray(aux, dtype=np.float64)
        lo = np.ascontiguousarray([int(b) for b in bc_lower], dtype=np.intc)
        up = np.ascontiguousarray([int(b) for b in bc_upper], dtype=np.intc)
        _lib.check(self._lib.claw2_patch_upload_aux(self.h, _lib.dptr(a), _lib.iptr(lo), _lib.iptr(up)))

    def push_auxbc(self, auxbc):
        """Upload an aux array with its ghost cells already filled on the host
        (claw2_patch_upload_auxbc)."""
        a = np.asfortranarray(auxbc, dtype=np.float64)
        _lib.check(self._lib.claw2_patch_upload_auxbc(self.h, _lib.dptr(a)))

    def upload_qbc(self, qbc):
        """Upload q with ghost cells filled on the host; the next step keeps
        them (claw2_patch_upload_qbc)."""
        a = np.asfortranarray(qbc, dtype=np.float64)
        _lib.check(self._lib.claw2_patch_upload_qbc(self.h, _lib.dptr(a)))
        self.host_dirty = False
        self.device_newer = False

    def write_ascii_async(self, path, append, header):
        """Queue the current state's ascii frame file (claw2_patch_write_ascii_async)."""
        _lib.check(self._lib.claw2_patch_write_ascii_async(self.h, path.encode(), 1 if append else 0,
                                                           header.encode(), 0))

    def wait_output(self):
        _lib.check(self._lib.claw2_patch_wait_output(self.h))

    def gather(self, cells):
        """q at the interior cells [(i, j), ...] of the current device state,
        shape (len(cells), num_eqn) (claw2_patch_gather_q)."""
        ij = np.ascontiguousarray(np.asarray(cells, dtype=np.intc).reshape(-1, 2))
        out = np.empty((len(ij), self.shape[0]))
        _lib.check(self._lib.claw2_patch_gather_q(self.h, len(ij), _lib.iptr(ij), _lib.dptr(out)))
        return out

    def linear_source(self, matrix, dt):
        """q <- q + dt M q on the device's current state (claw2_patch_linear_source)."""
        M = np.ascontiguousarray(matrix, dtype=np.float64)
        _lib.check(self._lib.claw2_patch_linear_source(self.h, _lib.dptr(M), M.shape[0], ctypes.c_double(dt)))
        self.device_newer = True

    def euler_axisymmetric_source(self, gamma, radius_aux, dt):
        """Axisymmetric Euler source step on the device's current state."""
        _lib.check(self._lib.claw2_patch_euler_axisymmetric_source(self.h, ctypes.c_double(gamma),
                                                                    int(radius_aux), ctypes.c_double(dt)))
        self.device_newer = True

    # ---- stepping -----------------------------------------------------------
    def set_cparam(self, vals):
        arr = (ctypes.c_double * len(vals))(*vals)
        _lib.check(self._lib.claw2_patch_set_cparam(self.h, arr, len(vals)))

    def step(self, dt, want_cfl=True):
        if want_cfl:
            _lib.check(self._lib.claw2_patch_step(self.h, ctypes.c_double(dt), ctypes.byref(self._cfl)))
            return self._cfl.value
        _lib.check(self._lib.claw2_patch_step(self.h, ctypes.c_double(dt), None))
        return None

    def step_part(self, dt, part, want_cfl=True):
        """One half of a step split around a halo exchange
        (claw2_patch_step_part): part 1 the interior row blocks, part 2 the
        ghost corners and the first and last row blocks; part 2 returns the
        Courant number (waits) unless want_cfl is False."""
        if part == 2 and want_cfl:
            _lib.check(self._lib.claw2_patch_step_part(self.h, ctypes.c_double(dt), 2, ctypes.byref(self._cfl)))
            return self._cfl.value
        _lib.check(self._lib.claw2_patch_step_part(self.h, ctypes.c_double(dt), int(part), None))
        return None

    def run_host(self, q_in, q_out, dt):
        """Independent steps from host arrays: q_out[k] = step of q_in[k] with
        dt[k] (claw2_patch_run_host; copies overlap compute).  q_in / q_out
        are lists of (num_eqn, mx, my) Fortran-order float64 arrays (pinned
        for overlap); an input must not be an earlier step's output array.
        Returns the Courant numbers."""
        n = len(q_in)
        if len(q_out) != n or len(dt) != n:
            raise ValueError("q_in, q_out and dt need one entry per step")
        for a in list(q_in) + list(q_out):
            if a.shape != self.shape or a.dtype != np.float64 or not a.flags.f_contiguous:
                raise ValueError("arrays must be float64 %s in Fortran order" % (self.shape,))
        pin = (ctypes.c_void_p * n)(*[a.ctypes.data for a in q_in])
        pout = (ctypes.c_void_p * n)(*[a.ctypes.data for a in q_out])
        dts = np.ascontiguousarray(dt, dtype=np.float64)
        cfl = np.zeros(n)
        _lib.check(self._lib.claw2_patch_run_host(self.h, n, pin, pout, _lib.dptr(dts), _lib.dptr(cfl)))
        self.device_newer = True
        self.host_dirty = False
        return cfl

    def evolve(self, es):
        """Run the device-resident time loop on ``es`` (a Claw2EvolveState,
        updated in place; claw2_patch_evolve).  The status code comes back
        unchecked so the caller can restore its own state first."""
        rc = self._lib.claw2_patch_evolve(self.h, ctypes.byref(es))
        if es.attempts > 0:
            self.device_newer = True
        return rc

    def accept(self, accept):
        _lib.check(self._lib.claw2_patch_accept(self.h, 1 if accept else 0))
        if accept:
            self.device_newer = True

    def cfl(self):
        _lib.check(self._lib.claw2_patch_cfl(self.h, ctypes.byref(self._cfl)))
        return self._cfl.value

    def set_stream(self, stream_ptr):
        _lib.check(self._lib.claw2_patch_set_stream(self.h, ctypes.c_void_p(stream_ptr or None)))

    def set_timing(self, on):
        _lib.check(self._lib.claw2_patch_set_timing(self.h, 1 if on else 0))

    def kernel_ms(self):
        ms = ctypes.c_float(0.0)
        _lib.check(self._lib.claw2_patch_kernel_ms(self.h, ctypes.byref(ms)))
        return ms.value

    def sync(self):
        _lib.check(self._lib.claw2_patch_sync(self.h))
