"""Batches of independent 2D problems stepped together on one GPU.

A user of the reference runs many independent problems as a host loop of
``Controller.run()`` / ``Solver.evolve_to_time`` calls, one problem at a time
(src/pyclaw/solver.py:554-666).  ``Batch`` steps all of them at once: every
batch step is one ghost-fill launch, one persistent step kernel over the tiles
of all problems and one per-problem accept/reject + dt update, all on the
device, and a run of many steps is one CUDA graph launch (claw2_batch_* in
include/claw2.h).  Each problem keeps the reference's own dt rule
(dt <- min(dt_max, dt * cfl_desired / cfl), reject when cfl > cfl_max).
"""
import ctypes

import numpy as np

from . import _lib


class Batch(object):
    """``Batch(claws)``: ``claws`` are Controllers built for the unsplit CUDA
    ClawSolver2D that share Riemann solver, method, BCs and parameters."""

    def __init__(self, claws, device=0):
        self._lib = _lib.load()
        descs = (_lib.Claw2Desc * len(claws))()
        self.claws = claws
        self.shapes = []
        for i, claw in enumerate(claws):
            s, sol = claw.solver, claw.solution
            s._check_cfl_settings()
            s._set_mthlim()
            s._set_method(sol.state)
            s.device = device
            descs[i] = s._device_desc(sol)
            self.shapes.append((sol.state.num_eqn,) + tuple(sol.state.grid.num_cells))
        h = ctypes.c_void_p()
        _lib.check(self._lib.claw2_batch_create(descs, len(claws), ctypes.byref(h)))
        self.h = h
        self.n = len(claws)
        self.upload()
        s0 = claws[0].solver
        self.set_time([c.solver.dt_initial for c in claws], 0.0, 1e99, s0.cfl_desired, s0.cfl_max, s0.dt_max)

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self._lib.claw2_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def upload(self):
        for i, claw in enumerate(self.claws):
            q = np.asfortranarray(claw.solution.state.get_q_global())
            _lib.check(self._lib.claw2_batch_upload_q(self.h, i, _lib.dptr(q)))

    def q(self, i):
        q = np.empty(self.shapes[i], order='F')
        _lib.check(self._lib.claw2_batch_download_q(self.h, i, _lib.dptr(q)))
        return q

    def set_time(self, dt0, t0, tend, cfl_desired=0.9, cfl_max=1.0, dt_max=1e99):
        arr = np.ascontiguousarray(dt0, dtype=np.float64)
        _lib.check(self._lib.claw2_batch_set_time(self.h, _lib.dptr(arr), t0, tend, cfl_desired, cfl_max, dt_max))

    def set_rows(self, rows):
        arr = np.ascontiguousarray(rows, dtype=np.intc)
        _lib.check(self._lib.claw2_batch_set_rows(self.h, _lib.iptr(arr)))

    def run(self, nsteps, mode=0):
        """nsteps batch steps; mode 0 = one CUDA graph, 1 = direct launches,
        2 = the plain per-problem launch loop.  Returns device ms."""
        ms = ctypes.c_float(0.0)
        _lib.check(self._lib.claw2_batch_run(self.h, int(nsteps), int(mode), ctypes.byref(ms)))
        return ms.value

    def state(self):
        n = self.n
        t, dt, cfl = np.zeros(n), np.zeros(n), np.zeros(n)
        ns, nr, stat = (np.zeros(n, dtype=np.intc) for _ in range(3))
        _lib.check(self._lib.claw2_batch_get_state(self.h, _lib.dptr(t), _lib.dptr(dt), _lib.iptr(ns),
                                                   _lib.iptr(nr), _lib.dptr(cfl), _lib.iptr(stat)))
        return {"t": t, "dt": dt, "nsteps": ns, "nreject": nr, "cfl": cfl, "failed": (stat & 1) != 0}

    def tiles(self):
        nt, grid = ctypes.c_int(0), ctypes.c_int(0)
        _lib.check(self._lib.claw2_batch_tiles(self.h, ctypes.byref(nt), ctypes.byref(grid)))
        return nt.value, grid.value


def size_buckets(sides, edges=(128, 256)):
    """Bucket index of every problem by its larger side."""
    return np.searchsorted(np.asarray(edges), np.asarray(sides), side="right")


def autotune_rows(batch, sides, candidates=(8, 12, 16, 24, 32, 48, 64), steps=2, dt0=None):
    """Row-block height per size bucket, chosen by measurement (coordinate
    descent over buckets, timing `steps` graph-free batch steps per trial).
    The trial steps advance the problems; the caller re-uploads its initial
    data afterwards (Batch.upload + set_time).  Returns (rows, trials)."""
    b = size_buckets(sides)
    nb = int(b.max()) + 1
    choice = [0] * nb  # 0 = the library heuristic
    trials = {}
    for k in range(nb):
        best = None
        for h in (0,) + tuple(candidates):
            c = list(choice)
            c[k] = h
            rows = np.array([c[x] for x in b], dtype=np.intc)
            batch.set_rows(rows)
            batch.run(1, mode=1)  # warm
            ms = batch.run(steps, mode=1) / steps
            trials[(k, h)] = ms
            if best is None or ms < best[0]:
                best = (ms, h)
        choice[k] = best[1]
    rows = np.array([choice[x] for x in b], dtype=np.intc)
    batch.set_rows(rows)
    return rows, trials, choice


def partition_instances(cells, world):
    """Split a batch over `world` ranks, balanced by cell count: instances in
    decreasing size, each to the rank with the fewest cells so far (greedy
    longest-processing-time order).  Instances are independent, so the ranks
    need no exchange; each builds a Batch of its own list.  Returns one sorted
    index list per rank; deterministic for equal inputs on every rank."""
    cells = np.asarray(cells, dtype=np.int64)
    order = sorted(range(len(cells)), key=lambda i: (-int(cells[i]), i))
    load = [0] * world
    parts = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += int(cells[i])
    return [sorted(p) for p in parts]
