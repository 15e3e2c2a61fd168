"""Controller: runs a solver through a list of output times and collects the
frames (the user surface of src/pyclaw/controller.py:85-409).

Each output time is one ``evolve_to_time`` call (on the device time loop, one
library call per output time), after which the frame is recorded: a host copy
when ``keep_copy`` is set, PyClaw's ascii files when ``output_format`` is set
(a frame whose q is on the GPU is formatted by a host thread while the next
steps run; ``fileio.wait`` joins the last one before ``run`` returns), and the
functional file when ``compute_F`` is set.  Output styles, file names and the
F-file line format are the reference's, since post-processing reads them.
"""
import copy
import logging
import os

import numpy as np


class Controller(object):
    def __init__(self):
        self.logger = logging.getLogger('pyclaw.controller')
        self.solver = None
        self.solution = None
        # output: fort.tNNNN / fort.qNNNN files under outdir (output_format None: no files)
        self.outdir = './_output'
        self.output_format = 'ascii'
        self.output_file_prefix = None
        self.output_options = {}
        self.overwrite = True
        self.write_aux_init = False
        self.write_aux_always = False
        self.compute_p = None          # derived quantity written under outdir/_p
        self.file_prefix_p = 'claw_p'
        self.compute_F = None          # functionals appended to outdir/F.txt
        self.F_file_name = 'F'
        self.keep_copy = False         # in-memory frames
        self.frames = []
        # output times: 1 = num_output_times equal intervals to tfinal,
        # 2 = the list out_times, 3 = every nstepout steps, num_output_times times
        self.output_style = 1
        self.num_output_times = 10
        self.out_times = np.linspace(0.0, 1.0, 11)
        self.nstepout = 1
        self.tfinal = 1.0
        self.start_frame = 0
        self.verbosity = 0
        self.setplot = None

    @property
    def outdir_p(self):
        return os.path.join(self.outdir, '_p')

    @property
    def F_path(self):
        return os.path.join(self.outdir, self.F_file_name + '.txt')

    @property
    def t(self):
        return None if self.solution is None else self.solution.t

    def check_validity(self):
        ok, why = self.solver.is_valid()
        if not ok:
            raise Exception("the solver is not ready to run: %s" % why)
        if not self.solution.is_valid():
            raise Exception("the initial solution is not valid")

    def write_F(self, mode='a'):
        """compute_F fills state.F; one line `t F_0 F_1 ...` (sums of absolute
        values per functional) goes to outdir/F.txt (controller.py:399-409)."""
        if self.compute_F is None:
            return
        state = self.solution.state
        self.compute_F(state)
        sums = [state.sum_F(i) for i in range(state.mF)]
        os.makedirs(self.outdir, exist_ok=True)
        with open(self.F_path, mode) as f:
            f.write(" ".join([str(self.solution.t)] + [str(v) for v in sums]) + "\n")

    def output_times(self):
        """The times a run records, the current time first."""
        style = self.output_style
        if style == 1:
            return np.linspace(self.solution.t, self.tfinal, self.num_output_times + 1)
        if style == 2:
            return self.out_times
        if style == 3:  # only their number matters: each is nstepout single steps
            return np.ones(self.num_output_times + 1 - self.start_frame)
        raise Exception("output_style must be 1, 2 or 3 (got %r)" % style)

    def _advance(self, t):
        if self.output_style < 3:
            return self.solver.evolve_to_time(self.solution, t)
        status = None
        for _ in range(self.nstepout):
            status = self.solver.evolve_to_time(self.solution)
        return status

    def _record(self, frame, first):
        """What every output time leaves behind: the kept copy, the files (p
        first, then q, with aux on the first frame when write_aux_init), the
        functionals."""
        sol = self.solution
        if self.keep_copy:
            self.frames.append(copy.deepcopy(sol))
        if self.output_format is not None:
            if first and not self.overwrite and os.path.exists(self.outdir):
                raise Exception("output directory %s exists and controller.overwrite is False" % self.outdir)
            if self.compute_p is not None:
                self.compute_p(sol.state)
                sol.write(frame, self.outdir_p, self.output_format, self.file_prefix_p, write_aux=False,
                          options=self.output_options, write_p=True)
            aux = self.write_aux_always or (first and self.write_aux_init)
            sol.write(frame, self.outdir, self.output_format, self.output_file_prefix, aux, self.output_options)
        self.write_F('w' if first else 'a')

    def run(self):
        """Evolve to every output time, recording a frame at each
        (controller.py:275-397).  Returns the solver's last status."""
        if self.solver is None or self.solution is None:
            raise Exception("Controller.run needs both controller.solver and controller.solution")
        sol, solver = self.solution, self.solver
        self.start_frame = sol.start_frame
        grid = sol.state.grid
        if grid.gauges:
            grid.setup_gauge_files(self.outdir)
        if not solver._is_set_up:
            solver.setup(sol)
            solver.dt = solver.dt_initial
        self.check_validity()
        solver.write_gauge_values(sol)
        times = self.output_times()
        if len(times) == 0:
            return None
        frame = self.start_frame
        self._record(frame, first=True)
        status = None
        for t in times[1:]:
            status = self._advance(t)
            frame += 1
            self._record(frame, first=False)
            self.logger.info("frame %d at t = %f", frame, sol.t)
            for f in grid.gauge_files:
                f.flush()
        for f in grid.gauge_files:
            f.close()
        if self.output_format is not None:
            from . import fileio
            fileio.wait(sol)  # the last frame written from the GPU
        sol._start_frame = len(self.frames)
        return status
