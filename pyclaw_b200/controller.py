"""Controller: the output-time loop (host mirror of src/pyclaw/controller.py:85-397)."""
import copy
import logging

import numpy as np


class Controller(object):
    def __init__(self):
        self.logger = logging.getLogger('pyclaw.controller')
        self.solver = None
        self.solution = None
        self.outdir = './_output'
        self.output_format = 'ascii'  # fort.tNNNN / fort.qNNNN files under outdir (None: no files)
        self.output_file_prefix = None
        self.file_prefix_p = 'claw_p'
        self.output_options = {}
        self.write_aux_init = False
        self.write_aux_always = False
        self.keep_copy = False
        self.frames = []
        self.output_style = 1
        self.num_output_times = 10
        self.out_times = np.linspace(0.0, 1.0, 11)
        self.nstepout = 1
        self.tfinal = 1.0
        self.verbosity = 0
        self.setplot = None
        self.compute_p = None
        self.compute_F = None
        self.overwrite = True
        self.start_frame = 0
        self.F_file_name = 'F'

    @property
    def outdir_p(self):
        import os
        return os.path.join(self.outdir, '_p')

    @property
    def F_path(self):
        import os
        return os.path.join(self.outdir, self.F_file_name + '.txt')

    def write_F(self, mode='a'):
        """Functionals: compute_F fills state.F, whose sums of absolute values
        go to outdir/F.txt with the time (controller.py:399-409)."""
        if self.compute_F is not None:
            import os
            self.compute_F(self.solution.state)
            F = [self.solution.state.sum_F(i) for i in range(self.solution.state.mF)]
            os.makedirs(self.outdir, exist_ok=True)
            with open(self.F_path, mode) as f:
                f.write(str(self.solution.t) + ' ' + ' '.join(str(j) for j in F) + '\n')

    @property
    def t(self):
        return self.solution.t if self.solution is not None else None

    def check_validity(self):
        valid, reason = self.solver.is_valid()
        if not valid:
            raise Exception("The solver failed to initialize properly: %s" % reason)
        if not self.solution.is_valid():
            raise Exception("Initial solution is not valid.")

    def _write_frame(self, frame, write_aux):
        """controller.py:327-349: the derived quantities p (with compute_p)
        and the frame itself; a frame whose q is on the GPU is written behind
        the following steps."""
        if self.compute_p is not None:
            self.compute_p(self.solution.state)
            self.solution.write(frame, self.outdir_p, self.output_format, self.file_prefix_p, write_aux=False,
                                options=self.output_options, write_p=True)
        self.solution.write(frame, self.outdir, self.output_format, self.output_file_prefix, write_aux,
                            self.output_options)

    def run(self):
        """controller.py:275-397."""
        if self.solver is None or self.solution is None:
            raise Exception('To run, a Controller must have a Solver and a Solution.')
        self.start_frame = self.solution.start_frame
        grid = self.solution.state.grid
        if len(grid.gauges) > 0:
            grid.setup_gauge_files(self.outdir)
        frame = self.start_frame
        if not self.solver._is_set_up:
            self.solver.setup(self.solution)
            self.solver.dt = self.solver.dt_initial
        self.check_validity()
        self.solver.write_gauge_values(self.solution)  # initial gauge values
        if self.output_style == 1:
            output_times = np.linspace(self.solution.t, self.tfinal, self.num_output_times + 1)
        elif self.output_style == 2:
            output_times = self.out_times
        elif self.output_style == 3:
            output_times = np.ones((self.num_output_times + 1 - self.start_frame))
        else:
            raise Exception("Invalid output style %s" % self.output_style)
        if len(output_times) == 0:
            return None
        if self.keep_copy:
            self.frames.append(copy.deepcopy(self.solution))
        if self.output_format is not None:
            import os
            if os.path.exists(self.outdir) and self.overwrite is False:
                raise Exception("Refusing to overwrite existing output data. \nEither delete/move the directory "
                                "or set controller.overwrite=True.")
            self._write_frame(frame, self.write_aux_always or self.write_aux_init)
        self.write_F('w')
        status = None
        for t in output_times[1:]:
            if self.output_style < 3:
                status = self.solver.evolve_to_time(self.solution, t)
            else:
                for n in range(self.nstepout):
                    status = self.solver.evolve_to_time(self.solution)
            frame += 1
            if self.keep_copy:
                self.frames.append(copy.deepcopy(self.solution))
            if self.output_format is not None:
                self._write_frame(frame, self.write_aux_always)
            self.write_F()
            self.logger.info("Solution %s computed for time t=%f" % (frame, self.solution.t))
            for gfile in grid.gauge_files:
                gfile.flush()
        for gfile in grid.gauge_files:
            gfile.close()
        if self.output_format is not None:
            from . import fileio
            fileio.wait(self.solution)  # the last frame written from the GPU
        self.solution._start_frame = len(self.frames)
        return status
