"""Frames written from the GPU: the copy of the current state is queued
behind the steps already issued and a host thread formats the file while the
next steps run (claw2_patch_write_ascii_async).  The files must equal those
the host writer makes from the same frames."""
import os

import numpy as np
import pytest

from pyclaw_b200 import Solution, workloads

pytestmark = pytest.mark.gpu


def test_async_frames_equal_host_frames(tmp_path):
    a_dir, b_dir = str(tmp_path / "async"), str(tmp_path / "host")
    a = workloads.euler_quadrants_unsplit(n=300, tfinal=0.2)
    a.num_output_times = 5
    a.output_format, a.outdir, a.keep_copy = 'ascii', a_dir, False   # frames written from the device
    a.run()
    b = workloads.euler_quadrants_unsplit(n=300, tfinal=0.2)
    b.num_output_times = 5
    b.output_format, b.outdir, b.keep_copy = 'ascii', b_dir, True    # frames pulled to the host first
    b.run()
    for k in range(6):
        name = "fort.q%04d" % k
        with open(os.path.join(a_dir, name), "rb") as f:
            x = f.read()
        with open(os.path.join(b_dir, name), "rb") as f:
            y = f.read()
        assert x == y
        sol = Solution(k, path=a_dir)
        assert np.allclose(sol.state.q, b.frames[k].q, rtol=1e-8, atol=0)


def test_restart_from_written_frame(tmp_path):
    # a frame read back continues on the device like the original run
    d = str(tmp_path)
    a = workloads.euler_quadrants_unsplit(n=128, tfinal=0.2)
    a.num_output_times = 2
    a.output_format, a.outdir = 'ascii', d
    a.run()
    sol = Solution(1, path=d)
    assert abs(sol.t - 0.1) < 1e-12
    assert np.allclose(sol.state.q, a.frames[1].q, rtol=1e-8, atol=0)
