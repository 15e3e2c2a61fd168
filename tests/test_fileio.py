"""PyClaw's ascii frame files (src/pyclaw/fileio/ascii.py): reading the
reference's own frame files, writing them back byte for byte, and the
Controller's output loop.  The GPU form (frames written behind the next steps)
is in test_gpu_fileio.py."""
import os

import numpy as np
import pytest

FRAMES = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "frames")


def test_read_reference_frame(goldens):
    # fort.t0020 / fort.q0020 / fort.a0000 of the reference's variable-acoustics
    # I/O test: an old-style fort.t (no num_ghost / file_format lines)
    from pyclaw_b200 import Solution
    sol = Solution(20, path=FRAMES, read_aux=True)
    assert sol.t == 0.6
    assert sol.num_eqn == 3 and sol.num_aux == 2
    dims = sol.domain.grid.dimensions
    assert [d.num_cells for d in dims] == [50, 50]
    assert dims[0].lower == -1.0 and abs(dims[0].delta - 0.04) < 1e-15
    assert np.array_equal(sol.state.q, goldens["acoustics_variable_io_q20"])
    assert np.array_equal(sol.state.aux, goldens["acoustics_variable_io_aux0"])


def test_write_reproduces_reference_bytes(tmp_path):
    # the library's writer formats the values read from the reference's files
    # into the same bytes (patch header, "%18.8e" values, blank line per row)
    from pyclaw_b200 import Solution
    sol = Solution(20, path=FRAMES, read_aux=True)
    sol.write(20, path=str(tmp_path), write_aux=True)
    for ours, ref in (("fort.q0020", "fort.q0020"), ("fort.a0020", "fort.a0000")):
        with open(os.path.join(str(tmp_path), ours), "rb") as f:
            a = f.read()
        with open(os.path.join(FRAMES, ref), "rb") as f:
            b = f.read()
        assert a == b
    t = open(os.path.join(str(tmp_path), "fort.t0020")).read().splitlines()
    assert t[0].split() == ["6.00000000e-01", "time"] and t[-1].split() == ["ascii", "file_format"]


def _py_format(q):
    # the reference's write_array (ascii.py:99-123), value by value
    out = []
    for j in range(q.shape[2]):
        for i in range(q.shape[1]):
            out.append("".join("%18.8e" % q[m, i, j] for m in range(q.shape[0])) + "\n")
        out.append("\n")
    return "".join(out)


@pytest.mark.parametrize("nthreads", [1, 3, 0])
def test_threaded_writer_matches_python_formatting(tmp_path, nthreads):
    from pyclaw_b200 import _lib
    rng = np.random.default_rng(nthreads)
    q = np.asfortranarray(rng.standard_normal((4, 37, 29)) * 10.0 ** rng.integers(-120, 120, (4, 37, 29)))
    q[0, 3, 4] = 0.0
    q[1, 5, 6] = -0.0
    fname = str(tmp_path / "x.txt")
    _lib.check(_lib.load().claw2_write_ascii(fname.encode(), 0, b"HEAD\n", _lib.dptr(q), 4, 37, 29, nthreads))
    assert open(fname).read() == "HEAD\n" + _py_format(q)


def test_controller_writes_and_reads_back_frames(oracle, tmp_path):
    from pyclaw_b200 import Solution, workloads
    claw = workloads.acoustics_variable(oracle.make_solver_class(), n=40, tfinal=0.2, num_output_times=4)
    claw.output_format = 'ascii'
    claw.outdir = str(tmp_path)
    claw.write_aux_init = True
    claw.run()
    for k, frame in enumerate(claw.frames):
        sol = Solution(k, path=str(tmp_path), read_aux=True)
        assert abs(sol.t - frame.t) <= 1e-8 * max(1.0, frame.t)
        assert np.allclose(sol.state.q, frame.q, rtol=1e-8, atol=1e-300)
        assert np.allclose(sol.state.aux, frame.state.aux, rtol=1e-8)
    assert sorted(f for f in os.listdir(str(tmp_path)) if f.startswith("fort.t")) == \
        ["fort.t%04d" % k for k in range(5)]
