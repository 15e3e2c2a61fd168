"""Extract the reference's own 2D classic regression goldens into
tests/golden/reference_goldens.npz.

Run where the reference tree is mounted, with its path as the argument or in
the environment variable CLAW_REFERENCE:
    python tests/golden/make_golden.py <path to the reference tree>  Sources, all produced by the reference's
Fortran step2/step2ds with clawpack/riemann solvers:
  examples/advection_2d/expected_sols.npy            (test_2d_advection.py:9-35)
  examples/acoustics_2d_homogeneous/verify_classic.txt (test_2d_acoustics.py:6-15)
  examples/euler_2d/expected_sols.npy['quadrants_roe'] (test_euler2d.py:6-29)
  examples/shallow_2d/expected_sols.npy['radialdambreak_classic_roe'], [..._hlle]
                                                     (test_shallow2d.py:9-28)
  examples/acoustics_2d_variable/io_test_verification/fort.q0020, fort.a0000
                                                     (test_acoustics_2d_variable_io.py:7-58)
  examples/acoustics_2d_variable/pressure_classic.txt (test_acoustics_2d_variable.py:6-23)
  examples/advection_2d_annulus/expected_sols.npy['classic']
                                                     (test_2d_advection_annulus.py:8-30)
  examples/psystem_2d/verify_gauge*.txt              (test_2d_psystem.py:8-24)
  examples/advection_reaction_2d/advection_reaction.txt (test_advection_reaction.py:1-22)
  examples/euler_2d/expected_sols.npy['shock_bubble_interaction'] (test_euler2d.py:10-36)
and copies the frame files examples/acoustics_2d_variable/io_test_verification/
fort.t0020, fort.q0020, fort.a0000 (the reference's ascii writer's output) to
tests/golden/frames/ for the file-format tests.
"""
import os
import sys

import numpy as np

REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("CLAW_REFERENCE")
if not REF:
    sys.exit("usage: make_golden.py <path to the reference tree> (or set CLAW_REFERENCE)")
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_goldens.npz")


def read_ascii_frame(path, mx, my, nvar):
    """A PyClaw ascii frame file (fort.qNNNN / fort.aNNNN of one patch): an
    8-line header, then for each row j the mx cells' values, rows separated by
    blank lines; returns the array (nvar, mx, my)."""
    with open(path) as f:
        lines = f.read().splitlines()[8:]
    vals = [list(map(float, ln.split())) for ln in lines if ln.strip()]
    arr = np.array(vals)
    assert arr.shape == (mx * my, nvar), arr.shape
    return np.ascontiguousarray(arr.reshape(my, mx, nvar).transpose(2, 1, 0))


def main():
    ex = os.path.join(REF, "examples")
    adv = np.load(os.path.join(ex, "advection_2d", "expected_sols.npy"), allow_pickle=True).item()
    eul = np.load(os.path.join(ex, "euler_2d", "expected_sols.npy"), allow_pickle=True).item()
    sw = np.load(os.path.join(ex, "shallow_2d", "expected_sols.npy"), allow_pickle=True).item()
    ac = np.loadtxt(os.path.join(ex, "acoustics_2d_homogeneous", "verify_classic.txt"))
    out = {
        "advection_classic_dim_split": adv["classic_dim_split"],
        "advection_classic_unsplit_no_trans": adv["classic_unsplit_no_trans"],
        "advection_classic_unsplit_trans_inc": adv["classic_unsplit_trans_inc"],
        "advection_classic_unsplit_trans_cor": adv["classic_unsplit_trans_cor"],
        "acoustics_verify_classic": ac,
        "euler_quadrants_roe": eul["quadrants_roe"],
        "shallow_radialdambreak_classic_hlle": sw["radialdambreak_classic_hlle"],
        "shallow_radialdambreak_classic_roe": sw["radialdambreak_classic_roe"],
    }
    vio = os.path.join(ex, "acoustics_2d_variable", "io_test_verification")
    out["acoustics_variable_io_q20"] = read_ascii_frame(os.path.join(vio, "fort.q0020"), 50, 50, 3)
    out["acoustics_variable_io_aux0"] = read_ascii_frame(os.path.join(vio, "fort.a0000"), 50, 50, 2)
    out["acoustics_variable_pressure_classic"] = np.loadtxt(
        os.path.join(ex, "acoustics_2d_variable", "pressure_classic.txt"))
    ann = np.load(os.path.join(ex, "advection_2d_annulus", "expected_sols.npy"), allow_pickle=True).item()
    out["advection_annulus_classic"] = ann["classic"]
    for g in ("0.25_0.25", "17.85_1.25", "3.25_18.75", "11.75_11.75"):
        out["psystem_gauge" + g] = np.loadtxt(os.path.join(ex, "psystem_2d", "verify_gauge" + g + ".txt"))
    out["advection_reaction_density"] = np.loadtxt(os.path.join(ex, "advection_reaction_2d",
                                                                "advection_reaction.txt"))
    out["euler_shock_bubble"] = eul["shock_bubble_interaction"]
    import shutil
    fdir = os.path.join(os.path.dirname(OUT), "frames")
    os.makedirs(fdir, exist_ok=True)
    for name in ("fort.t0020", "fort.q0020", "fort.a0000"):
        shutil.copyfile(os.path.join(vio, name), os.path.join(fdir, name))
    np.savez_compressed(OUT, **{k: np.asarray(v, dtype=np.float64) for k, v in out.items()})
    print("wrote", OUT, {k: np.asarray(v).shape for k, v in out.items()})


if __name__ == "__main__":
    main()
