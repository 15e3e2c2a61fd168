"""The CPU oracle, driven by the package's host loop (Controller/Solver), against
the reference's own regression goldens (tests/golden/make_golden.py).

The reference's tolerances are the L1 norms of examples/*/test_*.py; the
oracle meets them by a wide margin, and the tighter bound asserted beside each
records how closely it is pinned (roundoff level where the golden was produced
by the same algorithm and dt sequence).
"""
import numpy as np
import pytest

from pyclaw_b200 import workloads


def _l1(claw, expected, comp=None):
    q = claw.frames[claw.num_output_times].state.get_q_global()
    if comp is not None:
        q = q[comp]
    dx, dy = claw.solution.domain.grid.delta
    return dx * dy * np.sum(np.abs(q.reshape([-1]) - expected))


@pytest.mark.parametrize("key,kw", [
    ("advection_classic_dim_split", dict(dimensional_split=True)),
    ("advection_classic_unsplit_no_trans", dict(dimensional_split=False, transverse_waves=0)),
    ("advection_classic_unsplit_trans_inc", dict(dimensional_split=False, transverse_waves=1)),
    ("advection_classic_unsplit_trans_cor", dict(dimensional_split=False, transverse_waves=2)),
])
def test_advection_step2_goldens(oracle, goldens, key, kw):
    # examples/advection_2d/test_2d_advection.py:21-35 (tolerance 1e-6)
    claw = workloads.advection_2d(oracle.make_solver_class(), **kw)
    claw.run()
    err = _l1(claw, goldens[key])
    assert err < 1e-6
    assert err < 1e-13


def test_acoustics_goldens(oracle, goldens):
    # examples/acoustics_2d_homogeneous/test_2d_acoustics.py:6-15 (check_diff reltol 1e-3)
    claw = workloads.acoustics_2d_homogeneous(oracle.make_solver_class())
    claw.run()
    exp = goldens["acoustics_verify_classic"]
    test = claw.frames[-1].q[0, :, :]
    rel = np.linalg.norm(exp - test) / np.linalg.norm(exp)
    assert rel < 1e-3


def test_euler_roe_goldens(oracle, goldens):
    # examples/euler_2d/test_euler2d.py:25-26 (tolerance 1e-6); pins the Roe
    # solver *with* the entropy fix (without it the error is 3.7e-5)
    claw = workloads.quadrants(oracle.make_solver_class())
    claw.run()
    err = _l1(claw, goldens["euler_quadrants_roe"], comp=0)
    assert err < 1e-6
    assert err < 1e-12


def test_euler_roe_goldens_need_efix(oracle, goldens):
    claw = workloads.quadrants(oracle.make_solver_class(), efix=False)
    claw.run()
    assert _l1(claw, goldens["euler_quadrants_roe"], comp=0) > 1e-6


def test_shallow_roe_goldens(oracle, goldens):
    # examples/shallow_2d/test_shallow2d.py:19-28 (tolerance 1e-5)
    claw = workloads.radial_dam_break(oracle.make_solver_class())
    claw.run()
    err = _l1(claw, goldens["shallow_radialdambreak_classic_roe"], comp=0)
    assert err < 1e-5
    assert err < 1e-12


def test_vc_acoustics_goldens(oracle, goldens):
    # examples/acoustics_2d_variable (classic, 50x50, unsplit trans_inc, two
    # materials in aux): frame 20 of the I/O verification run (reltol 1e-6,
    # test_acoustics_2d_variable_io.py:42) and the pressure of the classic test
    # (abstol 0.1 in max norm, test_acoustics_2d_variable.py:14-18)
    from pyclaw_b200 import workloads
    claw = workloads.acoustics_variable(oracle.make_solver_class(), n=50)
    claw.run()
    assert np.array_equal(claw.frames[0].state.aux, goldens["acoustics_variable_io_aux0"])
    q = claw.frames[20].q
    exp = goldens["acoustics_variable_io_q20"]
    rel = np.linalg.norm(exp - q) / np.linalg.norm(exp)
    assert rel < 1e-6
    assert rel < 1e-8  # the golden file has 8 significant digits
    assert np.max(np.abs(goldens["acoustics_variable_pressure_classic"] - q[0])) < 1e-14


def test_annulus_golden(oracle, goldens):
    # examples/advection_2d_annulus (classic, 40x120 polar grid, vc_advection_2D
    # with edge velocities and the cell area as capacity function, custom aux
    # BCs in r, unsplit trans_cor, van Leer): L1 difference weighted by the
    # physical cell area at t = 1, < 1e-6 in test_2d_advection_annulus.py:11-30
    from pyclaw_b200 import workloads
    claw = workloads.advection_annulus(oracle.make_solver_class())
    claw.run()
    q = claw.frames[claw.num_output_times].state.get_q_global().reshape([-1])
    dx, dy = claw.solution.domain.grid.delta
    area = claw.frames[0].state.aux[2].reshape([-1]) * dx * dy
    diff = np.sum(np.abs(area * (q - goldens["advection_annulus_classic"])))
    assert diff < 1e-6
    assert diff < 1e-13  # measured 1.8e-15


@pytest.mark.parametrize("device_source", [False, True])
def test_advection_reaction_golden(oracle, goldens, device_source):
    # examples/advection_reaction_2d (split step, the example's own vector
    # advection solver, time-dependent edge velocities from a before-step hook,
    # Godunov-split reaction source): species 0 at t = 4, relative 2-norm
    # < 1e-5 in test_advection_reaction.py:7-19; the source as the host
    # function and as a LinearSource (numpy on a host state)
    from pyclaw_b200 import workloads
    claw = workloads.advection_reaction(oracle.make_solver_class(), device_source=device_source)
    claw.run()
    q0 = claw.solution.state.get_q_global()[0]
    exp = goldens["advection_reaction_density"]
    rel = np.linalg.norm(exp - q0) / np.linalg.norm(exp)
    assert rel < 1e-5
    assert rel < 1e-14  # measured 4.5e-16


def test_shock_bubble_golden(oracle, goldens):
    # examples/euler_2d/shock_bubble_interaction (euler_5wave_2D with a tracer,
    # custom inflow BC, wall at the axis, geometric source by a Godunov-split
    # step, limiters [4,4,4,4,2]) at 160x40 to t = 0.2: L1 density difference
    # times dx dy < 1e-6 in test_euler2d.py:10-36
    from pyclaw_b200 import workloads
    claw = workloads.shock_bubble(oracle.make_solver_class(), mx=160, my=40, tfinal=0.2, num_output_times=1)
    claw.run()
    d = claw.frames[claw.num_output_times].state.get_q_global()[0].reshape([-1])
    dx, dy = claw.solution.domain.grid.delta
    diff = dx * dy * np.sum(np.abs(d - goldens["euler_shock_bubble"]))
    assert diff < 1e-6
    assert diff < 1e-13  # measured 1.0e-15


def test_shallow_hlle_goldens(oracle, goldens):
    # examples/shallow_2d/test_shallow2d.py:31-37 with the HLLE solver (tolerance 1e-5)
    claw = workloads.radial_dam_break(oracle.make_solver_class(), riemann_solver='hlle')
    claw.run()
    err = _l1(claw, goldens["shallow_radialdambreak_classic_hlle"], comp=0)
    assert err < 1e-5
    assert err < 1e-12  # measured 1.4e-14


PSYSTEM_GAUGES = ("0.25_0.25", "17.85_1.25", "3.25_18.75", "11.75_11.75")


def test_psystem_gauge_goldens(oracle, goldens, tmp_path):
    # examples/psystem_2d/test_2d_psystem.py:8-24 (np.allclose of each gauge's
    # time/stress/10*stress rows, in memory and in the files): f-waves, the
    # before-step hook writing the strain into aux, wall and extrapolation
    # sides for q and aux, superbee, unsplit with trans_inc
    claw = workloads.psystem(oracle.make_solver_class(), cells_per_layer=6, tfinal=1.,
                             outdir=str(tmp_path))
    claw.run()
    st = claw.solution.state
    for k, g in enumerate(PSYSTEM_GAUGES):
        expected = goldens["psystem_gauge" + g]
        mem = np.asarray(st.gauge_data[k])
        assert mem.shape == expected.shape
        assert np.allclose(expected, mem)
        assert np.allclose(expected, np.loadtxt(st.grid.gauge_files[k].name))
        # the files hold 12 significant digits; measured 4.9e-11 on the
        # corner gauge (|value| up to 98.6)
        assert np.max(np.abs(mem - expected)) <= 1e-9
