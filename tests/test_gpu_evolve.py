"""The device-resident time loop (claw2_patch_evolve): evolve_to_time with
get_dt, the CFL test, accept/reject and the clipping to the output time done
on the GPU.  It must take the same steps (same count, same rejections) with
the same dt as the host loop and give the same states and solver status.
The loop's step kernels are their own instantiations (dt read from the loop's
device record), and the compiler may fuse a multiply-add differently in two
instantiations of the same source, so states, Courant numbers and times are
compared to a few units in the last place (1e-13 relative), counts exactly."""
import numpy as np
import pytest

from helpers import max_rel
from pyclaw_b200 import workloads
from pyclaw_b200.solver import CFLError

pytestmark = pytest.mark.gpu


def _pair(make, **solver_kw):
    runs = []
    for device_loop in (True, False):
        claw = make()
        claw.solver.device_time_loop = device_loop
        for k, v in solver_kw.items():
            setattr(claw.solver, k, v)
        claw.run()
        runs.append(claw)
    return runs


ULP_RTOL = 1e-13


def _close(x, y):
    return x == y or abs(x - y) <= ULP_RTOL * max(abs(x), abs(y))


def _same(a, b):
    sa, sb = a.solver.status, b.solver.status
    assert sa['numsteps'] == sb['numsteps']
    for k in ('cflmax', 'dtmin', 'dtmax'):
        assert _close(sa[k], sb[k]), (k, sa[k], sb[k])
    assert _close(a.solver.dt, b.solver.dt)
    assert _close(a.solver.cfl.get_cached_max(), b.solver.cfl.get_cached_max())
    assert len(a.frames) == len(b.frames)
    for fa, fb in zip(a.frames, b.frames):
        assert _close(fa.t, fb.t)
        assert max_rel(fa.q, fb.q) <= ULP_RTOL


@pytest.mark.parametrize("name", ["euler_unsplit", "acoustics", "shallow_split", "vc_acoustics", "advection"])
def test_device_loop_equals_host_loop(name):
    make = {"euler_unsplit": lambda: workloads.euler_quadrants_unsplit(n=192, tfinal=0.3),
            "acoustics": lambda: workloads.acoustics_wall(n=150, tfinal=0.4),
            "shallow_split": lambda: workloads.radial_dam_break(mx=120, my=100),
            "vc_acoustics": lambda: workloads.acoustics_variable(n=80, tfinal=0.4, num_output_times=4),
            "advection": lambda: workloads.advection_2d(dimensional_split=False, transverse_waves=1, mx=90, my=60)}
    a, b = _pair(make[name])
    assert a.solver.status['numsteps'] > 10
    _same(a, b)


def test_rejected_steps_on_the_device():
    # a first dt far above the CFL limit: rejected and retaken inside the loop
    a, b = _pair(lambda: workloads.euler_quadrants_unsplit(n=128, tfinal=0.1), dt_initial=0.5)
    _same(a, b)


def test_fixed_dt_and_its_cfl_error():
    def make():
        claw = workloads.acoustics_wall(n=100, tfinal=0.2)
        claw.num_output_times = 2
        return claw
    a, b = _pair(make, dt_variable=False, dt_initial=0.002)
    _same(a, b)
    for device_loop in (True, False):
        claw = make()
        claw.solver.device_time_loop = device_loop
        claw.solver.dt_variable = False
        claw.solver.dt_initial = 0.02  # CFL 4: the first step already fails
        with pytest.raises(CFLError):
            claw.run()


def test_max_steps_reached():
    msgs = []
    for device_loop in (True, False):
        claw = workloads.acoustics_wall(n=100, tfinal=0.4)
        claw.num_output_times = 1   # one interval of many more than 7 steps
        claw.solver.device_time_loop = device_loop
        claw.solver.max_steps = 7
        with pytest.raises(Exception) as ei:
            claw.run()
        msgs.append((str(ei.value), claw.solution.t, claw.solver.status['numsteps']))
    assert msgs[0][2] == msgs[1][2] == 7
    assert _close(msgs[0][1], msgs[1][1])
    for m in msgs:
        assert m[0].startswith("max_steps = 7 steps taken"), m[0]


@pytest.mark.parametrize("variant,rows", [(1, 8), (2, 16), (4, 8)])
def test_device_loop_launch_variants(variant, rows):
    # the loop's own kernel instantiations for the 3-CTA register cap, a TMA
    # request (the loop loads rows directly) and the two-barrier tile
    from pyclaw_b200 import _lib, tune
    tune.set_shape(_lib.RP_EULER_ROE, variant, rows)
    try:
        a, b = _pair(lambda: workloads.euler_quadrants_unsplit(n=160, tfinal=0.15))
    finally:
        tune.set_shape(_lib.RP_EULER_ROE, 0, 0)
    assert a.solver.status['numsteps'] > 10
    _same(a, b)


def test_device_loop_capacity_form():
    # the annulus (capacity function, aux edge velocities) with extrapolated
    # aux ghost cells in r, so no host fill is needed between steps
    from pyclaw_b200.solver import BC

    def make():
        claw = workloads.advection_annulus(m_r=40, m_theta=120, tfinal=0.4, num_output_times=2)
        s = claw.solver
        s.aux_bc_lower[0] = s.aux_bc_upper[0] = BC.extrap
        return claw
    a, b = _pair(make)
    assert a.solver.status['numsteps'] > 5
    _same(a, b)
