"""The row-slab decomposition's device path on one GPU: 2 and 3 slabs of one
problem, each a SlabClawSolver2D with its own device patch, stepped by threads
of one process that exchange halo rows through DevicePlanes (device copies
into the receiving patch's own planes) and reduce the Courant number through
a ThreadTransport.  The ghost fill skips the internal sides (CLAW2_BC_NONE),
the slabs take the same dt and accept decisions, and the result must equal
the single-domain device run bit for bit (every interface sees the same
inputs and sums its cell's increments in the same order, whatever the rows a
patch holds).  No kernel waits on another slab: the threads synchronise on
the host."""
import threading

import numpy as np
import pytest

from pyclaw_b200 import classic, slabs, workloads

pytestmark = pytest.mark.gpu


def _problem(name, cls=None):
    if name == "euler_extrap":
        return workloads.euler_quadrants_unsplit(cls, n=192)
    if name == "acoustics_wall":
        return workloads.acoustics_wall(cls, n=150, tfinal=1.0)
    if name == "advection_periodic":
        return workloads.advection_2d(cls, dimensional_split=False, transverse_waves=2, mx=90, my=61)
    if name == "shallow_split":
        return workloads.radial_dam_break(cls, mx=96, my=80)
    raise ValueError(name)


def _slab_run(name, world, nsteps, overlap=False):
    hub = slabs.ThreadTransport(world)
    out, errs = {}, []

    def worker(rank):
        try:
            import torch
            torch.cuda.set_device(0)
            cls = slabs.make_slab_solver_class(classic.ClawSolver2D)
            claw, (start, count) = slabs.localize(_problem(name, cls), rank, world)
            s, sol = claw.solver, claw.solution
            s.transport = hub.endpoint(rank)
            s.overlap = overlap
            s.setup(sol)
            s.dt = s.dt_initial
            dts = []
            for _ in range(nsteps):
                s.evolve_to_time(sol)
                dts.append(s.dt)
            out[rank] = (sol.state.get_q_global(), dts, sol.t, s.status['numsteps'])
        except BaseException as e:  # noqa: B902 -- any failure must release the other slabs
            errs.append(e)
            hub.barrier.abort()

    threads = [threading.Thread(target=worker, args=(r,)) for r in range(world)]
    for t in threads:
        t.start()
    for t in threads:
        t.join(300)
    assert not errs, errs
    assert len(out) == world
    return out


@pytest.mark.parametrize("overlap", [False, True])
@pytest.mark.parametrize("name,world", [("euler_extrap", 2), ("euler_extrap", 3), ("acoustics_wall", 2),
                                        ("advection_periodic", 3), ("shallow_split", 2)])
def test_device_slabs_equal_single_domain(name, world, overlap):
    # overlap: each step in two parts around the halo exchange (interior row
    # blocks, then ghost corners and edge row blocks; claw2_patch_step_part)
    nsteps = 10
    parts = _slab_run(name, world, nsteps, overlap)
    q_slabs = np.concatenate([parts[r][0] for r in range(world)], axis=2)
    claw = _problem(name)
    s, sol = claw.solver, claw.solution
    s.setup(sol)
    s.dt = s.dt_initial
    dts = []
    for _ in range(nsteps):
        s.evolve_to_time(sol)
        dts.append(s.dt)
    for r in range(world):
        assert parts[r][1] == dts and parts[r][2] == sol.t and parts[r][3] == s.status['numsteps']
    assert np.array_equal(q_slabs, sol.state.get_q_global())


@pytest.mark.parametrize("name,rows", [("euler_extrap", 8), ("acoustics_wall", 4), ("euler_extrap", 0),
                                       ("advection_periodic", 4)])  # 61 rows: a last block of one row
def test_step_in_two_parts_equals_whole_step(name, rows):
    # one patch, no internal sides: part 1 (every ghost cell, interior row
    # blocks) + part 2 (edge row blocks) gives claw2_patch_step's result bit
    # for bit, on several row heights (rows 0: the heuristic)
    from pyclaw_b200 import _lib, tune
    rp = _problem(name).solver.rp.rp_id
    tune.set_shape(rp, 0, rows)
    try:
        outs = []
        for split in (False, True):
            claw = _problem(name)
            s, sol = claw.solver, claw.solution
            s.setup(sol)
            dev = s._dev
            dt = 0.4 * min(sol.state.grid.delta) / 3.0
            cfls = []
            for _ in range(4):
                if split:
                    dev.step_part(dt, 1)
                    cfls.append(dev.step_part(dt, 2))
                else:
                    cfls.append(dev.step(dt))
                dev.accept(True)
            outs.append((sol.state.get_q_global(), cfls))
        assert outs[0][1] == outs[1][1]
        assert np.array_equal(outs[0][0], outs[1][0])
    finally:
        tune.set_shape(rp, 0, 0)


def test_step_part_order_is_checked():
    from pyclaw_b200 import _lib
    claw = _problem("acoustics_wall")
    s, sol = claw.solver, claw.solution
    s.setup(sol)
    dev = s._dev
    with pytest.raises(_lib.Claw2Error):
        dev.step_part(1e-3, 2)          # part 2 without part 1
    dev.step_part(1e-3, 1)
    with pytest.raises(_lib.Claw2Error):
        dev.step(1e-3)                  # a whole step while part 1 waits for its part 2
    with pytest.raises(_lib.Claw2Error):
        dev.step_part(1e-3, 1)          # part 1 twice
    dev.step_part(1e-3, 2)
    dev.accept(True)
