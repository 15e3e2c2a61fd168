"""Row-slab decomposition on CPU ranks (gloo, world size 2 and 3): the
package's halo exchange, boundary bookkeeping and global CFL, with the oracle
as the local step, must reproduce the single-domain oracle run exactly (every
interface sees the same inputs, so the results are bitwise equal)."""
import datetime
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _oracle_slab_class():
    import torch
    from oracle import pyoracle
    from pyclaw_b200 import slabs
    Orc = pyoracle.make_solver_class()

    class OracleSlab(Orc):
        def __init__(self, riemann_solver=None, claw_package=None):
            self.slab = None
            self.global_delta = None
            self.transport = None
            super().__init__(riemann_solver, claw_package)

        def step_hyperbolic(self, solution):
            rank, world, periodic, group = self.slab
            state = solution.states[0]
            dx, dy = self.global_delta
            my = state.grid.num_cells[1]
            qbc = self.qbc
            qbc[:, 2:-2, 2:-2] = state._q
            t = torch.from_numpy(qbc)  # (meqn, mx+4, my+4); rows are the last axis
            slabs.exchange_rows(lambda a, b: t[:, :, a:b].contiguous(),
                                lambda a, b, x: t[:, :, a:b].copy_(x), my, rank, world, periodic, group,
                                self.transport)
            lo, up = slabs.local_bcs(self.bc_lower, self.bc_upper, rank, world)
            pyoracle.bc_fill(qbc, lo, up)
            qold = qbc.copy(order="F")
            cp = self.rp.cparam(state.problem_data)
            cfl = pyoracle.step2(qold, qbc, dx, dy, self.dt, self._method, self._mthlim, self.rp.rp_id, cp)
            self.cfl.update_global_max(slabs.global_cfl(cfl, group=group, transport=self.transport))
            state._q = np.asfortranarray(qbc[:, 2:-2, 2:-2].copy())

    return OracleSlab


def _problem(name, cls):
    from pyclaw_b200 import workloads
    if name == "acoustics_wall":
        return workloads.acoustics_wall(cls, n=36, tfinal=1.0)
    if name == "advection_periodic":
        return workloads.advection_2d(cls, dimensional_split=False, transverse_waves=2, mx=30, my=33)
    if name == "euler_extrap":
        return workloads.euler_quadrants_unsplit(cls, n=40)
    raise ValueError(name)


def _worker(rank, world, port, name, nsteps, outdir):
    import sys
    sys.path.insert(0, ROOT)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        from pyclaw_b200 import slabs
        claw = _problem(name, _oracle_slab_class())
        claw, (start, count) = slabs.localize(claw, rank, world)
        s, sol = claw.solver, claw.solution
        s.setup(sol)
        s.dt = s.dt_initial
        dts = []
        for _ in range(nsteps):
            s.evolve_to_time(sol)
            dts.append(s.dt)
        np.savez(os.path.join(outdir, "rank%d.npz" % rank), q=sol.state.get_q_global(), start=start,
                 dts=np.array(dts), t=sol.t)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("name,world", [("acoustics_wall", 2), ("advection_periodic", 2),
                                        ("advection_periodic", 3), ("euler_extrap", 3)])
def test_slab_run_equals_single_domain(oracle, tmp_path, name, world):
    nsteps = 12
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, name, nsteps, str(tmp_path)))
             for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    parts = [np.load(os.path.join(tmp_path, "rank%d.npz" % r)) for r in range(world)]
    q_slabs = np.concatenate([p["q"] for p in parts], axis=2)

    claw = _problem(name, oracle.make_solver_class())
    s, sol = claw.solver, claw.solution
    s.setup(sol)
    s.dt = s.dt_initial
    dts = []
    for _ in range(nsteps):
        s.evolve_to_time(sol)
        dts.append(s.dt)
    assert np.array_equal(parts[0]["dts"], np.array(dts))
    assert float(parts[0]["t"]) == sol.t
    assert np.array_equal(q_slabs, sol.state.get_q_global())


@pytest.mark.parametrize("name,world", [("euler_extrap", 2), ("advection_periodic", 3)])
def test_thread_transport_slabs_equal_single_domain(oracle, name, world):
    # the same decomposition with the in-process transport (threads, one
    # mailbox and barrier) that the one-GPU device test uses
    import threading
    from pyclaw_b200 import slabs
    nsteps = 8
    hub = slabs.ThreadTransport(world)
    out, errs = {}, []

    def worker(rank):
        try:
            claw, (start, count) = slabs.localize(_problem(name, _oracle_slab_class()), rank, world)
            s, sol = claw.solver, claw.solution
            s.transport = hub.endpoint(rank)
            s.setup(sol)
            s.dt = s.dt_initial
            for _ in range(nsteps):
                s.evolve_to_time(sol)
            out[rank] = (sol.state.get_q_global(), sol.t)
        except BaseException as e:  # noqa: B902
            errs.append(e)
            hub.barrier.abort()

    threads = [threading.Thread(target=worker, args=(r,)) for r in range(world)]
    for t in threads:
        t.start()
    for t in threads:
        t.join(120)
    assert not errs, errs
    claw = _problem(name, oracle.make_solver_class())
    s, sol = claw.solver, claw.solution
    s.setup(sol)
    s.dt = s.dt_initial
    for _ in range(nsteps):
        s.evolve_to_time(sol)
    assert np.array_equal(np.concatenate([out[r][0] for r in range(world)], axis=2), sol.state.get_q_global())
    assert all(out[r][1] == sol.t for r in range(world))


def test_partition_and_bcs():
    from pyclaw_b200 import slabs
    rows = [slabs.partition(10, 3, r) for r in range(3)]
    assert rows == [(0, 4), (4, 3), (7, 3)]
    assert slabs.local_bcs([1, 3], [1, 3], 0, 2) == ([1, 3], [1, -1])
    assert slabs.local_bcs([1, 3], [1, 3], 1, 2) == ([1, -1], [1, 3])
    assert slabs.local_bcs([2, 2], [2, 2], 0, 2) == ([2, -1], [2, -1])
    assert slabs.neighbours(0, 3, True) == (2, 1) and slabs.neighbours(0, 3, False) == (None, 1)


def test_batch_partition_balances_cells_over_ranks():
    # the batched workload's seeded sides (512 problems, side in {64, 80, ..., 512})
    from pyclaw_b200.batch import partition_instances
    rng = np.random.default_rng(2024)
    sides = []
    for _ in range(512):
        sides.append(int(rng.choice(tuple(range(64, 513, 16)))))
        rng.uniform(0.3, 0.7, size=2)
        for _q in range(4):
            rng.uniform(0.1, 2.0, size=2)
            rng.uniform(-1.0, 1.0, size=2)
    cells = np.array(sides) ** 2
    for world in (1, 2, 4, 8):
        parts = partition_instances(cells, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(512))
        loads = np.array([cells[p].sum() for p in parts])
        assert loads.max() <= loads.mean() + cells.max()
        assert loads.max() / loads.mean() < 1.01
        assert parts == partition_instances(cells, world)
