"""Row-slab domain decomposition: one process per GPU.

The reference's only parallel path is petclaw (src/petclaw/): a PETSc DMDA
splits the grid; before each step ``globalToLocal`` fills every patch's ghost
cells from its neighbours (src/petclaw/state.py:205-229, stencil width =
num_ghost), physical boundary conditions apply only on the true domain
boundary (src/pyclaw/solver.py:377-437 with geometry on_lower/upper_boundary,
src/petclaw/geometry.py:30-40), and the CFL number is a global maximum
(src/petclaw/cfl.py:15-35).

Here rank r owns a contiguous band of rows (the y direction) of the global
grid.  Per step:
  1. halo exchange: the first and last two interior rows go to the lower and
     upper neighbours (torch.distributed point-to-point: NCCL over NVLink for
     device tensors, gloo for host tensors), wrapping around for periodic y;
  2. the device ghost fill applies the x rule everywhere and the y rule only
     on true boundaries (internal sides carry CLAW2_BC_NONE);
  3. the local step;
  4. one all-reduce (MAX) of the Courant number, so every rank takes the same
     accept/reject decision and the same next dt.
The halo rows land in the receiving rank's own buffers before the step reads
them; no kernel reads another GPU's memory.
"""
import numpy as np

BC_NONE = -1


def partition(n, world, rank):
    """Rows [start, start + count) of an n-row grid owned by ``rank``."""
    base, extra = divmod(n, world)
    count = base + (1 if rank < extra else 0)
    start = rank * base + min(rank, extra)
    return start, count


def neighbours(rank, world, periodic):
    lower = rank - 1 if rank > 0 else (world - 1 if periodic else None)
    upper = rank + 1 if rank < world - 1 else (0 if periodic else None)
    return lower, upper


class DistTransport(object):
    """Halo messages and the Courant-number reduction over torch.distributed:
    NCCL over NVLink for device tensors, gloo for host tensors."""

    def __init__(self, group=None):
        self.group = group

    def exchange(self, sends, recvs):
        """Post every send ``(tensor, dst)`` and receive ``(buffer, src)`` of one
        phase together and wait for all of them."""
        import torch.distributed as dist
        ops = [dist.P2POp(dist.isend, t, dst, self.group) for t, dst in sends]
        ops += [dist.P2POp(dist.irecv, b, src, self.group) for b, src in recvs]
        for r in dist.batch_isend_irecv(ops) if ops else []:
            r.wait()

    def max(self, value, device=None):
        import torch
        import torch.distributed as dist
        if not dist.is_initialized() or dist.get_world_size(self.group) == 1:
            return float(value)
        t = torch.tensor([float(value)], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX, group=self.group)
        return float(t.item())


class ThreadTransport(object):
    """The same two operations between slabs stepped by threads of one
    process (several slabs on one device, or on the host): a shared mailbox
    and a barrier.  Device rows are complete before they are posted (the
    poster synchronises the device), so no kernel ever waits on another
    slab's kernels."""

    def __init__(self, world, timeout=120.0):
        import threading
        self.world = world
        self.barrier = threading.Barrier(world, timeout=timeout)  # a failed slab breaks it for all
        self.box = {}
        self.vals = [0.0] * world

    def endpoint(self, rank):
        return _ThreadEndpoint(self, rank)


class _ThreadEndpoint(object):
    def __init__(self, hub, rank):
        self.hub, self.rank = hub, rank

    def exchange(self, sends, recvs):
        import torch
        hub = self.hub
        if any(t.is_cuda for t, _ in sends):
            torch.cuda.synchronize()
        for t, dst in sends:
            hub.box[(self.rank, dst)] = t
        hub.barrier.wait()
        for b, src in recvs:
            b.copy_(hub.box[(src, self.rank)])
        if any(b.is_cuda for b, _ in recvs):
            torch.cuda.synchronize()
        hub.barrier.wait()
        for t, dst in sends:
            del hub.box[(self.rank, dst)]
        hub.barrier.wait()

    def max(self, value, device=None):
        hub = self.hub
        hub.vals[self.rank] = float(value)
        hub.barrier.wait()
        m = max(hub.vals)
        hub.barrier.wait()
        return m


def exchange_rows(get_rows, set_rows, my_local, rank, world, periodic, group=None, transport=None):
    """Fill the two ghost rows on each internal side from the neighbours.

    ``get_rows(j0, j1)`` returns a contiguous tensor with padded rows
    [j0, j1) of the local array (padded row = interior row + 2);
    ``set_rows(j0, j1, t)`` stores one.  Two phases, each with at most one
    message per ordered pair of ranks, so matching never depends on tags
    (NCCL ignores them): first every rank sends its top rows up, then its
    bottom rows down.  ``transport`` carries the messages (default: a
    DistTransport over ``group``).
    """
    if world == 1:
        return
    tr = transport if transport is not None else DistTransport(group)
    lower, upper = neighbours(rank, world, periodic)
    # phase 1: top interior rows -> upper neighbour's lower halo
    sends = [(get_rows(my_local, my_local + 2), upper)] if upper is not None else []
    recv = get_rows(0, 2).clone() if lower is not None else None
    tr.exchange(sends, [(recv, lower)] if recv is not None else [])
    if recv is not None:
        set_rows(0, 2, recv)
    # phase 2: bottom interior rows -> lower neighbour's upper halo
    sends = [(get_rows(2, 4), lower)] if lower is not None else []
    recv = get_rows(my_local + 2, my_local + 4).clone() if upper is not None else None
    tr.exchange(sends, [(recv, upper)] if recv is not None else [])
    if recv is not None:
        set_rows(my_local + 2, my_local + 4, recv)


def global_cfl(local_cfl, device=None, group=None, transport=None):
    """MAX of the Courant number over ranks (src/petclaw/cfl.py:34-35)."""
    tr = transport if transport is not None else DistTransport(group)
    return tr.max(local_cfl, device=device)


def local_bcs(bc_lower, bc_upper, rank, world):
    """Boundary codes of one slab: internal y sides become BC_NONE (their
    ghost rows come from the halo exchange; periodic y across ranks too)."""
    lo, up = list(bc_lower), list(bc_upper)
    if world > 1:
        if rank > 0 or lo[1] == 2:
            lo[1] = BC_NONE
        if rank < world - 1 or up[1] == 2:
            up[1] = BC_NONE
    return lo, up


def slice_rows(q, start, count):
    """Rows [start, start+count) of a global q (num_eqn, mx, my), F-order."""
    return np.asfortranarray(q[:, :, start:start + count])


def localize(claw, rank, world, group=None):
    """Turn a Controller built for the global grid into this rank's slab:
    its Solution keeps rows partition(my, world, rank) of q; the solver (a
    make_slab_solver_class class) learns its rank, the y periodicity and the
    global cell sizes.  Returns the controller and (first row, row count)."""
    from .geometry import Dimension, Domain
    from .solution import Solution
    from .solver import BC
    from .state import State
    sol = claw.solution
    st = sol.state
    mx, my = st.grid.num_cells
    xdim, ydim = st.grid.dimensions
    start, count = partition(my, world, rank)
    if world > 1 and count < 2:
        raise ValueError("each slab needs at least 2 rows (my=%d, %d ranks)" % (my, world))
    dy = ydim.delta
    ly = Dimension(ydim.lower + start * dy, ydim.lower + (start + count) * dy, count, name=ydim.name)
    dom = Domain([xdim, ly])
    lst = State(dom, st.num_eqn)
    lst.problem_data = dict(st.problem_data)
    lst.t = st.t
    lst.q = st.get_q_global()[:, :, start:start + count]
    claw.solution = Solution(lst, dom)
    periodic = claw.solver.bc_lower[1] == BC.periodic
    claw.solver.slab = (rank, world, periodic, group)
    claw.solver.global_delta = (xdim.delta, dy)
    return claw, (start, count)


class DevicePlanes(object):
    """Torch view of a patch's current device q planes [num_eqn, my+4, pitch]
    (for the halo exchange on device memory)."""

    def __init__(self, patch):
        import ctypes
        import torch
        from . import _lib
        ptr = ctypes.POINTER(ctypes.c_double)()
        lay = (ctypes.c_longlong * 4)()
        _lib.check(patch._lib.claw2_patch_device_q(patch.h, ctypes.byref(ptr), lay))
        ny, pitch, plane = int(lay[1]), int(lay[2]), int(lay[3])
        meqn = patch.desc.num_eqn
        addr = ctypes.cast(ptr, ctypes.c_void_p).value

        class _Iface(object):
            __cuda_array_interface__ = {"shape": (meqn, ny, pitch), "typestr": "<f8",
                                        "data": (addr, False), "version": 2,
                                        "strides": (plane * 8, pitch * 8, 8)}
        self.t = torch.as_tensor(_Iface(), device="cuda")

    def get_rows(self, j0, j1):
        return self.t[:, j0:j1, :].contiguous()

    def set_rows(self, j0, j1, x):
        self.t[:, j0:j1, :].copy_(x)


def make_slab_solver_class(base):
    """A ClawSolver2D subclass (of ``base``) that steps one slab of a
    row-decomposed grid: halo exchange before the step, global CFL after."""

    class SlabClawSolver2D(base):
        def __init__(self, riemann_solver=None, claw_package=None):
            self.slab = None          # (rank, world, periodic_y, group)
            self.global_delta = None  # (dx, dy) of the global grid
            self.transport = None     # halo/CFL transport (None: torch.distributed over the group)
            self.overlap = False      # step the interior row blocks while the halo rows move
            self._stream_set = False  # the patch runs on torch's current stream (with the halo copies)
            self._side = None         # the halo exchange's stream when overlapping
            super().__init__(riemann_solver, claw_package)

        def _device_desc(self, solution):
            d = super()._device_desc(solution)
            rank, world, periodic, group = self.slab
            if self.global_delta is not None:
                d.dx, d.dy = self.global_delta
            lo, up = local_bcs([d.bc_lower[0], d.bc_lower[1]], [d.bc_upper[0], d.bc_upper[1]], rank, world)
            d.bc_lower[1], d.bc_upper[1] = lo[1], up[1]
            return d

        def step_hyperbolic(self, solution):
            rank, world, periodic, group = self.slab
            state = solution.states[0]
            dev = self._dev
            if dev is None or state._mirror is not dev:
                self._make_device_patch(solution)
                dev = self._dev
            if dev.host_dirty:
                dev.push(state)
            if not self._stream_set:
                import torch
                dev.set_stream(torch.cuda.current_stream().cuda_stream)  # one stream for NCCL + kernels
                self._stream_set = True
            my = state.grid.num_cells[1]
            if world > 1 and self.overlap:
                # interior row blocks on the patch's stream while the halo rows
                # move on a side stream (the interior neither reads nor writes
                # them), then the ghost corners and the edge row blocks
                import torch
                main = torch.cuda.current_stream()
                if self._side is None:
                    self._side = torch.cuda.Stream()
                ready = torch.cuda.Event()
                ready.record(main)              # the current q (last step accepted) is complete
                dev.step_part(self.dt, 1)
                with torch.cuda.stream(self._side):
                    self._side.wait_event(ready)
                    planes = DevicePlanes(dev)
                    exchange_rows(planes.get_rows, planes.set_rows, my, rank, world, periodic, group, self.transport)
                    moved = torch.cuda.Event()
                    moved.record(self._side)
                main.wait_event(moved)
                cfl = dev.step_part(self.dt, 2)
            else:
                if world > 1:
                    planes = DevicePlanes(dev)
                    exchange_rows(planes.get_rows, planes.set_rows, my, rank, world, periodic, group,
                                  self.transport)
                cfl = dev.step(self.dt)
            self.cfl.update_global_max(global_cfl(cfl, device="cuda", group=group, transport=self.transport))

    return SlabClawSolver2D
