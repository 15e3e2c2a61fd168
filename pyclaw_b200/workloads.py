"""Problem setups: the reference's 2D classic regression examples and the
benchmark workloads, each returning a ready-to-run Controller.

The regression examples restate the setups of the reference's examples
(initial data evaluated with the same numpy expressions, so the grids match
bit for bit):
  advection_2d              examples/advection_2d/advection_2d.py:19-81
  acoustics_2d_homogeneous  examples/acoustics_2d_homogeneous/acoustics_2d.py:20-106
  quadrants                 examples/euler_2d/quadrants.py:73-126
  radial_dam_break          examples/shallow_2d/radial_dam_break.py:23-87
  acoustics_variable        examples/acoustics_2d_variable/acoustics_2d_interface.py:23-96
  advection_annulus         examples/advection_2d_annulus/advection_annulus.py:22-213
  psystem                   examples/psystem_2d/psystem_2d.py:26-235
  advection_reaction        examples/advection_reaction_2d/advection_reaction.py:37-114
  shock_bubble              examples/euler_2d/shock_bubble_interaction.py:36-220
The benchmark workloads are the acoustics, Euler-quadrant and shallow-water
dam-break problems at the benchmark sizes (unsplit step, transverse
corrections, MC limiter).

``solver_class`` lets tests run the same setup through another ClawSolver2D
subclass; by default the CUDA solver is used.
"""
import numpy as np

from . import riemann
from .classic import ClawSolver2D
from .controller import Controller
from .geometry import Dimension, Domain
from .limiters import tvd
from .solution import Solution
from .solver import BC
from .state import State


def _controller(solver, solution, tfinal, num_output_times=10, keep_copy=True):
    claw = Controller()
    claw.solution = solution
    claw.solver = solver
    claw.tfinal = tfinal
    claw.num_output_times = num_output_times
    claw.keep_copy = keep_copy
    claw.output_format = None
    return claw


def advection_2d(solver_class=None, dimensional_split=True, transverse_waves=0, mx=50, my=50):
    cls = solver_class or ClawSolver2D
    solver = cls(riemann.advection_2D)
    solver.dimensional_split = dimensional_split
    solver.transverse_waves = transverse_waves
    solver.limiters = tvd.vanleer
    solver.bc_lower[0] = BC.periodic
    solver.bc_upper[0] = BC.periodic
    solver.bc_lower[1] = BC.periodic
    solver.bc_upper[1] = BC.periodic
    if not dimensional_split and not transverse_waves:
        solver.cfl_max = 0.5
        solver.cfl_desired = 0.45
    else:
        solver.cfl_max = 1.0
        solver.cfl_desired = 0.9
    x = Dimension(0.0, 1.0, mx, name='x')
    y = Dimension(0.0, 1.0, my, name='y')
    domain = Domain([x, y])
    state = State(domain, 1)
    state.problem_data['u'] = 0.5
    state.problem_data['v'] = 1.0
    X, Y = state.grid.p_centers
    state.q[0, :, :] = 0.9 * (0.1 < X) * (X < 0.6) * (0.1 < Y) * (Y < 0.6) + 0.1
    return _controller(solver, Solution(state, domain), 2.0)


def acoustics_2d_homogeneous(solver_class=None, mx=100, my=100):
    cls = solver_class or ClawSolver2D
    solver = cls(riemann.acoustics_2D)
    solver.dimensional_split = True
    solver.cfl_max = 0.5
    solver.cfl_desired = 0.45
    solver.limiters = tvd.MC
    solver.bc_lower[0] = BC.extrap
    solver.bc_upper[0] = BC.extrap
    solver.bc_lower[1] = BC.extrap
    solver.bc_upper[1] = BC.extrap
    x = Dimension(-1.0, 1.0, mx, name='x')
    y = Dimension(-1.0, 1.0, my, name='y')
    domain = Domain([x, y])
    state = State(domain, 3)
    rho = 1.0
    bulk = 4.0
    cc = np.sqrt(bulk / rho)
    zz = rho * cc
    state.problem_data['rho'] = rho
    state.problem_data['bulk'] = bulk
    state.problem_data['zz'] = zz
    state.problem_data['cc'] = cc
    solver.dt_initial = np.min(domain.grid.delta) / state.problem_data['cc'] * solver.cfl_desired
    X, Y = state.grid.p_centers
    r = np.sqrt(X ** 2 + Y ** 2)
    width = 0.2
    state.q[0, :, :] = (np.abs(r - 0.5) <= width) * (1. + np.cos(np.pi * (r - 0.5) / width))
    state.q[1, :, :] = 0.
    state.q[2, :, :] = 0.
    return _controller(solver, Solution(state, domain), 0.12)


def quadrants(solver_class=None, mx=100, my=100, efix=None):
    cls = solver_class or ClawSolver2D
    solver = cls(riemann.euler_4wave_2D)
    solver.transverse_waves = 2
    solver.all_bcs = BC.extrap
    domain = Domain([0., 0.], [1., 1.], [mx, my])
    solution = Solution(4, domain)
    gamma = 1.4
    solution.problem_data['gamma'] = gamma
    if efix is not None:
        solution.problem_data['efix'] = efix
    xx, yy = domain.grid.p_centers
    l = xx < 0.8
    r = xx >= 0.8
    b = yy < 0.8
    t = yy >= 0.8
    q = solution.q
    q[0, ...] = 1.5 * r * t + 0.532258064516129 * l * t \
        + 0.137992831541219 * l * b \
        + 0.532258064516129 * r * b
    u = 0.0 * r * t + 1.206045378311055 * l * t \
        + 1.206045378311055 * l * b \
        + 0.0 * r * b
    v = 0.0 * r * t + 0.0 * l * t \
        + 1.206045378311055 * l * b \
        + 1.206045378311055 * r * b
    p = 1.5 * r * t + 0.3 * l * t + 0.029032258064516 * l * b + 0.3 * r * b
    q[1, ...] = q[0, ...] * u
    q[2, ...] = q[0, ...] * v
    q[3, ...] = 0.5 * q[0, ...] * (u ** 2 + v ** 2) + p / (gamma - 1.0)
    return _controller(solver, solution, 0.8)


def radial_dam_break(solver_class=None, mx=150, my=150, h_in=2., h_out=1., dam_radius=0.5, riemann_solver='roe'):
    cls = solver_class or ClawSolver2D
    rs = {'roe': riemann.shallow_roe_with_efix_2D, 'hlle': riemann.shallow_hlle_2D}[riemann_solver.lower()]
    solver = cls(rs)
    solver.limiters = tvd.MC
    solver.dimensional_split = 1
    solver.bc_lower[0] = BC.extrap
    solver.bc_upper[0] = BC.wall
    solver.bc_lower[1] = BC.extrap
    solver.bc_upper[1] = BC.wall
    x = Dimension(-2.5, 2.5, mx, name='x')
    y = Dimension(-2.5, 2.5, my, name='y')
    domain = Domain([x, y])
    state = State(domain, 3)
    state.problem_data['grav'] = 1.0
    X, Y = state.p_centers
    r = np.sqrt((X - 0.) ** 2 + (Y - 0.) ** 2)
    state.q[0, :, :] = h_in * (r <= dam_radius) + h_out * (r > dam_radius)
    state.q[1, :, :] = 0.
    state.q[2, :, :] = 0.
    return _controller(solver, Solution(state, domain), 2.5)


# ---------------------------------------------------------------------------
# Benchmark workloads (unsplit step2 with transverse corrections)
# ---------------------------------------------------------------------------
def acoustics_wall(solver_class=None, n=200, tfinal=0.6):
    """Linear acoustics, rho=1, K=4 (c=2), [-1,1]^2, wall BCs, MC limiter,
    unsplit trans_cor, CFL 0.9; p = exp(-100((x-0.25)^2 + y^2)), u = v = 0."""
    cls = solver_class or ClawSolver2D
    solver = cls(riemann.acoustics_2D)
    solver.dimensional_split = False
    solver.transverse_waves = 2
    solver.limiters = tvd.MC
    solver.cfl_max = 1.0
    solver.cfl_desired = 0.9
    solver.all_bcs = BC.wall
    domain = Domain([-1.0, -1.0], [1.0, 1.0], [n, n])
    state = State(domain, 3)
    rho, bulk = 1.0, 4.0
    cc = np.sqrt(bulk / rho)
    state.problem_data.update(rho=rho, bulk=bulk, cc=cc, zz=rho * cc)
    X, Y = state.grid.p_centers
    state.q[0, ...] = np.exp(-100.0 * ((X - 0.25) ** 2 + Y ** 2))
    state.q[1, ...] = 0.0
    state.q[2, ...] = 0.0
    solver.dt_initial = np.min(domain.grid.delta) / cc * solver.cfl_desired
    return _controller(solver, Solution(state, domain), tfinal)


def acoustics_variable(solver_class=None, n=50, tfinal=0.6, num_output_times=20):
    """Acoustics in two materials (vc_acoustics_2D, aux = density and sound
    speed): rho = 4, K = 4 for x < 0 and rho = 1, K = 4 for x >= 0 on
    [-1,1]^2; a pressure ring of radius 0.25 around (-0.5, 0); wall BCs at
    the lower and extrapolation at the upper sides for q and aux; MC limiter,
    unsplit with the reference's default transverse mode (trans_inc)."""
    cls = solver_class or ClawSolver2D
    solver = cls(riemann.vc_acoustics_2D)
    solver.dimensional_split = False
    solver.limiters = tvd.MC
    solver.bc_lower[0] = BC.wall
    solver.bc_upper[0] = BC.extrap
    solver.bc_lower[1] = BC.wall
    solver.bc_upper[1] = BC.extrap
    solver.aux_bc_lower[0] = BC.wall
    solver.aux_bc_upper[0] = BC.extrap
    solver.aux_bc_lower[1] = BC.wall
    solver.aux_bc_upper[1] = BC.extrap
    x = Dimension(-1.0, 1.0, n, name='x')
    y = Dimension(-1.0, 1.0, n, name='y')
    domain = Domain([x, y])
    state = State(domain, 3, 2)
    X, Y = state.grid.p_centers
    rho_left, rho_right, bulk_left, bulk_right = 4.0, 1.0, 4.0, 4.0
    c_left, c_right = np.sqrt(bulk_left / rho_left), np.sqrt(bulk_right / rho_right)
    state.aux[0, :, :] = rho_left * (X < 0.) + rho_right * (X >= 0.)
    state.aux[1, :, :] = c_left * (X < 0.) + c_right * (X >= 0.)
    x0, y0 = -0.5, 0.
    r = np.sqrt((X - x0) ** 2 + (Y - y0) ** 2)
    width, rad = 0.1, 0.25
    state.q[0, :, :] = (np.abs(r - rad) <= width) * (1. + np.cos(np.pi * (r - rad) / width))
    state.q[1, :, :] = 0.
    state.q[2, :, :] = 0.
    return _controller(solver, Solution(state, domain), tfinal, num_output_times=num_output_times)


def _annulus_map(xc, yc):
    """Polar mapping of the annulus: computational (r, theta) -> physical."""
    return [xc * np.cos(yc), xc * np.sin(yc)]


def _annulus_stream(xp, yp):
    """Stream function of the rigid rotation, one turn per unit time."""
    return np.pi * (xp ** 2 + yp ** 2)


def annulus_edge_aux(xn, yn, dx, dy):
    """aux of the cells spanned by the physical corner arrays xn, yn
    (ncells + 1 per axis): [0] the velocity through each cell's left edge and
    [1] through its bottom edge, differences of the stream function over the
    edge divided by the computational edge length; [2] the capacity, the
    physical area of the quadrilateral (shoelace formula) over dx dy."""
    mx, my = xn.shape[0] - 1, xn.shape[1] - 1
    aux = np.empty((3, mx, my), order='F')
    x0, y0 = xn[:mx, :my], yn[:mx, :my]   # lower left
    x1, y1 = xn[:mx, 1:], yn[:mx, 1:]     # upper left
    x2, y2 = xn[1:, 1:], yn[1:, 1:]       # upper right
    x3, y3 = xn[1:, :my], yn[1:, :my]     # lower right
    aux[0, :mx, :my] = (_annulus_stream(x1, y1) - _annulus_stream(x0, y0)) / dy
    aux[1, :mx, :my] = -(_annulus_stream(x3, y3) - _annulus_stream(x0, y0)) / dx
    area = 1. / 2. * ((y0 + y1) * (x1 - x0) + (y1 + y2) * (x2 - x1) +
                      (y2 + y3) * (x3 - x2) + (y3 + y0) * (x0 - x3))
    aux[2, :mx, :my] = area / (dx * dy)
    return aux


def _annulus_aux_lower(state, dim, t, qbc, auxbc, num_ghost):
    """Ghost cells inside the inner radius: the same edge velocities and
    areas, from the mapped corners of the ghost cells."""
    grid = state.grid
    if dim != grid.dimensions[0]:
        raise Exception('Custom BC for this boundary is not appropriate!')
    dx, dy = grid.delta
    xn, yn = grid.p_nodes_with_ghost(num_ghost=2)
    auxbc[:, 0:num_ghost, :] = annulus_edge_aux(xn[0:num_ghost + 1, :], yn[0:num_ghost + 1, :], dx, dy)


def _annulus_aux_upper(state, dim, t, qbc, auxbc, num_ghost):
    """Ghost cells outside the outer radius (see _annulus_aux_lower)."""
    grid = state.grid
    if dim != grid.dimensions[0]:
        raise Exception('Custom BC for this boundary is not appropriate!')
    dx, dy = grid.delta
    xn, yn = grid.p_nodes_with_ghost(num_ghost=2)
    auxbc[:, -num_ghost:, :] = annulus_edge_aux(xn[-num_ghost - 1:, :], yn[-num_ghost - 1:, :], dx, dy)


def advection_annulus(solver_class=None, m_r=40, m_theta=120, tfinal=1.0, num_output_times=10):
    """Advection by a rigid rotation on the annulus 0.2 <= r <= 1 (a mapped
    polar grid): vc_advection_2D with edge velocities in aux[0:2] and the
    cell area as capacity function in aux[2] (index_capa = 2); extrapolation
    in r and periodic in theta for q, custom (geometric) aux BCs in r;
    unsplit, transverse corrections, van Leer limiter, cfl 0.4 / 0.5; two
    Gaussian pulses of opposite sign."""
    cls = solver_class or ClawSolver2D
    solver = cls(riemann.vc_advection_2D)
    solver.dimensional_split = False
    solver.transverse_waves = 2
    solver.order = 2
    solver.bc_lower[0] = BC.extrap
    solver.bc_upper[0] = BC.extrap
    solver.bc_lower[1] = BC.periodic
    solver.bc_upper[1] = BC.periodic
    solver.aux_bc_lower[0] = BC.custom
    solver.aux_bc_upper[0] = BC.custom
    solver.user_aux_bc_lower = _annulus_aux_lower
    solver.user_aux_bc_upper = _annulus_aux_upper
    solver.aux_bc_lower[1] = BC.periodic
    solver.aux_bc_upper[1] = BC.periodic
    solver.dt_initial = 0.1
    solver.cfl_max = 0.5
    solver.cfl_desired = 0.4
    solver.limiters = tvd.vanleer
    r = Dimension(0.2, 1.0, m_r, name='r')
    theta = Dimension(0.0, np.pi * 2.0, m_theta, name='theta')
    domain = Domain([r, theta])
    domain.grid.mapc2p = _annulus_map
    domain.grid.num_ghost = solver.num_ghost
    state = State(domain, 1)
    xp, yp = state.grid.p_centers
    pulse = [(1., 40., -0.5, 0.), (-1., 40., 0.5, 0.)]  # amplitude, decay, x, y of the centre
    state.q[0, :, :] = sum(a * np.exp(-b * (np.square(xp - x0) + np.square(yp - y0))) for a, b, x0, y0 in pulse)
    dx, dy = state.grid.delta
    xn, yn = state.grid.p_nodes
    state.aux = annulus_edge_aux(xn, yn, dx, dy)
    state.index_capa = 2
    return _controller(solver, Solution(state, domain), tfinal, num_output_times=num_output_times)


def psystem_checkerboard_aux(x, y, KA=1., KB=4., rhoA=1., rhoB=4., stress_rel=2):
    """aux (4, len(x), len(y)) of the p-system's checkerboard medium of unit
    period: density and bulk modulus A in the squares where x and y are both
    in the lower or both in the upper half of their period, B elsewhere; the
    stress-strain relation; 0 for the strain slot that the step hook fills."""
    half = 0.5
    xf = x - np.floor(x / 1.) * 1.
    yf = y - np.floor(y / 1.) * 1.
    yg, xg = np.meshgrid(yf, xf)
    aux = np.zeros((4, len(x), len(y)), order='F')
    same = (xg <= half) * (yg <= half), (xg > half) * (yg > half)
    other = (xg > half) * (yg <= half), (xg <= half) * (yg > half)
    aux[0, :, :] = rhoA * same[0] + rhoA * same[1] + rhoB * other[0] + rhoB * other[1]
    aux[1, :, :] = KA * same[0] + KA * same[1] + KB * other[0] + KB * other[1]
    aux[2, :, :] = stress_rel
    return aux


def _psystem_strain_to_aux(solver, state):
    """Before each step: the strain into aux[3], where the transverse solver
    reads it."""
    state.aux[3, :, :] = state.q[0, :, :]


def _psystem_gauge_stress(q, aux):
    p = np.exp(q[0] * aux[1]) - 1
    return [p, 10 * p]


def _psystem_stress(state):
    K, rel, eps = state.aux[1, :, :], state.aux[2, :, :], state.q[0, :, :]
    state.p[0, :, :] = np.where(rel == 1, 1, 0) * K * eps + np.where(rel == 2, 1, 0) * (np.exp(eps * K) - 1)


def _psystem_energy(state):
    rho, K = state.aux[0, :, :], state.aux[1, :, :]
    u, v = state.q[1, :, :] / rho, state.q[2, :, :] / rho
    kinetic = rho * (u ** 2 + v ** 2) / 2.
    eps = state.q[0, :, :]
    sigma = np.exp(K * eps) - 1.
    potential = (sigma - np.log(sigma + 1.)) / K
    dx, dy = state.grid.delta
    state.F[0, :, :] = (potential + kinetic) * dx * dy


def psystem(solver_class=None, cells_per_layer=6, tfinal=1., outdir='./_output', num_output_times=10):
    """The 2D p-system in a checkerboard medium (psystem_2D, f-waves): a
    Gaussian stress pulse of amplitude 10 in the corner of [0.25, 20.25]^2,
    wall BCs at the lower and extrapolation at the upper sides (q and aux),
    superbee limiter, unsplit, cfl 0.8 / 0.9; a before-step hook copies the
    strain into aux[3]; four stress gauges kept in memory and written under
    outdir/_gauges; the energy functional written to outdir/F.txt."""
    cls = solver_class or ClawSolver2D
    solver = cls(riemann.psystem_2D)
    solver.dimensional_split = False
    solver.cfl_max = 0.9
    solver.cfl_desired = 0.8
    solver.limiters = tvd.superbee
    solver.bc_lower[0] = BC.wall
    solver.bc_upper[0] = BC.extrap
    solver.bc_lower[1] = BC.wall
    solver.bc_upper[1] = BC.extrap
    solver.aux_bc_lower[0] = BC.wall
    solver.aux_bc_upper[0] = BC.extrap
    solver.aux_bc_lower[1] = BC.wall
    solver.aux_bc_upper[1] = BC.extrap
    solver.fwave = True
    solver.before_step = _psystem_strain_to_aux
    x_lower, x_upper, y_lower, y_upper = 0.25, 20.25, 0.25, 20.25
    mx = int((x_upper - x_lower) * cells_per_layer)
    my = int((y_upper - y_lower) * cells_per_layer)
    domain = Domain([Dimension(x_lower, x_upper, mx, name='x'), Dimension(y_lower, y_upper, my, name='y')])
    state = State(domain, 3, 4)
    state.mF = 1
    state.mp = 1
    grid = state.grid
    state.aux = psystem_checkerboard_aux(grid.x.centers, grid.y.centers)
    # Gaussian stress, zero velocities (the first coordinate array of
    # c_centers is x; the pulse is symmetric in x and y)
    A, x0, y0, varx, vary = 10., 0.25, 0.25, 0.5, 0.5
    cx, cy = grid.c_centers
    stress = A * np.exp(-(cy - x0) ** 2 / (2 * varx) - (cx - y0) ** 2 / (2 * vary))
    rel, K = state.aux[2, :], state.aux[1, :]
    state.q[0, :, :] = np.where(rel == 1, 1, 0) * stress / K + np.where(rel == 2, 1, 0) * np.log(stress + 1) / K
    state.q[1, :, :] = 0
    state.q[2, :, :] = 0
    claw = _controller(solver, Solution(state, domain), tfinal, num_output_times=num_output_times)
    claw.outdir = outdir
    claw.compute_F = _psystem_energy
    claw.compute_p = _psystem_stress
    grid.add_gauges([[0.25, 0.25], [17.85, 1.25], [3.25, 18.75], [11.75, 11.75]])
    solver.compute_gauge_values = _psystem_gauge_stress
    state.keep_gauges = True
    return claw


REACTION_PERIOD = 4.0
REACTION_RATE = 0.1


def _reaction_source(solver, state, dt):
    """Forward-Euler step of the reaction p' = eps q, q' = eps p."""
    qq = state.q.copy()
    state.q[0, :, :] = state.q[0, :, :] + REACTION_RATE * dt * qq[1, :, :]
    state.q[1, :, :] = state.q[1, :, :] + REACTION_RATE * dt * qq[0, :, :]


def _reaction_psi(x, y):
    """Stream function of the swirling velocity field."""
    return (np.sin(np.pi * x)) ** 2 * (np.sin(np.pi * y)) ** 2 / np.pi


def _reaction_edge_velocities(aux, xn, yn, dx, dy):
    """u on the left and v on the bottom edge of every cell from the stream
    function at the cell corners."""
    aux[0, :, :] = - (_reaction_psi(xn[:-1, 1:], yn[:-1, 1:]) - _reaction_psi(xn[:-1, :-1], yn[:-1, :-1])) / dy
    aux[1, :, :] = (_reaction_psi(xn[1:, :-1], yn[1:, :-1]) - _reaction_psi(xn[:-1, :-1], yn[:-1, :-1])) / dx


def _reaction_velocities(solver, state):
    """Before each step: the velocity field at the middle of the step, the
    steady field scaled by cos(2 pi t / T)."""
    v_t = np.cos(2 * np.pi * (state.t + solver.dt / 2) / REACTION_PERIOD)
    xn, yn = state.grid.p_nodes
    dx, dy = state.grid.delta
    _reaction_edge_velocities(state.aux, xn, yn, dx, dy)
    state.aux[:] = v_t * state.aux[:]


def advection_reaction(solver_class=None, n=100, tfinal=REACTION_PERIOD, device_source=False,
                       num_output_times=10):
    """Two species carried by a time-periodic swirl with edge velocities
    (vc_advection_vector_2D, split step, no limiter choice: minmod) and a
    linear reaction coupling them through a Godunov-split source step;
    extrapolation BCs for q and aux; species 0 = 1 left of x = 0.5, species 1
    = 1 below y = 0.5.  device_source: the reaction as a LinearSource, which
    stays on the device, instead of the host function."""
    from .sources import LinearSource
    cls = solver_class or ClawSolver2D
    solver = cls(riemann.vc_advection_vector_2D)
    solver.dimensional_split = 1
    solver.all_bcs = BC.extrap
    solver.aux_bc_lower[0] = BC.extrap
    solver.aux_bc_upper[0] = BC.extrap
    solver.aux_bc_lower[1] = BC.extrap
    solver.aux_bc_upper[1] = BC.extrap
    domain = Domain((0., 0.), (1., 1.), (n, n))
    solver.num_eqn = 2
    solver.num_waves = 1
    solver.fwave = False
    state = State(domain, solver.num_eqn, 2)
    xn, yn = domain.grid.p_nodes
    xc, yc = domain.grid.p_centers
    dx, dy = domain.grid.delta
    _reaction_edge_velocities(state.aux, xn, yn, dx, dy)
    solver.before_step = _reaction_velocities
    solver.step_source = (LinearSource([[0., REACTION_RATE], [REACTION_RATE, 0.]]) if device_source
                          else _reaction_source)
    solver.source_split = 1
    state.q[0, :, :] = (xc <= 0.5)
    state.q[1, :, :] = (yc <= 0.5)
    return _controller(solver, Solution(state, domain), tfinal, num_output_times=num_output_times)


BUBBLE_GAMMA = 1.4
BUBBLE_CENTER, BUBBLE_RADIUS = (0.5, 0.), 0.2


def _post_shock_state(pinf=5., gamma=BUBBLE_GAMMA):
    """Density, velocity and energy behind a shock of pressure ratio pinf
    moving into gas at rest with unit density and pressure."""
    gamma1 = gamma - 1.
    rinf = (gamma1 + pinf * (gamma + 1.)) / ((gamma + 1.) + gamma1 * pinf)
    vinf = 1. / np.sqrt(gamma) * (pinf - 1.) / np.sqrt(0.5 * ((gamma + 1.) / gamma) * pinf + 0.5 * gamma1 / gamma)
    einf = 0.5 * rinf * vinf ** 2 + pinf / gamma1
    return rinf, vinf, einf


def _bubble_height(x, ymin, ymax):
    """Height of the part of the bubble (a disc) above x that lies in [ymin, ymax]."""
    x0, y0 = BUBBLE_CENTER
    r0 = BUBBLE_RADIUS
    if ((x - x0) ** 2) < (r0 ** 2):
        return max(min(y0 + np.sqrt(r0 ** 2 - (x - x0) ** 2), ymax) - ymin, 0.)
    return 0


def _bubble_qinit(state, rhoin=0.1, pinf=5.):
    """The shock at x = 0.2 moving right, a low-density bubble ahead of it;
    cells cut by the bubble's edge get the area-weighted mixture (quadrature
    of the disc's height over the cell)."""
    from scipy import integrate
    gamma = BUBBLE_GAMMA
    gamma1 = gamma - 1.
    grid = state.grid
    rhoout, pout, pin, xshock = 1., 1., 1., 0.2
    rinf, vinf, einf = _post_shock_state(pinf)
    X, Y = grid.p_centers
    x0, y0 = BUBBLE_CENTER
    r0 = BUBBLE_RADIUS
    r = np.sqrt((X - x0) ** 2 + (Y - y0) ** 2)
    state.q[0, :, :] = rinf * (X < xshock) + rhoin * (r <= r0) + rhoout * (r > r0) * (X >= xshock)
    state.q[1, :, :] = rinf * vinf * (X < xshock)
    state.q[2, :, :] = 0.
    state.q[3, :, :] = einf * (X < xshock) + (pin * (r <= r0) + pout * (r > r0) * (X >= xshock)) / gamma1
    state.q[4, :, :] = 1. * (r <= r0)
    d2 = np.linalg.norm(state.grid.delta) / 2.
    dx, dy = state.grid.delta
    dx2, dy2 = dx / 2., dy / 2.
    q = state.q
    for i in range(q.shape[1]):
        for j in range(q.shape[2]):
            ydown, yup = Y[i, j] - dy2, Y[i, j] + dy2
            if abs(r[i, j] - r0) < d2:
                infrac, _ = integrate.quad(_bubble_height, X[i, j] - dx2, X[i, j] + dx2, args=(ydown, yup),
                                           epsabs=1.e-8, epsrel=1.e-5)
                infrac = infrac / (dx * dy)
                q[0, i, j] = rhoin * infrac + rhoout * (1. - infrac)
                q[3, i, j] = (pin * infrac + pout * (1. - infrac)) / gamma1
                q[4, i, j] = 1. * infrac


def _incoming_shock(state, dim, t, qbc, auxbc, num_ghost):
    """Left boundary: the post-shock state flows in."""
    rinf, vinf, einf = _post_shock_state()
    for i in range(num_ghost):
        qbc[0, i, ...] = rinf
        qbc[1, i, ...] = rinf * vinf
        qbc[2, i, ...] = 0.
        qbc[3, i, ...] = einf
        qbc[4, i, ...] = 0.


def _euler_radial_source(solver, state, dt):
    """Geometric source of the axisymmetric Euler equations (r = aux[0] the
    radial coordinate): two-stage second-order Runge-Kutta over the step."""
    gamma = BUBBLE_GAMMA
    dt2 = dt / 2.
    q = state.q
    rad = state.aux[0, :, :]
    rho = q[0, :, :]
    u = q[1, :, :] / rho
    v = q[2, :, :] / rho
    press = (gamma - 1.) * (q[3, :, :] - 0.5 * rho * (u ** 2 + v ** 2))
    qstar = np.empty(q.shape)
    qstar[0, :, :] = q[0, :, :] - dt2 / rad * q[2, :, :]
    qstar[1, :, :] = q[1, :, :] - dt2 / rad * rho * u * v
    qstar[2, :, :] = q[2, :, :] - dt2 / rad * rho * v * v
    qstar[3, :, :] = q[3, :, :] - dt2 / rad * v * (q[3, :, :] + press)
    rho = qstar[0, :, :]
    u = qstar[1, :, :] / rho
    v = qstar[2, :, :] / rho
    press = (gamma - 1.) * (qstar[3, :, :] - 0.5 * rho * (u ** 2 + v ** 2))
    q[0, :, :] = q[0, :, :] - dt / rad * qstar[2, :, :]
    q[1, :, :] = q[1, :, :] - dt / rad * rho * u * v
    q[2, :, :] = q[2, :, :] - dt / rad * rho * v * v
    q[3, :, :] = q[3, :, :] - dt / rad * v * (qstar[3, :, :] + press)


def shock_bubble(solver_class=None, mx=320, my=80, tfinal=0.6, num_output_times=10, device_source=False):
    """A planar shock hitting a low-density bubble, in r-z coordinates with
    cylindrical symmetry (euler_5wave_2D with a tracer marking the bubble):
    unsplit, MC on the Euler families and superbee on the tracer, cfl 0.45 /
    0.5; inflow of the post-shock state on the left (custom BC), wall at the
    axis, extrapolation elsewhere; the geometric source by a Godunov-split
    step.  device_source: the source as EulerAxisymmetricSource, which stays on
    the device, instead of the host function."""
    from .sources import EulerAxisymmetricSource
    cls = solver_class or ClawSolver2D
    solver = cls(riemann.euler_5wave_2D)
    solver.step_source = (EulerAxisymmetricSource(BUBBLE_GAMMA, radius_aux=0) if device_source
                          else _euler_radial_source)
    solver.source_split = 1
    solver.limiters = [4, 4, 4, 4, 2]
    solver.cfl_max = 0.5
    solver.cfl_desired = 0.45
    domain = Domain([Dimension(0.0, 2.0, mx, name='x'), Dimension(0.0, 0.5, my, name='y')])
    state = State(domain, 5, 1)
    state.problem_data['gamma'] = BUBBLE_GAMMA
    _bubble_qinit(state)
    y = state.grid.y.centers
    for j, r in enumerate(y):
        state.aux[0, :, j] = r
    solver.user_bc_lower = _incoming_shock
    solver.bc_lower[0] = BC.custom
    solver.bc_upper[0] = BC.extrap
    solver.bc_lower[1] = BC.wall
    solver.bc_upper[1] = BC.extrap
    solver.aux_bc_lower[0] = BC.extrap
    solver.aux_bc_upper[0] = BC.extrap
    solver.aux_bc_lower[1] = BC.extrap
    solver.aux_bc_upper[1] = BC.extrap
    return _controller(solver, Solution(state, domain), tfinal, num_output_times=num_output_times)


QUADRANT_STATES = {  # (rho, u, v, p) per quadrant, split at x = y = 0.8
    'NE': (1.5, 0.0, 0.0, 1.5),
    'NW': (0.5323, 1.206, 0.0, 0.3),
    'SW': (0.138, 1.206, 1.206, 0.029),
    'SE': (0.5323, 0.0, 1.206, 0.3),
}


def euler_quadrants_unsplit(solver_class=None, n=1024, tfinal=0.8, split=(0.8, 0.8), states=None,
                            gamma=1.4):
    """Four-quadrant Euler Riemann problem on [0,1]^2, Roe 4-wave solver,
    extrapolation BCs, MC limiter, unsplit with transverse corrections."""
    cls = solver_class or ClawSolver2D
    solver = cls(riemann.euler_4wave_2D)
    solver.dimensional_split = False
    solver.transverse_waves = 2
    solver.limiters = tvd.MC
    solver.all_bcs = BC.extrap
    domain = Domain([0., 0.], [1., 1.], [n, n])
    solution = Solution(4, domain)
    solution.problem_data['gamma'] = gamma
    st = states or QUADRANT_STATES
    xx, yy = domain.grid.p_centers
    xs, ys = split
    masks = {'NE': (xx >= xs) & (yy >= ys), 'NW': (xx < xs) & (yy >= ys),
             'SW': (xx < xs) & (yy < ys), 'SE': (xx >= xs) & (yy < ys)}
    rho = np.zeros_like(xx)
    u = np.zeros_like(xx)
    v = np.zeros_like(xx)
    p = np.zeros_like(xx)
    for k, msk in masks.items():
        rho[msk], u[msk], v[msk], p[msk] = st[k]
    q = solution.q
    q[0, ...] = rho
    q[1, ...] = rho * u
    q[2, ...] = rho * v
    q[3, ...] = 0.5 * rho * (u ** 2 + v ** 2) + p / (gamma - 1.0)
    return _controller(solver, solution, tfinal)


def shallow_dam_break_unsplit(solver_class=None, n=4096, tfinal=1.0):
    """Radial dam break, g=1, [-2.5,2.5]^2, h=2 for r<0.5 else 1, Roe solver
    with entropy fix, extrapolation BCs, MC limiter, unsplit trans_cor, CFL 0.9."""
    cls = solver_class or ClawSolver2D
    solver = cls(riemann.shallow_roe_with_efix_2D)
    solver.dimensional_split = False
    solver.transverse_waves = 2
    solver.limiters = tvd.MC
    solver.cfl_desired = 0.9
    solver.cfl_max = 1.0
    solver.all_bcs = BC.extrap
    domain = Domain([-2.5, -2.5], [2.5, 2.5], [n, n])
    state = State(domain, 3)
    state.problem_data['grav'] = 1.0
    X, Y = state.p_centers
    r = np.sqrt(X ** 2 + Y ** 2)
    state.q[0, ...] = 2.0 * (r < 0.5) + 1.0 * (r >= 0.5)
    state.q[1, ...] = 0.0
    state.q[2, ...] = 0.0
    return _controller(solver, Solution(state, domain), tfinal)


def batched_quadrants(n_instances=512, seed=2024, sides=tuple(range(64, 513, 16)), solver_class=None):
    """The batched workload: independent four-quadrant Euler problems on
    [0,1]^2, side drawn uniformly from `sides` (multiples of 16), split point
    uniform in [0.3,0.7]^2, per quadrant rho and p uniform in [0.1,2] and u, v
    uniform in [-1,1]; Roe solver, MC, unsplit trans_cor, extrapolation BCs.
    Each problem's first dt is 0.45 of its cell-speed CFL limit at t = 0 (the
    Roe-averaged speed at a quadrant interface can exceed both sides')"""
    rng = np.random.default_rng(seed)
    claws, drawn = [], []
    for i in range(n_instances):
        side = int(rng.choice(sides))
        xs, ys = rng.uniform(0.3, 0.7, size=2)
        states = {}
        for quad in ('NE', 'NW', 'SW', 'SE'):
            rho, p = rng.uniform(0.1, 2.0, size=2)
            u, v = rng.uniform(-1.0, 1.0, size=2)
            states[quad] = (rho, u, v, p)
        claw = euler_quadrants_unsplit(solver_class, n=side, split=(xs, ys), states=states)
        smax = max(abs(u) + np.sqrt(1.4 * p / rho) for rho, u, v, p in states.values())
        smax = max(smax, max(abs(v) + np.sqrt(1.4 * p / rho) for rho, u, v, p in states.values()))
        claw.solver.dt_initial = 0.45 * (1.0 / side) / smax
        claws.append(claw)
        drawn.append(side)
    return claws, np.array(drawn)
