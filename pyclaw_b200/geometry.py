"""Grid geometry: Dimension, Grid, Patch, Domain.

Host-side mirror of src/pyclaw/geometry.py (Dimension :476-640, Grid :16-470,
Patch :647-743, Domain :744-800) restricted to what the classic 2D step and its
callers use: cell sizes, centers, nodes and the serial on-boundary flags.
"""
import numpy as np


class Dimension(object):
    """One coordinate direction: ``Dimension(lower, upper, num_cells, name='x')``
    (geometry.py:476-560)."""

    def __init__(self, lower, upper, num_cells, name='x', on_lower_boundary=None,
                 on_upper_boundary=None, units=None):
        if upper <= lower:
            raise ValueError('Dimension.upper must be greater than lower')
        if int(num_cells) < 1:
            raise ValueError('Dimension.num_cells must be positive')
        self._lower = float(lower)
        self._upper = float(upper)
        self.num_cells = int(num_cells)
        self.name = name
        self.units = units
        self.on_lower_boundary = True if on_lower_boundary is None else on_lower_boundary
        self.on_upper_boundary = True if on_upper_boundary is None else on_upper_boundary

    lower = property(lambda self: self._lower)
    upper = property(lambda self: self._upper)

    @property
    def delta(self):
        """(upper - lower) / num_cells (geometry.py:521-523)."""
        return (self.upper - self.lower) / float(self.num_cells)

    @property
    def nodes(self):
        return np.array([self.lower + i * self.delta for i in range(self.num_cells + 1)])

    @property
    def centers(self):
        """lower + (i + 1/2) delta, evaluated like geometry.py:547-554."""
        return np.array([self.lower + (i + 0.5) * self.delta for i in range(self.num_cells)])

    def centers_with_ghost(self, num_ghost):
        """Centers of the ghost cells below, the cells, and the ghost cells
        above, the outer ones measured from lower / upper (geometry.py:583-589)."""
        pre = self.lower + (np.arange(-num_ghost, 0) + 0.5) * self.delta
        post = self.upper + self.delta * (np.arange(num_ghost) + 0.5)
        return np.hstack((pre, self.centers, post))

    def nodes_with_ghost(self, num_ghost):
        """Edges including those of the ghost cells (geometry.py:591-597)."""
        pre = np.linspace(self.lower - num_ghost * self.delta, self.lower - self.delta, num_ghost)
        post = np.linspace(self.upper + self.delta, self.upper + num_ghost * self.delta, num_ghost)
        return np.hstack((pre, self.nodes, post))

    def __str__(self):
        return "Dimension %s:  (num_cells,delta,[lower,upper]) = (%s,%s,[%s,%s])" % (
            self.name, self.num_cells, self.delta, self.lower, self.upper)


def identity_map_2d(x, y):
    """The default mapping (computational = physical coordinates); a
    module-level function so frames can pickle it (geometry.py:249)."""
    return [x, y]


def identity_map_1d(x):
    return [x]


def identity_map_3d(x, y, z):
    return [x, y, z]


_IDENTITY = {1: identity_map_1d, 2: identity_map_2d, 3: identity_map_3d}


class Grid(object):
    """Cartesian product of Dimensions (geometry.py:16-470)."""

    def __init__(self, dimensions):
        if isinstance(dimensions, Dimension):
            dimensions = [dimensions]
        self._dims = list(dimensions)
        self.gauges = []            # cell indices of the gauges (add_gauges)
        self.gauge_file_names = []
        self.gauge_files = []
        self.gauge_dir_name = '_gauges'
        self.mapc2p = _IDENTITY.get(len(self._dims), identity_map_2d)

    dimensions = property(lambda self: list(self._dims))
    num_dim = property(lambda self: len(self._dims))
    num_cells = property(lambda self: [d.num_cells for d in self._dims])
    delta = property(lambda self: [d.delta for d in self._dims])
    lower = property(lambda self: [d.lower for d in self._dims])
    upper = property(lambda self: [d.upper for d in self._dims])
    on_lower_boundary = property(lambda self: [d.on_lower_boundary for d in self._dims])
    on_upper_boundary = property(lambda self: [d.on_upper_boundary for d in self._dims])

    def get_dim_attribute(self, attr):
        return [getattr(d, attr) for d in self._dims]

    @property
    def c_centers(self):
        """Cell-center coordinate arrays, indexing 'ij' (geometry.py:165-300)."""
        idx = np.indices(self.num_cells)
        return [d.centers[idx[i, ...]] for i, d in enumerate(self._dims)]

    @property
    def c_nodes(self):
        idx = np.indices([n + 1 for n in self.num_cells])
        return [d.nodes[idx[i, ...]] for i, d in enumerate(self._dims)]

    @property
    def p_centers(self):
        return self.mapc2p(*self.c_centers)

    @property
    def p_nodes(self):
        return self.mapc2p(*self.c_nodes)

    def c_centers_with_ghost(self, num_ghost):
        """Cell centers including ghost cells (geometry.py:335-348)."""
        idx = np.indices([n + 2 * num_ghost for n in self.num_cells])
        return [d.centers_with_ghost(num_ghost)[idx[i, ...]] for i, d in enumerate(self._dims)]

    def c_nodes_with_ghost(self, num_ghost):
        """Cell corners including those of ghost cells (geometry.py:350-363)."""
        idx = np.indices([n + 2 * num_ghost + 1 for n in self.num_cells])
        return [d.nodes_with_ghost(num_ghost)[idx[i, ...]] for i, d in enumerate(self._dims)]

    def p_centers_with_ghost(self, num_ghost):
        return self.mapc2p(*self.c_centers_with_ghost(num_ghost))

    def p_nodes_with_ghost(self, num_ghost):
        return self.mapc2p(*self.c_nodes_with_ghost(num_ghost))

    def add_gauges(self, gauge_coords):
        """Record the cell index of every gauge inside this grid (lower <= x <
        upper in each dimension) and its file name (geometry.py:392-405)."""
        for gauge in gauge_coords:
            if all(self.lower[n] <= gauge[n] < self.upper[n] for n in range(self.num_dim)):
                index = [int((gauge[n] - self.lower[n]) // self.delta[n]) for n in range(self.num_dim)]
                self.gauge_file_names.append('gauge' + '_'.join(str(c) for c in gauge) + '.txt')
                self.gauges.append(index)

    def setup_gauge_files(self, outdir):
        """Open one file per gauge under outdir/_gauges, replacing old ones
        (geometry.py:407-423)."""
        import os
        path = os.path.join(outdir, self.gauge_dir_name)
        os.makedirs(path, exist_ok=True)
        for name in self.gauge_file_names:
            f = os.path.join(path, name)
            if os.path.isfile(f):
                os.remove(f)
            self.gauge_files.append(open(f, 'a'))

    def __getattr__(self, name):
        # grid.x, grid.y address the dimensions by name, as in the reference
        for d in self.__dict__.get('_dims', []):
            if d.name == name:
                return d
        raise AttributeError(name)


class Patch(object):
    """A logically rectangular piece of the domain (geometry.py:647-743)."""

    def __init__(self, dimensions):
        self.grid = Grid(dimensions)
        self.level = 1
        self.patch_index = 1

    def __deepcopy__(self, memo={}):
        """A new patch on copies of the dimensions with the same mapping; gauges
        and their open files stay with the original (geometry.py:725-734)."""
        import copy
        result = self.__class__(copy.deepcopy(self.dimensions))
        result.grid.mapc2p = self.grid.mapc2p
        result.level = self.level
        result.patch_index = self.patch_index
        return result

    num_dim = property(lambda self: self.grid.num_dim)
    dimensions = property(lambda self: self.grid.dimensions)
    delta = property(lambda self: self.grid.delta)
    num_cells_global = property(lambda self: self.grid.num_cells)
    lower_global = property(lambda self: self.grid.lower)
    upper_global = property(lambda self: self.grid.upper)


class Domain(object):
    """``Domain(lower, upper, num_cells)`` or ``Domain([dims])`` / ``Domain(patch)``
    (geometry.py:744-800)."""

    def __init__(self, *arg):
        if len(arg) > 1:
            lower, upper, n = arg[0], arg[1], arg[2]
            names = ['x', 'y', 'z'][:len(n)]
            self.patches = [Patch([Dimension(lo, up, nn, name=nm)
                                   for lo, up, nn, nm in zip(lower, upper, n, names)])]
        else:
            geom = arg[0]
            if not isinstance(geom, (list, tuple)):
                geom = [geom]
            if isinstance(geom[0], Patch):
                self.patches = list(geom)
            elif isinstance(geom[0], Dimension):
                self.patches = [Patch(geom)]
            else:
                raise TypeError("Domain needs Dimensions, Patches or (lower, upper, num_cells)")

    patch = property(lambda self: self.patches[0])
    grid = property(lambda self: self.patches[0].grid)
    num_dim = property(lambda self: self.patches[0].num_dim)
