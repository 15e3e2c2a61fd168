"""Frame files in PyClaw's ascii format (src/pyclaw/fileio/ascii.py).

``write`` produces the reference's fort.tNNNN, fort.qNNNN, fort.aNNNN (with
write_aux) and fort.pklNNNN files; the q and aux arrays are formatted by the
library (claw2_write_ascii, several threads), and when the current q lives on
the GPU its copy to the host and the file writing run behind the next steps
(claw2_patch_write_ascii_async; ``wait`` collects the result).  ``read``
loads such a frame back into a Solution (restart, comparison with the
reference's files).
"""
import os
import pickle

import numpy as np

from . import _lib


def _patch_header(patch):
    """write_patch_header (ascii.py:86-97)."""
    lines = ["%5i                  patch_number\n" % patch.patch_index,
             "%5i                  AMR_level\n" % patch.level]
    for dim in patch.dimensions:
        lines.append("%5i                  m%s\n" % (dim.num_cells, dim.name))
    for dim in patch.dimensions:
        lines.append("%18.8e     %slow\n" % (dim.lower, dim.name))
    for dim in patch.dimensions:
        lines.append("%18.8e     d%s\n" % (dim.delta, dim.name))
    lines.append("\n")
    return "".join(lines)


def _write_host(fname, append, header, arr):
    a = np.asfortranarray(arr, dtype=np.float64)
    nvar, mx, my = a.shape
    _lib.check(_lib.load().claw2_write_ascii(fname.encode(), 1 if append else 0, header.encode(), _lib.dptr(a),
                                             nvar, mx, my, 0))


def wait(solution):
    """Wait for the frame files still being written from the GPU."""
    for state in solution.states:
        m = getattr(state, '_mirror', None)
        if m is not None:
            m.wait_output()


def write(solution, frame, path, file_prefix='fort', write_aux=False, options={}, write_p=False):
    """ascii.py:17-83: fort.t, fort.q (q or p), fort.a (aux) and fort.pkl."""
    num_eqn = solution.state.mp if write_p else solution.num_eqn
    with open(os.path.join(path, '%s.t%s' % (file_prefix, str(frame).zfill(4))), 'w') as f:
        f.write("%18.8e     time\n" % solution.t)
        f.write("%5i                  num_eqn\n" % num_eqn)
        f.write("%5i                  nstates\n" % len(solution.states))
        f.write("%5i                  num_aux\n" % solution.num_aux)
        f.write("%5i                  num_dim\n" % solution.domain.num_dim)
        f.write("%5i                  num_ghost\n" % 0)
        f.write("%s                  file_format\n" % "ascii")
    qname = os.path.join(path, '%s.q%s' % (file_prefix, str(frame).zfill(4)))
    for k, state in enumerate(solution.states):
        header = _patch_header(state.patch)
        m = getattr(state, '_mirror', None)
        if not write_p and m is not None and m.device_newer and len(solution.states) == 1:
            m.write_ascii_async(qname, False, header)   # the device's copy, behind the next steps
        else:
            _write_host(qname, k > 0, header, state.p if write_p else state._read_q())
    if solution.num_aux > 0 and write_aux:
        aname = os.path.join(path, '%s.a%s' % (file_prefix, str(frame).zfill(4)))
        for k, state in enumerate(solution.states):
            _write_host(aname, k > 0, _patch_header(state.patch), state.aux)
    sol_dict = {'t': solution.t, 'num_eqn': num_eqn, 'nstates': len(solution.states),
                'num_aux': solution.num_aux, 'num_dim': solution.domain.num_dim, 'write_aux': write_aux,
                'problem_data': solution.problem_data, 'mapc2p': solution.state.grid.mapc2p}
    pname = os.path.join(path, '%s.pkl' % file_prefix) + str(frame).zfill(4)
    with open(pname, 'wb') as f:
        try:
            pickle.dump(sol_dict, f)
        except (pickle.PicklingError, AttributeError, TypeError):
            # a mapping defined inside a function cannot be pickled: keep the rest
            sol_dict['mapc2p'] = None
            f.seek(0)
            f.truncate()
            pickle.dump(sol_dict, f)


def read_t(frame, path='./', file_prefix='fort'):
    """ascii.py:219-268: t, num_eqn, nstates, num_aux, num_dim, num_ghost, file_format."""
    fname = os.path.join(path, '%s.t' % file_prefix) + str(frame).zfill(4)
    with open(fname) as f:
        lines = [ln.split() for ln in f.read().splitlines() if ln.strip()]
    t = float(lines[0][0])
    ints = [int(lines[k][0]) for k in range(1, 5)]
    num_ghost = int(lines[5][0]) if len(lines) > 5 else 0
    file_format = lines[6][0] if len(lines) > 6 else None
    return [t] + ints + [num_ghost, file_format]


def _read_blocks(fname, nstates, num_dim, nvar):
    """(patch header fields, array) for each patch of a fort.q / fort.a file."""
    from .geometry import Dimension, Patch
    with open(fname) as f:
        tokens = f.read().split()
    pos = 0
    out = []
    names = ['x', 'y', 'z']
    for _ in range(nstates):
        head = tokens[pos:pos + 2 * (2 + 3 * num_dim)]   # "value label" pairs
        patch_index, level = int(head[0]), int(head[2])
        k = 4
        n, lower, d = [], [], []
        for _ in range(num_dim):
            n.append(int(head[k]))
            k += 2
        for _ in range(num_dim):
            lower.append(float(head[k]))
            k += 2
        for _ in range(num_dim):
            d.append(float(head[k]))
            k += 2
        pos += k
        count = nvar * int(np.prod(n))
        vals = np.array(tokens[pos:pos + count], dtype=np.float64)
        if vals.size != count:
            raise IOError('Unexpected EOF in %s' % fname)
        pos += count
        arr = np.asfortranarray(vals.reshape(list(reversed(n)) + [nvar]).transpose())
        patch = Patch([Dimension(lower[i], lower[i] + n[i] * d[i], n[i], name=names[i]) for i in range(num_dim)])
        patch.patch_index, patch.level = patch_index, level
        out.append((patch, arr))
    return out


def read(solution, frame, path='./', file_prefix='fort', read_aux=False, options={}):
    """ascii.py:126-216: the states, domain, problem_data and mapping of a frame."""
    from .geometry import Domain
    from .state import State
    problem_data, mapc2p = None, None
    pname = os.path.join(path, '%s.pkl' % file_prefix) + str(frame).zfill(4)
    if os.path.exists(pname):
        with open(pname, 'rb') as f:
            d = pickle.load(f)
        problem_data, mapc2p = d.get('problem_data', None), d.get('mapc2p', None)
    t, num_eqn, nstates, num_aux, num_dim, num_ghost, file_format = read_t(frame, path, file_prefix)
    qname = os.path.join(path, '%s.q' % file_prefix) + str(frame).zfill(4)
    patches = []
    for patch, q in _read_blocks(qname, nstates, num_dim, num_eqn):
        state = State(patch, num_eqn, num_aux)
        state.t = t
        state.problem_data = problem_data if problem_data is not None else {}
        if mapc2p is not None:
            state.grid.mapc2p = mapc2p
        if num_aux > 0:
            state.aux[:] = np.nan
        state.q = q
        solution.states.append(state)
        patches.append(state.patch)
    solution.domain = Domain(patches)
    if num_aux > 0 and read_aux:
        a1 = os.path.join(path, '%s.a' % file_prefix) + str(frame).zfill(4)
        a0 = os.path.join(path, '%s.a' % file_prefix) + str(0).zfill(4)
        fname = a1 if os.path.exists(a1) else (a0 if os.path.exists(a0) else None)
        if fname is not None:
            for state, (patch, aux) in zip(solution.states, _read_blocks(fname, nstates, num_dim, num_aux)):
                for dim, adim in zip(state.patch.dimensions, patch.dimensions):
                    assert dim.num_cells == adim.num_cells, "aux file header does not match the q file"
                state.aux = aux
