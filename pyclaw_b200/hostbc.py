"""Ghost cells filled on the host, for boundary conditions that are user
functions (BC.custom).

The device fills ghost cells itself for extrap / periodic / wall
(claw2_patch_step for q, claw2_patch_upload_aux for aux).  A custom BC is a
Python function, so the host builds the arrays with ghost cells the way
Solver._apply_bcs does (src/pyclaw/solver.py:351-437): interiors from State.q
and State.aux (state.py:288-303), then dimension by dimension the lower side
and the upper side, on each side aux before q, each either the user function
or the built-in rule (solver.py:439-519: a wall negates the normal momentum of
q, reflect_index, and mirrors aux unchanged).  The results go to the device
whole (claw2_patch_upload_qbc, claw2_patch_upload_auxbc).

With only aux BCs custom (``fill_auxbc``) q stays on the device and the user
function receives qbc = None.
"""
import numpy as np

from .solver import BC


def _builtin(bc_type, arr, ng, lower, reflect=None):
    """One side of one dimension; ``arr`` has that dimension on axis 1;
    ``reflect`` is the component a wall negates (None for aux)."""
    if bc_type == BC.extrap:
        for i in range(ng):
            if lower:
                arr[:, i, ...] = arr[:, ng, ...]
            else:
                arr[:, -i - 1, ...] = arr[:, -ng - 1, ...]
    elif bc_type == BC.periodic:
        if lower:
            arr[:, :ng, ...] = arr[:, -2 * ng:-ng, ...]
        else:
            arr[:, -ng:, ...] = arr[:, ng:2 * ng, ...]
    elif bc_type == BC.wall:
        for i in range(ng):
            if lower:
                arr[:, i, ...] = arr[:, 2 * ng - 1 - i, ...]
                if reflect is not None:
                    arr[reflect, i, ...] = -arr[reflect, 2 * ng - 1 - i, ...]
            else:
                arr[:, -i - 1, ...] = arr[:, -2 * ng + i, ...]
                if reflect is not None:
                    arr[reflect, -i - 1, ...] = -arr[reflect, -2 * ng + i, ...]
    elif bc_type is None:
        raise Exception('%s boundary condition not specified for either q or aux.'
                        % ('Lower' if lower else 'Upper'))
    else:
        raise NotImplementedError("Boundary condition %s not implemented" % bc_type)


def needs_host_fill(solver):
    """Some aux BC is a user function."""
    return any(b == BC.custom for b in list(solver.aux_bc_lower) + list(solver.aux_bc_upper))


def has_custom_q(solver):
    """Some q BC is a user function."""
    return any(b == BC.custom for b in list(solver.bc_lower) + list(solver.bc_upper))


def _call(solver, fun, state, dim, qbc, auxbc, arr, ng, which):
    if fun is None:
        raise Exception('%s custom BC function has not been set.' % which)
    if getattr(solver, '_use_old_bc_sig', False):
        fun(state, dim, state.t, arr, ng)
    else:
        fun(state, dim, state.t, qbc, auxbc, ng)


def fill_bcs(solver, state, qbc, auxbc):
    """Fill the ghost cells of ``qbc`` (num_eqn, mx + 2 ng, my + 2 ng) and, if
    not None, ``auxbc``, both Fortran order, in place, interiors included."""
    ng = solver.num_ghost
    qbc[:, ng:-ng, ng:-ng] = state._read_q()
    if auxbc is not None:
        auxbc[:, ng:-ng, ng:-ng] = state.aux
    grid = state.grid
    for idim, dim in enumerate(grid.dimensions):
        for lower in (True, False):
            on = grid.on_lower_boundary[idim] if lower else grid.on_upper_boundary[idim]
            if not on:
                continue
            arrays = []
            if auxbc is not None:
                arrays.append(('aux', auxbc, solver.aux_bc_lower if lower else solver.aux_bc_upper,
                               solver.user_aux_bc_lower if lower else solver.user_aux_bc_upper, None))
            arrays.append(('q', qbc, solver.bc_lower if lower else solver.bc_upper,
                           solver.user_bc_lower if lower else solver.user_bc_upper, solver.reflect_index[idim]))
            for name, arr, types, fun, reflect in arrays:
                bc_type = types[idim]
                if bc_type == BC.custom:
                    _call(solver, fun, state, dim, qbc, auxbc, arr, ng, 'Lower' if lower else 'Upper')
                else:
                    _builtin(bc_type, np.rollaxis(arr, idim + 1, 1), ng, lower, reflect)
    return qbc, auxbc


def fill_auxbc(solver, state, auxbc):
    """Fill ``auxbc`` (num_aux, mx + 2 ng, my + 2 ng), Fortran order, in place
    (aux BCs only; a custom function gets qbc = None)."""
    ng = solver.num_ghost
    auxbc[:, ng:-ng, ng:-ng] = state.aux
    grid = state.grid
    for idim, dim in enumerate(grid.dimensions):
        for lower in (True, False):
            on = grid.on_lower_boundary[idim] if lower else grid.on_upper_boundary[idim]
            if not on:
                continue
            bc_type = (solver.aux_bc_lower if lower else solver.aux_bc_upper)[idim]
            if bc_type == BC.custom:
                _call(solver, solver.user_aux_bc_lower if lower else solver.user_aux_bc_upper, state, dim, None,
                      auxbc, auxbc, ng, 'Lower' if lower else 'Upper')
            else:
                _builtin(bc_type, np.rollaxis(auxbc, idim + 1, 1), ng, lower)
    return auxbc
