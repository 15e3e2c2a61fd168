"""Ghost cells of the aux array filled on the host, for aux boundary
conditions that are user functions (BC.custom).

The device fills aux ghost cells itself for extrap / periodic / wall
(claw2_patch_upload_aux).  A custom aux BC is a Python function, so the host
builds auxbc the way Solver._apply_bcs does for aux (src/pyclaw/solver.py:
351-437): interior from State.aux (state.py:288-303), then dimension by
dimension the lower side and the upper side, each either the user function or
the built-in rule (solver.py:439-519 with name 'aux': a wall mirrors without a
sign change).  The result goes to the device whole (claw2_patch_upload_auxbc).
q lives on the device, so the user function gets qbc = None.
"""
import numpy as np

from .solver import BC


def _builtin(bc_type, arr, ng, lower):
    """One side of one dimension; ``arr`` has that dimension on axis 1."""
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
            else:
                arr[:, -i - 1, ...] = arr[:, -2 * ng + i, ...]
    elif bc_type is None:
        raise Exception('%s boundary condition not specified for either q or aux.'
                        % ('Lower' if lower else 'Upper'))
    else:
        raise NotImplementedError("Boundary condition %s not implemented" % bc_type)


def needs_host_fill(solver):
    return any(b == BC.custom for b in list(solver.aux_bc_lower) + list(solver.aux_bc_upper))


def fill_auxbc(solver, state, auxbc):
    """Fill ``auxbc`` (num_aux, mx + 2 ng, my + 2 ng), Fortran order, in place."""
    ng = solver.num_ghost
    auxbc[:, ng:-ng, ng:-ng] = state.aux
    grid = state.grid
    old_sig = getattr(solver, '_use_old_bc_sig', False)
    for idim, dim in enumerate(grid.dimensions):
        for lower in (True, False):
            on = grid.on_lower_boundary[idim] if lower else grid.on_upper_boundary[idim]
            if not on:
                continue
            bc_type = (solver.aux_bc_lower if lower else solver.aux_bc_upper)[idim]
            if bc_type == BC.custom:
                fun = solver.user_aux_bc_lower if lower else solver.user_aux_bc_upper
                if fun is None:
                    raise Exception('%s custom aux BC function has not been set.' % ('Lower' if lower else 'Upper'))
                if old_sig:
                    fun(state, dim, state.t, auxbc, ng)
                else:
                    fun(state, dim, state.t, None, auxbc, ng)
            else:
                _builtin(bc_type, np.rollaxis(auxbc, idim + 1, 1), ng, lower)
    return auxbc
