"""``Equation`` / ``equation()`` (gridfoam ``core/equation.py:6-68``).

Pairs a target field with its solve matrix, applying the immersed
Dirichlet (Gibou) cell constraints after assembly.  The constraint
selection is geometric and cached in the field's boundary table; the
prescribed values are gathered from the current boundary state.
"""

from __future__ import annotations

import torch

from gridfoam_b200._lib import GfBcAux, call, ptr, stream_ptr
from gridfoam_b200.core.field import CellField
from gridfoam_b200.core.fvmatrix import FvMatrix


def immersed_dirichlet_constraints(field: CellField) -> tuple[torch.Tensor, torch.Tensor]:
    """boundary_ops.py:440-535: ``(cells[K], values[K, *comp])``."""
    grid = field.grid
    cells, faces, _ = field.table.constraints()
    n = int(cells.numel())
    nc = field.num_components
    if n == 0:
        return cells.long(), torch.zeros((0, *field.component_shape), dtype=torch.float64, device=grid.device)
    aux = GfBcAux()
    phi = grid.get_facefield("phi")
    if phi is not None:
        aux.phi_bnd = ptr(phi.boundary_store)
    field.evaluate_bc(aux)
    vals = torch.empty((nc, n), dtype=torch.float64, device=grid.device)
    call("gf_gather_bnd", grid.num_bnd, nc, n, ptr(faces), ptr(field.table.refv), ptr(vals), stream_ptr())
    values = vals[0] if field.component_shape == () else vals.t()
    return cells.long(), values


class Equation:
    def __init__(self, target: CellField, fv_matrix: FvMatrix):
        self.name = target.name
        self.target = target
        cells, values = immersed_dirichlet_constraints(target)
        _, _, mask = target.table.constraints()
        # differentiable coefficients: the elimination carries their graph
        # (FvMatrix.with_fixed_values)
        self.fv_matrix = fv_matrix.with_fixed_values(cells, values, mask=mask) if cells.numel() else fv_matrix


def equation(target: CellField, fv_matrix: FvMatrix) -> Equation:
    return Equation(target, fv_matrix)


def apply_immersed_dirichlet_values(field: CellField) -> None:
    """boundary_ops.py:538-542."""
    cells, values = immersed_dirichlet_constraints(field)
    n = int(cells.numel())
    if n == 0:
        return
    grid = field.grid
    nc = field.num_components
    vals = values.reshape(n, nc).t().contiguous()
    c32 = cells.to(torch.int32).contiguous()
    call("gf_set_cell_values", grid.num_cells, nc, n, ptr(c32), ptr(vals), n, ptr(field.store), stream_ptr())
