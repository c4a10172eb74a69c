"""Velocity-potential initialisation (gridfoam ``pre/potential_flow.py``).

OpenFOAM ``potentialFoam``: build ``phi`` from ``U``, solve
``laplacian(Phi) = div(phi)`` (with the configured non-orthogonal
correctors), correct the flux like the pressure projection, reconstruct
``U`` from it and balance the outflow.  ``Phi`` takes Dirichlet conditions
where ``p`` has them and zero gradient elsewhere.  Every step runs on the
device through the same kernels as the pressure-velocity algorithms.
"""

from __future__ import annotations

import ctypes
import logging

import torch

from gridfoam_b200._lib import GfBcAux, call, ptr, stream_ptr
from gridfoam_b200.core.boundary import DirichletBC, NeumannBC
from gridfoam_b200.core.equation import apply_immersed_dirichlet_values, equation
from gridfoam_b200.core.field import CellField, get_or_create_cellfield, get_or_create_facefield
from gridfoam_b200.fv import fvc, fvm
from gridfoam_b200.fv.adjust_phi import adjust_phi
from gridfoam_b200.meta.config import BoundaryConditionType, FieldRole
from gridfoam_b200.solvers.factory import create_solver

logger = logging.getLogger(__name__)


def _name(base: str, phase: str | None) -> str:
    return base if not phase else f"{base}.{phase}"


class PotentialFlow:
    """potential_flow.py:40-214."""

    def __init__(self, grid, phase: str | None = None):
        sim = grid.sim_config
        if sim.fvSolution.potentialFlow is None:
            raise ValueError("potentialFlow configuration in fvSolution is required.")
        self.grid = grid
        self.U = get_or_create_cellfield(grid, _name("U", phase), FieldRole.LOCAL, (3,))
        self.p = get_or_create_cellfield(grid, _name("p", phase), FieldRole.LOCAL, ())
        self.phi = get_or_create_facefield(grid, _name("phi", phase), FieldRole.LOCAL, ())
        p_condition = sim.get_field_condition(self.p.name)
        if p_condition is None:
            raise ValueError("pressure boundaryConditions are required.")
        self.p_bc_configs = list(p_condition.iter_bc_configs())
        self.config = sim.fvSolution.potentialFlow
        self.solver_configs = sim.fvSolution.solvers
        self.adjust_phi_enabled = sim.fvSolution.adjustPhi

    def _set_Phi_bcs(self, Phi: CellField) -> None:
        """potential_flow.py:87-117: Dirichlet p patches -> Dirichlet Phi,
        every other p patch -> zero gradient."""
        bcs = {}
        for cfg in self.p_bc_configs:
            for patch in cfg.patches:
                if cfg.type == BoundaryConditionType.DIRICHLET:
                    bcs[patch] = DirichletBC(cfg.value)
                else:
                    bcs[patch] = NeumannBC(0.0)
        Phi.add_boundary_conditions(bcs)

    @staticmethod
    def _eval(field) -> None:
        aux = GfBcAux()
        phi = field.grid.get_facefield("phi")
        if phi is not None:
            aux.phi_bnd = ptr(phi.boundary_store)
        field.evaluate_bc(aux)

    def solve(self) -> CellField:
        """potential_flow.py:122-214; returns ``Phi``."""
        g = self.grid
        fvc.face_flux(self.phi, self.U)  # correct_flux(phi, U, update_internal=True)
        div_phi = fvc.div(self.phi).data.clone()
        Phi = CellField(g, "Phi", FieldRole.LOCAL, ())
        self._set_Phi_bcs(Phi)
        if "Phi" not in self.solver_configs:
            raise KeyError("Solver configuration for 'Phi' not found")
        solver = create_solver(self.solver_configs["Phi"])
        needs_ref = not any(isinstance(bc, DirichletBC) for bc in Phi.bcs.values())
        n = int(self.config.nNonOrthogonalCorrectors)
        ref_cell = self.config.phiRefCell
        ref_value = self.config.phiRefValue if self.config.phiRefValue is not None else 0.0
        source = div_phi * g.cell_volumes
        mat = None
        for _ in range(n + 1):
            mat = fvm.laplacian(1.0, Phi)
            mat.source = mat.source + source
            if needs_ref:
                if ref_cell is None:
                    raise ValueError("phiRefCell is required when Phi needs a reference value")
                d = mat.diag_store[ref_cell].clone()
                mat.diag_store[ref_cell] += d
                mat.source_store[0, ref_cell] += d * ref_value
            Phi.data = solver.solve(equation(Phi, mat)).solution
        # correct_phi(phi, predicted, -mat, Phi, 1): the pressure projection's
        # flux correction with a unit coefficient (incl. fixed-cell closure).
        self._eval(Phi)
        t = Phi.table
        predicted = self.phi.store.clone()
        ones = torch.ones(g.num_cells, dtype=torch.float64, device=g.device)
        s = stream_ptr()
        call("gf_correct_phi", ctypes.byref(g.cmesh), ptr(predicted), ptr(ones), ptr(Phi.store), ptr(t.kind),
             ptr(t.frac), ptr(t.refv), ptr(t.refg), -1.0, 0, None, ptr(mat._ffc), ptr(self.phi.store), s)
        faces, frac = t.fixed_faces()
        if faces.numel():
            scratch = torch.zeros(faces.numel(), dtype=torch.float64, device=g.device)
            call("gf_close_fixed_flux", ctypes.byref(g.cmesh), int(faces.numel()), ptr(faces), ptr(frac),
                 ptr(self.phi.store), ptr(scratch), s)
        fvc.reconstruct(self.phi, self.U)
        apply_immersed_dirichlet_values(self.U)
        if self.adjust_phi_enabled:
            adjust_phi(self.phi, self.U)
        self.Phi = Phi
        return Phi
