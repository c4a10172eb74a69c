"""CPU oracle of fvc.reconstruct and the potential-flow initialisation
(test infrastructure).

Restates ``fv/fvc/reconstruct.py:28-117`` and
``pre/potential_flow.py:40-214`` of the reference on the oracle's
primitives: the velocity potential ``Phi`` takes Dirichlet conditions where
``p`` has them and zero gradient elsewhere, ``laplacian(Phi) = div(phi)``
is solved with the configured correctors, the flux is corrected like the
pressure projection and ``U`` is reconstructed from it.
"""

from __future__ import annotations

import numpy as np

from oracle.algorithms import correct_phi, needs_reference_value, set_reference_value
from oracle.case import CellField, DirichletBC, FaceField, NeumannBC, apply_immersed_dirichlet_values, scatter_add
from oracle.ops import adjust_phi, correct_flux, equation_matrix, fvc_div, fvm_laplacian
from oracle.solvers import solve


def fvc_reconstruct(phi: FaceField, U: CellField) -> np.ndarray:
    """reconstruct.py:28-117: ``(sum |Sf| n n^T)^-1 sum n phi`` per cell
    over every face of the cell, both sides of internal faces with the same
    sign; diagonal on an axis-aligned grid."""
    c = phi.case
    numer = np.zeros((c.num_cells, 3))
    denom = np.zeros((c.num_cells, 3))

    def acc(cells, Sf, flux):
        mag = np.linalg.norm(Sf, axis=1)
        n = Sf / mag[:, None]
        numer[:] += scatter_add(c.num_cells, cells, flux[:, None] * n)
        denom[:] += scatter_add(c.num_cells, cells, mag[:, None] * n * n)

    acc(c.owner_s, c.Sf_s, phi.single_data)
    acc(c.neighbour_s, c.Sf_s, phi.single_data)
    acc(c.domain_bnd_owner, c.domain_bnd_Sf, phi.domain_bnd_data)
    if c.num_immersed_faces > 0:
        imm = c.ap_is_immersed_faces
        acc(c.owner[imm], c.Sf[imm], phi.immersed_upper)
        acc(c.neighbour[imm], -c.Sf[imm], phi.immersed_lower)
    u = numer / denom
    U.data = u
    return u


def potential_flow(case, U: CellField, p: CellField, phi: FaceField) -> CellField:
    """potential_flow.py:122-214; returns ``Phi``."""
    pf_cfg = case.sim["fvSolution"]["potentialFlow"]
    correct_flux(phi, U, update_internal=True)
    div_phi = fvc_div(phi)
    Phi = CellField(case, "Phi", "local", ())
    for patch, bc in p.bcs.items():
        Phi.bcs[patch] = DirichletBC(bc.value) if isinstance(bc, DirichletBC) else NeumannBC(0.0)
    cfg = case.solver_config("Phi")
    ref = needs_reference_value(Phi)
    source = div_phi * case.cell_volumes
    mat = None
    for _ in range(int(pf_cfg.get("nNonOrthogonalCorrectors", 0)) + 1):
        mat = fvm_laplacian(1.0, Phi)
        mat.source = mat.source + source
        if ref:
            set_reference_value(mat, int(pf_cfg["phiRefCell"]), float(pf_cfg.get("phiRefValue") or 0.0))
        solve_mat = equation_matrix(Phi, mat)
        x, _ = solve(solve_mat, solve_mat.source, Phi.data, cfg)
        Phi.data = x
    predicted = FaceField(case, "potential_predicted_flux")
    predicted.single_data = phi.single_data.copy()
    predicted.domain_bnd_data = phi.domain_bnd_data.copy()
    predicted.immersed_upper = phi.immersed_upper.copy()
    predicted.immersed_lower = phi.immersed_lower.copy()
    coeff = CellField(case, "potential_coefficient", "local", ())
    coeff.data = np.ones(case.num_cells)
    correct_phi(phi, predicted, -mat, Phi, coeff)
    fvc_reconstruct(phi, U)
    apply_immersed_dirichlet_values(U)
    if case.sim["fvSolution"].get("adjustPhi", True):
        adjust_phi(phi, U)
    return Phi
