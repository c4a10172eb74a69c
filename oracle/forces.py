"""CPU oracle of the immersed-surface force integral (test infrastructure).

Restates ``post/forces/sampling.py:69-168`` and
``post/forces/integration.py:76-187`` of the reference: every AP boundary
sample (upper and lower side of the patch's immersed faces) whose outward
direction points into the body is kept; its force is the pressure force
``rho p_b Sf`` plus the viscous force ``-rho nu (gradU + gradU^T) Sf`` with
``gradU = (U_b - U_P) / wall_dist (x) n_surface``.  The surface normals per
anchor stand in for the surface mesh's face area vectors.
"""

from __future__ import annotations

import numpy as np

from oracle.case import CellField, boundary_batches, boundary_state


def _side_value(field: CellField, batch) -> np.ndarray:
    """sampling.py:29-66: the value-fraction boundary value, or the cell
    value on patches without a boundary condition."""
    if batch.patch not in field.bcs:
        return field.data[batch.target_cells]
    return boundary_state(field, batch)[3]


def patch_force(p: CellField, U: CellField, nu_eff, patch: str, rho: float, cofr: np.ndarray,
                anchor_normals: np.ndarray):
    """Return ``(force[3], moment[3], pressure_force[A,3], viscous_force[A,3])``
    with per-anchor accumulations (A anchors, one per immersed face)."""
    case = U.case
    n_anchor = anchor_normals.shape[0]
    p_acc = np.zeros((n_anchor, 3))
    v_acc = np.zeros((n_anchor, 3))
    force = np.zeros(3)
    moment = np.zeros(3)
    nu = np.broadcast_to(np.asarray(nu_eff, dtype=np.float64), (case.num_cells,))
    batches = [b for b in boundary_batches(U) if b.patch == patch and b.kind in ("upper", "lower")]
    for b in batches:
        # p's batches on the patch carry the same faces in the same order
        pb_batch = next(x for x in boundary_batches(p) if x.patch == patch and x.kind == b.kind) \
            if patch in p.bcs else b
        anchor = np.nonzero(b.face_mask)[0]  # anchor = immersed ordinal
        n_hat = b.Sf / b.mag_Sf[:, None]
        S_body = -anchor_normals[anchor]
        keep = np.sum(n_hat * S_body, axis=1) > 0.0
        if not np.any(keep):
            continue
        area = np.linalg.norm(S_body, axis=1)
        n_surf = S_body / area[:, None]
        align = np.sum(n_hat * n_surf, axis=1)
        wall = b.mag_d[keep] * np.maximum(align[keep], 1.0e-12)
        U_b = _side_value(U, b)[keep]
        U_c = U.data[b.target_cells][keep]
        p_b = _side_value(p, pb_batch)[keep]
        dudn = (U_b - U_c) / wall[:, None]
        grad = dudn[:, :, None] * n_surf[keep, None, :]
        stress = rho * nu[b.target_cells][keep, None, None] * (grad + np.transpose(grad, (0, 2, 1)))
        pf = (rho * p_b)[:, None] * b.Sf[keep]
        vf = -(stress * b.Sf[keep, None, :]).sum(axis=-1)
        ff = pf + vf
        np.add.at(p_acc, anchor[keep], pf)
        np.add.at(v_acc, anchor[keep], vf)
        centers = case.cell_centers[b.target_cells][keep] + b.mag_d[keep, None] * n_hat[keep]
        force += ff.sum(axis=0)
        moment += np.cross(centers - cofr, ff).sum(axis=0)
    return force, moment, p_acc, v_acc
