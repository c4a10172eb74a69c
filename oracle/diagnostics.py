"""CPU oracle of the per-step continuity diagnostics (test infrastructure).

Restates ``post/diagnostics/continuity.py:11-49`` of the reference:
``contErr = fvc.div(phi)`` per cell, then the volume-weighted averages
``local = dt * sum(|contErr| V) / sum(V)`` and ``global = dt * sum(contErr
V) / sum(V)``; the collector (``post/diagnostics/collector.py:190-229``)
accumulates ``global`` into the cumulative column.
"""

from __future__ import annotations

import numpy as np

from oracle.case import Case, get_facefield
from oracle.ops import fvc_div


def set_packed(face, packed: np.ndarray) -> None:
    """Fill a face field from the packed ``[single | domain | imm_upper |
    imm_lower]`` order."""
    c = face.case
    a = c.num_single
    b = a + c.num_domain_bnd_faces
    k = c.num_immersed_faces
    face.single_data[...] = packed[:a]
    face.domain_bnd_data[...] = packed[a:b]
    face.immersed_upper[...] = packed[b:b + k]
    face.immersed_lower[...] = packed[b + k:b + 2 * k]


def continuity_error(case: Case, packed_phi: np.ndarray, delta_t: float) -> tuple[float, float]:
    """continuity.py:11-49 on a packed face flux."""
    phi = get_facefield(case, "phi_diagnostics")
    set_packed(phi, packed_phi)
    cont = fvc_div(phi)
    vol = case.cell_volumes
    total = np.sum(vol)
    return delta_t * (np.sum(np.abs(cont) * vol) / total), delta_t * (np.sum(cont * vol) / total)


def continuity_rows(case: Case, packed_phis: list[np.ndarray], delta_t: float) -> np.ndarray:
    """``[time, local, global, cumulative]`` rows of the collector for a
    continuity interval of one step."""
    rows, cum = [], 0.0
    for k, phi in enumerate(packed_phis, start=1):
        loc, glo = continuity_error(case, phi, delta_t)
        cum += glo
        rows.append([k * delta_t, loc, glo, cum])
    return np.array(rows)
