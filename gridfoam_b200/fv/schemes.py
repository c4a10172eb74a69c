"""Scheme selection (gridfoam ``fv/schemes/selection.py:23-113``) and the
time-scheme weights (``fv/schemes/ddt.py:13-58``)."""

from __future__ import annotations

import logging
import math

from gridfoam_b200.meta.config import (
    DdtScheme,
    DivScheme,
    FieldRole,
    GradScheme,
    LaplacianScheme,
    SnGradScheme,
)

logger = logging.getLogger(__name__)

LAPLACIAN_ALIASES = {
    LaplacianScheme.LINEAR: LaplacianScheme.CORRECTED,
    LaplacianScheme.GAUSS_LINEAR_CORRECTED: LaplacianScheme.CORRECTED,
    LaplacianScheme.GAUSS_LINEAR_UNCORRECTED: LaplacianScheme.UNCORRECTED,
}
HARMONIC = {LaplacianScheme.GAUSS_HARMONIC_CORRECTED, LaplacianScheme.GAUSS_HARMONIC_UNCORRECTED}
# Schemes that add the explicit hanging-face skewness correction.
CORRECTED = {LaplacianScheme.CORRECTED, LaplacianScheme.GAUSS_HARMONIC_CORRECTED}


def _lookup(table, key: str, default, warning: str | None = None):
    if table is None:
        return default
    v = table.get(key)
    if v is None:
        v = table.get("default")
    if v is None:
        if warning:
            logger.warning(warning, key)
        return default
    return v


def div_scheme(sim, phi_name: str, field_name: str) -> DivScheme:
    return DivScheme(
        _lookup(
            sim.fvSchemes.divSchemes,
            f"div({phi_name}, {field_name})",
            DivScheme.UPWIND,
            "Div scheme for %s not found. Using UPWIND scheme.",
        )
    )


def grad_scheme(sim, field_name: str) -> GradScheme:
    return GradScheme(_lookup(sim.fvSchemes.gradSchemes, f"grad({field_name})", GradScheme.LEASTSQUARE))


def laplacian_scheme(sim, field_name: str) -> LaplacianScheme:
    s = LaplacianScheme(
        _lookup(sim.fvSchemes.laplacianSchemes, f"laplacian({field_name})", LaplacianScheme.CORRECTED)
    )
    return LAPLACIAN_ALIASES.get(s, s)


def sn_grad_scheme(sim, field_name: str) -> SnGradScheme:
    return SnGradScheme(_lookup(sim.fvSchemes.snGradSchemes, f"snGrad({field_name})", SnGradScheme.CORRECTED))


def ddt_coefficients(field) -> tuple[float, float, float]:
    """``(a, b, c)`` of ``(a x - b x_old + c x_older) / dt`` (ddt.py:13-58)."""
    grid = field.grid
    dt = grid.dt
    if not math.isfinite(dt) or dt <= 0:
        raise ValueError("Time step must be finite and positive")
    scheme = DdtScheme(_lookup(grid.sim_config.fvSchemes.ddtSchemes, f"ddt({field.name})", DdtScheme.EULER))
    if scheme == DdtScheme.EULER:
        return 1.0, 1.0, 0.0
    if field.role != FieldRole.TRANSIENT:
        raise ValueError("backward ddt requires a TRANSIENT cell field")
    if field.older_store is None:
        return 1.0, 1.0, 0.0
    dt0 = field.previous_dt
    if dt0 is None or not math.isfinite(dt0) or dt0 <= 0:
        raise ValueError("backward ddt requires a finite positive previous time step")
    ratio = dt / dt0
    a = 1.0 + dt / (dt + dt0)
    c = ratio * dt / (dt + dt0)
    return a, a + c, c
