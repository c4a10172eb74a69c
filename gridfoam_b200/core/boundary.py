"""Boundary conditions in value-fraction form, compiled to per-face tables.

The classes mirror gridfoam's ``boundaries/**`` (constructor arguments,
``type`` and ``assignable``).  Instead of evaluating on every call with
tensor code, a field's conditions are compiled once into a per-boundary-face
kind/value table that ``gf_bc_state`` evaluates on the device
(``fv/boundary_ops.py:311-326``).

``DirichletBC`` additionally accepts a per-face value array
``[F_patch, *component_shape]`` on a domain patch (e.g. a parabolic inlet),
which in the reference needs a user ``BoundaryCondition`` subclass.
"""

from __future__ import annotations

import numpy as np
import torch

from gridfoam_b200 import _lib
from gridfoam_b200.meta.config import BoundaryConditionType


class BoundaryCondition:
    """Base class (boundaries/base.py:19-106)."""

    kind: int = _lib.BC_NONE

    @property
    def type(self) -> BoundaryConditionType:
        raise NotImplementedError

    @property
    def assignable(self) -> bool:
        return True

    def face_values(self, n_faces: int, comp: tuple[int, ...]) -> np.ndarray:
        """Per-face value column written into the table ``[n, *comp]``."""
        return np.zeros((n_faces,) + comp)


def _as_array(value) -> np.ndarray:
    if isinstance(value, torch.Tensor):
        return value.detach().to("cpu", torch.float64).numpy()
    return np.asarray(value, dtype=np.float64)


class DirichletBC(BoundaryCondition):
    """Fixed value (boundaries/basic/dirichlet.py:30-73)."""

    kind = _lib.BC_DIRICHLET

    def __init__(self, value):
        self.value = value

    @property
    def type(self):
        return BoundaryConditionType.DIRICHLET

    @property
    def assignable(self) -> bool:
        return False

    def face_values(self, n_faces, comp):
        v = _as_array(self.value)
        if v.shape == comp:
            return np.broadcast_to(v, (n_faces,) + comp).copy()
        if v.shape == (n_faces,) + comp:
            return v.copy()
        raise ValueError(f"dirichlet value shape {v.shape} does not match {comp} or {(n_faces,) + comp}")


class NeumannBC(BoundaryCondition):
    """Fixed gradient (boundaries/basic/neumann.py:30-73)."""

    kind = _lib.BC_NEUMANN

    def __init__(self, grad_value):
        self.grad_value = grad_value

    @property
    def type(self):
        return BoundaryConditionType.NEUMANN

    def face_values(self, n_faces, comp):
        v = _as_array(self.grad_value)
        if v.shape != comp:
            raise ValueError(f"neumann value shape {v.shape} does not match {comp}")
        return np.broadcast_to(v, (n_faces,) + comp).copy()


class EmptyBC(BoundaryCondition):
    """2-D empty patch (boundaries/basic/empty.py:20-51): excluded."""

    kind = _lib.BC_NONE

    @property
    def type(self):
        return BoundaryConditionType.EMPTY


class SlipBC(BoundaryCondition):
    """Slip wall (boundaries/basic/slip.py:27-101)."""

    kind = _lib.BC_SLIP

    @property
    def type(self):
        return BoundaryConditionType.SLIP

    @property
    def assignable(self) -> bool:
        return False


class InletOutletBC(BoundaryCondition):
    """Inflow value / outflow zero gradient (derived/inlet_outlet.py:27-123)."""

    kind = _lib.BC_INLET_OUTLET

    def __init__(self, inlet_value, phase: str | None = None):
        self.inlet_value = inlet_value
        self.phase = phase
        self.phi_name = "phi" if phase is None else f"phi.{phase}"

    @property
    def type(self):
        return BoundaryConditionType.INLET_OUTLET

    def face_values(self, n_faces, comp):
        v = _as_array(self.inlet_value)
        if v.shape != comp:
            raise ValueError(f"inlet value shape {v.shape} does not match {comp}")
        return np.broadcast_to(v, (n_faces,) + comp).copy()


class FixedFluxPressure(BoundaryCondition):
    """Pressure gradient matching the velocity flux (derived/fixed_flux_pressure.py:127-252)."""

    kind = _lib.BC_FIXED_FLUX_P

    def __init__(self, phase: str | None = None):
        self.phase = phase

    @property
    def type(self):
        return BoundaryConditionType.FIXED_FLUX_PRESSURE


def create_boundary_condition(bc_config, dtype=torch.float64, device=None) -> BoundaryCondition:
    """boundaries/factory.py:25-69."""
    t = bc_config.type
    if t == BoundaryConditionType.DIRICHLET:
        if bc_config.value is None:
            raise ValueError("Boundary condition value is required.")
        return DirichletBC(np.asarray(bc_config.value, dtype=np.float64))
    if t == BoundaryConditionType.NEUMANN:
        if bc_config.value is None:
            raise ValueError("Boundary condition value is required.")
        return NeumannBC(np.asarray(bc_config.value, dtype=np.float64))
    if t == BoundaryConditionType.EMPTY:
        return EmptyBC()
    if t == BoundaryConditionType.SLIP:
        return SlipBC()
    if t == BoundaryConditionType.INLET_OUTLET:
        if bc_config.value is None:
            raise ValueError("Boundary condition value is required.")
        return InletOutletBC(np.asarray(bc_config.value, dtype=np.float64), phase=bc_config.phase)
    if t == BoundaryConditionType.FIXED_FLUX_PRESSURE:
        return FixedFluxPressure(phase=bc_config.phase)
    raise ValueError(f"Unsupported boundary condition type: {t}")
