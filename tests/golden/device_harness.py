"""Build device (gridfoam_b200) cases from ``tests/golden/cases.py``."""

from __future__ import annotations

import copy

import numpy as np
import torch

from tests.golden.cases import ALL_CASES, build_mesh, inlet_profile_values

TRANSIENT = {"piso", "pimple"}


def device_case(name: str | None = None, case_def: dict | None = None, device: str = "cuda"):
    """Return ``(case_def, mesh, grid, algorithm)`` on the device."""
    from gridfoam_b200.algorithms.pressure_velocity import create_algorithm
    from gridfoam_b200.core.boundary import DirichletBC
    from gridfoam_b200.core.field import CellField
    from gridfoam_b200.core.grid import AxisProjectedGrid
    from gridfoam_b200.meta.config import FieldRole, SimulatorConfig

    case_def = copy.deepcopy(case_def or ALL_CASES[name]())
    mesh = build_mesh(case_def["mesh"], device=device)
    sim = SimulatorConfig.model_validate(case_def["simulator"])
    grid = AxisProjectedGrid(sim, mesh, device=device)
    kind = case_def["simulator"]["fvSolution"]["algorithm"]["type"]
    role = FieldRole.TRANSIENT if kind in TRANSIENT else FieldRole.LOCAL
    U = CellField(grid, "U", role, (3,))
    profile = case_def.get("inlet_profile")
    if profile is not None:
        U.add_boundary_conditions({profile["patch"]: DirichletBC(inlet_profile_values(mesh, profile))})
    algo = create_algorithm(grid)
    return case_def, mesh, grid, algo


def to_np(t: torch.Tensor) -> np.ndarray:
    return t.detach().to("cpu").numpy()
