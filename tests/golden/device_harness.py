"""Build device (gridfoam_b200) cases from ``tests/golden/cases.py``."""

from __future__ import annotations

import numpy as np
import torch

from gridfoam_b200.cases import create_case
from tests.golden.cases import ALL_CASES


def device_case(name: str | None = None, case_def: dict | None = None, device: str = "cuda"):
    """Return ``(case_def, mesh, grid, algorithm)`` on the device."""
    case_def = case_def or ALL_CASES[name]()
    mesh, grid, algo = create_case(case_def, device=device)
    return case_def, mesh, grid, algo


def to_np(t: torch.Tensor) -> np.ndarray:
    return t.detach().to("cpu").numpy()
