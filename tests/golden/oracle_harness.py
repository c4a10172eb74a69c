"""Build CPU-oracle cases from ``tests/golden/cases.py`` definitions."""

from __future__ import annotations

import copy

import numpy as np

from oracle.algorithms import create_algorithm
from oracle.case import Case, CellField, DirichletBC
from tests.golden.cases import ALL_CASES, build_mesh, inlet_profile_values

TRANSIENT = {"piso", "pimple"}


def oracle_case(name: str, case_def: dict | None = None):
    """Return ``(case_def, mesh, oracle Case, oracle algorithm)``."""
    case_def = copy.deepcopy(case_def or ALL_CASES[name]())
    mesh = build_mesh(case_def["mesh"])
    case = Case(mesh, case_def["simulator"])
    kind = case_def["simulator"]["fvSolution"]["algorithm"]["type"]
    role = "transient" if kind in TRANSIENT else "local"
    U = CellField(case, "U", role, (3,))
    profile = case_def.get("inlet_profile")
    if profile is not None:
        U.bcs[profile["patch"]] = DirichletBC(inlet_profile_values(mesh, profile))
    algo = create_algorithm(case)
    return case_def, mesh, case, algo


def load_golden(name: str) -> dict:
    import pathlib

    path = pathlib.Path(__file__).resolve().parent / f"{name}.npz"
    with np.load(path) as data:
        return {k: data[k] for k in data.files}
