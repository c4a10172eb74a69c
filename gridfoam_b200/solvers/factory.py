"""Solver factory and ``*Final`` resolution (solvers/factory.py, resolver.py)."""

from __future__ import annotations

from gridfoam_b200.meta.config import SolverConfig, SolverType
from gridfoam_b200.solvers.base import LinearSolver
from gridfoam_b200.solvers.krylov import BiCGSTABSolver, CGSolver


def create_solver(config: SolverConfig) -> LinearSolver:
    """solvers/factory.py:9-35 (PyAMG is not part of the device path)."""
    match config.method:
        case SolverType.CG:
            return CGSolver(config)
        case SolverType.BiCGSTAB:
            return BiCGSTABSolver(config)
        case SolverType.PyAMG:
            raise NotImplementedError("the PyAMG host solver is not part of the device path")
        case _:
            raise ValueError(f"Unknown solver method: {config.method}")


def resolve_solver(solvers: dict, field_name: str, *, is_final: bool = False):
    """solvers/resolver.py:46-80."""
    if is_final:
        for key in (f"{field_name}Final", f"{field_name}_final"):
            if key in solvers:
                return solvers[key]
    if field_name not in solvers:
        raise KeyError(f"Solver for {field_name!r} not found")
    return solvers[field_name]
