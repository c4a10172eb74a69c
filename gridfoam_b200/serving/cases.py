"""Cavity case set-up for the solve server.

``cavity_simulator`` is the SIMPLE lid-driven cavity in gridfoam's YAML
schema (the reference's examples/cavity configuration: relaxation U 0.7 /
p 0.3, Jacobi-PCG pressure, Jacobi-BiCGStab momentum, linear convection,
least-squares gradients, corrected Laplacian) with ``residualControl`` on
``p`` (absolute, algorithms/simple.py:245-271).  ``TopologyCache`` builds
each grid size once; cases share its read-only device arrays through
``AxisProjectedGrid.with_config``.
"""

from __future__ import annotations

import threading

import torch

from gridfoam_b200.meta.config import SimulatorConfig

_WALLS = ["x_minus", "x_plus", "y_minus", "z_minus", "z_plus"]
_ALL = ["x_minus", "x_plus", "y_minus", "y_plus", "z_minus", "z_plus"]


def cavity_simulator(nu: float, lid: float, *, p_tol: float = 1e-6, p_solver_tol: float = 1e-6,
                     p_solver_rtol: float = 0.0, max_outer: int = 2000, inner_precision: str = "float64",
                     device: str = "cuda") -> SimulatorConfig:
    """``p_tol``: residualControl on p (the RHS-normalised initial residual,
    algorithms/utils/residual.py:12-36); ``p_solver_tol``: absolute CG
    tolerance of the pressure solve.  The normalised residual cannot fall
    much below ``p_solver_tol / |b|``, so a tight ``p_tol`` needs a tight
    solver tolerance (or a relative one, ``p_solver_rtol``); otherwise the
    run ends at ``max_outer`` (endTime).
    ``inner_precision="float32"`` runs the pressure CG's inner iterations in
    FP32 inside FP64 iterative refinement."""
    sim = {
        "control": {
            "deltaT": 1.0,
            "endTime": float(max_outer),
            "writeInterval": 1000000,
            "output": {"output_dir": "/tmp/gridfoam_b200_serving", "base_name": "cavity"},
            "precision": "float64",
        },
        "fvSchemes": {
            "divSchemes": {"default": "linear"},
            "gradSchemes": {"default": "leastsquare"},
            "laplacianSchemes": {"default": "corrected"},
        },
        "fvSolution": {
            "adjustPhi": True,
            "algorithm": {
                "type": "simple",
                "nNonOrthogonalCorrectors": 0,
                "relaxationFactors": {"equations": {"U": 0.7, "p": 0.3}},
                "residualControl": {"p": p_tol},
                "pRefCell": 0,
                "pRefValue": 0.0,
            },
            "solvers": {
                "U": {"method": "bicgstab", "preconditioner": "jacobi", "tolerance": 1e-8,
                      "rel_tolerance": 0.1, "max_iter": 1000},
                "p": {"method": "cg", "preconditioner": "jacobi", "tolerance": p_solver_tol,
                      "rel_tolerance": p_solver_rtol, "max_iter": 2000, "inner_precision": inner_precision},
            },
        },
        "conditions": {
            "U": {
                "internal": [0.0, 0.0, 0.0],
                "boundary": {
                    "wall": {"type": "dirichlet", "patches": _WALLS, "value": [0.0, 0.0, 0.0]},
                    "lid": {"type": "dirichlet", "patches": ["y_plus"], "value": [float(lid), 0.0, 0.0]},
                },
            },
            "p": {
                "internal": 0.0,
                "boundary": {"wall": {"type": "neumann", "patches": _ALL, "value": 0.0}},
            },
        },
        "properties": {
            "transport": {"type": "newtonian", "nu": float(nu)},
            "turbulence": {"type": "laminar"},
        },
        "device": device,
    }
    return SimulatorConfig.model_validate(sim)


class TopologyCache:
    """One base grid per cavity size and device, built on first use."""

    def __init__(self, device: torch.device):
        self.device = torch.device(device)
        self._grids: dict[int, object] = {}
        self._lock = threading.Lock()

    def grid(self, n: int, sim: SimulatorConfig):
        from gridfoam_b200.core.grid import AxisProjectedGrid
        from gridfoam_b200.mesh.builder import build_uniform_mesh

        with self._lock:
            base = self._grids.get(n)
            if base is None:
                mesh = build_uniform_mesh((0.0, 0.0, 0.0), (1.0, 1.0, 1.0), (n, n, n))
                base = AxisProjectedGrid(sim, mesh, device=self.device)
                self._grids[n] = base
        return base.with_config(sim)
