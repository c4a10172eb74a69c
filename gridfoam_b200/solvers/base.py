"""Linear-solver interface (gridfoam ``solvers/base.py:15-162``).

``LinearSolver.solve(eq)`` returns a ``SolveResult`` whose ``stats`` hold one
``SolveStats`` per component.  The device solvers never synchronise inside a
solve: the statistics are copied asynchronously to pinned host memory and
materialise on first access, so a whole algorithm step runs without a host
round trip.
"""

from __future__ import annotations

from abc import ABC, abstractmethod
from dataclasses import dataclass
from typing import Literal

import torch

from gridfoam_b200 import _lib

GradientMode = Literal["adjoint", "unrolled"]

_STATUS = {
    _lib.GF_OK: "ok",
    _lib.GF_MAX_ITER: "max_iter",
    _lib.GF_BREAKDOWN: "breakdown",
    _lib.GF_NONFINITE: "nonfinite",
    _lib.GF_ERR_TIMEOUT: "timeout",
}


class _StatsBuffer:
    """Pinned host copy of a device ``[ncomp, 5]`` statistics block."""

    def __init__(self, device_stats: torch.Tensor):
        self.host = torch.empty(device_stats.shape, dtype=torch.float64, pin_memory=True)
        self.host.copy_(device_stats, non_blocking=True)
        self.event = torch.cuda.Event()
        self.event.record()
        self._ready = False

    def ready(self) -> bool:
        """True once the copy has landed (never blocks)."""
        if not self._ready and self.event.query():
            self._ready = True
        return self._ready

    def row(self, k: int) -> torch.Tensor:
        if not self._ready:
            self.event.synchronize()
            self._ready = True
        return self.host[k]


class SolveStats:
    """Statistics of one component solve (solvers/base.py:15-47).

    Attributes ``initial_residual``, ``final_residual`` (unnormalised norms),
    ``iterations`` and ``converged`` read the device result on first access.
    ``status`` is ``"ok"``, ``"max_iter"``, ``"breakdown"``, ``"nonfinite"``
    or ``"timeout"``.
    """

    def __init__(self, solver: str, buffer: _StatsBuffer, k: int):
        self.solver = solver
        self._buf = buffer
        self._k = k

    def ready(self) -> bool:
        """True once the statistics are on the host (never blocks)."""
        return self._buf.ready()

    @property
    def initial_residual(self) -> float:
        return float(self._buf.row(self._k)[0])

    @property
    def final_residual(self) -> float:
        return float(self._buf.row(self._k)[1])

    @property
    def iterations(self) -> int:
        return int(self._buf.row(self._k)[2])

    @property
    def converged(self) -> bool:
        return bool(self._buf.row(self._k)[3])

    @property
    def status(self) -> str:
        return _STATUS.get(int(self._buf.row(self._k)[4]), "error")

    def __repr__(self) -> str:
        return (
            f"SolveStats(solver={self.solver!r}, initial_residual={self.initial_residual:.3e}, "
            f"final_residual={self.final_residual:.3e}, iterations={self.iterations}, "
            f"converged={self.converged})"
        )


@dataclass(frozen=True)
class SolveResult:
    solution: torch.Tensor
    stats: tuple[SolveStats, ...]


class LinearSolver(ABC):
    """Abstract linear solver (solvers/base.py:70-137)."""

    atol: float
    rtol: float
    grad_mode: GradientMode = "adjoint"

    def solve(self, eq) -> SolveResult:
        return self._solve_primal(eq)

    @abstractmethod
    def _solve_primal(self, eq) -> SolveResult: ...

    @abstractmethod
    def solve_transpose(self, A_T, rhs: torch.Tensor) -> torch.Tensor: ...


def residual_threshold(atol: float, rtol: float, ref_norm: float) -> float:
    """solvers/base.py:140-162."""
    return max(atol, rtol * ref_norm)
