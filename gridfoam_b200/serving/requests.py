"""Synthetic request stream: cavity solves arriving as a Poisson process.

Each request is a lid-driven cubic cavity (unit cube, ``n^3`` uniform
cells) with Reynolds number log-uniform in ``re_range`` and lid speed
uniform in ``lid_range``; the viscosity follows as ``nu = lid * L / Re``
with ``L = 1``.  Inter-arrival gaps are exponential with mean ``1/rate``.
All draws come from one seeded ``numpy.random.default_rng``.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

SIZES = (16, 24, 32, 48, 64, 96)


@dataclass(frozen=True)
class CavityRequest:
    id: int
    n: int
    re: float
    lid: float
    arrival: float  # seconds after the stream starts

    @property
    def nu(self) -> float:
        return self.lid / self.re

    @property
    def cells(self) -> int:
        return self.n**3


def poisson_stream(count: int, rate: float = 50.0, sizes=SIZES, re_range=(10.0, 1000.0),
                   lid_range=(0.5, 2.0), seed: int = 0) -> list[CavityRequest]:
    """``count`` requests, arrivals at rate ``rate`` per second (first at 0)."""
    if count < 0 or rate <= 0:
        raise ValueError("count must be >= 0 and rate > 0")
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, size=count)
    arrivals = np.concatenate([[0.0], np.cumsum(gaps[1:])]) if count else np.zeros(0)
    n = rng.choice(np.asarray(sizes, dtype=np.int64), size=count)
    re = np.exp(rng.uniform(np.log(re_range[0]), np.log(re_range[1]), size=count))
    lid = rng.uniform(lid_range[0], lid_range[1], size=count)
    return [CavityRequest(i, int(n[i]), float(re[i]), float(lid[i]), float(arrivals[i])) for i in range(count)]
