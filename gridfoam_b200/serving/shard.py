"""Sharding the request stream over GPU replicas.

One process per GPU serves its own share of the stream; cases never span
GPUs, so the data path has no collective.  Every rank computes the same
assignment from the same stream (greedy by estimated work, in arrival
order), so the split needs no communication either; only the final
summaries are gathered for reporting.
"""

from __future__ import annotations

import numpy as np

from gridfoam_b200.serving.requests import CavityRequest


def estimated_work(req: CavityRequest) -> float:
    """Work of one request in cell-iterations per unit of iteration count
    (every request of a stream runs to the same iteration cap)."""
    return float(req.cells)


def shard_stream(requests: list[CavityRequest], world: int, rank: int,
                 work=estimated_work) -> list[CavityRequest]:
    """Requests of ``rank``: in arrival order, each goes to the rank with
    the least work assigned so far (lowest rank on ties)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("need 0 <= rank < world")
    load = np.zeros(world)
    mine = []
    for r in sorted(requests, key=lambda q: (q.arrival, q.id)):
        k = int(np.argmin(load))
        load[k] += work(r)
        if k == rank:
            mine.append(r)
    return mine


def merge_summaries(latencies: list[list[float]], firsts: list[float], lasts: list[float]) -> dict:
    """Whole-job throughput and latency percentiles from per-rank results:
    solves/s over the span from the first arrival to the last finish on any
    rank, percentiles over every request."""
    lat = np.concatenate([np.asarray(x, dtype=np.float64) for x in latencies]) if latencies else np.zeros(0)
    if lat.size == 0:
        return {"completed": 0}
    span = max(lasts) - min(firsts)
    return {
        "completed": int(lat.size),
        "solves_per_s": float(lat.size / max(span, 1e-12)),
        "p50_latency_s": float(np.percentile(lat, 50)),
        "p99_latency_s": float(np.percentile(lat, 99)),
        "makespan_s": float(span),
    }
