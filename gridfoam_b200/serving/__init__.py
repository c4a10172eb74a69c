"""Continuous-batching solve server for many cavity cases on one GPU.

Requests (lid-driven cavity solves of uneven grid sizes, each a SIMPLE run
to a pressure-residual tolerance) arrive over time.  The engine keeps each
admitted case's fields, matrices and workspaces resident on the device in a
*slot* with its own CUDA stream, captures one SIMPLE iteration of the slot
into a CUDA graph, and replays the graphs of all slots round-robin, so the
kernels of many cases overlap on the device while the host only replays
graphs and reads one residual per iteration.  New requests are admitted as
slots and the HBM budget free up; p50/p99 latency (arrival to result on the
host) and solves/s are reported.  ``serve_sequential`` is the one-at-a-time
FP64 baseline through the plain algorithm API.  ``BatchedEngine`` runs the
resident cases in lockstep instead: the same-phase Krylov solves of every
case go into one batched launch, and each batched iteration is one CUDA
graph.
"""

from gridfoam_b200.serving.batched import BatchedEngine, blocks_for
from gridfoam_b200.serving.engine import ServeResult, ServingEngine, serve_sequential, summarize
from gridfoam_b200.serving.requests import SIZES, CavityRequest, poisson_stream

__all__ = [
    "BatchedEngine",
    "SIZES",
    "blocks_for",
    "CavityRequest",
    "ServeResult",
    "ServingEngine",
    "poisson_stream",
    "serve_sequential",
    "summarize",
]
