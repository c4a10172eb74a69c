"""Continuous-batching engine: resident slots, CUDA-graph iterations.

Life of a request:

1. *Queued* at its arrival time.
2. *Admitted* when a slot is free and its estimated device footprint fits
   the HBM budget.  The slot builds the case on the shared topology of its
   grid size (``TopologyCache``), runs the first SIMPLE iteration eagerly
   on its own stream (this allocates every workspace), then captures one
   iteration into a CUDA graph.
3. *Running*: the host loop replays each slot's graph, copies the recorded
   pressure residual to pinned memory and records an event; when the event
   has fired it applies the reference's stopping rule (simple.py:245-271:
   stop after the iteration whose pressure residual is below
   ``residualControl``) or the ``endTime`` cap, otherwise replays again.
   Only one iteration per slot is in flight, so every case runs exactly the
   iterations it would run alone.
4. *Draining*: U and p are copied to pinned host memory; the slot is freed
   (graph, fields and workspaces go back to the caching allocator) when that
   copy has landed, which is the request's finish time.

The kernels of all running slots overlap on the device (one stream each);
the persistent Krylov kernels of small grids use few blocks, so several
fit side by side.  Each case's launches have the same shapes alone and in
the mix, so its result does not depend on what else runs.
"""

from __future__ import annotations

import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np
import torch

from gridfoam_b200.serving.cases import TopologyCache, cavity_simulator
from gridfoam_b200.serving.requests import CavityRequest


@dataclass
class ServeResult:
    id: int
    n: int
    arrival: float
    admitted: float
    finished: float
    iterations: int
    converged: bool
    residual: float
    U: np.ndarray | None = field(default=None, repr=False)
    p: np.ndarray | None = field(default=None, repr=False)

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


# Resident blocks per SM of the persistent CG launch shapes (variants 0-5)
# and of BiCGStab; a slot's block cap is a share of these.
_BLOCKS_PER_SM = {0: 4, 1: 4, 2: 2, 3: 1, 4: 1, 5: 1}


class _Slot:
    """One admitted case: its fields and matrices stay on the device."""

    def __init__(self, engine: "ServingEngine", req: CavityRequest, now: float):
        from gridfoam_b200.algorithms.pressure_velocity import create_algorithm

        self.req = req
        self.admitted = now
        self.engine = engine
        self.stream = torch.cuda.Stream(engine.device)
        self.iterations = 0
        self.residual = float("inf")
        self.graph = None
        self.done = False
        self.draining = False
        sim = cavity_simulator(req.nu, req.lid, p_tol=engine.p_tol, p_solver_tol=engine.p_solver_tol,
                               p_solver_rtol=engine.p_solver_rtol, max_outer=engine.max_outer,
                               inner_precision=engine.inner_precision, device=str(engine.device.type))
        self.max_outer = engine.max_outer
        self.tol = engine.p_tol
        with torch.cuda.stream(self.stream):
            grid = engine.topologies.grid(req.n, sim)
            self.algo = create_algorithm(grid)
            self.algo.set_host_readback(False)
            variant = engine.variants.get(req.n)
            if variant is not None:
                self.algo.solvers["p"].variant = variant
            if engine.gpu_share < 1.0:
                for name, s in self.algo.solvers.items():
                    v = s.variant if s.variant is not None else 0
                    per_sm = 2 if s.bicgstab else _BLOCKS_PER_SM.get(v, 1)
                    s.block_cap = max(1, int(engine.gpu_share * engine.sms * per_sm))
            self.res_host = torch.empty(1, dtype=torch.float64, pin_memory=True)
            self.event = torch.cuda.Event()
            # First iteration eagerly: allocates every workspace and cache.
            self.algo.step()
            self._post()
            if engine.use_graphs:
                self.graph = torch.cuda.CUDAGraph()
                self.graph.capture_begin()
                self.algo.step()
                self.graph.capture_end()

    def _post(self) -> None:
        self.res_host.copy_(self.algo.p_residual, non_blocking=True)
        self.event.record(self.stream)

    def launch(self) -> None:
        with torch.cuda.stream(self.stream):
            if self.graph is not None:
                self.graph.replay()
            else:
                self.algo.step()
            self._post()

    def ready(self) -> bool:
        return self.event.query()

    def finish_iteration(self) -> None:
        """The iteration in flight has completed: apply the stopping rule."""
        self.iterations += 1
        self.residual = float(self.res_host[0])
        if self.residual < self.tol or self.iterations >= self.max_outer or not np.isfinite(self.residual):
            self.done = True

    def start_drain(self) -> None:
        with torch.cuda.stream(self.stream):
            self.U_host = torch.empty(self.algo.U.data.shape, dtype=torch.float64, pin_memory=True)
            self.p_host = torch.empty(self.algo.p.data.shape, dtype=torch.float64, pin_memory=True)
            self.U_host.copy_(self.algo.U.data, non_blocking=True)
            self.p_host.copy_(self.algo.p.data, non_blocking=True)
            self.event.record(self.stream)
        self.draining = True

    def result(self, now: float, keep_fields: bool) -> ServeResult:
        r = self.req
        return ServeResult(r.id, r.n, r.arrival, self.admitted, now, self.iterations,
                           bool(self.residual < self.tol), self.residual,
                           self.U_host.numpy().copy() if keep_fields else None,
                           self.p_host.numpy().copy() if keep_fields else None)

    def release(self) -> None:
        self.graph = None
        self.algo = None


class ServingEngine:
    """Admit, run and retire cavity solves on one device.

    ``hbm_budget``: bytes the resident cases may hold (default 80 % of the
    device memory free at construction); ``max_slots``: cases in flight at
    once; ``use_graphs``: replay captured iterations (False: eager steps).
    """

    def __init__(self, device="cuda", *, hbm_budget: int | None = None, max_slots: int = 8,
                 use_graphs: bool = True, p_tol: float = 1e-6, p_solver_tol: float = 1e-6,
                 p_solver_rtol: float = 0.0, max_outer: int = 2000, inner_precision: str = "float64",
                 keep_fields: bool = False, gpu_share: float = 1.0):
        self.device = torch.device(device)
        if self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        if hbm_budget is None:
            free, _ = torch.cuda.mem_get_info(self.device)
            hbm_budget = int(0.8 * free)
        self.hbm_budget = int(hbm_budget)
        self.max_slots = int(max_slots)
        self.use_graphs = bool(use_graphs)
        self.p_tol = float(p_tol)
        self.p_solver_tol = float(p_solver_tol)
        self.p_solver_rtol = float(p_solver_rtol)
        self.inner_precision = str(inner_precision)
        # Share of the GPU one case's persistent Krylov kernels may occupy
        # (< 1 leaves SMs free for the kernels of other slots).
        self.gpu_share = float(gpu_share)
        self.sms = torch.cuda.get_device_properties(self.device).multi_processor_count
        self.max_outer = int(max_outer)
        self.keep_fields = bool(keep_fields)
        self.topologies = TopologyCache(self.device)
        self.footprint: dict[int, int] = {}
        self.variants: dict[int, int] = {}

    # ------------------------------------------------------------------
    def prepare(self, sizes, *, autotune: bool = True) -> None:
        """Start-up for each grid size: build the topology, pick the
        pressure-CG launch shape with the autotuner and measure one case's
        device footprint (fields, matrices, workspaces, graph pool)."""
        from gridfoam_b200.solvers.autotune import PERSISTENT_VARIANTS, BoxSystem, best_variant

        for n in sorted(set(int(s) for s in sizes)):
            sim = cavity_simulator(1e-2, 1.0, p_tol=self.p_tol, p_solver_tol=self.p_solver_tol,
                                   p_solver_rtol=self.p_solver_rtol, max_outer=self.max_outer,
                                   inner_precision=self.inner_precision, device=str(self.device.type))
            self.topologies.grid(n, sim)
            if autotune:
                sysm = BoxSystem(n, n, n, device=self.device)
                # each iteration is one captured graph: single-launch variants only
                self.variants[n] = best_variant(sysm, sysm.diag, sysm.val, sysm.rhs, symmetric=True,
                                                mixed=self.inner_precision == "float32",
                                                variants=PERSISTENT_VARIANTS)
                del sysm
            torch.cuda.synchronize(self.device)
            before = torch.cuda.memory_allocated(self.device)
            slot = _Slot(self, CavityRequest(-1, n, 100.0, 1.0, 0.0), 0.0)
            torch.cuda.synchronize(self.device)
            used = torch.cuda.memory_allocated(self.device) - before
            slot.release()
            del slot
            self.footprint[n] = int(1.1 * used) + (1 << 20)

    def estimate(self, n: int) -> int:
        if n in self.footprint:
            return self.footprint[n]
        return 4096 * n**3 + (64 << 20)

    # ------------------------------------------------------------------
    def run(self, requests: list[CavityRequest], *, clock=time.perf_counter) -> list[ServeResult]:
        """Serve ``requests`` (arrival times relative to the call); returns
        results in completion order."""
        pending = deque(sorted(requests, key=lambda r: r.arrival))
        queue: deque = deque()
        active: list[_Slot] = []
        results: list[ServeResult] = []
        used = 0
        t0 = clock()
        while pending or queue or active:
            now = clock() - t0
            while pending and pending[0].arrival <= now:
                queue.append(pending.popleft())
            while queue and len(active) < self.max_slots:
                need = self.estimate(queue[0].n)
                if active and used + need > self.hbm_budget:
                    break
                req = queue.popleft()
                used += need
                # The slot's first iteration is already in flight.
                slot = _Slot(self, req, clock() - t0)
                slot.need = need
                active.append(slot)
            progressed = False
            for slot in list(active):
                if not slot.ready():
                    continue
                progressed = True
                if slot.draining:
                    results.append(slot.result(clock() - t0, self.keep_fields))
                    slot.release()
                    used -= slot.need
                    active.remove(slot)
                    continue
                slot.finish_iteration()
                if slot.done:
                    slot.start_drain()
                else:
                    slot.launch()
            if not progressed and not queue:
                if pending and not active:
                    time.sleep(max(0.0, min(1e-3, pending[0].arrival - (clock() - t0))))
                else:
                    time.sleep(2e-5)
        return results


def serve_sequential(requests: list[CavityRequest], device="cuda", *, p_tol: float = 1e-6,
                     p_solver_tol: float = 1e-6, p_solver_rtol: float = 0.0, max_outer: int = 2000,
                     keep_fields: bool = False,
                     topologies: TopologyCache | None = None, variants: dict | None = None,
                     clock=time.perf_counter) -> list[ServeResult]:
    """One-at-a-time FP64 baseline through the plain algorithm API: each
    request starts when it has arrived and the previous one has finished,
    and runs ``step()`` / ``has_converged()`` on the default stream."""
    from gridfoam_b200.algorithms.pressure_velocity import create_algorithm

    dev = torch.device(device)
    topo = topologies or TopologyCache(dev)
    results = []
    t0 = clock()
    for req in sorted(requests, key=lambda r: r.arrival):
        now = clock() - t0
        if req.arrival > now:
            time.sleep(req.arrival - now)
        admitted = clock() - t0
        sim = cavity_simulator(req.nu, req.lid, p_tol=p_tol, p_solver_tol=p_solver_tol,
                               p_solver_rtol=p_solver_rtol, max_outer=max_outer, device=str(dev.type))
        algo = create_algorithm(topo.grid(req.n, sim))
        if variants and req.n in variants:
            algo.solvers["p"].variant = variants[req.n]
        its, res = 0, float("inf")
        while its < max_outer:
            algo.step()
            its += 1
            if algo.has_converged():
                break
        res = float(algo.res_buf[0].item())
        converged = res < p_tol
        U = algo.U.data.cpu().numpy() if keep_fields else None
        p = algo.p.data.cpu().numpy() if keep_fields else None
        torch.cuda.synchronize(dev)
        results.append(ServeResult(req.id, req.n, req.arrival, admitted, clock() - t0, its, converged, res, U, p))
        del algo
    return results


def summarize(results: list[ServeResult]) -> dict:
    """Throughput and latency percentiles of a served stream."""
    if not results:
        return {"completed": 0}
    lat = np.array([r.latency for r in results])
    first = min(r.arrival for r in results)
    last = max(r.finished for r in results)
    statuses: dict = {}
    for r in results:
        st = getattr(r, "status", "converged" if r.converged else "end_time")
        statuses[st] = statuses.get(st, 0) + 1
    return {
        "completed": len(results),
        "converged": int(sum(r.converged for r in results)),
        "statuses": statuses,
        "solves_per_s": len(results) / max(last - first, 1e-12),
        "p50_latency_s": float(np.percentile(lat, 50)),
        "p99_latency_s": float(np.percentile(lat, 99)),
        "mean_iterations": float(np.mean([r.iterations for r in results])),
        "makespan_s": last - first,
    }
