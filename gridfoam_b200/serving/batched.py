"""Lockstep solve server: the same-phase Krylov solves of every resident case
in ONE launch, each batched iteration captured in a CUDA graph; cases above
``solo_cells`` cells run beside that lane as solo slots.

Life of a request:

1. *Queued* at its arrival time.
2. *Admitted* when a slot is free, its estimated device footprint fits the
   HBM budget and its persistent blocks fit beside the resident cases'
   (``blocks_for``: a fixed share per grid size, so a case's solves do not
   depend on what else runs).  The slot builds its case on the shared
   topology of its size and runs its first SIMPLE iteration eagerly (this
   allocates every workspace).
3. *Running*: one batched iteration advances every resident case by one
   SIMPLE iteration.  Each case's step pauses at its Krylov solves
   (``SIMPLE.step_phases`` with deferred solves); the cases' assembly and
   correction kernels run on one stream per case, and at every solve phase
   the cases' systems go into one ``gf_bicgstab_solve_batched`` /
   ``gf_pcg_solve_batched`` launch on the engine stream (fork/join by
   events).  The whole iteration, the copy of every case's pressure
   residual to pinned memory included, is captured once per set of
   resident cases and replayed; the set changes when a case retires or a
   new one is admitted.  After each replay the host applies the reference's
   stopping rule (simple.py:245-271: stop after the iteration whose
   pressure residual is below ``residualControl``) or the ``endTime`` cap.
4. *Draining*: U and p are copied to pinned host memory; the slot is freed
   when the copy has landed (the request's finish time).

Large cases (more than ``solo_cells`` cells, default 200,000: the 64^3 and
96^3 cavities) are bandwidth-bound and already fill the GPU alone; in the
batched launch their fixed block share makes them slower than alone and
holds the lockstep back.  They run as *solo slots* instead
(``serving.engine``'s slot: the case's own stream, its single-system Krylov
kernels, one captured graph an iteration, at most ``max_solo`` at once),
asynchronously beside the lockstep lane of the small cases; the host loop
polls the lane and every solo slot and relaunches whichever has finished.

Failure handling: a request whose footprint can never fit the budget, or
whose first iteration raises (an allocation failure, a NaN input), is
rejected with ``status`` set and does not stop the others; a non-finite
pressure residual ends that request with status ``nonfinite``.
"""

from __future__ import annotations

import ctypes
import time
from collections import deque

import numpy as np
import torch

from gridfoam_b200._lib import GfKrylov, call, load
from gridfoam_b200.serving.cases import TopologyCache, cavity_simulator
from gridfoam_b200.serving.engine import ServeResult
from gridfoam_b200.serving.requests import CavityRequest


def blocks_for(n_cells: int, bicgstab: bool) -> int:
    """Persistent blocks of one case's solves in a batched launch: about
    1024 cells a 256-thread CG block (at most 296, two an SM) and 8192 cells
    a 512-thread BiCGStab block (at most 74).  A fixed count per grid size
    keeps a case's iterates independent of what else shares the launch;
    fewer, fuller blocks (4096 and 65536 cells) made the small cases'
    solves latency-bound at about twice the time an iteration."""
    if bicgstab:
        return int(min(74, max(1, -(-n_cells // 8192))))
    return int(min(296, max(1, -(-n_cells // 1024))))


class _Case:
    """One admitted case: its fields, matrices and workspaces stay resident."""

    def __init__(self, engine: "BatchedEngine", req: CavityRequest, now: float):
        from gridfoam_b200.algorithms.pressure_velocity import create_algorithm

        self.req = req
        self.admitted = now
        self.stream = torch.cuda.Stream(engine.device)
        self.iterations = 0
        self.residual = float("inf")
        self.status = "running"
        sim = cavity_simulator(req.nu, req.lid, p_tol=engine.p_tol, p_solver_tol=engine.p_solver_tol,
                               p_solver_rtol=engine.p_solver_rtol, max_outer=engine.max_outer,
                               inner_precision=engine.inner_precision, device=str(engine.device.type))
        with torch.cuda.stream(self.stream):
            self.algo = create_algorithm(engine.topologies.grid(req.n, sim))
            self.algo.set_host_readback(False)
        self.cg_blocks = blocks_for(req.n**3, False)
        self.bicg_blocks = blocks_for(req.n**3, True)

    @property
    def n_cells(self) -> int:
        return self.req.n**3


class BatchedEngine:
    """Admit, run and retire cavity solves on one device in lockstep.

    ``hbm_budget``: bytes the resident cases may hold (default 80 % of the
    free device memory); ``max_slots``: resident cases (at most 16, the
    batched launch's limit); ``p_tol``: residualControl on p (normalised
    initial residual); ``p_solver_tol`` / ``p_solver_rtol``: the pressure
    CG's absolute and relative tolerances.
    """

    MAX_SLOTS = 16

    def __init__(self, device="cuda", *, hbm_budget: int | None = None, max_slots: int = 8,
                 use_graphs: bool = True, p_tol: float = 1e-6, p_solver_tol: float = 1e-12,
                 p_solver_rtol: float = 0.01, max_outer: int = 2000, inner_precision: str = "float64",
                 keep_fields: bool = False, solo_cells: int | None = 200_000, max_solo: int = 2):
        self.device = torch.device(device)
        if self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        if hbm_budget is None:
            free, _ = torch.cuda.mem_get_info(self.device)
            hbm_budget = int(0.8 * free)
        self.hbm_budget = int(hbm_budget)
        self.max_slots = int(min(max_slots, self.MAX_SLOTS))
        self.use_graphs = bool(use_graphs)
        self.p_tol = float(p_tol)
        self.p_solver_tol = float(p_solver_tol)
        self.p_solver_rtol = float(p_solver_rtol)
        self.inner_precision = str(inner_precision)
        self.max_outer = int(max_outer)
        self.keep_fields = bool(keep_fields)
        self.topologies = TopologyCache(self.device)
        self.footprint: dict[int, int] = {}
        # Solo slots (see the module doc); None: every case in the lane.
        self.solo_cells = None if solo_cells is None else int(solo_cells)
        self.max_solo = int(max_solo)
        self.variants: dict[int, int] = {}
        self.gpu_share = 1.0
        self.sms = torch.cuda.get_device_properties(self.device).multi_processor_count
        self.stream = torch.cuda.Stream(self.device)
        with torch.cuda.device(self.device):
            lib = load()
            self.cg_capacity = int(lib.gf_batch_max_blocks(0))
            self.bicg_capacity = int(lib.gf_batch_max_blocks(1))
        if self.cg_capacity < 1 or self.bicg_capacity < 1:
            raise RuntimeError("batched solve kernels are not available on this device")
        self._res_dev = torch.zeros(self.MAX_SLOTS, dtype=torch.float64, device=self.device)
        self._res_host = torch.zeros(self.MAX_SLOTS, dtype=torch.float64, pin_memory=True)
        self.launches = 0
        self.captures = 0
        # Fault-injection hooks for tests: admission_hook(request) runs just
        # before a case is built (an exception there rejects the request);
        # case_hook(case) runs after (e.g. to plant a NaN in its fields).
        self.admission_hook = None
        self.case_hook = None

    # ------------------------------------------------------------------
    def prepare(self, sizes) -> None:
        """Start-up per grid size: build the topology and measure one case's
        device footprint (fields, matrices, workspaces)."""
        from gridfoam_b200.serving.engine import _Slot

        for n in sorted(set(int(s) for s in sizes)):
            torch.cuda.synchronize(self.device)
            before = torch.cuda.memory_allocated(self.device)
            req = CavityRequest(-1, n, 100.0, 1.0, 0.0)
            if self.is_solo(n):
                slot = _Slot(self, req, 0.0)
                torch.cuda.synchronize(self.device)
                used = torch.cuda.memory_allocated(self.device) - before
                slot.release()
                del slot
            else:
                case = _Case(self, req, 0.0)
                self._iteration([case], capture=False)
                torch.cuda.synchronize(self.device)
                used = torch.cuda.memory_allocated(self.device) - before
                del case
            self.footprint[n] = int(1.1 * used) + (1 << 20)

    def is_solo(self, n: int) -> bool:
        return self.solo_cells is not None and n**3 > self.solo_cells

    def estimate(self, n: int) -> int:
        if n in self.footprint:
            return self.footprint[n]
        return 4096 * n**3 + (64 << 20)

    # ------------------------------------------------------------------
    def _batched_solve(self, entries: list) -> None:
        """One launch for the deferred solves ``[(case, solver, k), ...]``."""
        bicg = entries[0][1].bicgstab
        if any(s.bicgstab != bicg for _, s, _ in entries):
            raise RuntimeError("cases reached different solve phases")
        arr = (GfKrylov * len(entries))(*[k for _, _, k in entries])
        blocks = (ctypes.c_int32 * len(entries))(*[c.bicg_blocks if bicg else c.cg_blocks for c, _, _ in entries])
        name = "gf_bicgstab_solve_batched" if bicg else "gf_pcg_solve_batched"
        call(name, arr, len(entries), blocks, ctypes.c_void_p(self.stream.cuda_stream))
        self.launches += 1

    def _iteration(self, cases: list[_Case], *, capture: bool) -> None:
        """Enqueue one SIMPLE iteration of every case (see module doc)."""
        main = self.stream
        fork = torch.cuda.Event()
        fork.record(main)
        gens = []
        for c in cases:
            c.stream.wait_event(fork)
            c.algo._deferred = []
            gens.append(c.algo.step_phases())
        try:
            while True:
                entries, finished = [], 0
                for c, g in zip(cases, gens):
                    with torch.cuda.stream(c.stream):
                        try:
                            next(g)
                        except StopIteration:
                            finished += 1
                            continue
                    solver, k = c.algo._deferred.pop()
                    entries.append((c, solver, k))
                if finished == len(cases):
                    break
                if finished:
                    raise RuntimeError("cases reached different solve phases")
                for c in cases:
                    ev = torch.cuda.Event()
                    ev.record(c.stream)
                    main.wait_event(ev)
                with torch.cuda.stream(main):
                    self._batched_solve(entries)
                done = torch.cuda.Event()
                done.record(main)
                for c in cases:
                    c.stream.wait_event(done)
        finally:
            for c in cases:
                c.algo._deferred = None
        for i, c in enumerate(cases):
            with torch.cuda.stream(c.stream):
                self._res_dev[i].copy_(c.algo.p_residual[0])
            ev = torch.cuda.Event()
            ev.record(c.stream)
            main.wait_event(ev)
        with torch.cuda.stream(main):
            self._res_host[: len(cases)].copy_(self._res_dev[: len(cases)], non_blocking=True)

    # ------------------------------------------------------------------
    def _result(self, c: _Case, now: float) -> ServeResult:
        r = c.req
        U = p = None
        if self.keep_fields:
            U, p = c.U_host.numpy().copy(), c.p_host.numpy().copy()
        res = ServeResult(r.id, r.n, r.arrival, c.admitted, now, c.iterations,
                          c.status == "converged", c.residual, U, p)
        res.status = c.status
        return res

    def _reject(self, req: CavityRequest, now: float, status: str) -> ServeResult:
        res = ServeResult(req.id, req.n, req.arrival, now, now, 0, False, float("nan"))
        res.status = status
        return res

    def run(self, requests: list[CavityRequest], *, clock=time.perf_counter) -> list[ServeResult]:
        """Serve ``requests`` (arrival times relative to the call); returns
        results in completion order (rejected requests included, with
        ``status`` set)."""
        from gridfoam_b200.serving.engine import _Slot

        pending = deque(sorted(requests, key=lambda r: r.arrival))
        queue: deque = deque()
        lane: list[_Case] = []
        solos: list = []
        results: list[ServeResult] = []
        used = 0
        graph = None
        graph_set: tuple = ()
        # lane state: "idle" | "eager" (an uncaptured iteration in flight) |
        # "replay" (a graph replay in flight)
        state = "idle"
        lane_ev = torch.cuda.Event()
        t0 = clock()

        def now() -> float:
            return clock() - t0

        def retire_lane() -> None:
            nonlocal used
            for c in [c for c in lane if c.status != "running"]:
                with torch.cuda.stream(c.stream):
                    c.stream.wait_stream(self.stream)
                    c.U_host = torch.empty(c.algo.U.data.shape, dtype=torch.float64, pin_memory=True)
                    c.p_host = torch.empty(c.algo.p.data.shape, dtype=torch.float64, pin_memory=True)
                    c.U_host.copy_(c.algo.U.data, non_blocking=True)
                    c.p_host.copy_(c.algo.p.data, non_blocking=True)
                c.stream.synchronize()
                results.append(self._result(c, now()))
                lane.remove(c)
                used -= c.need
                c.algo = None

        while pending or queue or lane or solos:
            while pending and pending[0].arrival <= now():
                queue.append(pending.popleft())
            # Admission (first admissible request in arrival order) by slots,
            # HBM budget, persistent blocks and, for the lane, an idle lane.
            admitted = True
            while admitted and queue and len(lane) + len(solos) < self.max_slots:
                admitted = False
                for req in list(queue):
                    need = self.estimate(req.n)
                    if need > self.hbm_budget:
                        queue.remove(req)
                        results.append(self._reject(req, now(), "rejected_memory"))
                        admitted = True
                        break
                    if (lane or solos) and used + need > self.hbm_budget:
                        continue
                    solo = self.is_solo(req.n)
                    if solo and len(solos) >= self.max_solo:
                        continue
                    if not solo:
                        cg = sum(c.cg_blocks for c in lane) + blocks_for(req.n**3, False)
                        bi = sum(c.bicg_blocks for c in lane) + blocks_for(req.n**3, True)
                        if state != "idle" or (lane and (cg > self.cg_capacity or bi > self.bicg_capacity)):
                            continue
                    queue.remove(req)
                    admitted = True
                    try:
                        if self.admission_hook is not None:
                            self.admission_hook(req)
                        case = _Slot(self, req, now()) if solo else _Case(self, req, now())
                        if self.case_hook is not None:
                            self.case_hook(case)
                    except (RuntimeError, ValueError, torch.cuda.OutOfMemoryError) as exc:
                        results.append(self._reject(req, now(), f"rejected: {type(exc).__name__}"))
                        break
                    case.need = need
                    used += need
                    (solos if solo else lane).append(case)
                    break
            progressed = False
            # Solo slots: one captured iteration in flight each.
            for slot in list(solos):
                if not slot.ready():
                    continue
                progressed = True
                if slot.draining:
                    res = slot.result(now(), self.keep_fields)
                    res.status = "converged" if res.converged else (
                        "nonfinite" if not np.isfinite(res.residual) else "end_time")
                    results.append(res)
                    slot.release()
                    used -= slot.need
                    solos.remove(slot)
                    continue
                slot.finish_iteration()
                if slot.done:
                    slot.start_drain()
                else:
                    slot.launch()
            # The lockstep lane.
            if state != "idle" and lane_ev.query():
                progressed = True
                self._finish(lane, now())
                running = not any(c.status != "running" for c in lane)
                if state == "eager" and running and self.use_graphs:
                    g = torch.cuda.CUDAGraph()
                    with torch.cuda.graph(g, stream=self.stream):
                        self._iteration(lane, capture=True)
                    self.captures += 1
                    graph, graph_set = g, tuple(id(c) for c in lane)
                state = "idle"
                retire_lane()
                if tuple(id(c) for c in lane) != graph_set:
                    graph = None
            if state == "idle" and lane:
                progressed = True
                key = tuple(id(c) for c in lane)
                if graph is not None and key == graph_set:
                    with torch.cuda.stream(self.stream):
                        graph.replay()
                    state = "replay"
                else:
                    # a new set of resident cases: one eager iteration (new
                    # cases allocate their workspaces), captured after it
                    graph = None
                    self._iteration(lane, capture=False)
                    state = "eager"
                lane_ev.record(self.stream)
            if not progressed:
                if pending and not (lane or solos or queue):
                    time.sleep(max(0.0, min(1e-3, pending[0].arrival - now())))
                else:
                    time.sleep(2e-5)
        return results

    def _finish(self, cases: list[_Case], now: float) -> None:
        """After an iteration: residuals, the stopping rule and the cap."""
        res = self._res_host[: len(cases)].numpy()
        for c, r in zip(cases, res):
            c.iterations += 1
            c.residual = float(r)
            if not np.isfinite(c.residual):
                c.status = "nonfinite"
            elif c.residual < self.p_tol:
                c.status = "converged"
            elif c.iterations >= self.max_outer:
                c.status = "end_time"


def serve_batched(requests, device="cuda", **kw) -> list[ServeResult]:
    eng = BatchedEngine(device, **kw)
    eng.prepare({r.n for r in requests})
    return eng.run(requests)
