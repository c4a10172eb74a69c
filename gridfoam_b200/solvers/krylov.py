"""Device CG and BiCGStab solvers (solvers/cg.py, bicgstab.py, krylov.py).

All components of a field are solved by one persistent cooperative launch
(``gf_pcg_solve`` / ``gf_bicgstab_solve``) that shares the matrix reads
between components; the reference loops over components serially
(``solvers/krylov.py:75-79``).  Convergence is decided on the device with the
reference's rule ``|r| < max(atol, rtol |r0|)``; the BiCGStab breakdown
restarts follow ``solvers/bicgstab.py:123-272``.
"""

from __future__ import annotations

import ctypes
import os

import torch

from gridfoam_b200 import _lib
from gridfoam_b200._lib import LAUNCHES, GfKrylov, call, load, ptr, stream_ptr
from gridfoam_b200.meta.config import NormType, PrecisionType, PreconditionerType, SolverConfig
from gridfoam_b200.solvers.adjoint import attach_implicit_adjoint
from gridfoam_b200.solvers.autotune import SPLIT_VARIANTS
from gridfoam_b200.solvers.base import LinearSolver, SolveResult, SolveStats, _StatsBuffer

def workspace(cache: dict, device: torch.device, n: int, ncomp: int, kind: int) -> torch.Tensor:
    """Per-shape workspace held in ``cache`` (allocated once, reused by
    every solve of its owner).

    Each solver owns its cache: solves on different streams (concurrent
    cases) must never share scratch.  ``kind``: 0 CG, 1 BiCGStab,
    ``2 + 100 * width`` mixed-precision CG, ``3 + 100 * width``
    mixed-precision BiCGStab.
    """
    key = (str(device), n, ncomp, kind)
    ws = cache.get(key)
    if ws is None:
        size = load().gf_krylov_workspace_size(n, ncomp, kind)
        ws = torch.empty(size, dtype=torch.float64, device=device)
        cache[key] = ws
    return ws


def _split_graph_loop() -> bool:
    """Whether the library runs the split CG's iterations as a CUDA graph
    while-loop (outside stream capture, unless GF_SPLIT_GRAPH=0)."""
    return os.environ.get("GF_SPLIT_GRAPH", "1")[:1] != "0" and not torch.cuda.is_current_stream_capturing()


def default_variant(n: int, mixed: bool, symmetric: bool, box: bool = True) -> int:
    """CG launch shape by system size, from fixed-iteration timings on B200
    (``python -m gridfoam_b200.solvers.autotune``).  FP64 up to ~400K cells:
    one grid reduction and a halo sync with the neighbouring blocks per
    iteration, vectors in shared memory (6.9 against 9.8 us an iteration
    for 256-thread register blocks at 48^3, 8.0 against 8.2 for the
    q-recurrence form at 64^3); then, up to ~1.3M cells, the q-recurrence
    form (q = A z + beta q, z alone gathered; 14.7 us at 1M cells); above
    that the shared-memory tiled kernel for symmetric boxes, else the split
    CG (two plain kernels an iteration, variant 29).  FP32-inner (mixed) solves: 256-thread register
    blocks below ~32K cells (6.5 us an inner iteration at 24^3, as for the
    shared-memory forms); then, up to ~1.3M cells, the single-reduction
    form with the halo sync (6.7 against 7.0 us for the q-recurrence form
    and 8.9 for the register blocks at 48^3, 7.5 against 7.8 at 64^3, 11.6
    either way at 1M cells; it falls back to the q-recurrence form where its
    six shared-memory arrays do not fit); then 512-thread blocks."""
    if mixed:
        if n < 32768:
            return 0
        return 10 if n <= 1300000 else 2
    if n <= 400000:
        return 10
    if n <= 1300000:
        return 8
    # Above ~1.3M cells (beyond L2): the staged tiles on symmetric boxes;
    # on other rows the split CG, two plain kernels an iteration, with
    # q = A p by recurrence (the rows gather z alone), x += alpha p in the
    # row kernel, the update kernel on pairs of cells, and each thread's
    # first cell prefetched into L2 while the kernel sums the previous
    # kernel's partials (fixed 100 iterations on the 4.08M-cell
    # cylinder-wake octree: 152.4-152.7 us an iteration against 155.7-156.2
    # without the prefetch (159.6 prefetching two cells), 158.5-159.6 with x
    # updated in the update kernel, 163.0 with q gathered from p, 163.0 with
    # the update one cell at a time and 164.5 for the 512-thread persistent
    # kernel).
    return 5 if symmetric and box else 29


class DeviceKrylov(LinearSolver):
    method: str = ""
    bicgstab: bool = False

    def __init__(self, config: SolverConfig):
        self.config = config
        self.solver_name = config.method.value
        self.precon_type = config.preconditioner
        self.atol = float(config.tolerance)
        self.rtol = float(config.rel_tolerance)
        self.max_iter = int(config.max_iter)
        self.max_restart = int(config.max_restart)
        self.norm_inf = config.norm_type == NormType.L_inf
        self.log_interval = config.log_interval
        self.mixed = config.inner_precision == PrecisionType.FLOAT32
        self.max_outer = int(config.max_outer)
        self.inner_eta = float(config.inner_eta)
        self.inner_margin = float(config.inner_margin)
        self._stats_dev: dict[tuple, torch.Tensor] = {}
        self._workspaces: dict[tuple, torch.Tensor] = {}
        # Optional list receiving (start event, end event, stats) per solve.
        self.profile_events: list | None = None
        # Upper bound on persistent blocks (0: one wave at full occupancy).
        self.block_cap = 0
        # Box-layout CG kernel variant (launch shape, see gf_krylov.cu and
        # solvers/autotune.py); None: chosen by system size.
        self.variant: int | None = None
        # FP64 CG with one grid reduction per iteration (Chronopoulos-Gear).
        self.single_reduction = False
        # False: no pinned statistics copy per solve (stream capture into a
        # CUDA graph); the statistics stay in the device buffer.
        self.host_stats = True
        # > 0: polls after which a device-side wait gives up and the solve
        # reports status "timeout" (0: the library default, about a second).
        self.spin_limit = 0

    def solve_arrays(self, grid, diag: torch.Tensor, val: torch.Tensor, rhs: torch.Tensor,
                     x: torch.Tensor, *, symmetric: bool = False) -> tuple[SolveStats, ...]:
        """Solve in place: ``x [ncomp, C]`` holds the guess and gets the solution.

        ``symmetric`` declares that ``A`` is symmetric (the pressure system),
        which lets CG on a uniform box read only three coefficient arrays.
        """
        k, stats = self.describe(grid, diag, val, rhs, x, symmetric=symmetric)
        nc = rhs.shape[0]
        ev = None
        if self.profile_events is not None:
            ev = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
            ev[0].record()
        call("gf_bicgstab_solve" if self.bicgstab else "gf_pcg_solve", ctypes.byref(k), stream_ptr())
        split = k.variant in SPLIT_VARIANTS and not self.bicgstab and not k.mixed and nc == 1 and not k.single_reduction
        graph_loop = split and _split_graph_loop()
        if split and not graph_loop:
            # inside a stream capture the split CG enqueues an initial
            # kernel, two a permitted iteration and a final one (those after
            # the stop return at once)
            LAUNCHES["gf_pcg_solve"] += 2 * k.max_iter + 1
        if ev is not None:
            ev[1].record()
        if not self.host_stats:
            return ()
        buf = _StatsBuffer(stats)
        out = tuple(SolveStats(self.solver_name, buf, i) for i in range(nc))
        if graph_loop and _lib.TRACK_DEFERRED:
            # the graph loop runs its two kernels iterations + 1 times
            _lib.DEFERRED_LAUNCHES.append(lambda st=out[0]: 2 * (st.iterations + 1))
        if ev is not None:
            self.profile_events.append((ev[0], ev[1], out))
        return out

    def describe(self, grid, diag: torch.Tensor, val: torch.Tensor, rhs: torch.Tensor,
                 x: torch.Tensor, *, symmetric: bool = False) -> tuple[GfKrylov, torch.Tensor]:
        """The solve's descriptor (workspace and statistics buffer included)
        without launching it: ``solve_arrays`` launches it alone, the solve
        server batches the descriptors of many cases into one launch."""
        nc, n = rhs.shape
        key = (str(grid.device), nc)
        stats = self._stats_dev.get(key)
        if stats is None:
            stats = torch.zeros((nc, 5), dtype=torch.float64, device=grid.device)
            self._stats_dev[key] = stats
        # FP32 inner cycles: CG for one system, BiCGStab for every component
        mixed = self.mixed and (nc == 1 or self.bicgstab)
        if mixed:
            kind = (3 if self.bicgstab else 2) + 100 * grid.ell_width
        else:
            kind = int(self.bicgstab)
        ws = workspace(self._workspaces, grid.device, n, nc, kind)
        k = GfKrylov()
        k.n = n
        k.width = grid.ell_width
        k.ncomp = nc
        k.max_iter = self.max_iter
        k.max_restart = self.max_restart
        k.norm_inf = int(self.norm_inf)
        k.jacobi = int(self.precon_type == PreconditionerType.JACOBI)
        k.atol = self.atol
        k.rtol = self.rtol
        k.nbr = ptr(grid.dev["ell_nbr"])
        if "ell_len" in grid.dev:
            k.row_len = ptr(grid.dev["ell_len"])
        k.diag = ptr(diag)
        k.val = ptr(val)
        k.rhs = ptr(rhs)
        k.x = ptr(x)
        k.work = ptr(ws)
        k.work_len = ws.numel()
        k.stats = ptr(stats)
        k.mixed = int(mixed)
        k.max_outer = self.max_outer
        k.inner_eta = self.inner_eta
        k.inner_margin = self.inner_margin
        k.block_cap = int(self.block_cap)
        k.spin_limit = int(self.spin_limit)
        box = getattr(grid, "box_strides", None)
        k.variant = (int(self.variant) if self.variant is not None
                     else default_variant(n, mixed, symmetric, box is not None))
        k.single_reduction = int(self.single_reduction and not mixed and not self.bicgstab and nc == 1)
        if box is not None and not self.bicgstab and nc == 1:
            k.stride_y, k.stride_z = box
            k.symmetric = int(symmetric)
        return k, stats

    def _solve_matrix(self, A, rhs_store: torch.Tensor, x0_store: torch.Tensor) -> SolveResult:
        x = x0_store.contiguous().clone()
        stats = self.solve_arrays(A.grid, A.diag_store, A.val, rhs_store.contiguous(), x)
        sol = x[0] if A.field.component_shape == () else x.t()
        return SolveResult(solution=sol, stats=stats)

    def solve(self, eq) -> SolveResult:
        """solvers/base.py:96-122: with ``grad_mode="adjoint"`` (default) and
        differentiable coefficients, the solve is detached and the implicit
        adjoint attached; with ``"unrolled"`` the iterations run as
        differentiable device tensor algebra (``solvers/unrolled.py``)."""
        A = eq.fv_matrix
        if torch.is_grad_enabled() and A.requires_grad:
            if self.grad_mode == "unrolled":
                from gridfoam_b200.solvers.unrolled import solve_unrolled

                sol, stats = solve_unrolled(self, A, A.source, eq.target.data.detach())
                return SolveResult(solution=sol, stats=stats)
            if self.grad_mode != "adjoint":
                raise ValueError(f"unknown grad_mode {self.grad_mode!r}")
            with torch.no_grad():
                res = self._solve_primal(eq)
            sol = attach_implicit_adjoint(A, res.solution, solve_transpose=self.solve_transpose)
            return SolveResult(solution=sol, stats=res.stats)
        return self._solve_primal(eq)

    def _solve_primal(self, eq) -> SolveResult:
        A = eq.fv_matrix
        return self._solve_matrix(A, A.source_store, eq.target.store)

    def solve_transpose(self, A_T, rhs: torch.Tensor) -> torch.Tensor:
        nc = A_T.num_components
        r = (rhs.reshape(1, -1) if nc == 1 else rhs.t()).contiguous()
        res = self._solve_matrix(A_T, r, torch.zeros_like(r))
        return res.solution


class CGSolver(DeviceKrylov):
    """Jacobi-preconditioned CG (solvers/cg.py:23-174)."""

    bicgstab = False


class BiCGSTABSolver(DeviceKrylov):
    """Right-preconditioned BiCGStab with restarts (solvers/bicgstab.py:23-272)."""

    bicgstab = True
