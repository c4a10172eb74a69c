"""Launch-shape autotuner and fixed-iteration timing of the CG kernels.

The box-layout CG kernels (uniform lexicographic grids, implicit
neighbours) come in variants that differ in threads per block and cells per
thread per pass (``gf_krylov.cu``: ``box_kernel``).  Which one is fastest
depends on the system size: small systems are bound by the two grid
barriers of each iteration, where fewer and larger blocks arrive faster,
and large ones by memory latency.  ``best_variant`` times a fixed number of
iterations of every variant on the caller's own matrix and caches the
winner per (device, cells, strides, symmetric, precision).  That cache is
the package's only global state and a lock guards it.

Run as a module it times one synthetic box system, or the pressure system
of the cylinder wake's octree after one PISO step (``--wake``), for
profiling a single fixed-length kernel launch::

    python -m gridfoam_b200.solvers.autotune --box 64 64 256 --iters 200
    python -m gridfoam_b200.solvers.autotune --wake 192 120 24 --iters 40 --variant 19
"""

from __future__ import annotations

import argparse
import json
import threading
from dataclasses import dataclass, field

import torch

from gridfoam_b200.meta.config import PrecisionType, PreconditionerType, SolverConfig, SolverType

# Variants 0-7 differ only in launch shape and memory placement (their
# iterates differ by the order of the dot-product partial sums); 8 and 9
# form q = A p by recurrence.
N_VARIANTS = 32
VARIANTS = {
    0: "256 threads x 1 cell/pass",
    1: "256 threads x 2 cells/pass",
    2: "512 threads x 1 cell/pass",
    3: "1024 threads x 1 cell/pass",
    4: "1024 threads x 2 cells/pass",
    5: "512 threads, shared-memory tiles by bulk async copy (symmetric FP64 only)",
    6: "512 threads, own-cell vectors resident in shared memory (up to ~1.3M cells)",
    7: "1024 threads, own-cell vectors resident in shared memory (up to ~1.3M cells)",
    8: "1024 threads, shared-memory vectors, q = A z + beta q recurrence, 1 cell/pass",
    9: "1024 threads, shared-memory vectors, q = A z + beta q recurrence, 2 cells/pass",
    10: "1024 threads, shared-memory vectors, one grid reduction and a halo sync per iteration, 1 cell/pass (FP32-inner: same form)",
    11: "1024 threads, shared-memory vectors, one grid reduction and a halo sync per iteration, 2 cells/pass",
    12: "512 threads x 2 a SM, vectors in global memory, q = A z + beta q recurrence (any size, FP64)",
    13: "1024 threads, vectors in global memory, q = A z + beta q recurrence (any size, FP64)",
    14: "256 threads x 4 a SM, vectors in global memory, q = A z + beta q recurrence (any size, FP64)",
    15: "ELL rows (box: as 2), lean 32-bit form, x update deferred: 256 threads x 4 a SM, row loads in groups of 8",
    16: "ELL rows (box: as 2), lean 32-bit form: 256 threads x 5 a SM, groups of 8",
    17: "ELL rows (box: as 2), lean 32-bit form: 256 threads x 6 a SM, groups of 4",
    18: "ELL rows (box: as 2), lean 32-bit form: 256 threads x 6 a SM, groups of 4, next cell prefetched to L2",
    19: "split: two plain kernels an iteration (no grid barrier), 256 threads x 8 a SM (FP64, large systems)",
    20: "split: two plain kernels an iteration (no grid barrier), 256 threads x 6 a SM (FP64, large systems)",
    21: "split, update kernel on pairs of cells (16-byte accesses), 256 threads x 8 a SM (FP64, large systems)",
    22: "split, update kernel on pairs of cells (16-byte accesses), 256 threads x 7 a SM (FP64, large systems)",
    23: "split, pairs, ELL slots loaded two at a time, 256 threads x 7 a SM (FP64, large systems)",
    24: "split, pairs, ELL slots loaded four at a time, 256 threads x 6 a SM (FP64, large systems)",
    25: "split, pairs, q = A z + beta q by recurrence (one gathered vector), 256 threads x 8 a SM (FP64, large systems)",
    26: "split, q = A z + beta q by recurrence, update one cell at a time, 256 threads x 8 a SM (FP64, large systems)",
    27: "split as 25, x += alpha p in the row kernel (update kernel reads neither x nor p) (FP64, large systems)",
    28: "split as 21, x += alpha p in the row kernel (update kernel reads neither x nor p) (FP64, large systems)",
    29: "split as 27, first cell's data prefetched into L2 while the partials are summed (FP64, large systems)",
    30: "split as 27, first two cells' data prefetched into L2 while the partials are summed (FP64, large systems)",
    31: "split as 29, prefetches and scalar reads ahead of the loop control reads and partial sums (FP64, large systems)",
}

_LOCK = threading.Lock()
_CACHE: dict[tuple, int] = {}


@dataclass
class BoxSystem:
    """A symmetric 7-point system on an ``nx x ny x nz`` lexicographic box.

    It carries what ``DeviceKrylov.solve_arrays`` reads from a grid
    (``device``, ``ell_width``, ``dev["ell_nbr"]``, ``box_strides``) plus the
    matrix: unit couplings between face neighbours, Dirichlet ends in z, so
    ``-A`` is an M-matrix (the sign of gridfoam's pressure Laplacian).
    """

    nx: int
    ny: int
    nz: int
    device: torch.device
    ell_width: int = 6
    dev: dict = field(default_factory=dict)
    box_strides: tuple[int, int] = (0, 0)

    def __post_init__(self):
        nx, ny, nz = self.nx, self.ny, self.nz
        n = nx * ny * nz
        c = torch.arange(n, device=self.device, dtype=torch.int64)
        i, j, k = c % nx, (c // nx) % ny, c // (nx * ny)
        sy, sz = nx, nx * ny
        self.box_strides = (sy, sz)
        nbr = torch.empty((6, n), dtype=torch.int64, device=self.device)
        val = torch.zeros((6, n), dtype=torch.float64, device=self.device)
        for s, (has, off) in enumerate(((i > 0, -1), (i < nx - 1, 1), (j > 0, -sy), (j < ny - 1, sy),
                                        (k > 0, -sz), (k < nz - 1, sz))):
            nbr[s] = torch.where(has, c + off, c)
            val[s] = has.to(torch.float64)
        self.dev["ell_nbr"] = nbr.to(torch.int32).contiguous()
        ends = (k == 0).to(torch.float64) + (k == nz - 1).to(torch.float64)
        self.diag = -(val.sum(0) + 2.0 * ends)
        self.val = val.contiguous()
        g = torch.Generator(device="cpu").manual_seed(0)
        self.rhs = torch.randn((1, n), generator=g, dtype=torch.float64).to(self.device)

    @property
    def num_cells(self) -> int:
        return self.nx * self.ny * self.nz


def _solver(iters: int, mixed: bool, variant: int, single_reduction: bool = False):
    from gridfoam_b200.solvers.krylov import CGSolver

    cfg = SolverConfig(
        method=SolverType.CG,
        preconditioner=PreconditionerType.JACOBI,
        tolerance=0.0,
        rel_tolerance=0.0,
        max_iter=iters,
        inner_precision=PrecisionType.FLOAT32 if mixed else PrecisionType.FLOAT64,
    )
    s = CGSolver(cfg)
    s.variant = variant
    s.single_reduction = single_reduction
    return s


def time_variant(grid, diag, val, rhs, *, symmetric: bool, mixed: bool, variant: int,
                 iters: int = 100, repeats: int = 3, single_reduction: bool = False) -> tuple[float, int]:
    """Microseconds per CG iteration of one variant (best of ``repeats``).

    Tolerances are zero, so FP64 runs exactly ``iters`` iterations; the
    mixed solver is normalised by the iterations its statistics report.
    ``x`` is a scratch zero vector; the caller's data are only read.
    """
    s = _solver(iters, mixed, variant, single_reduction)
    x = torch.zeros_like(rhs)
    s.solve_arrays(grid, diag, val, rhs, x, symmetric=symmetric)  # warm-up
    best, its = float("inf"), 0
    for _ in range(repeats):
        x.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        st = s.solve_arrays(grid, diag, val, rhs, x, symmetric=symmetric)
        e1.record()
        e1.synchronize()
        its = max(1, st[0].iterations)
        best = min(best, 1e3 * e0.elapsed_time(e1) / its)
    return best, its


SPLIT_VARIANTS = (19, 20, 21, 22, 23, 24, 25, 26, 27, 28, 29, 30, 31)
# The persistent single-launch variants: the ones a captured CUDA graph
# holds as one kernel node (the split CG, 19 and 20, enqueues every
# permitted iteration when it is captured).
PERSISTENT_VARIANTS = tuple(v for v in range(N_VARIANTS) if v not in SPLIT_VARIANTS)


def best_variant(grid, diag, val, rhs, *, symmetric: bool, mixed: bool, iters: int = 60,
                 variants=None) -> int:
    """Fastest box CG variant for this system shape among ``variants``
    (default all; timed once, then cached)."""
    cands = tuple(range(N_VARIANTS) if variants is None else variants)
    key = (str(grid.device), torch.cuda.get_device_name(grid.device), grid.num_cells,
           tuple(grid.box_strides), bool(symmetric), bool(mixed), cands)
    with _LOCK:
        hit = _CACHE.get(key)
        if hit is not None:
            return hit
        times = {v: time_variant(grid, diag, val, rhs, symmetric=symmetric, mixed=mixed, variant=v,
                                 iters=iters, repeats=2)[0] for v in cands}
        best = min(cands, key=lambda v: times[v])
        _CACHE[key] = best
        return best


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--box", type=int, nargs=3, default=[64, 64, 256], metavar=("NX", "NY", "NZ"))
    ap.add_argument("--iters", type=int, default=200)
    ap.add_argument("--repeats", type=int, default=3)
    ap.add_argument("--variant", type=int, default=-1, help="one variant; -1 times all of them")
    ap.add_argument("--precision", choices=["float64", "float32"], default="float64",
                    help="float32: FP32 inner CG inside FP64 refinement")
    ap.add_argument("--single-reduction", action="store_true",
                    help="FP64 Chronopoulos-Gear CG (one grid reduction per iteration)")
    ap.add_argument("--wake", type=int, nargs=3, default=None, metavar=("NX", "NY", "NZ"),
                    help="the cylinder wake's pressure system on this base grid (2 refinement levels)")
    args = ap.parse_args()
    dev = torch.device("cuda")
    mixed = args.precision == "float32"
    variants = range(N_VARIANTS) if args.variant < 0 else [args.variant]
    if args.wake is not None:
        from gridfoam_b200.cases import create_case, cylinder_wake_case

        _, grid, algo = create_case(cylinder_wake_case(tuple(args.wake)), device=dev)
        algo.step()
        torch.cuda.synchronize()
        diag, val, rhs = algo.pEqn.diag_store, algo.pEqn.val, algo.pEqn.source_store
        n, f, label = grid.num_cells, grid.num_internal_faces, {"wake": args.wake}
        sysm = grid
    else:
        sysm = BoxSystem(*args.box, device=dev)
        diag, val, rhs = sysm.diag, sysm.val, sysm.rhs
        n = sysm.num_cells
        nx, ny, nz = args.box
        f = (nx - 1) * ny * nz + nx * (ny - 1) * nz + nx * ny * (nz - 1)
        label = {"box": args.box}
    for v in variants:
        us, its = time_variant(sysm, diag, val, rhs, symmetric=True, mixed=mixed, variant=v,
                               iters=args.iters, repeats=args.repeats, single_reduction=args.single_reduction)
        # Algorithmic bytes of one fused symmetric PCG-Jacobi iteration:
        # 14 C s + F (s + 8), F the internal faces.
        s = 4 if mixed else 8
        gbs = (14 * n * s + f * (s + 8)) / (us * 1e-6) / 1e9
        print(json.dumps({**label, "cells": n, "faces": f, "precision": args.precision,
                          "single_reduction": args.single_reduction, "variant": v,
                          "shape": VARIANTS[v], "iterations": its, "us_per_iter": round(us, 3),
                          "algorithmic_GBps": round(gbs, 1)}))


if __name__ == "__main__":
    main()
