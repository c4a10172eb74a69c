"""Benchmark: cell-iterations/s of the cylinder wake on a 3-level octree
(domain 30D x 20D x 4D, base 256 x 160 x 32 cells refined two levels within
2D of an immersed cylinder of diameter D = 1: 4,079,808 cells, 12.2M
internal faces, hanging faces at both level interfaces), inflow 1,
nu = 0.01 (Re 100), PISO at CFL 0.5 on the finest cell, two correctors,
float64, on one B200.

One step is one PISO time step (momentum BiCGStab + 2 pressure CG solves to
tolerance).  ``value`` is device-timed with inputs resident in HBM; ``e2e``
times the public API with the step's state copied host->device from pinned
memory and the result read back every step.  ``--impl reference`` times the
CPU path (the reference algorithm restated in numpy with its Krylov solves
and repeated scatter-adds in multi-threaded C) on the same mesh and case,
on every host core.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
"""

from __future__ import annotations

import argparse
import json
import os
import pathlib
import statistics
import subprocess
import sys
import tempfile
import time

REPO = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(REPO))

METRIC = "cell-iters/s"
BASE = (256, 160, 32)
WORKLOAD = f"cylinder_wake_{BASE[0]}x{BASE[1]}x{BASE[2]}_piso"
ALGORITHM = ("piso nCorrectors=2, dt=CFL 0.5 on the finest cell, upwind, p cg+jacobi tol 1e-7 rel 0.01 "
             "(pFinal rel 0), U bicgstab+jacobi tol 1e-8 rel 0.1")


def workload_case() -> dict:
    from gridfoam_b200.cases import cylinder_wake_case

    return cylinder_wake_case(BASE)


def workload_config(mesh, world: int) -> dict:
    """The bench line's ``config``: a function of the mesh and the case only,
    so the GPU arm and the reference arm print the same dictionary."""
    import numpy as np

    F = int(np.asarray(mesh.internal_faces_owner).shape[0])
    imm = int(np.asarray(mesh.ap.is_immersed_face).sum())
    return {
        "workload": WORKLOAD,
        "cells": int(mesh.n_cells),
        "internal_faces": F,
        "immersed_faces": imm,
        "algorithm": ALGORITHM,
        "l2": "working set (8 GB) larger than L2 (126 MB), no flush",
        "parallelism": f"replicas x{world}",
    }


def peaks() -> tuple[float, str]:
    path = REPO / "MEASURED_PEAKS.json"
    try:
        data = json.loads(path.read_text())
        return float(data["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    QUERY = (
        "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
        "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
        "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"
    )

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = tempfile.NamedTemporaryFile(prefix="gf_clocks_", suffix=".csv", delete=False).name

    def start(self) -> None:
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "200"],
                stdout=self.fh, stderr=subprocess.DEVNULL,
            )
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in pathlib.Path(self.path).read_text().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        return {
            "sm_mhz": statistics.median(sm) if sm else None,
            "sm_max_mhz": max(smax) if smax else None,
            "reasons": sorted(reasons),
            "samples": len(sm),
        }


def pcg_bytes_per_iter(C: int, F: int, s: int = 8) -> float:
    """Algorithmic bytes of one fused Jacobi-PCG iteration (int32 indices):
    14 C s + F (s + 8)."""
    return 14 * C * s + F * (s + 8)


def pcg_bytes_setup(C: int, F: int, s: int = 8) -> float:
    """Initial residual pass: x, b, diag read; r, p written; matrix once."""
    return 5 * C * s + F * (s + 8)


# Measured DRAM bytes (read + write) per cell per iteration of the pressure
# CG on the cylinder-wake octree, by split-CG variant: one k_cgs_a plus one
# k_cgs_b launch in an ncu capture on the 192x120x24 base (1,729,632 cells;
# the working set exceeds L2, so the traffic grows in proportion to the
# cells), against 159.8 B of the byte model.  Variant 25 (q by recurrence):
# 204.6 + 83.5 MB (the recurrence reads q of the own cell); variant 27 (the
# same with x += alpha p in the row kernel): 231.0 + 43.4 MB; variant 29
# (27 with L2 prefetches of each thread's first cell): 229.1 + 42.4 MB.
PCG_DRAM_BYTES_PER_CELL_ITER = {25: 166.6, 27: 158.6, 29: 157.0}


def _oracle_threads() -> int:
    from oracle import native

    return native.num_threads()


def oracle_step_sample(mesh, case_def: dict, steps: int = 1):
    """The CPU oracle (numpy restatement, Krylov solves and repeated
    scatter-adds in multi-threaded C) on ``mesh``: ``steps`` PISO steps from
    the initial state.  Returns (seconds, algorithm)."""
    from oracle import native
    from oracle.algorithms import create_algorithm
    from oracle.case import Case, CellField

    native.enable()
    case = Case(mesh, case_def["simulator"])
    CellField(case, "U", "transient", (3,))
    algo = create_algorithm(case)
    t0 = time.perf_counter()
    for _ in range(steps):
        algo.step()
    return time.perf_counter() - t0, algo


def cpu_baseline(mesh, case_def: dict) -> tuple[dict, object]:
    """One PISO step of the workload itself (full mesh, from the initial
    state) on the host: a bounded sample of about half a minute."""
    el, algo = oracle_step_sample(mesh, case_def, 1)
    its = [s.iterations for s in algo.last_stats["p"]]
    line = {
        "value": mesh.n_cells / el,
        "unit": METRIC,
        "cores": _oracle_threads(),
        "kind": "port",
        "sample": f"oracle (reference algorithm restated; Krylov and scatter-adds in OpenMP C), {WORKLOAD}, "
                  f"the first PISO step from the initial state on the full mesh ({mesh.n_cells} cells) in "
                  f"{el:.1f} s, pFinal CG iterations {its}",
    }
    return line, algo


def run_reference(args) -> None:
    """The reference arm: the reference algorithm (the oracle port) on the
    same mesh and case as the GPU arm, every host core, W untimed and K
    timed PISO steps.  Under torchrun rank 0 alone runs it."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    from oracle import native

    native.build()
    from gridfoam_b200.cases import build_mesh

    case = workload_case()
    mesh = build_mesh(case["mesh"])
    from oracle.algorithms import create_algorithm
    from oracle.case import Case, CellField

    native.enable()
    ocase = Case(mesh, case["simulator"])
    CellField(ocase, "U", "transient", (3,))
    algo = create_algorithm(ocase)
    for _ in range(args.warmup):
        algo.step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        algo.step()
    el = time.perf_counter() - t0
    value = mesh.n_cells * args.steps / el
    cores = _oracle_threads()
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": METRIC,
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1e3 * el / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": workload_config(mesh, world),
        "cpu_baseline": {
            "value": value,
            "unit": METRIC,
            "cores": cores,
            "kind": "port",
            "sample": f"the whole run: {args.warmup} untimed and {args.steps} timed PISO steps of {WORKLOAD} on the "
                      f"full mesh, oracle port (numpy; Krylov and scatter-adds in OpenMP C on {cores} threads)",
        },
        "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def _timed_steps(algo, steps: int, torch) -> float:
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        algo.step()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1)


def _rel(a, b) -> float:
    import numpy as np

    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(np.asarray(b)), 1e-300))


# Drag and lift of the cylinder (diameter 1, span 4, inflow 1): force
# scale 0.5 rho U^2 D span.
FORCE_PATCH, FORCE_SCALE, FORCE_COFR = "cylinder", 0.5 * 1.0 * 1.0 * 4.0, (10.0, 10.0, 2.0)


def gpu_coefficients(grid, algo) -> dict:
    """Cd / Cl of the cylinder from the device force integral."""
    import numpy as np

    from gridfoam_b200.post.forces import patch_force

    r = patch_force(grid, algo.p, algo.U, algo.nu, FORCE_PATCH, 1.0, np.asarray(FORCE_COFR))
    return {"Cd": float(r.force[0] / FORCE_SCALE), "Cl": float(r.force[1] / FORCE_SCALE)}


def oracle_coefficients(oalgo, mesh) -> dict:
    import numpy as np

    from oracle.forces import patch_force

    f, _, _, _ = patch_force(oalgo.p, oalgo.U, oalgo.nu, FORCE_PATCH, 1.0, np.asarray(FORCE_COFR),
                             mesh.ap.anchor_normal)
    return {"Cd": float(f[0] / FORCE_SCALE), "Cl": float(f[1] / FORCE_SCALE)}


def mixed_variant(args, local: int, torch, first_fp64, oracle_first) -> dict:
    """The workload with FP32 inner iterations of the pressure CG inside FP64
    iterative refinement.  Errors: after the first step against the FP64
    oracle (when it ran) and the FP64 GPU path; after warm-up plus the timed
    steps against the FP64 GPU path run over the same steps."""
    from gridfoam_b200.cases import create_case

    case = workload_case()
    for key in ("p", "pFinal"):
        case["simulator"]["fvSolution"]["solvers"][key]["inner_precision"] = "float32"
    _, grid, algo = create_case(case, device=f"cuda:{local}")
    algo.step()
    torch.cuda.synchronize()
    U1, p1 = algo.U.data.cpu().numpy(), algo.p.data.cpu().numpy()
    out = {"rel_l2_U_vs_fp64_gpu_step1": _rel(U1, first_fp64[0]),
           "rel_l2_p_vs_fp64_gpu_step1": _rel(p1, first_fp64[1]),
           "coefficients_step1": gpu_coefficients(grid, algo)}
    if oracle_first is not None:
        out["rel_l2_U_vs_fp64_oracle_step1"] = _rel(U1, oracle_first[0])
        out["rel_l2_p_vs_fp64_oracle_step1"] = _rel(p1, oracle_first[1])
    for _ in range(max(0, args.warmup - 1)):
        algo.step()
    ms = _timed_steps(algo, args.steps, torch)
    its = [s.iterations for s in algo.last_stats["p"]]
    out["coefficients_after_all_steps"] = gpu_coefficients(grid, algo)
    out.update({
        "value": grid.num_cells * args.steps / (ms * 1e-3),
        "unit": METRIC,
        "ms_per_step": ms / args.steps,
        "last_pfinal_iterations": its,
    })
    return out, algo


def serving_bench(args, local: int, dist=None, rank: int = 0, world: int = 1) -> dict:
    """Solve-server stream (cavity SIMPLE solves of uneven sizes arriving as
    a Poisson process, each to residualControl p 1e-6): the lockstep engine
    (same-phase Krylov solves of all resident cases in one batched launch,
    each batched iteration a CUDA graph) in FP64 and with FP32 inner
    pressure-CG iterations, against one-at-a-time FP64 solves through the
    plain API, on the same requests and solver settings (p CG absolute 1e-12,
    relative 0.01).  With several GPUs each rank serves its share of the one
    stream (no collective on the data path) and the summaries are merged."""
    import numpy as np
    import torch

    from gridfoam_b200.serving import (SIZES, BatchedEngine, ServingEngine, poisson_stream, serve_sequential,
                                       summarize)
    from gridfoam_b200.serving.shard import merge_summaries, shard_stream

    stream = poisson_stream(args.serve_requests, rate=50.0, sizes=SIZES, seed=0)
    reqs = shard_stream(stream, world, rank)

    def whole(res):
        if dist is None:
            return summarize(res)
        part = ([r.latency for r in res], min((r.arrival for r in res), default=0.0),
                max((r.finished for r in res), default=0.0))
        parts = [None] * world
        dist.all_gather_object(parts, part)
        return merge_summaries([p[0] for p in parts], [p[1] for p in parts], [p[2] for p in parts])
    common = dict(max_outer=args.serve_end_time, p_tol=1e-6, p_solver_tol=1e-12, p_solver_rtol=0.01,
                  keep_fields=True)
    out = {
        "workload": "cavity SIMPLE stream: sizes uniform over 16^3..96^3, Re log-uniform [10,1000], "
                    "lid U uniform [0.5,2], Poisson arrivals 50/s, residualControl p 1e-6 (normalised), "
                    "p cg+jacobi tol 1e-12 rel 0.01",
        "requests": len(stream),
        "replicas": world,
        "end_time": args.serve_end_time,
        "sample": f"{len(reqs)} of the 1024-request stream",
    }
    runs = {}
    for name, prec in (("batched_fp64", "float64"), ("batched_mixed", "float32")):
        eng = BatchedEngine(device=f"cuda:{local}", max_slots=args.serve_slots, inner_precision=prec, **common)
        t0 = time.perf_counter()
        eng.prepare(SIZES)
        prep = time.perf_counter() - t0
        res = eng.run(reqs)
        runs[name] = {r.id: r for r in res}
        out[name] = {**whole(res), "prepare_s": prep, "slots": args.serve_slots,
                     "batched_launches": eng.launches, "graph_captures": eng.captures}
        del eng
        torch.cuda.empty_cache()
    # Per-case graphs on concurrent streams (no lockstep): each slot's
    # iteration is one graph replay, the slots' kernels overlap on the GPU.
    for name, prec in (("slots_fp64", "float64"), ("slots_mixed", "float32")):
        eng = ServingEngine(device=f"cuda:{local}", max_slots=args.serve_slots, inner_precision=prec, **common)
        t0 = time.perf_counter()
        eng.prepare(SIZES)
        prep = time.perf_counter() - t0
        res = eng.run(reqs)
        runs[name] = {r.id: r for r in res}
        out[name] = {**whole(res), "prepare_s": prep, "slots": args.serve_slots}
        del eng
        torch.cuda.empty_cache()
    seq = serve_sequential(reqs, device=f"cuda:{local}", **common)
    runs["sequential_fp64"] = {r.id: r for r in seq}
    out["sequential_fp64"] = whole(seq)

    def max_err(a: str, b: str) -> float:
        # at equal residual: requests that converged in both runs
        errs = [float(np.linalg.norm(runs[a][i].U - runs[b][i].U) / max(np.linalg.norm(runs[b][i].U), 1e-300))
                for i in runs[a] if runs[a][i].U is not None and i in runs[b] and runs[b][i].U is not None
                and runs[a][i].converged and runs[b][i].converged]
        m = max(errs, default=0.0)
        if dist is not None:
            both = [None] * world
            dist.all_gather_object(both, m)
            m = max(both)
        return m
    # Converged results at equal residual: the FP64 engine against the plain
    # API (other CG kernels) and the FP32-inner engine against both.
    out["batched_fp64"]["max_rel_l2_U_vs_sequential_fp64"] = max_err("batched_fp64", "sequential_fp64")
    out["batched_mixed"]["max_rel_l2_U_vs_batched_fp64"] = max_err("batched_mixed", "batched_fp64")
    out["batched_mixed"]["max_rel_l2_U_vs_sequential_fp64"] = max_err("batched_mixed", "sequential_fp64")
    out["slots_fp64"]["max_rel_l2_U_vs_sequential_fp64"] = max_err("slots_fp64", "sequential_fp64")
    out["slots_mixed"]["max_rel_l2_U_vs_slots_fp64"] = max_err("slots_mixed", "slots_fp64")
    out["slots_mixed"]["max_rel_l2_U_vs_sequential_fp64"] = max_err("slots_mixed", "sequential_fp64")
    for k in ("batched_fp64", "batched_mixed", "slots_fp64", "slots_mixed"):
        out[k]["speedup_solves_per_s_vs_sequential"] = (
            out[k]["solves_per_s"] / out["sequential_fp64"]["solves_per_s"])
    return out


def pipe_variant(args, local: int, torch) -> dict:
    """The immersed Hagen-Poiseuille pipe (64x64x256 cells, PISO dt 1e-3),
    FP64 and FP32-inner (pressure CG and momentum BiCGStab, each in FP64
    refinement): cell-iters/s over the timed steps, the pressure CG
    per iteration (its working set is L2-resident: against the measured
    floor of its two grid reductions, not HBM), and after ``pipe_steps``
    steps the relative L2 error of u_z against the analytic profile
    2 (1 - r^2 / 0.16) over the cells in the last quarter of the pipe."""
    import numpy as np

    from gridfoam_b200.cases import create_case, pipe_analytic_uz, pipe_case

    out = {}
    finals = {}
    for name, prec in (("fp64", "float64"), ("fp32_inner", "float32")):
        case = pipe_case(64, 256, 4.0)
        for key in ("p", "pFinal", "U"):
            if key in case["simulator"]["fvSolution"]["solvers"]:
                case["simulator"]["fvSolution"]["solvers"][key]["inner_precision"] = prec
        mesh, grid, algo = create_case(case, device=f"cuda:{local}")
        psolvers = [s for n, s in algo.solvers.items() if n.startswith("p")]
        for _ in range(args.warmup):
            algo.step()
        events: list = []
        for s in psolvers:
            s.profile_events = events
        ms = _timed_steps(algo, args.steps, torch)
        for s in psolvers:
            s.profile_events = None
        cg_ms = sum(a.elapsed_time(b) for a, b, _ in events)
        cg_its = sum(st[0].iterations for _, _, st in events)
        done = args.warmup + args.steps
        t0 = time.perf_counter()
        for _ in range(max(0, args.pipe_steps - done)):
            algo.step()
        torch.cuda.synchronize()
        run_s = time.perf_counter() - t0
        c = mesh.cell_centers
        uz = algo.U.data[:, 2].cpu().numpy()
        ref = pipe_analytic_uz(mesh, case["inlet_profile"])
        sel = (c[:, 2] > 3.0) & (ref > 0.0)
        finals[name] = algo.U.data.cpu().numpy()
        out[name] = {
            "value": grid.num_cells * args.steps / (ms * 1e-3),
            "unit": METRIC,
            "ms_per_step": ms / args.steps,
            "p_cg_us_per_iteration": 1e3 * cg_ms / max(1, cg_its),
            "steps_run": max(done, args.pipe_steps),
            "wall_s_after_timed": run_s,
            "rel_l2_uz_vs_analytic_last_quarter": float(np.linalg.norm(uz[sel] - ref[sel]) / np.linalg.norm(ref[sel])),
        }
        del algo, grid
        torch.cuda.empty_cache()
    out["workload"] = "ib_pipe_64x64x256_piso (1,048,576 cells)"
    out["p_cg_sync_floor_us"] = 4.7
    out["p_cg_sync_floor_note"] = ("two grid reductions of 1024-thread blocks on 148 SMs measured at 2.07 + 2.66 us "
                                   "(empty loop); the CG working set (~90 MB) is L2-resident at this size")
    out["rel_l2_U_fp32_inner_vs_fp64_gpu_final"] = _rel(finals["fp32_inner"], finals["fp64"])
    return out


def cavity_variant(local: int, torch) -> dict:
    """The lid-driven cavity at 32^3, SIMPLE for 300 iterations (the
    CPU-runnable config): wall time and cell-iters/s on the device."""
    from gridfoam_b200.cases import cavity_case, create_case

    case = cavity_case(32)
    _, grid, algo = create_case(case, device=f"cuda:{local}")
    algo.step()
    ms = _timed_steps(algo, 299, torch)
    return {"workload": "cavity_32^3_simple_300_iterations", "value": grid.num_cells * 299 / (ms * 1e-3),
            "unit": METRIC, "ms_per_iteration": ms / 299,
            "last_p_iterations": [s.iterations for s in algo.last_stats["p"]]}


BLUFF_BASE = (256, 64, 48)


def bluff_adjoint_variant(args, local: int, torch) -> dict:
    """The drag's shape gradient with respect to the body's 8 parameters on
    the bluff body's 4-level octree channel at base 128x32x24 (731,062
    cells; the full base 256x64x48 is the forward variant): the steady state
    converged with exact solves, the fixed-point adjoint, and central
    differences at h = 1e-4 of two parameters as a spot check."""
    import numpy as np

    from gridfoam_b200.cases import bluff_body_case, create_case
    from gridfoam_b200.mesh.builder import BLUFF_DEFAULT, BLUFF_PARAMS, bluff_body_sdf
    from gridfoam_b200.post.forces import patch_force
    from gridfoam_b200.solvers import shape_adjoint as sa

    base = (128, 32, 24)
    theta = np.array(BLUFF_DEFAULT)

    def make(params):
        return create_case(bluff_body_case(base, levels=3, params=params), device=f"cuda:{local}")

    def drag(grid, algo) -> float:
        return float(patch_force(grid, algo.p, algo.U, algo.nu, "body", 1.0, np.zeros(3)).force[0])

    mesh, grid, algo = make(BLUFF_DEFAULT)
    ext = torch.as_tensor(np.nonzero(bluff_body_sdf(0.0, theta)(np.asarray(mesh.cell_centers)) > 0)[0],
                          device=f"cuda:{local}")
    t0 = time.perf_counter()
    its = sa.converge_exact(algo, cells=ext)
    torch.cuda.synchronize()
    primal_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    g = sa.shape_gradient(algo, lambda t: bluff_body_sdf(0.0, t), theta, patch="body", extent=8.0)
    torch.cuda.synchronize()
    adjoint_s = time.perf_counter() - t0
    state = (algo.U.data.detach().clone(), algo.p.data.detach().clone(), algo.phi.store[0].detach().clone())
    imm0, near0 = np.asarray(grid.host.imm_faces), np.asarray(grid.host.bnd_near)
    spot = {}
    # (on this mesh a 1e-4 change of the side-view rounding or the clearance
    # moves some segment crossing past a cell centre -- another discrete
    # structure; width and the plan-view rounding do not)
    for j in (1, 3):
        J, same = [], True
        for sign in (1.0, -1.0):
            th = theta.copy()
            th[j] += sign * 1e-4
            _, gj, aj = make(th)
            same &= gj.num_cells == grid.num_cells and np.array_equal(np.asarray(gj.host.imm_faces), imm0) \
                and np.array_equal(np.asarray(gj.host.bnd_near), near0)
            if not same:
                break
            with torch.no_grad():
                aj.U.store.copy_(state[0].t())
                aj.p.store.copy_(state[1].reshape(1, -1))
                aj.phi.store[0].copy_(state[2])
            sa.converge_exact(aj, cells=ext)
            J.append(drag(gj, aj))
            del aj, gj
        if not same:
            spot[BLUFF_PARAMS[j]] = {"adjoint": float(g.grad[j]), "discrete_structure_unchanged": False}
            continue
        fd = (J[0] - J[1]) / 2e-4
        spot[BLUFF_PARAMS[j]] = {"fd_h1e-4": fd, "adjoint": float(g.grad[j]),
                                 "rel": abs(fd - g.grad[j]) / abs(fd), "discrete_structure_unchanged": True}
    area = 0.39 * 0.29
    out = {
        "workload": "bluff_body_128x32x24_l3_simple_shape_gradient",
        "cells": grid.num_cells,
        "hanging_faces": grid.num_hanging,
        "immersed_faces": grid.num_immersed_faces,
        "drag": g.objective,
        "Cd": g.objective / (0.5 * area),
        "grad_drag": dict(zip(BLUFF_PARAMS, (float(v) for v in g.grad))),
        "primal_iterations_configured_then_exact": list(its),
        "primal_s": primal_s,
        "adjoint_sweeps": g.adjoint_sweeps,
        "adjoint_s": adjoint_s,
        "spot_check": spot,
    }
    del algo, grid
    torch.cuda.empty_cache()
    return out


def bluff_variant(args, local: int, torch) -> dict:
    """The slanted bluff body (length 1, width 0.39, height 0.29, front
    rounding 0.1, rear slant 25 deg over 0.222) in a channel on a 4-level
    octree (base 256x64x48, levels 0-3), inflow 1, nu 0.0024 (Re 418), steady SIMPLE
    (SIMPLEC): cell-iters/s of the SIMPLE iterations after warm-up, the
    mesh set-up time and the drag coefficient on the body."""
    import numpy as np

    from gridfoam_b200.cases import bluff_body_case, create_case
    from gridfoam_b200.post.forces import patch_force

    case = bluff_body_case(BLUFF_BASE)
    t0 = time.perf_counter()
    mesh, grid, algo = create_case(case, device=f"cuda:{local}")
    torch.cuda.synchronize()
    setup = time.perf_counter() - t0
    for _ in range(args.warmup):
        algo.step()
    ms = _timed_steps(algo, args.steps, torch)
    r = patch_force(grid, algo.p, algo.U, algo.nu, "body", 1.0, np.zeros(3))
    area = 0.39 * 0.29
    out = {
        "workload": f"bluff_body_{BLUFF_BASE[0]}x{BLUFF_BASE[1]}x{BLUFF_BASE[2]}_l3_simple",
        "cells": grid.num_cells,
        "internal_faces": grid.num_internal_faces,
        "hanging_faces": grid.num_hanging,
        "immersed_faces": grid.num_immersed_faces,
        "setup_s": setup,
        "value": grid.num_cells * args.steps / (ms * 1e-3),
        "unit": METRIC,
        "ms_per_iteration": ms / args.steps,
        "last_p_iterations": [s.iterations for s in algo.last_stats["p"]],
        "Cd_after_all_iterations": float(r.force[0] / (0.5 * area)),
        "note": "forward; the drag's shape gradient: bluff_body_shape_gradient (same channel, base 128x32x24)",
    }
    del algo, grid
    torch.cuda.empty_cache()
    return out


def run_gpu(args) -> None:
    import numpy as np
    import torch

    import gridfoam_b200._lib as gl
    from gridfoam_b200.cases import create_case
    from gridfoam_b200.solvers.krylov import default_variant

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    case = workload_case()
    t0 = time.perf_counter()
    mesh, grid, algo = create_case(case, device=f"cuda:{local}")
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t0
    C, F = grid.num_cells, grid.num_internal_faces
    algo.step()
    torch.cuda.synchronize()
    first = (algo.U.data.cpu().numpy(), algo.p.data.cpu().numpy())
    coeff_first = gpu_coefficients(grid, algo)
    for _ in range(max(0, args.warmup - 1)):
        algo.step()
    torch.cuda.synchronize()

    # Per-launch events around every pressure solve (the dominant kernel).
    psolvers = [s for name, s in algo.solvers.items() if name.startswith("p")]
    events: list = []
    for s in psolvers:
        s.profile_events = events

    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.4)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    gl.clear_launches()
    gl.TRACK_DEFERRED = True
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.nvtx.range_push("timed_steps")  # for profilers' range filters
    start.record()
    for _ in range(args.steps):
        algo.step()
    stop.record()
    torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    launches = gl.launch_total()
    gl.TRACK_DEFERRED = False
    gl.clear_launches()
    ms = start.elapsed_time(stop)
    for s in psolvers:
        s.profile_events = None
    clocks = sampler.stop()
    if dist is not None:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    final = (algo.U.data.cpu().numpy(), algo.p.data.cpu().numpy())
    coeff_final = gpu_coefficients(grid, algo)

    # Roofline of the pressure CG launches (HBM-bound at this size).
    durations, iters = [], []
    for ev0, ev1, st in events:
        durations.append(ev0.elapsed_time(ev1) * 1e-3)
        iters.append(st[0].iterations)
    total_bytes = sum(pcg_bytes_setup(C, F) + it * pcg_bytes_per_iter(C, F) for it in iters)
    total_time = sum(durations)
    peak, peak_kind = peaks()
    achieved = total_bytes / total_time / 1e9 if total_time > 0 else 0.0
    variant = default_variant(C, False, True, False)
    step_bytes = total_bytes / args.steps

    # End-to-end through the public API on the same trajectory: a second
    # case from the same initial state, the same warm-up, then the same
    # steps, each taking U and p in from pinned host memory and reading them
    # back into the same buffers (stream-ordered).
    _, _, algo2 = create_case(workload_case(), device=f"cuda:{local}")
    for _ in range(args.warmup):
        algo2.step()
    U_h = algo2.U.data.detach().cpu().pin_memory()
    p_h = algo2.p.data.detach().cpu().pin_memory()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        algo2.U.data = U_h.to(algo2.U.store.device, non_blocking=True)
        algo2.p.data = p_h.to(algo2.p.store.device, non_blocking=True)
        algo2.step()
        U_h.copy_(algo2.U.data, non_blocking=True)
        p_h.copy_(algo2.p.data, non_blocking=True)
    e1.record()
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1) / args.steps
    h2d = U_h.numel() * 8 + p_h.numel() * 8
    del algo2
    torch.cuda.empty_cache()

    per_launch_traffic = None
    if variant in PCG_DRAM_BYTES_PER_CELL_ITER and iters:
        per_launch_traffic = PCG_DRAM_BYTES_PER_CELL_ITER[variant] * C * sum(iters) / len(iters)
    value = C * world * args.steps / (ms * 1e-3)
    line = {
        "metric": METRIC,
        "value": value,
        "unit": METRIC,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": workload_config(mesh, world),
        "workload_detail": {
            "hanging_faces": grid.num_hanging,
            "ell_width": grid.ell_width,
            "setup_s": setup_s,
            "p_iterations_per_solve": (sum(iters) / len(iters)) if iters else None,
            "p_solve_share_of_step": total_time * 1e3 / ms if ms > 0 else None,
            "cylinder_coefficients_after_warmup_and_timed_steps": coeff_final,
            "algorithmic_bytes_per_step_pcg": step_bytes,
            "algorithmic_GBps_per_step_pcg": step_bytes / (ms / args.steps * 1e-3) / 1e9,
        },
        "roofline": {
            "kernel": (f"pressure CG, variant {variant}: " + (
                "split Jacobi-PCG (k_cgs_a: " + ("x += alpha p, " if variant in (27, 28, 29, 30, 31) else "") +
                ("p update + q = A z + beta q + p.q partials; " if variant in (25, 26, 27, 29, 30, 31)
                 else "p update + SpMV + p.q partials; ") +
                ("k_cgs_b: r/z update + partials" if variant in (27, 28, 29, 30, 31) else "k_cgs_b: x/r/z update + partials") +
                ("; first cell prefetched into L2" if variant in (29, 31) else "") +
                "), octree ELL rows, fp64" if 19 <= variant <= 31 else
                "persistent Jacobi-PCG on the octree ELL rows, fp64")),
            "bound": "hbm",
            "achieved": achieved,
            "peak": peak,
            "peak_source": peak_kind,
            "unit": "GB/s",
            "frac": achieved / peak if peak else None,
            "traffic": per_launch_traffic,
            "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum per cell-iteration of fixed-length "
                              "launches on the 192x120x24-base wake (1.73M cells, above L2), scaled to this "
                              "launch's cells and mean iterations",
            "bytes_model": "per iteration 14 C s + F (s + 8), s = 8, plus one initial pass 5 C s + F (s + 8)",
            "launches": len(durations),
            "avg_launch_ms": 1e3 * total_time / max(1, len(durations)),
        },
        "clocks": clocks,
        "gpu_launches": launches,
        "e2e": {
            "value": C * world / (e2e_ms * 1e-3),
            "unit": METRIC,
            "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": h2d,
        },
    }
    del algo
    torch.cuda.empty_cache()
    oracle_first = None
    if rank == 0 and not args.no_cpu_baseline and world == 1:
        cpu, oalgo = cpu_baseline(mesh, case)
        line["cpu_baseline"] = cpu
        oracle_first = (oalgo.U.data, oalgo.p.data)
        line["parity_first_step_vs_fp64_oracle"] = {
            "rel_l2_U": _rel(first[0], oracle_first[0]),
            "rel_l2_p": _rel(first[1], oracle_first[1]),
            "coefficients_gpu": coeff_first,
            "coefficients_oracle": oracle_coefficients(oalgo, mesh),
            "note": "full mesh, first PISO step from the initial state; p solves stop at rel_tolerance 0.01 "
                    "(p) and 1e-7 absolute (pFinal), so two correct implementations differ inside that band",
        }
        del oalgo
    if not args.no_variants:
        mixed, malgo = mixed_variant(args, local, torch, first, oracle_first)
        mixed["rel_l2_U_vs_fp64_gpu_after_all_steps"] = _rel(malgo.U.data.cpu().numpy(), final[0])
        mixed["rel_l2_p_vs_fp64_gpu_after_all_steps"] = _rel(malgo.p.data.cpu().numpy(), final[1])
        del malgo
        torch.cuda.empty_cache()
        line["variants"] = {"mixed_fp32_inner": mixed,
                            "ib_pipe_64x64x256": pipe_variant(args, local, torch),
                            "cavity_32": cavity_variant(local, torch),
                            "bluff_body": bluff_variant(args, local, torch),
                            "bluff_body_shape_gradient": bluff_adjoint_variant(args, local, torch)}
    if not args.no_serving:
        line["serving"] = serving_bench(args, local, dist, rank, world)
    if rank == 0:
        print(json.dumps(line))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="gridfoam_b200")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-variants", action="store_true")
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--pipe-steps", type=int, default=2000,
                    help="PISO steps of the pipe variant before its error against the analytic profile")
    ap.add_argument("--serve-requests", type=int, default=48)
    ap.add_argument("--serve-end-time", type=int, default=1500)
    ap.add_argument("--serve-slots", type=int, default=12)
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
