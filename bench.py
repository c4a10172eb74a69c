"""Benchmark: cell-iterations/s of the immersed-boundary Hagen-Poiseuille
pipe (box 1x1x4 on 64x64x256 cells, cylindrical IB r = 0.4 along z,
parabolic inlet with mean velocity 1, nu = 0.02, PISO dt = 1e-3, two
correctors, upwind convection), float64 on one B200.

One step is one PISO time step (momentum BiCGStab + 2 pressure CG solves to
tolerance).  ``value`` is device-timed with inputs resident in HBM; ``e2e``
times the public API with the step's state copied host->device from pinned
memory and the result read back every step.  ``--impl reference`` times the
CPU oracle (the reference algorithm restated in numpy) on a bounded sample.

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
WORKLOAD = "ib_pipe_64x64x256_piso"


def pipe_config(n: int = 64, nz: int = 256, length: float = 4.0) -> dict:
    from tests.golden.cases import pipe_case

    return pipe_case(n, nz, length)


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


def pcg_bytes_per_iter(C: int, F: int) -> float:
    """Algorithmic bytes of one fused Jacobi-PCG iteration (fp64, int32 indices):
    14 C s + F (s + 8), s = 8."""
    return 14 * C * 8 + F * (8 + 8)


# Measured DRAM bytes (read + write) of the pressure CG kernel
# (k_pcg1_qrec_box<1, 1024, 1>) on a 64x64x256 box, from two ncu captures of
# fixed-length launches: 51.91 MB at 50 iterations, 51.88 MB at 400.  The
# global working set, x included, stays in the 126 MB L2, so a launch costs
# a one-time read of its arrays and no DRAM traffic per iteration.
PCG_DRAM_BYTES_PER_ITER = 0.0
PCG_DRAM_BYTES_PER_LAUNCH = (51905280 + 51882240) / 2


def pcg_bytes_setup(C: int, F: int) -> float:
    """Initial residual pass: x, b, diag read; r, p written; matrix once."""
    return 5 * C * 8 + F * (8 + 8)


def cpu_baseline(seconds: float = 15.0) -> dict:
    """The CPU oracle on a bounded sample: a 16x16x64 downscale of the pipe."""
    import numpy as np  # noqa: F401

    from tests.golden.oracle_harness import oracle_case

    case = pipe_config(16, 64, 4.0)
    _, mesh, _, algo = oracle_case("pipe_cpu", case_def=case)
    algo.step()
    steps, t0 = 0, time.perf_counter()
    while True:
        algo.step()
        steps += 1
        el = time.perf_counter() - t0
        if el > seconds or steps >= 200:
            break
    return {
        "value": mesh.n_cells * steps / el,
        "unit": METRIC,
        "cores": 1,
        "kind": "port",
        "sample": f"numpy oracle, pipe 16x16x64 ({mesh.n_cells} cells) PISO, {steps} steps in {el:.1f} s",
    }


def _reference_worker(steps: int, warmup: int) -> tuple[int, float]:
    """One CPU replica of the reference arm: the oracle pipe downscale,
    ``warmup`` untimed and ``steps`` timed PISO steps; returns (cells, s)."""
    from tests.golden.oracle_harness import oracle_case

    case = pipe_config(32, 128, 4.0)
    _, mesh, _, algo = oracle_case("pipe_ref", case_def=case)
    for _ in range(warmup):
        algo.step()
    t0 = time.perf_counter()
    for _ in range(steps):
        algo.step()
    return int(mesh.n_cells), time.perf_counter() - t0


def run_reference(args) -> None:
    """The reference arm: the reference algorithm (the numpy oracle port)
    on every host core at once, one independent replica per core (numpy's
    scatter-heavy steps are single-threaded), spawned processes."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import multiprocessing as mp

    cores = max(1, min(os.cpu_count() or 1, 64))
    for var in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
        os.environ.setdefault(var, "1")
    with mp.get_context("spawn").Pool(cores) as pool:
        res = pool.starmap(_reference_worker, [(args.steps, args.warmup)] * cores)
    cells = res[0][0]
    el = max(r[1] for r in res)
    value = cells * args.steps * cores / el
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
        "config": {"workload": WORKLOAD, "sample": f"pipe 32x32x128 per step, {cores} replicas (bounded sample)"},
        "cpu_baseline": {
            "value": value,
            "unit": METRIC,
            "cores": cores,
            "kind": "port",
            "sample": f"numpy oracle (reference algorithm restated), pipe 32x32x128 ({cells} cells) PISO, "
                      f"{args.steps} steps on each of {cores} cores; slowest replica's time",
        },
        "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def mixed_variant(args, local: int, ref_algo, torch) -> dict:
    """Same workload with the pressure CG in FP32 inside FP64 refinement.

    Both runs start from the same initial state and take the same number of
    steps; the reported errors are relative L2 norms against the FP64 run.
    """
    from tests.golden.device_harness import device_case

    case = pipe_config()
    for key in ("p", "pFinal"):
        case["simulator"]["fvSolution"]["solvers"][key]["inner_precision"] = "float32"
    _, _, grid, algo = device_case(case_def=case, device=f"cuda:{local}")
    _, _, _, ref = device_case(case_def=pipe_config(), device=f"cuda:{local}")
    n_steps = args.warmup + args.steps
    for _ in range(args.warmup):
        algo.step()
        ref.step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        algo.step()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    for _ in range(args.steps):
        ref.step()
    torch.cuda.synchronize()
    du = torch.linalg.vector_norm(algo.U.data - ref.U.data) / torch.linalg.vector_norm(ref.U.data)
    dp = torch.linalg.vector_norm(algo.p.data - ref.p.data) / torch.linalg.vector_norm(ref.p.data)
    its = [s.iterations for s in algo.last_stats["p"]]
    return {
        "value": grid.num_cells * args.steps / (ms * 1e-3),
        "unit": METRIC,
        "ms_per_step": ms / args.steps,
        "steps_compared": n_steps,
        "rel_l2_U_vs_fp64": float(du),
        "rel_l2_p_vs_fp64": float(dp),
        "last_p_iterations": its,
    }


def octree_variant(args, local: int, torch) -> dict:
    """Cylinder wake on a 3-level octree (hanging faces, general ELL path):
    the cylinder-wake config at a 96x64x12 base, refined 2 levels within 2D
    of the cylinder."""
    from tests.golden.cases import cylinder_wake_case
    from tests.golden.device_harness import device_case

    case = cylinder_wake_case()
    t0 = time.perf_counter()
    _, _, grid, algo = device_case(case_def=case, device=f"cuda:{local}")
    setup = time.perf_counter() - t0
    for _ in range(args.warmup):
        algo.step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    its = []
    e0.record()
    for _ in range(args.steps):
        algo.step()
        its.append(algo.last_stats["p"])
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    return {
        "workload": case["name"] + "_piso",
        "value": grid.num_cells * args.steps / (ms * 1e-3),
        "unit": METRIC,
        "ms_per_step": ms / args.steps,
        "cells": grid.num_cells,
        "internal_faces": grid.num_internal_faces,
        "hanging_faces": grid.num_hanging,
        "immersed_faces": grid.num_immersed_faces,
        "ell_width": grid.ell_width,
        "p_iterations_last_step": [s.iterations for s in its[-1]] if its else None,
        "setup_s": setup,
    }


def serving_bench(args, local: int, dist=None, rank: int = 0, world: int = 1) -> dict:
    """Solve-server stream (cavity SIMPLE solves of uneven sizes arriving as
    a Poisson process): the continuous-batching engine (FP64, and FP32-inner
    pressure CG) against one-at-a-time FP64 solves through the plain API,
    on the same requests.  With several GPUs each rank serves its share of
    the one stream (no collective on the data path) and the summaries are
    merged: solves/s over the whole job, percentiles over every request."""
    import numpy as np
    import torch

    from gridfoam_b200.serving import SIZES, ServingEngine, poisson_stream, serve_sequential, summarize
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
    common = dict(max_outer=args.serve_end_time, p_tol=1e-6, p_solver_tol=1e-6, keep_fields=True)
    out = {
        "workload": "cavity SIMPLE stream: sizes uniform over 16^3..96^3, Re log-uniform [10,1000], "
                    "lid U uniform [0.5,2], Poisson arrivals 50/s, p cg tol 1e-6, residualControl p 1e-6",
        "requests": len(stream),
        "replicas": world,
        "end_time": args.serve_end_time,
        "sample": f"{len(reqs)} of the 1024-request stream, endTime capped at {args.serve_end_time} iterations",
    }
    runs = {}
    for name, kw in (("engine_fp64", {}), ("engine_mixed", {"inner_precision": "float32"})):
        eng = ServingEngine(device=f"cuda:{local}", max_slots=args.serve_slots, gpu_share=args.serve_share,
                            **common, **kw)
        t0 = time.perf_counter()
        eng.prepare(SIZES)
        prep = time.perf_counter() - t0
        res = eng.run(reqs)
        runs[name] = {r.id: r for r in res}
        if name == "engine_fp64":
            fp_variants = dict(eng.variants)
        out[name] = {**whole(res), "prepare_s": prep, "slots": args.serve_slots, "gpu_share": args.serve_share,
                     "autotuned_variants": {str(k): v for k, v in eng.variants.items()}}
        del eng
        torch.cuda.empty_cache()
    seq = serve_sequential(reqs, device=f"cuda:{local}", variants=fp_variants, **common)
    runs["sequential_fp64"] = {r.id: r for r in seq}
    out["sequential_fp64"] = whole(seq)
    fp = runs["engine_fp64"]
    seq_d = [float(np.linalg.norm(fp[i].U - runs["sequential_fp64"][i].U) /
                   max(np.linalg.norm(runs["sequential_fp64"][i].U), 1e-300)) for i in fp]
    errs = []
    for i, r in runs["engine_mixed"].items():
        ref = fp[i].U
        errs.append(float(np.linalg.norm(r.U - ref) / max(np.linalg.norm(ref), 1e-300)))
    # Same algorithm and iterations; the engine's block caps change only the
    # order of the dot-product partial sums.
    if dist is not None:
        both = [None] * world
        dist.all_gather_object(both, (max(seq_d, default=0.0), max(errs, default=0.0)))
        seq_d, errs = [b[0] for b in both], [b[1] for b in both]
    out["engine_fp64"]["max_rel_l2_U_vs_sequential"] = max(seq_d) if seq_d else None
    out["engine_mixed"]["max_rel_l2_U_vs_fp64"] = max(errs) if errs else None
    for k in ("engine_fp64", "engine_mixed"):
        out[k]["speedup_solves_per_s_vs_sequential"] = (
            out[k]["solves_per_s"] / out["sequential_fp64"]["solves_per_s"])
    return out


def run_gpu(args) -> None:
    import torch

    import gridfoam_b200._lib as gl
    from tests.golden.device_harness import device_case

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    case = pipe_config()
    _, mesh, grid, algo = device_case(case_def=case, device=f"cuda:{local}")
    C, F = grid.num_cells, grid.num_internal_faces
    for _ in range(args.warmup):
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
    gl.LAUNCHES.clear()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    stats = []
    start.record()
    for _ in range(args.steps):
        algo.step()
        stats.append(algo.last_stats)
    stop.record()
    torch.cuda.synchronize()
    launches = sum(gl.LAUNCHES.values())
    ms = start.elapsed_time(stop)
    for s in psolvers:
        s.profile_events = None
    clocks = sampler.stop()
    if dist is not None:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())

    # Roofline of the pressure PCG launches.
    durations, iters = [], []
    for ev0, ev1, st in events:
        durations.append(ev0.elapsed_time(ev1) * 1e-3)
        iters.append(st[0].iterations)
    total_bytes = sum(pcg_bytes_setup(C, F) + it * pcg_bytes_per_iter(C, F) for it in iters)
    total_time = sum(durations)
    peak, peak_kind = peaks()
    achieved = total_bytes / total_time / 1e9 if total_time > 0 else 0.0

    # End-to-end through the public API on the same trajectory as the timed
    # region: a second case from the same initial state, the same warm-up,
    # then the same steps, each taking U and p in from pinned host memory
    # and reading them back into the same buffers (stream-ordered, so the
    # next step's upload sees this step's result).
    _, _, _, algo = device_case(case_def=pipe_config(), device=f"cuda:{local}")
    for _ in range(args.warmup):
        algo.step()
    U_h = algo.U.data.detach().cpu().pin_memory()
    p_h = algo.p.data.detach().cpu().pin_memory()
    e2e_steps = args.steps
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(e2e_steps):
        algo.U.data = U_h.to(algo.U.store.device, non_blocking=True)
        algo.p.data = p_h.to(algo.p.store.device, non_blocking=True)
        algo.step()
        U_h.copy_(algo.U.data, non_blocking=True)
        p_h.copy_(algo.p.data, non_blocking=True)
    e1.record()
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1) / e2e_steps
    h2d = U_h.numel() * 8 + p_h.numel() * 8

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
        "config": {
            "workload": WORKLOAD,
            "cells": C,
            "internal_faces": F,
            "immersed_faces": grid.num_immersed_faces,
            "algorithm": "piso nCorrectors=2, dt=1e-3, upwind, p cg+jacobi tol 1e-7 rel 0.01 (pFinal rel 0), "
                         "U bicgstab+jacobi tol 1e-8 rel 0.1",
            "l2": "working set larger than L2 (126 MB), no flush",
            "parallelism": f"replicas x{world}",
            "p_iterations_per_solve": (sum(iters) / len(iters)) if iters else None,
        },
        "roofline": {
            "kernel": "k_pcg1_qrec_box (persistent Jacobi-PCG, fp64, q by recurrence)",
            "bound": "hbm",
            "achieved": achieved,
            "peak": peak,
            "peak_source": peak_kind,
            "unit": "GB/s",
            "frac": achieved / peak if peak else None,
            "traffic": (PCG_DRAM_BYTES_PER_LAUNCH + PCG_DRAM_BYTES_PER_ITER * sum(iters) / len(iters))
                       if iters else None,
            "traffic_source": "ncu dram bytes of 50- and 400-iteration launches of the same kernel on the same box "
                              "(equal within 0.05 %: a fixed part per launch, nothing per iteration)",
            "note": "working set mostly L2-resident at 1M cells: DRAM traffic is well below the algorithmic "
                    "bytes; the kernel is bound by L2 latency and two grid barriers per iteration",
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
    if not args.no_variants:
        line["variants"] = {"mixed_fp32_inner": mixed_variant(args, local, algo, torch),
                            "octree_cylinder_wake": octree_variant(args, local, torch)}
    if not args.no_serving:
        line["serving"] = serving_bench(args, local, dist, rank, world)
    if rank == 0 and not args.no_cpu_baseline and world == 1:
        line["cpu_baseline"] = cpu_baseline(args.cpu_seconds)
    if rank == 0:
        print(json.dumps(line))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="gridfoam_b200")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-variants", action="store_true")
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--serve-requests", type=int, default=64)
    ap.add_argument("--serve-end-time", type=int, default=100)
    ap.add_argument("--serve-slots", type=int, default=8)
    ap.add_argument("--serve-share", type=float, default=1.0)
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
