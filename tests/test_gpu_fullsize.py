"""GPU parity at the benchmark configs' full sizes, with the default kernel
selection (no forced CG launch shape), against the reference's own float64
CPU run of the same mesh and case (``make_golden.py --fullsize``).

* cavity 32^3, 300 SIMPLE iterations (the CPU-runnable config in full);
* immersed pipe 64x64x256, the first 20 PISO steps;
* cylinder wake on the 3-level octree (base 256x160x32, 4.08M cells), the
  first 10 PISO steps;
* the slanted bluff body on its 4-level octree, downscaled to base
  64x16x12 (96,344 cells, hanging and immersed faces), the first 20 steady
  SIMPLE(C) iterations (``make_golden.py --downscaled``).

The fixtures hold per-step Krylov iteration counts and field norms, a fixed
sample of cells at some steps and (cavity) the final fields in full.  The
pressure solves of the pipe and the wake stop at ``rel_tolerance`` 0.01
(pFinal: 1e-7 absolute), so two correct implementations that round
differently stop at different iterates inside that band: fields are
compared at 1e-4 relative there and iteration counts within a few.

The FP32-inner pressure CG (FP64 refinement) takes a different Krylov path
that stops elsewhere inside the same stopping band, so after a fixed number
of SIMPLE iterations its fields differ from the FP64 run by the width of
that band (about 3e-4 in U on the cavity at 300 iterations); its 1e-5
velocity target is checked at equal residual, both runs converged to
residualControl (tests/test_serving.py).
"""

from __future__ import annotations

import pathlib

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

GOLDEN = pathlib.Path(__file__).resolve().parent / "golden"


def rel(a, b) -> float:
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(np.asarray(b)), 1e-300))


def _fixture(key: str, prefix: str = "fullsize") -> dict:
    path = GOLDEN / f"{prefix}_{key}.npz"
    if not path.exists():
        pytest.skip(f"fixture {path.name} not generated")
    with np.load(path) as d:
        return {k: d[k] for k in d.files}


@pytest.fixture(autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")


def _run(case: dict, ref: dict, n_steps: int, *, field_tol: float, its_slack: int, inner: str = "float64"):
    from gridfoam_b200.cases import create_case

    for key in ("p", "pFinal"):
        if key in case["simulator"]["fvSolution"]["solvers"]:
            case["simulator"]["fvSolution"]["solvers"][key]["inner_precision"] = inner
    mesh, grid, algo = create_case(case, device="cuda")
    assert grid.num_cells == int(ref["mesh_n_cells"])
    sample = torch.as_tensor(ref["sample_cells"], device="cuda")
    worst = {"its_p": 0, "U": 0.0, "p": 0.0, "norms": 0.0}
    for step in range(n_steps):
        algo.step()
        its_p = np.array([s.iterations for s in algo.last_stats["p"]])
        worst["its_p"] = max(worst["its_p"], int(np.abs(its_p - ref["its_p"][step]).max()))
        U, p = algo.U.data, algo.p.data
        norms = np.array([float(torch.linalg.vector_norm(U[:, k])) for k in range(3)]
                         + [float(torch.linalg.vector_norm(p))])
        scale = np.abs(ref["norms"][step]).max()
        worst["norms"] = max(worst["norms"], float(np.abs(norms - ref["norms"][step]).max() / scale))
        if f"step{step}_U_sample" in ref:
            worst["U"] = max(worst["U"], rel(U[sample].cpu().numpy(), ref[f"step{step}_U_sample"]))
            worst["p"] = max(worst["p"], rel(p[sample].cpu().numpy(), ref[f"step{step}_p_sample"]))
    assert worst["its_p"] <= its_slack, worst
    assert worst["U"] < field_tol and worst["norms"] < field_tol, worst
    assert worst["p"] < 10 * field_tol, worst
    return algo, worst


def test_cavity32_300_iterations_match_reference():
    from gridfoam_b200.cases import cavity_case

    ref = _fixture("cavity32_300")
    algo, _ = _run(cavity_case(32), ref, 300, field_tol=1e-7, its_slack=2)
    assert rel(algo.U.data.cpu().numpy(), ref["final_U"]) < 1e-7
    assert rel(algo.p.data.cpu().numpy(), ref["final_p"]) < 1e-6


def test_pipe_64x64x256_first_20_steps_match_reference():
    from gridfoam_b200.cases import pipe_case

    ref = _fixture("pipe64x256_20")
    # rel_tolerance 0.01: the trajectories drift apart inside the stopping
    # band, and the pressure iteration counts of later steps with them.
    _run(pipe_case(64, 256, 4.0), ref, 20, field_tol=1e-4, its_slack=12)


def test_cylinder_wake_full_first_10_steps_match_reference():
    from gridfoam_b200.cases import cylinder_wake_case

    ref = _fixture("wake256x160x32_10")
    _run(cylinder_wake_case((256, 160, 32)), ref, 10, field_tol=1e-4, its_slack=12)


def test_bluff_body_downscaled_first_20_iterations_match_reference():
    from gridfoam_b200.cases import bluff_body_case

    ref = _fixture("bluff64x16x12_20", prefix="downscaled")
    _run(bluff_body_case((64, 16, 12)), ref, 20, field_tol=1e-4, its_slack=12)
