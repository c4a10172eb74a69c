"""Pin the CPU oracle against golden vectors from the reference gridfoam.

The fixtures in ``tests/golden/*.npz`` were produced by running the
reference's own float64 PyTorch code (``tests/golden/make_golden.py``).
These tests check that the numpy restatement in ``oracle/`` reproduces them:
operator outputs to round-off, and whole algorithm steps to round-off on
tightly converged cases.  On the loosely converged pipe case (pressure
``rel_tolerance`` 0.01) two correct implementations that round differently
may stop the Krylov iteration at different iterates inside the stopping
band, so fields are compared at a tolerance derived from that band.
"""

from __future__ import annotations

import numpy as np
import pytest

from tests.golden.cases import STEPS
from tests.golden.oracle_harness import load_golden, oracle_case
from tests.golden.oracle_ops_check import oracle_operator_outputs

CASES = list(STEPS)
# Relative L2 tolerance of whole-step fields against the reference.
STEP_TOL = {"cavity8": 1e-12, "channel": 1e-11, "channel_ffp": 1e-11, "ibplane": 1e-12, "ibplane_io": 1e-12, "pipe10x20": 1e-4,
            "cavity_oct": 1e-11, "duct_oct": 1e-9, "ibcyl_oct": 1e-9}


def rel(a: np.ndarray, b: np.ndarray) -> float:
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("name", CASES)
def test_mesh_matches_fixture(name):
    golden = load_golden(name)
    _, mesh, _, _ = oracle_case(name)
    assert mesh.n_cells == int(golden["mesh_n_cells"])
    checksum = np.array(
        [
            float(mesh.internal_faces_owner.sum()),
            float(mesh.cell_centers.sum()),
            float(mesh.ap.dist_owner_to_bnd.sum()),
            float(mesh.ap.is_immersed_face.sum()),
        ]
    )
    np.testing.assert_allclose(checksum, golden["mesh_checksum"], rtol=1e-13)


@pytest.mark.parametrize("name", CASES)
def test_oracle_steps_match_reference(name):
    golden = load_golden(name)
    _, _, _, algo = oracle_case(name)
    np.testing.assert_allclose(algo.phi.pack(), golden["init_phi"], rtol=0, atol=1e-14)
    tol = STEP_TOL[name]
    for step in range(STEPS[name]):
        algo.step()
        assert rel(algo.U.data, golden[f"step{step}_U"]) < tol
        # p carries the Krylov stopping band (absolute tolerance 1e-9 on the
        # octree cases) more directly than U.
        ptol = 10 * tol if name.startswith("pipe") or name.endswith("_oct") else tol
        assert rel(algo.p.data, golden[f"step{step}_p"]) < ptol
        assert rel(algo.phi.pack(), golden[f"step{step}_phi"]) < tol
        its_u = [s.iterations for s in algo.last_stats["U"]]
        its_p = [s.iterations for s in algo.last_stats["p"]]
        slack = 1 if name.startswith("pipe") else 0
        assert np.all(np.abs(np.array(its_u) - golden[f"step{step}_stats_U"][:, 2]) <= slack)
        assert np.all(np.abs(np.array(its_p) - golden[f"step{step}_stats_p"][:, 2]) <= slack)


@pytest.mark.parametrize("name", CASES)
def test_oracle_operators_match_reference(name):
    out, golden = oracle_operator_outputs(name)
    flux_scale = np.abs(golden[f"step{STEPS[name]-1}_phi"]).max()
    for key, val in out.items():
        ref = golden[key]
        assert val.shape == ref.shape, key
        if key.endswith("_stats"):
            np.testing.assert_array_equal(val[:, 2], ref[:, 2], err_msg=key)
            continue
        if key == "op_div_phi":
            # Face-sum of a nearly divergence-free flux: compare against the
            # flux scale per unit volume, not the (cancelled) result.
            volume = 1.0 / np.abs(ref).size
            scale = max(np.abs(ref).max(), flux_scale / volume * 1e-3)
            assert np.abs(val - ref).max() <= 1e-10 * scale, key
            continue
        scale = max(np.abs(ref).max(), 1e-300)
        assert np.abs(val - ref).max() <= 1e-11 * scale, key


NATIVE_STEP_TOL = {"cavity8": 1e-10, "channel": 1e-9, "channel_ffp": 1e-9, "ibplane": 1e-10, "ibplane_io": 1e-10, "pipe10x20": 1e-4,
                   "cavity_oct": 1e-9, "duct_oct": 1e-8, "ibcyl_oct": 1e-8}


@pytest.fixture
def native_krylov():
    from oracle import native

    native.enable()
    yield
    native.disable()


@pytest.mark.parametrize("name", CASES)
def test_oracle_native_krylov_steps_match_reference(name, native_krylov):
    """The multi-threaded C Krylov restatement (``oracle/krylov.c``, used by
    the CPU baseline of large cases) gives the same whole steps."""
    golden = load_golden(name)
    _, _, _, algo = oracle_case(name)
    # Its sums run in another order, as on the GPU: the tolerances of the
    # GPU whole-step tests apply.
    tol = NATIVE_STEP_TOL[name]
    for step in range(STEPS[name]):
        algo.step()
        assert rel(algo.U.data, golden[f"step{step}_U"]) < tol
        assert rel(algo.p.data, golden[f"step{step}_p"]) < 10 * tol
        assert rel(algo.phi.pack(), golden[f"step{step}_phi"]) < tol
        slack = 1 if name.startswith("pipe") or name.endswith("_oct") else 0
        its_u = [s.iterations for s in algo.last_stats["U"]]
        its_p = [s.iterations for s in algo.last_stats["p"]]
        assert np.all(np.abs(np.array(its_u) - golden[f"step{step}_stats_U"][:, 2]) <= slack)
        assert np.all(np.abs(np.array(its_p) - golden[f"step{step}_stats_p"][:, 2]) <= slack)


@pytest.mark.parametrize("name", ["cavity8", "channel", "duct_oct", "ibcyl_oct"])
def test_oracle_grad_linear_steps_match_reference(name):
    """The oracle with the Green-Gauss ('linear') gradient scheme against
    the reference's run of the same cases."""
    from oracle.ops import eval_grad
    from tests.golden.cases import grad_linear_case

    golden = load_golden(f"gradlinear_{name}")
    _, _, _, algo = oracle_case(name, case_def=grad_linear_case(name))
    tol = NATIVE_STEP_TOL[name]
    for step in range(STEPS[name]):
        algo.step()
        assert rel(algo.U.data, golden[f"step{step}_U"]) < tol
        ptol = 10 * tol if name.endswith("_oct") else tol
        assert rel(algo.p.data, golden[f"step{step}_p"]) < ptol
        assert rel(algo.phi.pack(), golden[f"step{step}_phi"]) < tol
    gp = eval_grad(algo.p)
    scale = np.abs(golden["op_grad_p"]).max()
    # op_grad_* were taken on the reference's final state; the oracle's final
    # state agrees to the step tolerance above.
    assert np.abs(gp - golden["op_grad_p"]).max() <= max(1e-10, 100 * tol) * scale
