"""Adjoint (reverse-mode) checks of the device path.

* The implicit adjoint of the CG / BiCGStab solves against finite
  differences (torch.autograd.gradcheck), as the reference does in
  test_linear_solver_adjoint.py:141-191.
* Gradients through the hand-written reverse kernels of ``fvm.laplacian``
  (diffusivity) and the solves, against the reference's own autograd
  gradient on the same inputs (``tests/golden/adjoint_*.npz``, written by
  ``make_golden.py --adjoint``), on a uniform and an octree mesh.
* The transpose face flux (``fvm.div`` reverse in phi) against central
  finite differences.
"""

from __future__ import annotations

import pathlib

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from tests.golden.device_harness import device_case, to_np  # noqa: E402
from tests.golden.cases import STEPS  # noqa: E402
from tests.golden.oracle_harness import load_golden  # noqa: E402

pytestmark = pytest.mark.gpu

HERE = pathlib.Path(__file__).resolve().parent / "golden"


def rel(a, b) -> float:
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(np.asarray(b)), 1e-300))


@pytest.fixture(autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")


def _state(name):
    if name.endswith("_harmonic"):
        # the base case with harmonic diffusivity interpolation; its state
        # (after the reference's own harmonic steps) is in the fixture
        from tests.golden.cases import ALL_CASES

        case = ALL_CASES[name[: -len("_harmonic")]]()
        case["simulator"]["fvSchemes"]["laplacianSchemes"] = {"default": "Gauss harmonic corrected"}
        _, _, grid, algo = device_case(case_def=case)
        ref = np.load(HERE / f"adjoint_{name}.npz")
        algo.U.data = torch.as_tensor(ref["state_U"], device="cuda")
        algo.p.data = torch.as_tensor(ref["state_p"], device="cuda")
        algo.phi.unpack(torch.as_tensor(ref["state_phi"], device="cuda"))
        return grid, algo
    golden = load_golden(name)
    _, _, grid, algo = device_case(name)
    step = STEPS[name] - 1
    algo.U.data = torch.as_tensor(golden[f"step{step}_U"], device="cuda")
    algo.p.data = torch.as_tensor(golden[f"step{step}_p"], device="cuda")
    algo.phi.unpack(torch.as_tensor(golden[f"step{step}_phi"], device="cuda"))
    return grid, algo


def _solver(kind, tol=1e-13):
    from gridfoam_b200.meta.config import SolverConfig
    from gridfoam_b200.solvers.krylov import BiCGSTABSolver, CGSolver

    cfg = SolverConfig(method=kind, preconditioner="jacobi", tolerance=tol, rel_tolerance=0.0, max_iter=5000)
    return CGSolver(cfg) if kind == "cg" else BiCGSTABSolver(cfg)


@pytest.mark.parametrize(("kind", "symmetric", "seed"), [("cg", True, 0), ("bicgstab", False, 2)])
def test_krylov_adjoint_gradcheck(kind, symmetric, seed):
    from gridfoam_b200.core.equation import equation
    from gridfoam_b200.core.field import CellField
    from gridfoam_b200.core.fvmatrix import FvMatrix

    _, _, grid, _ = device_case("cavity8")
    p = CellField(grid, f"p_{kind}_adj", "local", ())
    A = FvMatrix(p)
    g = torch.Generator(device="cpu").manual_seed(seed)
    F, C = grid.num_internal_faces, grid.num_cells
    upper = (0.1 * torch.rand(F, generator=g, dtype=torch.float64)).cuda()
    lower = upper.clone() if symmetric else (0.05 * torch.rand(F, generator=g, dtype=torch.float64)).cuda()
    off = torch.zeros(C, dtype=torch.float64, device="cuda")
    off.index_add_(0, grid.owner, upper.abs())
    off.index_add_(0, grid.neighbour, lower.abs())
    diag = off + 1.0
    source = torch.randn(C, generator=g, dtype=torch.float64).cuda()
    eq = equation(p, A)
    solver = _solver(kind, 1e-12)

    def solve_fn(d, u, lo, s):
        A.diag, A.upper, A.lower, A.source = d, u, lo, s
        eq.target.data = torch.zeros(C, dtype=torch.float64, device="cuda")
        return solver.solve(eq).solution

    inputs = tuple(t.detach().requires_grad_(True) for t in (diag, upper, lower, source))
    assert torch.autograd.gradcheck(solve_fn, inputs, eps=1e-6, atol=1e-4, rtol=1e-3, fast_mode=True)


@pytest.mark.parametrize("name", ["cavity8", "cavity_oct", "cavity_oct_harmonic", "ibplane"])
def test_gradients_match_reference_autograd(name):
    from gridfoam_b200.core.equation import equation
    from gridfoam_b200.fv import fvm

    ref = np.load(HERE / f"adjoint_{name}.npz")
    grid, algo = _state(name)
    U, p, phi = algo.U, algo.p, algo.phi
    dev = dict(dtype=torch.float64, device="cuda")

    gamma = torch.as_tensor(ref["adj_gamma"], **dev).requires_grad_(True)
    pmat = -fvm.laplacian(gamma, p)
    pmat.source = pmat.source - torch.as_tensor(ref["adj_src"], **dev) * grid.cell_volumes
    if algo.p_needs_ref:
        # reference_value.py:33-51: the reference cell's diagonal doubles
        # (and its gradient with it).
        d = pmat.diag
        pmat.diag = d + torch.nn.functional.one_hot(torch.tensor(0), grid.num_cells).cuda() * d[0]
    p.data = torch.zeros(grid.num_cells, **dev)
    x = _solver("cg").solve(equation(p, pmat)).solution
    (torch.as_tensor(ref["adj_r"], **dev) * x).sum().backward()
    np.testing.assert_allclose(to_np(x), ref["adj_x"], rtol=0, atol=1e-9 * np.abs(ref["adj_x"]).max())
    g_ref = ref["adj_grad_gamma"]
    assert np.abs(to_np(gamma.grad) - g_ref).max() <= 1e-7 * np.abs(g_ref).max()

    nu = torch.as_tensor(ref["adj_nu"], **dev).requires_grad_(True)
    umat = fvm.div(phi, U) - fvm.laplacian(nu, U)
    umat.diag = umat.diag + grid.cell_volumes / 0.01
    umat.source = umat.source + torch.as_tensor(ref["adj_usrc"], **dev) * grid.cell_volumes[:, None]
    U.data = torch.zeros((grid.num_cells, 3), **dev)
    u = _solver("bicgstab").solve(equation(U, umat)).solution
    (torch.as_tensor(ref["adj_r3"], **dev) * u).sum().backward()
    np.testing.assert_allclose(to_np(u), ref["adj_u"], rtol=0, atol=1e-9 * np.abs(ref["adj_u"]).max())
    g_ref = ref["adj_grad_nu"]
    assert np.abs(to_np(nu.grad) - g_ref).max() <= 1e-7 * np.abs(g_ref).max()


@pytest.mark.parametrize("name", ["cavity8", "duct_oct"])
@pytest.mark.parametrize("scheme", ["linear", "upwind", "vanleer"])
def test_transpose_face_flux_matches_finite_differences(name, scheme):
    """d/dphi of sum(r * u), u solving div(phi, U) - laplacian(nu, U) + V/dt,
    along random directions: adjoint (transpose face flux + BiCGStab
    transpose solve) against central differences, h = 1e-6 relative."""
    from gridfoam_b200.core.equation import equation
    from gridfoam_b200.fv import fvm

    grid, algo = _state(name)
    U, phi = algo.U, algo.phi
    base = grid.sim_config
    grid.sim_config = base.model_copy(update={"fvSchemes": base.fvSchemes.model_copy(
        update={"divSchemes": {"default": scheme}})})
    dev = dict(dtype=torch.float64, device="cuda")
    rng = np.random.default_rng(3)
    r3 = torch.as_tensor(rng.standard_normal((grid.num_cells, 3)), **dev)
    usrc = torch.as_tensor(rng.standard_normal((grid.num_cells, 3)), **dev)
    solver = _solver("bicgstab")
    phi0 = phi.store.detach().clone()
    U0 = U.data.detach().clone()

    def loss():
        U.data = U0  # the advected field (TVD limiter) and the initial guess
        m = fvm.div(phi, U) - fvm.laplacian(algo.nu, U)
        m.diag = m.diag + grid.cell_volumes / 0.01
        m.source = m.source + usrc * grid.cell_volumes[:, None]
        return (r3 * solver.solve(equation(U, m)).solution).sum()

    # The face-flux store is the leaf: gradients w.r.t. phi on every face.
    phi.store.requires_grad_(True)
    loss().backward()
    g = phi.store.grad.detach().clone()
    phi.store.requires_grad_(False)
    phi.store.grad = None
    scale = phi0.abs().max().item()
    for k in range(3):
        h = 1e-6 * scale
        # Upwind/TVD are piecewise linear in phi: leave faces whose flux is
        # within 10 h of zero unperturbed, so no face changes sign.
        v = torch.as_tensor(rng.standard_normal(phi0.shape), **dev) * (phi0.abs() > 10 * h)
        with torch.no_grad():
            phi.store.copy_(phi0 + h * v)
            lp = loss().item()
            phi.store.copy_(phi0 - h * v)
            lm = loss().item()
            phi.store.copy_(phi0)
        fd = (lp - lm) / (2 * h)
        ad = float((g * v).sum())
        assert abs(ad - fd) <= 1e-5 * max(abs(fd), 1e-12), (k, ad, fd)
    grid.sim_config = base


def _piso_cavity(n: int = 8, dt: float = 0.02) -> dict:
    """The lid-driven cavity as a PISO case with tightly converged solves
    (so the implicit adjoint of each solve is that of the exact solve)."""
    import copy

    from tests.golden.cases import cavity_case

    case = copy.deepcopy(cavity_case(n))
    sim = case["simulator"]
    sim["control"]["deltaT"] = dt
    sim["control"]["endTime"] = 1.0
    sim["fvSolution"]["algorithm"] = {"type": "piso", "nCorrectors": 2, "pRefCell": 0, "pRefValue": 0.0}
    tight = {"tolerance": 1e-14, "rel_tolerance": 0.0, "max_iter": 5000}
    sim["fvSolution"]["solvers"] = {
        "U": {"method": "bicgstab", "preconditioner": "jacobi", **tight},
        "p": {"method": "cg", "preconditioner": "jacobi", **tight},
    }
    case["name"] = f"cavity{n}_piso"
    return case


def _objective(U):
    return (U[:, 0] ** 2 + 0.5 * U[:, 1] ** 2 + U[:, 0] * U[:, 2]).sum()


@pytest.mark.gpu
def test_differentiable_piso_step_matches_device_step():
    """The reverse sweep's differentiable re-execution of a PISO step gives
    the device algorithm's step (kernels) to round-off."""
    from gridfoam_b200.cases import create_case
    from gridfoam_b200.solvers.step_adjoint import DifferentiablePisoStep, _state

    _, _, algo = create_case(_piso_cavity(), device="cuda")
    for _ in range(2):
        algo.step()
    s = _state(algo)
    dstep = DifferentiablePisoStep(algo)
    with torch.no_grad():
        nu = torch.tensor(algo.nu, dtype=torch.float64, device="cuda")
        U, phi, p = dstep.step(s[0], s[1], s[2], nu)
    from gridfoam_b200.solvers.step_adjoint import _restore

    _restore(algo, s)
    algo.step()
    ref = _state(algo)
    for a, b in zip((U, phi, p), ref):
        err = float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))
        assert err < 1e-9, err


@pytest.mark.gpu
@pytest.mark.parametrize("checkpoint_every", [1, 2, 5])
def test_piso_gradient_through_steps_matches_central_differences(checkpoint_every):
    """d J(U_N) / d nu through N = 5 PISO steps (reverse sweep with
    checkpoint-and-recompute) against central finite differences with
    h = 1e-3 nu: 1e-4 relative."""
    from gridfoam_b200.cases import create_case
    from gridfoam_b200.solvers.step_adjoint import piso_gradient

    n_steps = 5
    _, _, algo = create_case(_piso_cavity(), device="cuda")
    nu0 = algo.nu
    res = piso_gradient(algo, n_steps, _objective, checkpoint_every=checkpoint_every)
    assert res.checkpoints == len(range(0, n_steps, checkpoint_every))

    def J(nu):
        _, _, a = create_case(_piso_cavity(), device="cuda")
        a.nu = nu
        for _ in range(n_steps):
            a.step()
        return float(_objective(a.U.data))

    h = 1e-3 * nu0
    fd = (J(nu0 + h) - J(nu0 - h)) / (2 * h)
    assert abs(res.objective - J(nu0)) <= 1e-12 * abs(res.objective)
    assert abs(res.grad_nu - fd) <= 1e-4 * abs(fd), (res.grad_nu, fd)


def test_unrolled_gradients_match_reference_autograd():
    """grad_mode="unrolled" (solvers/base.py:111-115): gradients through the
    CG and BiCGStab iterations that ran (relative tolerance 1e-3, so they
    differ from the implicit adjoint's by 6 % and 0.1 %), against the
    reference's own unrolled run on the same inputs."""
    from gridfoam_b200.core.equation import equation
    from gridfoam_b200.fv import fvm
    from gridfoam_b200.meta.config import SolverConfig
    from gridfoam_b200.solvers.krylov import BiCGSTABSolver, CGSolver

    ref = np.load(HERE / "adjoint_cavity8_unrolled.npz")
    grid, algo = _state("cavity8")
    U, p, phi = algo.U, algo.p, algo.phi
    dev = dict(dtype=torch.float64, device="cuda")
    loose = dict(preconditioner="jacobi", tolerance=0.0, rel_tolerance=1e-3, max_iter=5000)

    gamma = torch.as_tensor(ref["adj_gamma"], **dev).requires_grad_(True)
    pmat = -fvm.laplacian(gamma, p)
    pmat.source = pmat.source - torch.as_tensor(ref["adj_src"], **dev) * grid.cell_volumes
    if algo.p_needs_ref:
        d = pmat.diag
        pmat.diag = d + torch.nn.functional.one_hot(torch.tensor(0), grid.num_cells).cuda() * d[0]
    p.data = torch.zeros(grid.num_cells, **dev)
    cg = CGSolver(SolverConfig(method="cg", **loose))
    cg.grad_mode = "unrolled"
    res = cg.solve(equation(p, pmat))
    (torch.as_tensor(ref["adj_r"], **dev) * res.solution).sum().backward()
    assert rel(to_np(res.solution), ref["unr_x"]) < 1e-10
    assert rel(to_np(gamma.grad), ref["unr_grad_gamma"]) < 1e-8
    assert rel(to_np(gamma.grad), ref["adj_grad_gamma"]) > 1e-3  # not the implicit adjoint's

    nu = torch.as_tensor(ref["adj_nu"], **dev).requires_grad_(True)
    umat = fvm.div(phi, U) - fvm.laplacian(nu, U)
    umat.diag = umat.diag + grid.cell_volumes / 0.01
    umat.source = umat.source + torch.as_tensor(ref["adj_usrc"], **dev) * grid.cell_volumes[:, None]
    U.data = torch.zeros((grid.num_cells, 3), **dev)
    bi = BiCGSTABSolver(SolverConfig(method="bicgstab", **loose))
    bi.grad_mode = "unrolled"
    res = bi.solve(equation(U, umat))
    (torch.as_tensor(ref["adj_r3"], **dev) * res.solution).sum().backward()
    assert rel(to_np(res.solution), ref["unr_u"]) < 1e-10
    assert rel(to_np(nu.grad), ref["unr_grad_nu"]) < 1e-8
