"""GPU parity: the sm_100a path against the reference's golden vectors and
the CPU oracle.

Whole algorithm steps are compared with the reference's own float64 run
(``tests/golden/*.npz``).  On tightly converged cases the fields agree to
round-off amplified by the Krylov stopping rule; the pipe case stops its
pressure solves at ``rel_tolerance`` 0.01, so its fields are compared at a
tolerance derived from that band and iteration counts may differ by one.
"""

from __future__ import annotations

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from tests.golden.device_harness import device_case, to_np  # noqa: E402
from tests.golden.cases import DIV_SCHEMES, OCTREE_CASES, STEPS  # noqa: E402
from tests.golden.oracle_harness import load_golden  # noqa: E402

pytestmark = pytest.mark.gpu

CASES = list(STEPS)
# Relative L2 tolerance of whole-step fields against the reference run.
STEP_TOL = {"cavity8": 1e-10, "channel": 1e-9, "channel_ffp": 1e-9, "ibplane": 1e-10, "ibplane_io": 1e-10, "pipe10x20": 1e-4,
            "cavity_oct": 1e-9, "duct_oct": 1e-8, "ibcyl_oct": 1e-8}


def rel(a, b) -> float:
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")


@pytest.mark.parametrize("algorithm", ["pcg", "sr", "staged", "smem", "qrec"])
@pytest.mark.parametrize("name", CASES)
def test_steps_match_reference(name, algorithm):
    """pcg: two-reduction fused PCG; sr: single-reduction CG; staged: the
    shared-memory tiled box kernel (box grids; ELL grids fall back); smem:
    own-cell vectors in shared memory; qrec: the same with q = A p formed
    by recurrence."""
    golden = load_golden(name)
    _, _, _, algo = device_case(name)
    for s in algo.solvers.values():
        s.single_reduction = algorithm == "sr"
        s.variant = {"staged": 5, "smem": 7, "qrec": 9}.get(algorithm, 0)
    np.testing.assert_allclose(to_np(algo.phi.pack()), golden["init_phi"], rtol=0, atol=1e-13)
    tol = STEP_TOL[name]
    slack = 1 if name.startswith("pipe") or name in OCTREE_CASES else 0
    for step in range(STEPS[name]):
        algo.step()
        torch.cuda.synchronize()
        assert rel(to_np(algo.U.data), golden[f"step{step}_U"]) < tol, (step, "U")
        assert rel(to_np(algo.p.data), golden[f"step{step}_p"]) < 10 * tol, (step, "p")
        assert rel(to_np(algo.phi.pack()), golden[f"step{step}_phi"]) < tol, (step, "phi")
        its_u = np.array([s.iterations for s in algo.last_stats["U"]])
        its_p = np.array([s.iterations for s in algo.last_stats["p"]])
        assert np.all(np.abs(its_u - golden[f"step{step}_stats_U"][:, 2]) <= slack), (step, its_u)
        assert np.all(np.abs(its_p - golden[f"step{step}_stats_p"][:, 2]) <= slack), (step, its_p)
        assert all(s.converged for s in algo.last_stats["p"])


def _load_state(algo, golden, step):
    algo.U.data = torch.as_tensor(golden[f"step{step}_U"], device="cuda")
    algo.p.data = torch.as_tensor(golden[f"step{step}_p"], device="cuda")
    algo.phi.unpack(torch.as_tensor(golden[f"step{step}_phi"], device="cuda"))


def _check(val, ref, key, rtol=1e-11):
    val = to_np(val) if isinstance(val, torch.Tensor) else np.asarray(val)
    assert val.shape == ref.shape, (key, val.shape, ref.shape)
    scale = max(np.abs(ref).max(), 1e-300)
    err = np.abs(val - ref).max()
    assert err <= rtol * scale, (key, err / scale)


@pytest.mark.parametrize("name", CASES)
def test_operators_match_reference(name):
    from gridfoam_b200.core.equation import equation
    from gridfoam_b200.fv import fvc, fvm
    from gridfoam_b200.meta.config import SolverConfig
    from gridfoam_b200.solvers.krylov import BiCGSTABSolver, CGSolver

    golden = load_golden(name)
    _, _, grid, algo = device_case(name)
    _load_state(algo, golden, STEPS[name] - 1)
    U, p, phi = algo.U, algo.p, algo.phi
    nu_eff = torch.full((grid.num_cells,), algo.nu, dtype=torch.float64, device="cuda")

    def mat(prefix, m, rtol=1e-11):
        _check(m.diag, golden[f"{prefix}_diag"], prefix + "_diag", rtol)
        _check(m.upper, golden[f"{prefix}_upper"], prefix + "_upper", rtol)
        _check(m.lower, golden[f"{prefix}_lower"], prefix + "_lower", rtol)
        _check(m.source, golden[f"{prefix}_source"], prefix + "_source", rtol)

    mat("op_lap_U", fvm.laplacian(nu_eff, U))
    base = grid.sim_config
    for scheme in DIV_SCHEMES:
        schemes_cfg = base.fvSchemes.model_copy(update={"divSchemes": {"default": scheme}})
        grid.sim_config = base.model_copy(update={"fvSchemes": schemes_cfg})
        mat(f"op_div_{scheme}", fvm.div(phi, U), rtol=1e-10)
    grid.sim_config = base
    _check(fvc.grad(p).data, golden["op_grad_p"], "grad_p", 1e-10)
    _check(fvc.grad(U).data, golden["op_grad_U"], "grad_U", 1e-10)
    _check(fvc.interpolate(U).pack(), golden["op_interp_U"], "interp_U")
    flux_scale = np.abs(golden[f"step{STEPS[name]-1}_phi"]).max() * golden["op_div_phi"].size
    div_err = np.abs(to_np(fvc.div(phi).data) - golden["op_div_phi"]).max()
    assert div_err <= 1e-12 * flux_scale
    _check(fvc.sn_grad(p).pack(), golden["op_sngrad_p"], "sngrad_p")

    gamma = torch.as_tensor(golden["op_gamma"], device="cuda")
    pmat = -fvm.laplacian(gamma, p)
    rng = np.random.default_rng(0)
    rng.random(grid.num_cells)
    src = torch.as_tensor(rng.standard_normal(grid.num_cells), device="cuda")
    pmat.source = pmat.source - src * grid.cell_volumes
    if algo.p_needs_ref:
        d = pmat.diag[0].clone()
        pmat.diag[0] += d
        pmat.source[0] += d * 0.0
    mat("op_pmat", pmat)
    peq = equation(p, pmat)
    mat("op_pmat_solve", peq.fv_matrix)
    cg = CGSolver(SolverConfig(method="cg", preconditioner="jacobi", tolerance=1e-9, rel_tolerance=0.0))
    res = cg.solve(peq)
    assert res.stats[0].iterations == int(golden["op_cg_stats"][0, 2])
    _check(res.solution, golden["op_cg_x"], "cg_x", 1e-8)

    umat = fvm.div(phi, U) - fvm.laplacian(nu_eff, U)
    umat.diag = umat.diag + grid.cell_volumes / 0.01
    umat.source = umat.source + torch.as_tensor(
        rng.standard_normal((grid.num_cells, 3)), device="cuda"
    ) * grid.cell_volumes[:, None]
    ueq = equation(U, umat)
    mat("op_umat_solve", ueq.fv_matrix, rtol=1e-10)
    bi = BiCGSTABSolver(SolverConfig(method="bicgstab", preconditioner="jacobi", tolerance=1e-10, rel_tolerance=0.0))
    res = bi.solve(ueq)
    its = [s.iterations for s in res.stats]
    assert np.all(np.abs(np.array(its) - golden["op_bicg_stats"][:, 2]) <= 1), its
    _check(res.solution, golden["op_bicg_x"], "bicg_x", 1e-8)
    _check(umat.multiply(U.data), golden["op_spmv_U"], "spmv")
    _check(umat.H(U.data), golden["op_H_U"], "H", 1e-10)
    _check(umat.H1(), golden["op_H1_U"], "H1")
    _check((-pmat).flux(p.data), golden["op_flux_p"], "flux")


def test_transpose_identity():
    """``y . A x == (A^T y) . x`` (test_linear_solver_adjoint.py:121-138)."""
    from gridfoam_b200.fv import fvm

    _, _, grid, algo = device_case("channel")
    gen = torch.Generator(device="cpu").manual_seed(0)
    algo.phi.store.copy_(torch.randn(algo.phi.store.shape, generator=gen, dtype=torch.float64))
    A = fvm.div(algo.phi, algo.U) - fvm.laplacian(0.1, algo.U)
    x = torch.randn((grid.num_cells, 3), generator=gen, dtype=torch.float64).cuda()
    y = torch.randn((grid.num_cells, 3), generator=gen, dtype=torch.float64).cuda()
    lhs = float((y * A.multiply(x)).sum())
    rhs = float((A.as_transpose().multiply(y) * x).sum())
    assert abs(lhs - rhs) <= 1e-12 * max(abs(lhs), 1.0)


def test_krylov_zero_rhs_and_limits():
    """Zero right-hand side converges at iteration 0; max_iter and a
    non-finite input end with the right status instead of hanging."""
    from gridfoam_b200.fv import fvm
    from gridfoam_b200.meta.config import SolverConfig
    from gridfoam_b200.solvers.krylov import BiCGSTABSolver, CGSolver

    _, _, grid, algo = device_case("cavity8")
    A = -fvm.laplacian(1.0, algo.p)
    A.diag = A.diag + grid.cell_volumes
    n = grid.num_cells
    zero = torch.zeros((1, n), dtype=torch.float64, device="cuda")
    for cls, method in ((CGSolver, "cg"), (BiCGSTABSolver, "bicgstab")):
        s = cls(SolverConfig(method=method, preconditioner="jacobi", tolerance=1e-12, rel_tolerance=0.0))
        x = torch.zeros_like(zero)
        st = s.solve_arrays(grid, A.diag_store, A.val, zero, x)
        assert st[0].iterations == 0 and st[0].converged
        rhs = torch.ones((1, n), dtype=torch.float64, device="cuda")
        s2 = cls(SolverConfig(method=method, preconditioner="jacobi", tolerance=1e-30, rel_tolerance=0.0, max_iter=3))
        x = torch.zeros_like(zero)
        st = s2.solve_arrays(grid, A.diag_store, A.val, rhs, x)
        assert st[0].iterations == 3 and not st[0].converged and st[0].status == "max_iter"
        bad = rhs.clone()
        bad[0, 5] = float("nan")
        x = torch.zeros_like(zero)
        st = s2.solve_arrays(grid, A.diag_store, A.val, bad, x)
        assert not st[0].converged and st[0].status == "nonfinite"


@pytest.mark.parametrize("method,variant", [("cg", 0), ("cg", 10), ("cg", 8), ("bicgstab", None)])
def test_krylov_wait_timeout_reports_and_recovers(method, variant):
    """A device wait that runs out ends the solve with status "timeout"
    (GF_ERR_TIMEOUT) and returns; the next solve on the same stream runs
    normally.  The poll limit is cut to two polls, so some block gives up
    at a grid barrier or halo flag: the kernel sets the error flag, every
    other block leaves at its next bounded wait, nothing traps."""
    from gridfoam_b200.fv import fvm
    from gridfoam_b200.meta.config import SolverConfig
    from gridfoam_b200.solvers.krylov import BiCGSTABSolver, CGSolver
    from tests.golden.cases import pipe_case

    _, _, grid, algo = device_case(case_def=pipe_case(24, 48) if method == "cg" else pipe_case(48, 96))
    A = -fvm.laplacian(1.0, algo.p)
    # BiCGStab gets a diagonally dominant system: on the nearly singular
    # Laplacian it exhausts its breakdown restarts (as the reference's does).
    A.diag = A.diag * (1.0 if method == "cg" else 1.02) + 1e-3 * grid.cell_volumes
    n = grid.num_cells
    rhs = torch.linspace(-1.0, 1.0, n, dtype=torch.float64, device="cuda").reshape(1, n)
    cls = CGSolver if method == "cg" else BiCGSTABSolver
    cfg = SolverConfig(method=method, preconditioner="jacobi", tolerance=1e-10, rel_tolerance=0.0, max_iter=5000)
    ref = cls(cfg)
    ref.variant = variant
    x_ref = torch.zeros_like(rhs)
    st = ref.solve_arrays(grid, A.diag_store, A.val, rhs, x_ref, symmetric=True)
    assert st[0].converged and st[0].iterations > 5

    s = cls(cfg)
    s.variant = variant
    s.spin_limit = 2
    statuses = []
    for _ in range(10):  # a timeout needs one block to arrive > 2 polls early
        x = torch.zeros_like(rhs)
        st = s.solve_arrays(grid, A.diag_store, A.val, rhs, x, symmetric=True)
        statuses.append(st[0].status)
        if st[0].status == "timeout":
            break
    assert "timeout" in statuses, statuses
    assert not st[0].converged
    s.spin_limit = 0
    x = torch.zeros_like(rhs)
    st = s.solve_arrays(grid, A.diag_store, A.val, rhs, x, symmetric=True)
    torch.cuda.synchronize()
    assert st[0].status == "ok" and st[0].converged
    torch.testing.assert_close(x, x_ref, rtol=1e-12, atol=1e-14)


def test_cavity32_against_oracle():
    """Full-size cavity config (32^3, SIMPLE, linear): two steps against the
    oracle (the reference restatement) on the same mesh."""
    from tests.golden.cases import cavity_case
    from tests.golden.oracle_harness import oracle_case

    case = cavity_case(32)
    _, _, _, dalgo = device_case(case_def=case)
    _, _, _, oalgo = oracle_case("cavity32", case_def=case)
    for _ in range(2):
        dalgo.step()
        oalgo.step()
        torch.cuda.synchronize()
        assert rel(to_np(dalgo.U.data), oalgo.U.data) < 1e-9
        assert rel(to_np(dalgo.p.data), oalgo.p.data) < 1e-8
        assert [s.iterations for s in dalgo.last_stats["p"]] == [s.iterations for s in oalgo.last_stats["p"]]


@pytest.mark.parametrize("layout", ["box", "ell"])
@pytest.mark.parametrize("variant", [None, 6, 7, 8, 9])
def test_mixed_precision_pcg_meets_fp64_criterion(variant, layout):
    """FP32 inner CG inside FP64 refinement reaches the same FP64 true-residual
    threshold as the FP64 solver, and its solution agrees with the FP64
    solution to the accuracy that threshold implies.  Variants 6/7: the
    kernels with each block's FP32 vectors resident in shared memory."""
    _mixed_case(variant, layout, 16, 32)


@pytest.mark.parametrize("layout", ["box", "ell"])
@pytest.mark.parametrize("variant", [10, 11])
def test_mixed_halo_pcg_meets_fp64_criterion(variant, layout):
    """The FP32-inner solve in the single-reduction form with a halo sync
    (27,648 cells: enough for its flags) meets the same FP64 criterion."""
    _mixed_case(variant, layout, 24, 48)


def _mixed_case(variant, layout, nxy, nz):
    from gridfoam_b200.fv import fvm
    from gridfoam_b200.meta.config import SolverConfig
    from gridfoam_b200.solvers.krylov import CGSolver

    from tests.golden.cases import pipe_case

    _, _, grid, algo = device_case(case_def=pipe_case(nxy, nz))
    gamma = torch.full((grid.num_cells,), 0.3, dtype=torch.float64, device="cuda")
    A = -fvm.laplacian(gamma, algo.p)
    gen = torch.Generator(device="cpu").manual_seed(1)
    rhs = torch.randn((1, grid.num_cells), generator=gen, dtype=torch.float64).cuda() * 1e-3
    strides = grid.box_strides
    if layout == "ell":
        grid.box_strides = None
    try:
        for tol, rel_tol in ((1e-9, 0.0), (1e-7, 0.01)):
            base = dict(method="cg", preconditioner="jacobi", tolerance=tol, rel_tolerance=rel_tol, max_iter=5000)
            x64 = torch.zeros_like(rhs)
            s64 = CGSolver(SolverConfig(**base)).solve_arrays(grid, A.diag_store, A.val, rhs, x64)
            x32 = torch.zeros_like(rhs)
            mixed = CGSolver(SolverConfig(**base, inner_precision="float32"))
            mixed.variant = variant
            s32 = mixed.solve_arrays(grid, A.diag_store, A.val, rhs, x32, symmetric=layout == "box")
            _check_mixed(A, rhs, x32, s32, s64, tol, rel_tol)
    finally:
        grid.box_strides = strides


def _check_mixed(A, rhs, x32, s32, s64, tol, rel_tol):
    assert s64[0].converged and s32[0].converged, (s64, s32)
    # true FP64 residual of the mixed solution meets the same threshold
    r = rhs - A.multiply(x32[0]).reshape(1, -1)
    thresh = max(tol, rel_tol * s64[0].initial_residual)
    assert float(torch.linalg.vector_norm(r)) < thresh
    assert abs(s32[0].initial_residual - s64[0].initial_residual) <= 1e-12 * s64[0].initial_residual


@pytest.mark.parametrize("variant", [None, 7, 8])
def test_box_layout_matches_ell_layout(variant):
    """On a uniform box, CG with implicit neighbours (symmetric three-array
    coefficient reads) gives the same solve as the generic ELL path, in the
    register kernels and in the shared-memory-resident ones (7)."""
    from gridfoam_b200.fv import fvm
    from gridfoam_b200.meta.config import SolverConfig
    from gridfoam_b200.solvers.krylov import CGSolver

    from tests.golden.cases import pipe_case

    _, _, grid, algo = device_case(case_def=pipe_case(16, 32))
    assert grid.box_strides == (16, 256)
    gamma = torch.linspace(0.2, 0.4, grid.num_cells, dtype=torch.float64, device="cuda")
    A = -fvm.laplacian(gamma, algo.p)
    gen = torch.Generator(device="cpu").manual_seed(2)
    rhs = torch.randn((1, grid.num_cells), generator=gen, dtype=torch.float64).cuda()
    for precision in ("float64", "float32"):
        cfg = SolverConfig(method="cg", preconditioner="jacobi", tolerance=1e-10, rel_tolerance=0.0,
                           max_iter=4000, inner_precision=precision)
        x_box = torch.zeros_like(rhs)
        solver = CGSolver(cfg)
        solver.variant = variant
        s_box = solver.solve_arrays(grid, A.diag_store, A.val, rhs, x_box, symmetric=True)
        strides, grid.box_strides = grid.box_strides, None
        try:
            x_ell = torch.zeros_like(rhs)
            s_ell = solver.solve_arrays(grid, A.diag_store, A.val, rhs, x_ell)
        finally:
            grid.box_strides = strides
        assert s_box[0].converged and s_ell[0].converged
        assert s_box[0].iterations == s_ell[0].iterations
        torch.testing.assert_close(x_box, x_ell, rtol=0, atol=0)


@pytest.mark.parametrize("layout", ["box", "ell"])
def test_single_reduction_cg_matches_pcg(layout):
    """Chronopoulos-Gear CG (one reduction per iteration) against the
    two-reduction PCG on a symmetric 7-point system: same iteration count
    within one, solutions within the stopping tolerance, and the true
    residual of both below the threshold."""
    from gridfoam_b200.solvers.autotune import BoxSystem, _solver

    sysm = BoxSystem(24, 20, 28, device=torch.device("cuda"))
    if layout == "ell":
        sysm.box_strides = None
    out = {}
    for sr in (False, True):
        s = _solver(2000, False, 0, sr)
        s.atol, s.rtol = 0.0, 1e-10
        x = torch.zeros_like(sysm.rhs)
        st = s.solve_arrays(sysm, sysm.diag, sysm.val, sysm.rhs, x, symmetric=True)
        out[sr] = (x.clone(), st[0])
    (x0, s0), (x1, s1) = out[False], out[True]
    assert s0.converged and s1.converged
    assert abs(s0.iterations - s1.iterations) <= 1, (s0.iterations, s1.iterations)
    assert s0.initial_residual == pytest.approx(s1.initial_residual, rel=1e-14)
    assert rel(to_np(x1), to_np(x0)) < 1e-8
    # true residual of the single-reduction solution
    nb = sysm.dev["ell_nbr"].long()
    ax = sysm.diag * x1[0] + (sysm.val * x1[0][nb]).sum(0)
    r = torch.linalg.vector_norm(sysm.rhs[0] - ax).item()
    assert r < 1e-9 * s1.initial_residual


@pytest.mark.parametrize("variant", [5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 19, 20])
@pytest.mark.parametrize("shape", [(24, 20, 28), (64, 64, 40), (7, 5, 6), (130, 3, 4)])
def test_staged_box_cg_matches_register_kernel(shape, variant):
    """The shared-memory variants against the register kernel (variant 0):
    5 stages tiles by bulk async copy, 6/7 keep each block's own-cell
    vectors resident (512/1024 threads), 8/9 also form q = A p by
    recurrence, 10/11 take one grid reduction and a halo sync with the
    neighbouring blocks per iteration.  Same iteration count within one and
    the same solution to the stopping tolerance, on shapes with partial last
    tiles or chunks, odd strides and a y halo larger than a tile's x extent."""
    from gridfoam_b200.solvers.autotune import BoxSystem, _solver

    sysm = BoxSystem(*shape, device=torch.device("cuda"))
    out = {}
    for v in (0, variant):
        s = _solver(3000, False, v)
        s.atol, s.rtol = 0.0, 1e-10
        x = torch.zeros_like(sysm.rhs)
        st = s.solve_arrays(sysm, sysm.diag, sysm.val, sysm.rhs, x, symmetric=True)
        out[v] = (x.clone(), st[0])
    (x0, s0), (x1, s1) = out[0], out[variant]
    assert s0.converged and s1.converged, (s0.status, s1.status)
    assert abs(s0.iterations - s1.iterations) <= 1, (s0.iterations, s1.iterations)
    assert s0.initial_residual == pytest.approx(s1.initial_residual, rel=1e-13)
    assert rel(to_np(x1), to_np(x0)) < 1e-8


def test_staged_box_cg_fixed_iterations_match_register_kernel():
    """With tolerances 0 both kernels run exactly max_iter iterations; the
    SpMV products are bitwise those of BoxRows, so the two iterates differ
    only through the order of the dot-product partial sums."""
    from gridfoam_b200.solvers.autotune import BoxSystem, _solver

    sysm = BoxSystem(32, 16, 48, device=torch.device("cuda"))
    xs = []
    for v in (0, 5):
        s = _solver(50, False, v)
        x = torch.zeros_like(sysm.rhs)
        st = s.solve_arrays(sysm, sysm.diag, sysm.val, sysm.rhs, x, symmetric=True)
        assert st[0].iterations == 50 and st[0].status == "max_iter"
        xs.append(to_np(x))
    assert rel(xs[1], xs[0]) < 1e-11


@pytest.mark.parametrize("box", [True, False])
@pytest.mark.parametrize("variant", [6, 7])
def test_smem_resident_cg_fixed_iterations_match_register_kernel(variant, box):
    """Exactly 60 iterations (tolerances 0) of the shared-memory-resident CG
    (pair-interleaved z/p, inverse diagonal once per solve, L1-cached
    gathers) against the register kernel: the iterates differ only through
    the order of the dot-product partial sums."""
    from gridfoam_b200.solvers.autotune import BoxSystem, _solver

    sysm = BoxSystem(40, 36, 44, device=torch.device("cuda"))
    if not box:
        sysm.box_strides = None
    xs = []
    for v in (0, variant):
        s = _solver(60, False, v)
        x = torch.zeros_like(sysm.rhs)
        st = s.solve_arrays(sysm, sysm.diag, sysm.val, sysm.rhs, x, symmetric=True)
        assert st[0].iterations == 60 and st[0].status == "max_iter"
        xs.append(to_np(x))
    assert rel(xs[1], xs[0]) < 1e-11


@pytest.mark.parametrize("variant", [6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16, 17, 18, 19, 20])
def test_smem_resident_cg_on_ell_layout(variant):
    """The shared-memory-resident CG through the general ELL rows (the
    octree path), against the register ELL kernel."""
    from gridfoam_b200.solvers.autotune import BoxSystem, _solver

    sysm = BoxSystem(20, 18, 26, device=torch.device("cuda"))
    sysm.box_strides = None
    out = {}
    for v in (0, variant):
        s = _solver(3000, False, v)
        s.atol, s.rtol = 0.0, 1e-10
        x = torch.zeros_like(sysm.rhs)
        st = s.solve_arrays(sysm, sysm.diag, sysm.val, sysm.rhs, x, symmetric=True)
        out[v] = (x.clone(), st[0])
    (x0, s0), (x1, s1) = out[0], out[variant]
    assert s0.converged and s1.converged
    assert abs(s0.iterations - s1.iterations) <= 1
    assert rel(to_np(x1), to_np(x0)) < 1e-8


@pytest.mark.parametrize("box", [True, False])
@pytest.mark.parametrize("variant", [10, 11])
def test_halo_cg_fixed_iterations_match_register_kernel(variant, box):
    """Exactly 60 iterations (tolerances 0) of the single-reduction CG with
    the halo sync against the register kernel: the same iterates up to the
    rounding of alpha = gamma / (delta - beta gamma / alpha_old) instead of
    gamma / p.Ap and of the partial-sum order."""
    from gridfoam_b200.solvers.autotune import BoxSystem, _solver

    sysm = BoxSystem(40, 36, 44, device=torch.device("cuda"))
    if not box:
        sysm.box_strides = None
    xs = []
    for v in (0, variant):
        s = _solver(60, False, v)
        x = torch.zeros_like(sysm.rhs)
        st = s.solve_arrays(sysm, sysm.diag, sysm.val, sysm.rhs, x, symmetric=True)
        assert st[0].iterations == 60 and st[0].status == "max_iter"
        xs.append(to_np(x))
    assert rel(xs[1], xs[0]) < 1e-9


def test_halo_cg_on_scrambled_ell():
    """A randomly renumbered system: every block's rows read cells of
    nearly every other block, so each halo sync waits on ~all blocks (one
    polling thread each).  Same iterations within one and the same solution
    as the register kernel, mapped back to the original numbering."""
    from gridfoam_b200.solvers.autotune import BoxSystem, _solver

    sysm = BoxSystem(48, 40, 60, device=torch.device("cuda"))
    sysm.box_strides = None
    n = sysm.num_cells
    g = torch.Generator(device="cpu").manual_seed(11)
    perm = torch.randperm(n, generator=g).cuda()  # new -> old
    inv = torch.empty_like(perm)
    inv[perm] = torch.arange(n, device=perm.device)
    nbr = sysm.dev["ell_nbr"].long()
    sysm.dev["ell_nbr"] = inv[nbr[:, perm]].to(torch.int32).contiguous()
    sysm.val = sysm.val[:, perm].contiguous()
    sysm.diag = sysm.diag[perm].contiguous()
    sysm.rhs = sysm.rhs[:, perm].contiguous()
    out = {}
    for v in (0, 10):
        s = _solver(4000, False, v)
        s.atol, s.rtol = 0.0, 1e-10
        x = torch.zeros_like(sysm.rhs)
        st = s.solve_arrays(sysm, sysm.diag, sysm.val, sysm.rhs, x, symmetric=True)
        out[v] = (x.clone(), st[0])
    (x0, s0), (x1, s1) = out[0], out[10]
    assert s0.converged and s1.converged
    assert abs(s0.iterations - s1.iterations) <= 1, (s0.iterations, s1.iterations)
    assert rel(to_np(x1), to_np(x0)) < 1e-8


@pytest.mark.parametrize("name", ["pipe10x20", "channel"])
@pytest.mark.parametrize("with_ddt", [False, True])
def test_axis_face_flux_matches_generic_path(name, with_ddt):
    """The two-faces-per-thread face-flux kernel of axis-aligned grids
    (``face_axis`` given) against the generic one (``face_axis`` NULL, all
    three Sf components): the same bits, up to the sign of zero, with and
    without the ddtCorr history term."""
    import ctypes

    from gridfoam_b200._lib import GfDdtCorr, GfMesh, call, ptr, stream_ptr

    _, _, grid, algo = device_case(name)
    for _ in range(2):
        algo.step()
    U = algo.U
    generic = GfMesh()
    ctypes.memmove(ctypes.byref(generic), ctypes.byref(grid.cmesh), ctypes.sizeof(GfMesh))
    generic.face_axis = None
    d = None
    if with_ddt:
        gen = torch.Generator(device="cpu").manual_seed(5)
        rau = torch.rand(grid.num_cells, generator=gen, dtype=torch.float64).cuda() + 0.5
        u_old = U.store + 0.01 * torch.randn(U.store.shape, generator=gen, dtype=torch.float64).cuda()
        u_older = U.store - 0.02 * torch.randn(U.store.shape, generator=gen, dtype=torch.float64).cuda()
        phi_old = algo.phi.store[: grid.num_internal_faces].clone() * 1.01
        phi_older = algo.phi.store[: grid.num_internal_faces].clone() * 0.98
        d = GfDdtCorr()
        d.rau, d.u_old, d.u_older = ptr(rau), ptr(u_old), ptr(u_older)
        d.phi_old, d.phi_older = ptr(phi_old), ptr(phi_older)
        d.b, d.c, d.dt = 2.0, 0.5, 1e-3
    outs = []
    for mesh in (grid.cmesh, generic):
        out = torch.full_like(algo.phi.store, float("nan"))
        call("gf_face_flux", ctypes.byref(mesh), 1, ptr(U.store), ptr(U.table.kind), ptr(U.table.psib),
             None if d is None else ctypes.byref(d), None, ptr(out), stream_ptr())
        outs.append(out + 0.0)
    torch.cuda.synchronize()
    assert not torch.isnan(outs[0]).any()
    assert torch.equal(outs[0], outs[1])


@pytest.mark.parametrize("name", ["cavity8", "pipe10x20", "channel", "ibplane"])
def test_staged_assembly_matches_generic_kernel(name):
    """The staged six-slot assembly (uniform grids, upwind/linear schemes)
    against the generic per-slot kernel, which a face-flux-correction
    output forces: the same matrix bits for every assembly of a step."""
    import ctypes

    from gridfoam_b200._lib import call, ptr, stream_ptr
    from gridfoam_b200.fv import fvm

    _, _, grid, algo = device_case(name)
    algo.step()
    captured = []
    orig = fvm._run

    def spy(field, a):
        captured.append((field, a))
        orig(field, a)

    fvm._run = spy
    try:
        rau = torch.rand(grid.num_cells, dtype=torch.float64, device="cuda") + 0.5
        mats = [fvm.laplacian(rau, algo.p), fvm.laplacian(0.3, algo.p), fvm.div(algo.phi, algo.U),
                fvm.laplacian(algo.nu, algo.U)]
    finally:
        fvm._run = orig
    assert len(captured) >= len(mats)
    scratch = torch.zeros((3, grid.num_internal_faces), dtype=torch.float64, device="cuda")
    for field, a in captured:
        nc = a.ncomp
        C = grid.num_cells
        diag = torch.empty(C, dtype=torch.float64, device="cuda")
        val = torch.empty((grid.ell_width, C), dtype=torch.float64, device="cuda")
        src = torch.empty((nc, C), dtype=torch.float64, device="cuda")
        a.diag, a.val, a.source = ptr(diag), ptr(val), ptr(src)
        outs = []
        for ffc in (None, scratch):
            a.ffc = None if ffc is None else ptr(ffc)
            call("gf_assemble", ctypes.byref(grid.cmesh), ctypes.byref(a), stream_ptr())
            outs.append((diag.clone(), val.clone(), src.clone()))
        a.ffc = None
        for x, y in zip(*outs):
            assert torch.equal(x, y), field.name


@pytest.mark.parametrize("variant", [8, 9, 10, 11, 12, 13, 19])
@pytest.mark.parametrize("box", [True, False])
def test_qrec_cg_true_residual(variant, box):
    """The q-recurrence CG updates r from q = A z + beta q rather than from
    A p: after a solve to 1e-10 relative, the true residual b - A x must sit
    at the reported one (no residual gap beyond rounding)."""
    from gridfoam_b200.solvers.autotune import BoxSystem, _solver

    sysm = BoxSystem(48, 40, 96, device=torch.device("cuda"))
    if not box:
        sysm.box_strides = None
    s = _solver(6000, False, variant)
    s.atol, s.rtol = 0.0, 1e-10
    x = torch.zeros_like(sysm.rhs)
    st = s.solve_arrays(sysm, sysm.diag, sysm.val, sysm.rhs, x, symmetric=True)[0]
    assert st.converged
    nb = sysm.dev["ell_nbr"].long()
    ax = sysm.diag * x[0] + (sysm.val * x[0][nb]).sum(0)
    true = torch.linalg.vector_norm(sysm.rhs[0] - ax).item()
    assert true < 2e-10 * st.initial_residual, (true / st.initial_residual, st.iterations)


@pytest.mark.parametrize("box", [True, False])
@pytest.mark.parametrize("variant", [12, 13, 14])
def test_stream_cg_fixed_iterations_match_qrec(variant, box):
    """The streaming CG (vectors in global memory) runs the q-recurrence of
    the shared-memory form: exactly 60 iterations of each agree up to the
    order of the dot-product partial sums."""
    from gridfoam_b200.solvers.autotune import BoxSystem, _solver

    sysm = BoxSystem(40, 36, 44, device=torch.device("cuda"))
    if not box:
        sysm.box_strides = None
    xs = []
    for v in (8, variant):
        s = _solver(60, False, v)
        x = torch.zeros_like(sysm.rhs)
        st = s.solve_arrays(sysm, sysm.diag, sysm.val, sysm.rhs, x, symmetric=True)
        assert st[0].iterations == 60 and st[0].status == "max_iter"
        xs.append(to_np(x))
    assert rel(xs[1], xs[0]) < 1e-11


@pytest.mark.parametrize("variant", [2, 12, 13, 15, 17, 19])
def test_row_lengths_skip_only_empty_slots(variant):
    """On an octree grid (couplings first in every row) the CG with the
    row-length early exit gives the same iterations and solution as the
    same kernel reading every slot."""
    from gridfoam_b200.fv import fvm
    from gridfoam_b200.meta.config import SolverConfig
    from gridfoam_b200.solvers.krylov import CGSolver

    _, _, grid, algo = device_case("ibcyl_oct")
    assert grid.box_strides is None
    assert float(grid.dev["ell_len"].double().mean()) < grid.ell_width  # rows shorter than the widest
    A = -fvm.laplacian(1.0, algo.p)
    A.diag = A.diag + 1e-2 * grid.cell_volumes
    rhs = torch.linspace(-1.0, 1.0, grid.num_cells, dtype=torch.float64, device="cuda").reshape(1, -1)
    cfg = SolverConfig(method="cg", preconditioner="jacobi", tolerance=0.0, rel_tolerance=1e-10, max_iter=4000)
    out = []
    for use_len in (True, False):
        saved = None if use_len else grid.dev.pop("ell_len")
        s = CGSolver(cfg)
        s.variant = variant
        x = torch.zeros_like(rhs)
        st = s.solve_arrays(grid, A.diag_store, A.val, rhs, x, symmetric=True)[0]
        if saved is not None:
            grid.dev["ell_len"] = saved
        out.append((to_np(x), st.iterations, st.converged))
    assert out[0][2] and out[1][2]
    assert out[0][1] == out[1][1]
    assert rel(out[0][0], out[1][0]) < 1e-13


@pytest.mark.parametrize("name", ["cavity8", "channel", "duct_oct", "ibcyl_oct"])
def test_grad_linear_steps_and_operator_match_reference(name):
    """The Green-Gauss ('linear') gradient scheme (fv/schemes/grad.py:21-43):
    whole steps with gradSchemes default linear, and fvc.grad of p and U on
    the final state, against the reference's own run."""
    from gridfoam_b200.fv import fvc
    from tests.golden.cases import grad_linear_case

    golden = load_golden(f"gradlinear_{name}")
    _, _, _, algo = device_case(case_def=grad_linear_case(name))
    tol = STEP_TOL[name]
    for step in range(STEPS[name]):
        algo.step()
        torch.cuda.synchronize()
        assert rel(to_np(algo.U.data), golden[f"step{step}_U"]) < tol, (step, "U")
        assert rel(to_np(algo.p.data), golden[f"step{step}_p"]) < 10 * tol, (step, "p")
        assert rel(to_np(algo.phi.pack()), golden[f"step{step}_phi"]) < tol, (step, "phi")
        its_p = np.array([s.iterations for s in algo.last_stats["p"]])
        slack = 1 if name in OCTREE_CASES else 0
        assert np.all(np.abs(its_p - golden[f"step{step}_stats_p"][:, 2]) <= slack), (step, its_p)
    _load_state(algo, golden, STEPS[name] - 1)
    _check(fvc.grad(algo.p).data, golden["op_grad_p"], "grad_p", 1e-10)
    _check(fvc.grad(algo.U).data, golden["op_grad_U"], "grad_U", 1e-10)


@pytest.mark.parametrize("variant", [15, 16, 17, 18, 19, 20, 21, 22, 23, 24, 25, 26, 27, 28, 29, 30, 31])
def test_lean_ell_cg_fixed_iterations_match_register_kernel(variant):
    """The lean ELL CG (32-bit indices, x update moved into the next gather
    pass) and the split CG forms against the register kernel: exactly 60
    iterations agree up to the order of the dot-product partial sums (and,
    for variant 25, the rounding of q = A z + beta q by recurrence)."""
    from gridfoam_b200.solvers.autotune import BoxSystem, _solver

    sysm = BoxSystem(40, 36, 44, device=torch.device("cuda"))
    sysm.box_strides = None
    xs = []
    for v in (0, variant):
        s = _solver(60, False, v)
        x = torch.zeros_like(sysm.rhs)
        st = s.solve_arrays(sysm, sysm.diag, sysm.val, sysm.rhs, x, symmetric=True)
        assert st[0].iterations == 60 and st[0].status == "max_iter"
        xs.append(to_np(x))
    assert rel(xs[1], xs[0]) < (1e-9 if variant in (25, 26, 27, 29, 30, 31) else 1e-11)


@pytest.mark.parametrize("xa,base", [(27, 25), (28, 21), (29, 25), (30, 25), (31, 25)])
@pytest.mark.parametrize("max_iter,rtol", [(60, 0.0), (500, 1e-8)])
def test_split_cg_x_update_in_row_kernel_is_bitwise(xa, base, max_iter, rtol):
    """Variants 27/28 apply x += alpha p in the next row kernel (and, at the
    stop, in the kernel that ends the solve) instead of the update kernel:
    the same values in the same order, so x is bitwise that of 25/21, on a
    fixed-length solve and on one that converges, through the graph loop
    and enqueued inside a stream capture.  Variants 29-31 (27 with L2
    prefetches and earlier scalar reads) compute the same."""
    from gridfoam_b200.fv import fvm
    from gridfoam_b200.meta.config import SolverConfig
    from gridfoam_b200.solvers.krylov import CGSolver

    _, _, grid, algo = device_case("ibcyl_oct")
    A = -fvm.laplacian(1.0, algo.p)
    A.diag = A.diag + 1e-2 * grid.cell_volumes
    rhs = torch.linspace(-1.0, 1.0, grid.num_cells, dtype=torch.float64, device="cuda").reshape(1, -1)
    cfg = SolverConfig(method="cg", preconditioner="jacobi", tolerance=0.0, rel_tolerance=rtol, max_iter=max_iter)
    xs, its = [], []
    for v in (base, xa):
        s = CGSolver(cfg)
        s.variant = v
        x = torch.zeros_like(rhs)
        st = s.solve_arrays(grid, A.diag_store, A.val, rhs, x, symmetric=True)[0]
        its.append((st.iterations, st.status))
        xs.append(x)
    assert its[0] == its[1]
    assert (its[0][0] == max_iter) if rtol == 0.0 else (0 < its[0][0] < max_iter)
    assert torch.equal(xs[0], xs[1])
    caps = []
    for v in (base, xa):
        s = CGSolver(cfg)
        s.variant = v
        s.host_stats = False
        x = torch.zeros_like(rhs)
        stream = torch.cuda.Stream()
        stream.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(stream):
            s.solve_arrays(grid, A.diag_store, A.val, rhs, x, symmetric=True)  # workspace allocation
        torch.cuda.synchronize()
        x.zero_()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=stream):
            s.solve_arrays(grid, A.diag_store, A.val, rhs, x, symmetric=True)
        x.zero_()
        torch.cuda.synchronize()
        g.replay()
        torch.cuda.synchronize()
        stats = next(iter(s._stats_dev.values())).cpu().numpy()
        assert int(stats[0, 2]) == its[0][0]
        caps.append(x.clone())
        del g
    assert torch.equal(caps[0], caps[1])
    assert torch.equal(caps[1], xs[1])


def test_split_cg_limits_and_statuses():
    """The split CG (variant 19) reports iteration 0 on a zero right-hand
    side, max_iter and non-finite input like the persistent kernels."""
    from gridfoam_b200.fv import fvm
    from gridfoam_b200.meta.config import SolverConfig
    from gridfoam_b200.solvers.krylov import CGSolver

    _, _, grid, algo = device_case("cavity8")
    A = -fvm.laplacian(1.0, algo.p)
    A.diag = A.diag + grid.cell_volumes
    n = grid.num_cells
    zero = torch.zeros((1, n), dtype=torch.float64, device="cuda")
    s = CGSolver(SolverConfig(method="cg", preconditioner="jacobi", tolerance=1e-12, rel_tolerance=0.0))
    s.variant = 19
    st = s.solve_arrays(grid, A.diag_store, A.val, zero, torch.zeros_like(zero))
    assert st[0].iterations == 0 and st[0].converged
    s2 = CGSolver(SolverConfig(method="cg", preconditioner="jacobi", tolerance=1e-30, rel_tolerance=0.0, max_iter=3))
    s2.variant = 19
    rhs = torch.ones((1, n), dtype=torch.float64, device="cuda")
    st = s2.solve_arrays(grid, A.diag_store, A.val, rhs, torch.zeros_like(zero))
    assert st[0].iterations == 3 and not st[0].converged and st[0].status == "max_iter"
    bad = rhs.clone()
    bad[0, 5] = float("nan")
    st = s2.solve_arrays(grid, A.diag_store, A.val, bad, torch.zeros_like(zero))
    assert not st[0].converged and st[0].status == "nonfinite"


def test_split_cg_graph_loop_matches_captured_form():
    """Outside stream capture the split CG runs its iterations as a CUDA
    graph while-loop that ends on the device; inside a capture it enqueues
    every permitted iteration.  Both run the same kernels in the same order:
    the same iterations and the same bits, solve after solve."""
    from gridfoam_b200.fv import fvm
    from gridfoam_b200.meta.config import SolverConfig
    from gridfoam_b200.solvers.krylov import CGSolver

    _, _, grid, algo = device_case("ibcyl_oct")
    A = -fvm.laplacian(1.0, algo.p)
    A.diag = A.diag + 1e-2 * grid.cell_volumes
    rhs = torch.linspace(-1.0, 1.0, grid.num_cells, dtype=torch.float64, device="cuda").reshape(1, -1)
    cfg = SolverConfig(method="cg", preconditioner="jacobi", tolerance=0.0, rel_tolerance=1e-8, max_iter=500)
    s = CGSolver(cfg)
    s.variant = 19
    x_loop = torch.zeros_like(rhs)
    loops = []
    for _ in range(3):
        x_loop.zero_()
        loops.append(s.solve_arrays(grid, A.diag_store, A.val, rhs, x_loop, symmetric=True)[0].iterations)
    s_cap = CGSolver(cfg)
    s_cap.variant = 19
    s_cap.host_stats = False
    x_cap = torch.zeros_like(rhs)
    stream = torch.cuda.Stream()
    stream.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(stream):
        s_cap.solve_arrays(grid, A.diag_store, A.val, rhs, x_cap, symmetric=True)  # workspace allocation
    torch.cuda.synchronize()
    x_cap.zero_()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=stream):
        s_cap.solve_arrays(grid, A.diag_store, A.val, rhs, x_cap, symmetric=True)
    for _ in range(3):
        x_cap.zero_()
        torch.cuda.synchronize()
        g.replay()
        torch.cuda.synchronize()
    stats = next(iter(s_cap._stats_dev.values())).cpu().numpy()
    assert 0 < loops[0] < 500 and loops[0] == loops[1] == loops[2]
    assert int(stats[0, 2]) == loops[2]
    assert torch.equal(x_loop, x_cap)


def test_inlet_outlet_constraints_track_flow_reversal():
    """inletOutlet on near immersed faces constrains their cells only while
    the faces carry inflow (boundary_ops.py:440-535; the reference's
    tests/integration/fv/test_immersed_dirichlet.py flow-reversal case):
    no cells with outflow everywhere, the oracle's selection with inflow,
    none again after the reversal."""
    import oracle.case as oc
    from tests.golden.oracle_harness import oracle_case

    _, _, grid, algo = device_case("ibplane_io")
    _, _, ocase, oalgo = oracle_case("ibplane_io")
    F, Fb = grid.num_internal_faces, grid.num_domain_bnd_faces
    phi = grid.get_facefield("phi")
    counts = []
    for flux in (1.0, -1.0, 1.0):
        with torch.no_grad():
            phi.store[0, F + Fb:] = flux
        cells, faces, mask = algo.U.table.constraints()
        counts.append(int(cells.numel()))
        assert int(mask.sum()) == counts[-1]
        oalgo.phi.immersed_upper[:] = flux
        oalgo.phi.immersed_lower[:] = flux
        ocells, _ = oc.immersed_dirichlet_constraints(oalgo.U)
        assert np.array_equal(np.sort(to_np(cells).astype(np.int64)), np.sort(ocells))
    assert counts[0] == 0 and counts[1] > 0 and counts[2] == 0


@pytest.mark.parametrize("name", ["cavity8", "duct_oct"])
def test_mixed_bicgstab_reaches_fp64_residual(name):
    """FP32-inner BiCGStab in FP64 refinement (three velocity components in
    one launch): the true FP64 residual of every component below the same
    threshold as the FP64 solve, the solutions within the tolerance band of
    each other, the statistics reporting the inner iterations."""
    from gridfoam_b200.fv import fvm
    from gridfoam_b200.meta.config import SolverConfig
    from gridfoam_b200.solvers.krylov import BiCGSTABSolver

    _, _, grid, algo = device_case(name)
    for _ in range(2):
        algo.step()
    U, phi = algo.U, algo.phi
    A = fvm.div(phi, U) - fvm.laplacian(0.01, U)
    A.diag = A.diag + grid.cell_volumes / 0.01
    g = torch.Generator(device="cuda").manual_seed(3)
    rhs = torch.randn((3, grid.num_cells), dtype=torch.float64, device="cuda", generator=g)
    out = {}
    for prec in ("float64", "float32"):
        cfg = SolverConfig(method="bicgstab", preconditioner="jacobi", tolerance=0.0, rel_tolerance=1e-9,
                           max_iter=2000, inner_precision=prec)
        s = BiCGSTABSolver(cfg)
        x = torch.zeros_like(rhs)
        st = s.solve_arrays(grid, A.diag_store, A.val, rhs, x)
        assert all(c.converged and c.status == "ok" for c in st), [c.status for c in st]
        out[prec] = (x, st)
    x32, st32 = out["float32"]
    x64, st64 = out["float64"]
    r = rhs.t() - A.multiply(x32.t())
    for k in range(3):
        assert float(torch.linalg.vector_norm(r[:, k])) < 1e-9 * st64[k].initial_residual
        assert st32[k].iterations > 0
    assert rel(to_np(x32), to_np(x64)) < 1e-6
