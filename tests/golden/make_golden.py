"""Generate golden fixtures by running the reference gridfoam on CPU.

Run where the reference source tree is available, with ``GRIDFOAM_REF``
naming its ``src`` directory (required; there is no default)::

    GRIDFOAM_REF=<reference>/src python tests/golden/make_golden.py
    GRIDFOAM_REF=<reference>/src python tests/golden/make_golden.py --adjoint
    GRIDFOAM_REF=<reference>/src python tests/golden/make_golden.py --forces
    GRIDFOAM_REF=<reference>/src python tests/golden/make_golden.py --potential
    GRIDFOAM_REF=<reference>/src python tests/golden/make_golden.py --diagnostics
    GRIDFOAM_REF=<reference>/src python tests/golden/make_golden.py --fullsize
    GRIDFOAM_REF=<reference>/src python tests/golden/make_golden.py --downscaled

It imports the unmodified reference package (with the import stubs in
``tests/golden/refshim`` for its absent optional dependencies), builds each
case of ``tests/golden/cases.py`` on the synthetic fluxel-compatible mesh,
runs a few algorithm steps in float64 and dumps the per-step fields and
solver statistics plus operator-level outputs to ``tests/golden/<case>.npz``.
The fixtures are committed; nothing on the GPU side reads the reference.
"""

from __future__ import annotations

import os
import pathlib
import sys

HERE = pathlib.Path(__file__).resolve().parent
REPO = HERE.parents[1]
REF_SRC = os.environ.get("GRIDFOAM_REF")
if not REF_SRC:
    raise SystemExit("set GRIDFOAM_REF to the reference's src directory")
os.environ.setdefault("GRIDFOAM_RUNTIME_TYPE_CHECKS", "0")
sys.path[:0] = [str(HERE / "refshim"), REF_SRC, str(REPO)]

import numpy as np  # noqa: E402
import torch  # noqa: E402

torch.set_num_threads(max(1, os.cpu_count() or 1))

from gridfoam.algorithms.factory import create_algorithm  # noqa: E402
from gridfoam.boundaries import factory as bc_factory  # noqa: E402
from gridfoam.boundaries.basic.dirichlet import DirichletBC  # noqa: E402
from gridfoam.algorithms.utils.reference_value import (  # noqa: E402
    needs_reference_value,
    set_reference_value,
)
from gridfoam.core import field as ref_field  # noqa: E402
from gridfoam.core.equation import equation  # noqa: E402
from gridfoam.core.fvmatrix import FvMatrix  # noqa: E402
from gridfoam.core.grid.axis_projected import AxisProjectedGrid  # noqa: E402
from gridfoam.fv import fvc, fvm  # noqa: E402
from gridfoam.meta.config import SimulatorConfig, SolverConfig  # noqa: E402
from gridfoam.meta.enums import DomainBoundaryPatch  # noqa: E402
from gridfoam.solvers.bicgstab import BiCGSTABSolver  # noqa: E402
from gridfoam.solvers.cg import CGSolver  # noqa: E402

from tests.golden.cases import (  # noqa: E402
    ALL_CASES,
    DIV_SCHEMES,
    STEPS,
    bluff_body_case,
    build_mesh,
    cavity_case,
    cylinder_wake_case,
    pipe_case,
)



class ParabolicInletBC(DirichletBC):
    """Per-face Dirichlet velocity: a parabolic profile on a domain patch."""

    def __init__(self, profile: dict):
        super().__init__(torch.zeros(3, dtype=torch.float64))
        self.profile = profile

    def evaluate(self, field, patch_name, side=None):
        grid = field.grid
        mask = grid.get_domain_bnd_mask(patch_name)
        cells = grid.domain_bnd_owner[mask]
        c = grid.cell_centers[cells]
        cx, cy = self.profile["center"]
        r2 = (c[:, 0] - cx) ** 2 + (c[:, 1] - cy) ** 2
        uz = self.profile["umax"] * torch.clamp(
            1.0 - r2 / self.profile["radius"] ** 2, min=0.0
        )
        ref_v = torch.zeros((cells.shape[0], 3), dtype=grid.dtype)
        ref_v[:, 2] = uz
        fraction = torch.ones(cells.shape[0], dtype=grid.dtype)
        return fraction, ref_v, torch.zeros_like(ref_v)


def make_grid(case: dict) -> AxisProjectedGrid:
    sim = SimulatorConfig.model_validate(case["simulator"])
    mesh = build_mesh(case["mesh"])
    return AxisProjectedGrid(sim, mesh), mesh


def packed(face_field) -> np.ndarray:
    return face_field.pack().detach().numpy().copy()


def stats_array(stats) -> np.ndarray:
    return np.array(
        [
            [s.initial_residual, s.final_residual, s.iterations, float(s.converged)]
            for s in stats
        ]
    )


def reference_algorithm(case: dict):
    """The reference's grid and algorithm for a case definition, with the
    per-face parabolic inlet where the case has one; returns
    ``(grid, mesh, algo, captured)``, ``captured`` receiving each step's
    solver statistics."""
    profile = case["inlet_profile"]
    original = bc_factory.create_boundary_condition

    def patched(bc_config, dtype, device):
        if profile is not None and [str(p) for p in bc_config.patches] == [
            profile["patch"]
        ] and bc_config.type == "dirichlet" and bc_config.value is not None and len(
            np.atleast_1d(bc_config.value)
        ) == 3:
            return ParabolicInletBC(profile)
        return original(bc_config, dtype, device)

    ref_field.boundary_factory.create_boundary_condition = patched
    try:
        grid, mesh = make_grid(case)
        algo = create_algorithm(grid)
    finally:
        ref_field.boundary_factory.create_boundary_condition = original
    captured: list[dict] = []
    orig_finalize = algo._finalize_diagnostics

    def capture(phi, solve_stats):
        captured.append(dict(solve_stats))
        return orig_finalize(phi, solve_stats)

    algo._finalize_diagnostics = capture
    return grid, mesh, algo, captured


# Full-size runs of the benchmark configs (fewer steps than the configs
# name where the reference's CPU run would take hours): key -> (case
# builder, steps, keep the full final fields).
FULLSIZE = {
    "cavity32_300": (lambda: cavity_case(32), 300, True),
    "pipe64x256_20": (lambda: pipe_case(64, 256, 4.0), 20, False),
    "wake256x160x32_10": (lambda: cylinder_wake_case((256, 160, 32)), 10, False),
}

# Downscaled runs of benchmark configs whose full size the reference's CPU
# run cannot reach in reasonable time (same layout as FULLSIZE).
DOWNSCALED = {
    "bluff64x16x12_20": (lambda: bluff_body_case((64, 16, 12)), 20, False),
}


def fullsize_run(key: str) -> dict:
    """Per-step solver iterations, field norms and a fixed sample of cells of
    the reference's own run at a benchmark config's full size; the final
    fields in full where they are small."""
    build, n_steps, keep_full = FULLSIZE[key] if key in FULLSIZE else DOWNSCALED[key]
    case = build()
    grid, mesh, algo, captured = reference_algorithm(case)
    n = int(mesh.n_cells)
    # A seeded random sample: a regular stride can alias with the grid (on
    # the 64-wide pipe every 256th cell sits on the x = 0 wall, outside the
    # immersed pipe, where the velocity is zero).
    sample = np.sort(np.random.default_rng(0).choice(n, size=min(n, 4096), replace=False))
    out: dict[str, np.ndarray] = {"sample_cells": sample, "mesh_n_cells": np.array(n)}
    its_u, its_p, norms = [], [], []
    for step in range(n_steps):
        with torch.no_grad():
            algo.step()
        stats = captured[-1]
        its_u.append([s.iterations for s in stats["U"]])
        its_p.append([s.iterations for s in stats["p"]])
        U, p = algo.U.data.numpy(), algo.p.data.numpy()
        norms.append([np.linalg.norm(U[:, k]) for k in range(3)] + [np.linalg.norm(p)])
        if step in (0, n_steps - 1) or (n_steps <= 20 and step % 5 == 4) or (n_steps > 20 and step % 100 == 99):
            out[f"step{step}_U_sample"] = U[sample].copy()
            out[f"step{step}_p_sample"] = p[sample].copy()
        print(f"  {key} step {step}: U its {its_u[-1]}, p its {its_p[-1]}", flush=True)
    out["its_U"] = np.array(its_u)
    out["its_p"] = np.array(its_p)
    out["norms"] = np.array(norms)
    if keep_full:
        out["final_U"] = algo.U.data.numpy().copy()
        out["final_p"] = algo.p.data.numpy().copy()
    return out


def run_case(name: str, n_steps: int, case: dict | None = None) -> dict:
    case = case if case is not None else ALL_CASES[name]()
    out: dict[str, np.ndarray] = {}
    profile = case["inlet_profile"]
    original = bc_factory.create_boundary_condition

    def patched(bc_config, dtype, device):
        if profile is not None and [str(p) for p in bc_config.patches] == [
            profile["patch"]
        ] and bc_config.type == "dirichlet" and bc_config.value is not None and len(
            np.atleast_1d(bc_config.value)
        ) == 3:
            return ParabolicInletBC(profile)
        return original(bc_config, dtype, device)

    ref_field.boundary_factory.create_boundary_condition = patched
    try:
        grid, mesh = make_grid(case)
        algo = create_algorithm(grid)
    finally:
        ref_field.boundary_factory.create_boundary_condition = original

    captured: list[dict] = []
    orig_finalize = algo._finalize_diagnostics

    def capture(phi, solve_stats):
        captured.append(dict(solve_stats))
        return orig_finalize(phi, solve_stats)

    algo._finalize_diagnostics = capture

    out["init_U"] = algo.U.data.numpy().copy()
    out["init_p"] = algo.p.data.numpy().copy()
    out["init_phi"] = packed(algo.phi)
    for step in range(n_steps):
        with torch.no_grad():
            algo.step()
        out[f"step{step}_U"] = algo.U.data.numpy().copy()
        out[f"step{step}_p"] = algo.p.data.numpy().copy()
        out[f"step{step}_phi"] = packed(algo.phi)
        if step == 0:
            out["step0_HbyA"] = algo.HbyA.data.numpy().copy()
            out["step0_rAtU"] = algo.rAtU.data.numpy().copy()
            out["step0_phiHbyA"] = packed(algo.phi_hbya)
        stats = captured[-1]
        out[f"step{step}_stats_U"] = stats_array(stats["U"])
        out[f"step{step}_stats_p"] = stats_array(stats["p"])
    if hasattr(algo, "_current_residuals"):
        for key, val in getattr(algo, "_current_residuals").items():
            out[f"residual_{key}"] = np.array(val)

    out.update(operator_dumps(grid, algo))
    out["mesh_n_cells"] = np.array(mesh.n_cells)
    out["mesh_checksum"] = np.array(
        [
            float(mesh.internal_faces_owner.sum()),
            float(mesh.cell_centers.sum()),
            float(mesh.ap.dist_owner_to_bnd.sum()),
            float(mesh.ap.is_immersed_face.sum()),
        ]
    )
    return out


def matrix_dict(prefix: str, mat: FvMatrix) -> dict:
    d = {
        f"{prefix}_diag": mat.diag.detach().numpy().copy(),
        f"{prefix}_upper": mat.upper.detach().numpy().copy(),
        f"{prefix}_lower": mat.lower.detach().numpy().copy(),
        f"{prefix}_source": mat.source.detach().numpy().copy(),
    }
    if mat.face_flux_correction is not None:
        d[f"{prefix}_ffc"] = mat.face_flux_correction.detach().numpy().copy()
    return d


def operator_dumps(grid: AxisProjectedGrid, algo) -> dict:
    """Operator outputs evaluated on the final algorithm state."""
    out: dict[str, np.ndarray] = {}
    U, p, phi = algo.U, algo.p, algo.phi
    nu_eff = algo.turbulence.nu_eff()
    with torch.no_grad():
        out.update(matrix_dict("op_lap_U", fvm.laplacian(nu_eff, U)))
        base_cfg = grid.sim_config
        for scheme in DIV_SCHEMES:
            schemes = base_cfg.fvSchemes.model_copy(
                update={"divSchemes": {"default": scheme}}
            )
            grid.sim_config = base_cfg.model_copy(update={"fvSchemes": schemes})
            out.update(matrix_dict(f"op_div_{scheme}", fvm.div(phi, U)))
        grid.sim_config = base_cfg
        out["op_grad_p"] = fvc.grad(p).data.numpy().copy()
        out["op_grad_U"] = fvc.grad(U).data.numpy().copy()
        out["op_interp_U"] = packed(fvc.interpolate(U))
        out["op_div_phi"] = fvc.div(phi).data.numpy().copy()
        out["op_sngrad_p"] = packed(fvc.sn_grad(p))

        # Pressure-type system with a positive cell coefficient field.
        rng = np.random.default_rng(0)
        gamma = torch.from_numpy(0.5 + rng.random(grid.num_cells))
        out["op_gamma"] = gamma.numpy().copy()
        pmat = -fvm.laplacian(gamma, p)
        pmat.source = pmat.source - torch.from_numpy(
            rng.standard_normal(grid.num_cells)
        ) * grid.cell_volumes
        if needs_reference_value(p):
            set_reference_value(pmat, 0, 0.0)
        out.update(matrix_dict("op_pmat", pmat))
        peq = equation(p, pmat)
        out.update(matrix_dict("op_pmat_solve", peq.fv_matrix))
        cg = CGSolver(
            SolverConfig.model_validate(
                {"method": "cg", "preconditioner": "jacobi", "tolerance": 1e-9, "rel_tolerance": 0.0}
            )
        )
        res = cg._solve_primal(peq)
        out["op_cg_x"] = res.solution.numpy().copy()
        out["op_cg_stats"] = stats_array(res.stats)
        out["op_cg_x0"] = p.data.numpy().copy()

        # Momentum-type system: convection + diffusion + ddt-like diagonal.
        umat = fvm.div(phi, U) - fvm.laplacian(nu_eff, U)
        umat.diag = umat.diag + grid.cell_volumes / 0.01
        umat.source = umat.source + torch.from_numpy(
            rng.standard_normal((grid.num_cells, 3))
        ) * grid.cell_volumes[:, None]
        ueq = equation(U, umat)
        out.update(matrix_dict("op_umat_solve", ueq.fv_matrix))
        bi = BiCGSTABSolver(
            SolverConfig.model_validate(
                {"method": "bicgstab", "preconditioner": "jacobi", "tolerance": 1e-10, "rel_tolerance": 0.0}
            )
        )
        res = bi._solve_primal(ueq)
        out["op_bicg_x"] = res.solution.numpy().copy()
        out["op_bicg_stats"] = stats_array(res.stats)
        out["op_bicg_x0"] = U.data.numpy().copy()
        out["op_spmv_U"] = umat.multiply(U.data).numpy().copy()
        out["op_H_U"] = umat.H(U.data).numpy().copy()
        out["op_H1_U"] = umat.H1().numpy().copy()
        out["op_flux_p"] = (-pmat).flux(p.data).numpy().copy()
    return out




ADJOINT_CASES = ("cavity8", "cavity_oct", "cavity_oct_harmonic", "ibplane", "cavity8_unrolled")


def adjoint_case(name: str) -> dict:
    """Reference autograd gradients through assembly and implicit-adjoint
    solves, on the case's state after its golden steps:

    * ``L_p = sum(r * x)``, ``x`` the CG solution of
      ``-laplacian(gamma, p) x = b`` (pressure-type), gradient in ``gamma``;
    * ``L_U = sum(r3 * u)``, ``u`` the BiCGStab solution of
      ``div(phi, U) - laplacian(nu_eff, U) + V/dt``, gradient in ``nu_eff``.
    """
    harmonic = name.endswith("_harmonic")
    unrolled = name.endswith("_unrolled")
    base = name[: -len("_harmonic")] if harmonic else name[: -len("_unrolled")] if unrolled else name
    case = ALL_CASES[base]()
    if harmonic:
        case["simulator"]["fvSchemes"]["laplacianSchemes"] = {"default": "Gauss harmonic corrected"}
    grid, _ = make_grid(case)
    algo = create_algorithm(grid)
    for _ in range(STEPS[base]):
        with torch.no_grad():
            algo.step()
    U, p, phi = algo.U, algo.p, algo.phi
    C = grid.num_cells
    rng = np.random.default_rng(7)
    out: dict[str, np.ndarray] = {}
    if harmonic:
        # the state the gradients are taken at (the steps ran with the
        # harmonic scheme, so the base case's golden steps do not hold it)
        out.update(state_U=U.data.detach().numpy().copy(), state_p=p.data.detach().numpy().copy(),
                   state_phi=packed(phi))
    gamma = torch.from_numpy(0.5 + rng.random(C)).requires_grad_(True)
    src = torch.from_numpy(rng.standard_normal(C))
    r = torch.from_numpy(rng.standard_normal(C))
    pmat = -fvm.laplacian(gamma, p)
    pmat.source = pmat.source - src * grid.cell_volumes
    if needs_reference_value(p):
        set_reference_value(pmat, 0, 0.0)
    with torch.no_grad():
        p.data.zero_()
    cg = CGSolver(SolverConfig.model_validate(
        {"method": "cg", "preconditioner": "jacobi", "tolerance": 1e-13, "rel_tolerance": 0.0, "max_iter": 5000}))
    x = cg.solve(equation(p, pmat)).solution
    (r * x).sum().backward()
    out.update(adj_gamma=gamma.detach().numpy().copy(), adj_src=src.numpy().copy(), adj_r=r.numpy().copy(),
               adj_x=x.detach().numpy().copy(), adj_grad_gamma=gamma.grad.numpy().copy())

    nu = torch.from_numpy(algo.turbulence.nu_eff().detach().numpy() * (0.5 + rng.random(C))).requires_grad_(True)
    usrc = torch.from_numpy(rng.standard_normal((C, 3)))
    r3 = torch.from_numpy(rng.standard_normal((C, 3)))
    umat = fvm.div(phi, U) - fvm.laplacian(nu, U)
    umat.diag = umat.diag + grid.cell_volumes / 0.01
    umat.source = umat.source + usrc * grid.cell_volumes[:, None]
    with torch.no_grad():
        U.data.zero_()
    bi = BiCGSTABSolver(SolverConfig.model_validate(
        {"method": "bicgstab", "preconditioner": "jacobi", "tolerance": 1e-13, "rel_tolerance": 0.0,
         "max_iter": 5000}))
    u = bi.solve(equation(U, umat)).solution
    (r3 * u).sum().backward()
    out.update(adj_nu=nu.detach().numpy().copy(), adj_usrc=usrc.numpy().copy(), adj_r3=r3.numpy().copy(),
               adj_u=u.detach().numpy().copy(), adj_grad_nu=nu.grad.numpy().copy(),
               adj_phi=packed(phi))
    if unrolled:
        # grad_mode="unrolled" (solvers/base.py:111-115): gradients through
        # the iterations that ran, loose tolerances so the difference from
        # the implicit adjoint shows
        g2 = torch.from_numpy(out["adj_gamma"]).requires_grad_(True)
        pm = -fvm.laplacian(g2, p)
        pm.source = pm.source - src * grid.cell_volumes
        if needs_reference_value(p):
            set_reference_value(pm, 0, 0.0)
        with torch.no_grad():
            p.data.zero_()
        cgu = CGSolver(SolverConfig.model_validate(
            {"method": "cg", "preconditioner": "jacobi", "tolerance": 0.0, "rel_tolerance": 1e-3,
             "max_iter": 5000}))
        cgu.grad_mode = "unrolled"
        xu = cgu.solve(equation(p, pm)).solution
        (r * xu).sum().backward()
        n2 = torch.from_numpy(out["adj_nu"]).requires_grad_(True)
        um = fvm.div(phi, U) - fvm.laplacian(n2, U)
        um.diag = um.diag + grid.cell_volumes / 0.01
        um.source = um.source + usrc * grid.cell_volumes[:, None]
        with torch.no_grad():
            U.data.zero_()
        biu = BiCGSTABSolver(SolverConfig.model_validate(
            {"method": "bicgstab", "preconditioner": "jacobi", "tolerance": 0.0, "rel_tolerance": 1e-3,
             "max_iter": 5000}))
        biu.grad_mode = "unrolled"
        uu = biu.solve(equation(U, um)).solution
        (r3 * uu).sum().backward()
        out.update(unr_x=xu.detach().numpy().copy(), unr_grad_gamma=g2.grad.numpy().copy(),
                   unr_u=uu.detach().numpy().copy(), unr_grad_nu=n2.grad.numpy().copy())
    return out


class _StubSurfaceMesh:
    """Stand-in for the graphlow surface mesh the reference's force
    integration reads: one face per AP anchor (immersed face) whose area
    vector is the builder's body-outward unit normal there."""

    class _Geometry:
        def __init__(self, vectors):
            self._v = vectors

        def face_area_vectors(self):
            return self._v

    def __init__(self, normals: np.ndarray):
        self.geometry = self._Geometry(torch.from_numpy(np.ascontiguousarray(normals)))
        self.n_cells = normals.shape[0]
        self.cell_data: dict = {}


FORCE_CASES = ("ibcyl_oct",)


def force_case(name: str) -> dict:
    """The reference's immersed-surface force integral
    (post/forces/integration.py:125-187) on the case's state after its golden
    steps, with the surface-mesh normals taken from the mesh builder."""
    from gridfoam.post.forces.integration import integrate_patch_on_surface_mesh, reset_surface_force_data

    case = ALL_CASES[name]()
    grid, mesh = make_grid(case)
    algo = create_algorithm(grid)
    for _ in range(STEPS[name]):
        with torch.no_grad():
            algo.step()
    grid._mesh_path = "builder-normals"
    grid._surface_mesh_cache = _StubSurfaceMesh(mesh.ap.anchor_normal)
    reset_surface_force_data(grid)
    cofr = torch.tensor([0.5, 0.5, 0.25], dtype=torch.float64)
    nu_eff = algo.turbulence.nu_eff()
    with torch.no_grad():
        force, moment = integrate_patch_on_surface_mesh(
            grid, p=algo.p, U=algo.U, nu_eff=nu_eff, patch_name="cylinder", rho=1.2, center_of_rotation=cofr)
    cd = grid.surface_mesh.cell_data
    return {
        "force": force.numpy().copy(),
        "moment": moment.numpy().copy(),
        "pressure_force": cd["pressure_force"].numpy().copy(),
        "viscous_force": cd["viscous_force"].numpy().copy(),
        "U": algo.U.data.numpy().copy(),
        "p": algo.p.data.numpy().copy(),
        "phi": packed(algo.phi),
        "nu_eff": nu_eff.detach().numpy().copy() if isinstance(nu_eff, torch.Tensor) else np.array(nu_eff),
        "rho": np.array(1.2),
        "cofr": cofr.numpy().copy(),
    }


def potential_run(name: str) -> dict:
    """The reference's potentialFoam-style initialisation
    (pre/potential_flow.py:122-214) and fvc.reconstruct of the initial flux
    on the case's initial fields."""
    from gridfoam.fv.fvc.reconstruct import reconstruct
    from gridfoam.fv.flux import correct_flux
    from gridfoam.pre.potential_flow import PotentialFlow

    from tests.golden.cases import potential_case

    case = potential_case(name)
    grid, _ = make_grid(case)
    pf = PotentialFlow(grid)
    out: dict[str, np.ndarray] = {}
    with torch.no_grad():
        correct_flux(pf.phi, pf.U, update_internal=True)
        out["init_phi"] = packed(pf.phi)
        out["init_U"] = pf.U.data.numpy().copy()
        scratch = ref_field.get_or_create_cellfield(grid, "U_reconstructed", ref_field.FieldRole.LOCAL, (3,))
        out["reconstruct_init"] = reconstruct(pf.phi, scratch).numpy().copy()
        pf.solve()
    out["U"] = pf.U.data.numpy().copy()
    out["phi"] = packed(pf.phi)
    Phi = grid.get_cellfield("Phi")
    if Phi is not None:
        out["Phi"] = Phi.data.numpy().copy()
    return out


# Post-processing settings of the diagnostics fixtures: continuity every
# step, solver statistics every DIAG_SOLVER_INTERVAL steps (and the last).
DIAG_CASES = ("cavity8", "pipe10x20")
DIAG_SOLVER_INTERVAL = 3


class _CaptureUnstructuredGrid:
    """Records what the reference's io/vtu.py hands to pyvista."""

    def __init__(self, cells, cell_types, points):
        self.cells = np.asarray(cells)
        self.cell_types = np.asarray(cell_types)
        self.points = np.asarray(points)
        self.cell_data: dict = {}

    def save(self, path):
        pass


def diagnostics_run(name: str) -> dict:
    """The reference's DiagnosticsCollector (post/diagnostics/collector.py)
    attached to the case's algorithm for its golden steps, and its VTU export
    (io/vtu.py) of the final state through a pyvista stand-in that records
    the points, cells, cell types and cell data it is given."""
    import csv
    import tempfile
    import types

    import gridfoam.io.vtu as ref_vtu
    from gridfoam.meta.config import PostProcessingConfig
    from gridfoam.post.diagnostics import DiagnosticsCollector

    case = ALL_CASES[name]()
    profile = case["inlet_profile"]
    original = bc_factory.create_boundary_condition

    def patched(bc_config, dtype, device):
        if profile is not None and [str(p) for p in bc_config.patches] == [
            profile["patch"]
        ] and bc_config.type == "dirichlet" and bc_config.value is not None and len(
            np.atleast_1d(bc_config.value)
        ) == 3:
            return ParabolicInletBC(profile)
        return original(bc_config, dtype, device)

    ref_field.boundary_factory.create_boundary_condition = patched
    try:
        grid, _ = make_grid(case)
        algo = create_algorithm(grid)
    finally:
        ref_field.boundary_factory.create_boundary_condition = original
    n_steps = STEPS[name]
    dt = float(grid.sim_config.control.deltaT)
    cfg = PostProcessingConfig.model_validate(
        {"continuityError": {"writeInterval": 1}, "solverInfo": {"writeInterval": DIAG_SOLVER_INTERVAL}})
    out: dict[str, np.ndarray] = {}
    with tempfile.TemporaryDirectory() as tmp:
        diag = DiagnosticsCollector.from_config(grid, cfg, pathlib.Path(tmp), n_steps=n_steps, delta_t=dt)
        algo.attach_diagnostics(diag)
        for k in range(n_steps):
            with torch.no_grad():
                algo.step()
            out[f"step{k}_phi"] = packed(algo.phi)
        diag.close()
        with open(pathlib.Path(tmp) / "continuity_error.csv") as fh:
            rows = list(csv.reader(fh))
        out["continuity_header"] = np.array(rows[0])
        out["continuity"] = np.array(rows[1:], dtype=np.float64)
        with open(pathlib.Path(tmp) / "solver_info.csv") as fh:
            rows = list(csv.reader(fh))
        out["solver_info_header"] = np.array(rows[0])
        out["solver_info"] = np.array(rows[1:])
    saved = (ref_vtu.pv.UnstructuredGrid, getattr(ref_vtu.pv, "CellType", None))
    ref_vtu.pv.UnstructuredGrid = _CaptureUnstructuredGrid
    ref_vtu.pv.CellType = types.SimpleNamespace(HEXAHEDRON=12)
    try:
        ug = ref_vtu.save_export_fields_as_vtu(grid, "unused.vtu")
    finally:
        ref_vtu.pv.UnstructuredGrid = saved[0]
        if saved[1] is None:
            del ref_vtu.pv.CellType
        else:
            ref_vtu.pv.CellType = saved[1]
    out["vtu_points"] = ug.points
    out["vtu_cells"] = ug.cells
    out["vtu_cell_types"] = ug.cell_types
    out["vtu_fields"] = np.array(sorted(ug.cell_data))
    for key, val in ug.cell_data.items():
        out[f"vtu_data_{key}"] = np.asarray(val)
    out["delta_t"] = np.array(dt)
    out["n_steps"] = np.array(n_steps)
    return out


def main() -> None:
    args = sys.argv[1:]
    if args and args[0] == "--diagnostics":
        for name in args[1:] or DIAG_CASES:
            data = diagnostics_run(name)
            path = HERE / f"diagnostics_{name}.npz"
            np.savez_compressed(path, **data)
            print(f"diagnostics {name}: {sorted(data)} -> {path} ({path.stat().st_size} B)")
        return
    if args and args[0] == "--potential":
        from tests.golden.cases import POTENTIAL_CASES

        for name in args[1:] or POTENTIAL_CASES:
            data = potential_run(name)
            path = HERE / f"potential_{name}.npz"
            np.savez_compressed(path, **data)
            print(f"potential {name}: {sorted(data)} -> {path} ({path.stat().st_size} B)")
        return
    if args and args[0] == "--forces":
        for name in args[1:] or FORCE_CASES:
            data = force_case(name)
            path = HERE / f"forces_{name}.npz"
            np.savez_compressed(path, **data)
            print(f"forces {name}: {len(data)} arrays -> {path} ({path.stat().st_size} B)")
        return
    if args and args[0] == "--fullsize":
        for key in args[1:] or list(FULLSIZE):
            data = fullsize_run(key)
            path = HERE / f"fullsize_{key}.npz"
            np.savez_compressed(path, **data)
            print(f"fullsize {key}: {len(data)} arrays -> {path} ({path.stat().st_size} B)")
        return
    if args and args[0] == "--downscaled":
        for key in args[1:] or list(DOWNSCALED):
            data = fullsize_run(key)
            path = HERE / f"downscaled_{key}.npz"
            np.savez_compressed(path, **data)
            print(f"downscaled {key}: {len(data)} arrays -> {path} ({path.stat().st_size} B)")
        return
    if args and args[0] == "--gradlinear":
        # The Green-Gauss ('linear') gradient scheme: whole steps and the
        # fvc.grad operator outputs of the reference with gradSchemes
        # default linear.
        from tests.golden.cases import GRAD_LINEAR_CASES, grad_linear_case

        for name in args[1:] or GRAD_LINEAR_CASES:
            data = run_case(name, STEPS[name], case=grad_linear_case(name))
            keep = ("init_", "step", "op_grad", "mesh_", "residual_")
            data = {k: v for k, v in data.items() if k.startswith(keep)}
            path = HERE / f"gradlinear_{name}.npz"
            np.savez_compressed(path, **data)
            print(f"gradlinear {name}: {len(data)} arrays -> {path} ({path.stat().st_size} B)")
        return
    if args and args[0] == "--adjoint":
        for name in args[1:] or ADJOINT_CASES:
            data = adjoint_case(name)
            path = HERE / f"adjoint_{name}.npz"
            np.savez_compressed(path, **data)
            print(f"adjoint {name}: {len(data)} arrays -> {path} ({path.stat().st_size} B)")
        return
    names = args or list(STEPS)
    for name in names:
        data = run_case(name, STEPS[name])
        path = HERE / f"{name}.npz"
        np.savez_compressed(path, **data)
        print(f"{name}: {len(data)} arrays -> {path} ({path.stat().st_size} B)")


if __name__ == "__main__":
    main()
