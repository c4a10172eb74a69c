"""SIMPLE / PISO / PIMPLE steps of the CPU oracle.

Restates ``algorithms/simple.py:149-408``, ``algorithms/piso.py:136-326``,
``algorithms/pimple.py:151-454``, ``algorithms/utils/pressure_correction.py``
``:68-363``, ``algorithms/utils/residual.py:12-87`` and
``algorithms/utils/reference_value.py:10-51`` of the reference (paths
relative to ``src/gridfoam``).
"""

from __future__ import annotations

import numpy as np

from oracle.case import (
    Case,
    CellField,
    DirichletBC,
    apply_immersed_dirichlet_values,
    boundary_states,
    fixed_value_mask,
    get_cellfield,
    get_facefield,
    normal_gradient,
    scatter_add,
)
from oracle.ops import (
    LDU,
    adjust_phi,
    compute_phi_hbya,
    correct_flux,
    equation_matrix,
    fvc_ddt_corr,
    fvc_div,
    fvm_ddt,
    fvm_div,
    fvm_laplacian,
    grad,
    linear_internal_face_values,
    sn_grad_single,
)
from oracle.solvers import solve


def needs_reference_value(field: CellField) -> bool:
    """reference_value.py:10-30."""
    return not any(isinstance(bc, DirichletBC) for bc in field.bcs.values())


def set_reference_value(mat: LDU, cell: int, value: float) -> None:
    """reference_value.py:33-51."""
    d = mat.diag[cell]
    mat.diag[cell] += d
    mat.source[cell] += d * value


def field_initial_residual(mat: LDU, field: CellField) -> float:
    """residual.py:12-36."""
    res = mat.multiply(field.data) - mat.source
    return float(np.sqrt(np.sum(res * res)) / (np.sqrt(np.sum(mat.source**2)) + np.finfo(np.float64).eps))


def continuity_residual(phi) -> float:
    """residual.py:39-53."""
    d = fvc_div(phi)
    return float(np.sqrt(np.sum(d * d)))


def _add_boundary_sn_grad_flux(face_field, p: CellField, cell_coeff, sign: float) -> None:
    """pressure_correction.py:197-217."""
    for b, f, ref_v, ref_g, _ in boundary_states(p):
        corr = sign * cell_coeff[b.target_cells] * b.mag_Sf * normal_gradient(p, b, f, ref_v, ref_g)
        blk = face_field.block(b.kind)
        blk[b.face_mask] = blk[b.face_mask] + corr


def _close_fixed_cell_flux(phi, p: CellField) -> None:
    """pressure_correction.py:308-335."""
    case = p.case
    selected = []
    area_sum = np.zeros(case.num_cells)
    for b, f, _, _, _ in boundary_states(p):
        fixed = fixed_value_mask(p, b, f)
        if not fixed.any():
            continue
        area = np.where(fixed, b.mag_Sf, 0.0)
        area_sum += scatter_add(case.num_cells, b.target_cells, area)
        selected.append((b, area))
    if not selected:
        return
    imbalance = fvc_div(phi) * case.cell_volumes
    for b, area in selected:
        total = area_sum[b.target_cells]
        frac = area / np.where(total > 0, total, 1.0)
        blk = phi.block(b.kind)
        blk[b.face_mask] = blk[b.face_mask] - frac * imbalance[b.target_cells]


def solve_pressure_poisson(p, rAtU, div_phi_hbya, cfg, *, n_nonorth, needs_ref, ref_cell, ref_value, final_cfg=None):
    """pressure_correction.py:68-160."""
    case = p.case
    div_source = div_phi_hbya * case.cell_volumes
    mat = stats = init = last_init = None
    for corr in range(n_nonorth + 1):
        mat = -fvm_laplacian(rAtU.data, p)
        mat.source = mat.source - div_source
        if needs_ref:
            set_reference_value(mat, ref_cell, ref_value)
        solve_mat = equation_matrix(p, mat)
        last_init = field_initial_residual(solve_mat, p)
        if init is None:
            init = last_init
        pass_cfg = final_cfg if (final_cfg is not None and corr == n_nonorth) else cfg
        x, stats = solve(solve_mat, solve_mat.source, p.data, pass_cfg)
        p.data = x
    return mat, stats, init, last_init


def simplec_rAtU(UEqn: LDU, rAU: CellField) -> np.ndarray:
    """pressure_correction.py:163-194 (bounded)."""
    inv = 1.0 / rAU.data - UEqn.H1()
    inv = np.maximum(inv, 0.1 / rAU.data)
    return 1.0 / inv


def apply_simplec(phi_hbya, HbyA, p, rAU, rAtU) -> None:
    """pressure_correction.py:229-267."""
    c = p.case
    d_r = rAtU.data - rAU.data
    d_r_f = c.w_s * d_r[c.owner_s] + (1.0 - c.w_s) * d_r[c.neighbour_s]
    phi_hbya.single_data = phi_hbya.single_data + d_r_f * c.mag_Sf_s * sn_grad_single(p)
    _add_boundary_sn_grad_flux(phi_hbya, p, d_r, 1.0)
    HbyA.data = HbyA.data - (rAU.data - rAtU.data)[:, None] * grad(p)


def correct_phi(phi, phi_hbya, p_mat: LDU, p, rAtU) -> None:
    """pressure_correction.py:270-305."""
    phi.single_data = phi_hbya.single_data - (-p_mat).flux(p.data)
    phi.domain_bnd_data = phi_hbya.domain_bnd_data.copy()
    if p.case.num_immersed_faces > 0:
        phi.immersed_upper = phi_hbya.immersed_upper.copy()
        phi.immersed_lower = phi_hbya.immersed_lower.copy()
    _add_boundary_sn_grad_flux(phi, p, rAtU.data, -1.0)
    _close_fixed_cell_flux(phi, p)


def correct_velocity(U, HbyA, rAtU, p) -> None:
    """pressure_correction.py:338-363."""
    U.data = HbyA.data - rAtU.data[:, None] * grad(p)
    apply_immersed_dirichlet_values(U)


class _Base:
    """Shared set-up of the three algorithms (field creation, solvers)."""

    transient = False

    def __init__(self, case: Case):
        self.case = case
        role = "transient" if self.transient else "local"
        self.U = get_cellfield(case, "U", role, (3,))
        self.p = get_cellfield(case, "p", "local", ())
        self.phi = get_facefield(case, "phi")
        self.phi_hbya = get_facefield(case, "phiHbyA")
        self.rAU = get_cellfield(case, "rAU", "local", ())
        self.rAtU = get_cellfield(case, "rAtU", "local", ())
        self.HbyA = get_cellfield(case, "HbyA", "local", (3,))
        self.nu_t = get_cellfield(case, "nu_t", "local", ())
        alg = dict(case.sim["fvSolution"]["algorithm"])
        self.alg = alg
        self.n_nonorth = int(alg.get("nNonOrthogonalCorrectors", 0))
        self.adjust_phi_enabled = bool(case.sim["fvSolution"].get("adjustPhi", True))
        self.p_needs_ref = needs_reference_value(self.p)
        if self.p_needs_ref:
            if alg.get("pRefCell") is None or alg.get("pRefValue") is None:
                raise ValueError("pRefCell and pRefValue are required")
            self.p_ref_cell = int(alg["pRefCell"])
            self.p_ref_value = float(alg["pRefValue"])
        else:
            self.p_ref_cell, self.p_ref_value = None, None
        self.nu = float(case.sim["properties"]["transport"]["nu"])
        self.last_stats: dict = {}
        correct_flux(self.phi, self.U, update_internal=True)
        if self.transient:
            self.U.update_history(reset=True)
            self.phi.update_history(reset=True)

    def nu_eff(self) -> np.ndarray:
        """models/turbulence/laminar.py:29-45."""
        return self.nu + self.nu_t.data

    def solver_cfg(self, name: str, final: bool = False) -> dict:
        """solvers/resolver.py:46-80."""
        solvers = self.case.sim["fvSolution"]["solvers"]
        if final:
            for key in (f"{name}Final", f"{name}_final"):
                if key in solvers:
                    return self.case.solver_config(key)
        return self.case.solver_config(name)

    def _pressure_stage(self, UEqn: LDU, *, ddt: bool, consistent: bool, final: bool):
        """Shared corrector body of piso.py:262-317 / pimple.py:351-434."""
        c = self.case
        self.rAU.data = 1.0 / UEqn.A()
        self.HbyA.data = self.rAU.data[:, None] * UEqn.H(self.U.data)
        corr = None
        if ddt:
            rAU_f = linear_internal_face_values(self.rAU)
            corr = rAU_f * fvc_ddt_corr(self.U, self.phi)
        compute_phi_hbya(self.phi_hbya, self.HbyA, self.U, ddt_corr=corr)
        if self.adjust_phi_enabled:
            adjust_phi(self.phi_hbya, self.U, self.p)
        if consistent:
            self.rAtU.data = simplec_rAtU(UEqn, self.rAU)
            apply_simplec(self.phi_hbya, self.HbyA, self.p, self.rAU, self.rAtU)
        else:
            self.rAtU.data = self.rAU.data
        div = fvc_div(self.phi_hbya)
        mat, stats, init, last = solve_pressure_poisson(
            self.p, self.rAtU, div, self.solver_cfg("p"),
            n_nonorth=self.n_nonorth, needs_ref=self.p_needs_ref,
            ref_cell=self.p_ref_cell, ref_value=self.p_ref_value,
            final_cfg=self.solver_cfg("p", final=final) if ddt else None,
        )
        del c
        return mat, stats, init, last

    def _momentum(self, with_ddt: bool, relax: float | None):
        c = self.case
        UEqn = fvm_div(self.phi, self.U) - fvm_laplacian(self.nu_eff(), self.U)
        if with_ddt:
            UEqn = fvm_ddt(self.U) + fvm_div(self.phi, self.U) - fvm_laplacian(self.nu_eff(), self.U)
        if relax is not None:
            A_old = UEqn.diag.copy()
            UEqn.diag = A_old / relax
            UEqn.source = UEqn.source + (((1.0 - relax) / relax) * A_old)[:, None] * self.U.data
        grad_p = grad(self.p)
        pred = UEqn.with_source(UEqn.source - c.cell_volumes[:, None] * grad_p)
        pred = equation_matrix(self.U, pred)
        return UEqn, pred


class SIMPLE(_Base):
    """algorithms/simple.py:48-408."""

    def __init__(self, case: Case):
        super().__init__(case)
        alg = self.alg
        eqs = alg.get("relaxationFactors", {}).get("equations", {})
        self.alpha_U = float(eqs["U"])
        self.alpha_p = float(eqs["p"])
        self.consistent = bool(alg.get("consistent", False))

    def step(self) -> None:
        UEqn, pred = self._momentum(False, self.alpha_U)
        x, st_u = solve(pred, pred.source, self.U.data, self.solver_cfg("U"))
        self.U.data = x
        UEqn = equation_matrix(self.U, UEqn)
        self.rAU.data = 1.0 / UEqn.A()
        self.HbyA.data = self.rAU.data[:, None] * UEqn.H(self.U.data)
        compute_phi_hbya(self.phi_hbya, self.HbyA, self.U)
        if self.adjust_phi_enabled:
            adjust_phi(self.phi_hbya, self.U, self.p)
        if self.consistent:
            self.rAtU.data = simplec_rAtU(UEqn, self.rAU)
            apply_simplec(self.phi_hbya, self.HbyA, self.p, self.rAU, self.rAtU)
        else:
            self.rAtU.data = self.rAU.data
        p_old = self.p.data.copy()
        div = fvc_div(self.phi_hbya)
        mat, st_p, init, _ = solve_pressure_poisson(
            self.p, self.rAtU, div, self.solver_cfg("p"),
            n_nonorth=self.n_nonorth, needs_ref=self.p_needs_ref,
            ref_cell=self.p_ref_cell, ref_value=self.p_ref_value,
        )
        correct_phi(self.phi, self.phi_hbya, mat, self.p, self.rAtU)
        self.p.data = p_old + self.alpha_p * (self.p.data - p_old)
        apply_immersed_dirichlet_values(self.p)
        correct_velocity(self.U, self.HbyA, self.rAtU, self.p)
        self.last_stats = {"U": st_u, "p": st_p, "p_initial_residual": init}


class PISO(_Base):
    """algorithms/piso.py:44-326."""

    transient = True

    def __init__(self, case: Case):
        super().__init__(case)
        self.n_correctors = int(self.alg.get("nCorrectors", 2))

    def step(self) -> None:
        UEqn, pred = self._momentum(True, None)
        x, st_u = solve(pred, pred.source, self.U.data, self.solver_cfg("U"))
        self.U.data = x
        UEqn = equation_matrix(self.U, UEqn)
        st_p = None
        for i in range(self.n_correctors):
            mat, st_p, _, _ = self._pressure_stage(
                UEqn, ddt=True, consistent=False, final=(i == self.n_correctors - 1)
            )
            correct_phi(self.phi, self.phi_hbya, mat, self.p, self.rAtU)
            correct_velocity(self.U, self.HbyA, self.rAtU, self.p)
        self.U.update_history()
        self.phi.update_history()
        self.last_stats = {"U": st_u, "p": st_p}


class PIMPLE(_Base):
    """algorithms/pimple.py:50-454 (residualControl-free outer loop)."""

    transient = True

    def __init__(self, case: Case):
        super().__init__(case)
        alg = self.alg
        self.n_outer = int(alg.get("nOuterCorrectors", 1))
        self.n_correctors = int(alg.get("nCorrectors", 2))
        self.consistent = bool(alg.get("consistent", False))
        rc = alg.get("residualControl", {}) or {}
        self.residual_control = {
            k: (v if isinstance(v, dict) else {"tolerance": float(v), "rel_tolerance": 0.0})
            for k, v in rc.items()
        }
        self.initial_res: dict = {}
        self.current_res: dict = {}
        self.outer_converged = False

    def _check(self, allow_relative: bool) -> bool:
        """pimple.py:271-288."""
        if not self.residual_control:
            return False
        for name, entry in self.residual_control.items():
            r, r0 = self.current_res.get(name), self.initial_res.get(name)
            if r is None or r0 is None:
                return False
            rel = entry.get("rel_tolerance", 0.0) if allow_relative else 0.0
            if not (r < entry["tolerance"] or (rel > 0.0 and r < rel * r0)):
                return False
        return True

    def _record(self, name: str, value: float) -> None:
        self.initial_res.setdefault(name, value)
        self.current_res[name] = value

    def step(self) -> None:
        self.outer_converged = False
        self.initial_res.clear()
        self.current_res.clear()
        st_u = st_p = None
        for outer in range(self.n_outer):
            final_after = 0 < outer < self.n_outer - 1 and self._check(outer > 1)
            if final_after:
                self.outer_converged = True
            UEqn, pred = self._momentum(True, None)
            if "U" in self.residual_control:
                self._record("U", field_initial_residual(pred, self.U))
            x, st_u = solve(pred, pred.source, self.U.data, self.solver_cfg("U"))
            self.U.data = x
            UEqn = equation_matrix(self.U, UEqn)
            for inner in range(self.n_correctors):
                mat, st_p, init, last = self._pressure_stage(
                    UEqn, ddt=True, consistent=self.consistent,
                    final=(inner == self.n_correctors - 1),
                )
                if "p" in self.residual_control:
                    if inner == 0:
                        self._record("p", init)
                    self.current_res["p"] = last
                correct_phi(self.phi, self.phi_hbya, mat, self.p, self.rAtU)
                correct_velocity(self.U, self.HbyA, self.rAtU, self.p)
            if "phi" in self.residual_control:
                self._record("phi", continuity_residual(self.phi))
            if final_after:
                break
        self.U.update_history()
        self.phi.update_history()
        self.last_stats = {"U": st_u, "p": st_p}


def create_algorithm(case: Case):
    """algorithms/factory.py:9-38."""
    kind = case.sim["fvSolution"]["algorithm"]["type"]
    return {"simple": SIMPLE, "piso": PISO, "pimple": PIMPLE}[kind](case)
