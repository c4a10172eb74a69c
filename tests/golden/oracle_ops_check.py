"""Evaluate the oracle's operators on a golden end state.

``oracle_operator_outputs(name)`` loads the last stored reference state of a
case into the oracle fields and returns the same operator outputs that
``make_golden.operator_dumps`` recorded from the reference, keyed alike.
"""

from __future__ import annotations

import numpy as np

from oracle import ops, solvers
from oracle.algorithms import needs_reference_value, set_reference_value
from tests.golden.cases import DIV_SCHEMES, STEPS
from tests.golden.oracle_harness import load_golden, oracle_case


def unpack_into(face_field, packed: np.ndarray) -> None:
    n_s = face_field.single_data.shape[0]
    n_b = face_field.domain_bnd_data.shape[0]
    n_i = face_field.immersed_upper.shape[0]
    face_field.single_data = packed[:n_s].copy()
    face_field.domain_bnd_data = packed[n_s : n_s + n_b].copy()
    face_field.immersed_upper = packed[n_s + n_b : n_s + n_b + n_i].copy()
    face_field.immersed_lower = packed[n_s + n_b + n_i :].copy()


def load_state(algo, golden: dict, step: int) -> None:
    algo.U.data = golden[f"step{step}_U"].copy()
    algo.p.data = golden[f"step{step}_p"].copy()
    unpack_into(algo.phi, golden[f"step{step}_phi"])


def _mat(prefix: str, m) -> dict:
    d = {
        f"{prefix}_diag": m.diag,
        f"{prefix}_upper": m.upper,
        f"{prefix}_lower": m.lower,
        f"{prefix}_source": m.source,
    }
    if m.ffc is not None:
        d[f"{prefix}_ffc"] = m.ffc
    return d


def oracle_operator_outputs(name: str) -> tuple[dict, dict]:
    golden = load_golden(name)
    _, _, case, algo = oracle_case(name)
    load_state(algo, golden, STEPS[name] - 1)
    U, p, phi = algo.U, algo.p, algo.phi
    out: dict[str, np.ndarray] = {}
    nu_eff = algo.nu_eff()
    out.update(_mat("op_lap_U", ops.fvm_laplacian(nu_eff, U)))
    base = case.sim.get("fvSchemes", {})
    for scheme in DIV_SCHEMES:
        case.sim["fvSchemes"] = dict(base, divSchemes={"default": scheme})
        out.update(_mat(f"op_div_{scheme}", ops.fvm_div(phi, U)))
    case.sim["fvSchemes"] = base
    out["op_grad_p"] = ops.grad(p)
    out["op_grad_U"] = ops.grad(U)
    out["op_interp_U"] = ops.interpolate_linear(U).pack()
    out["op_div_phi"] = ops.fvc_div(phi)
    out["op_sngrad_p"] = ops.fvc_sn_grad(p).pack()

    rng = np.random.default_rng(0)
    gamma = 0.5 + rng.random(case.num_cells)
    pmat = -ops.fvm_laplacian(gamma, p)
    pmat.source = pmat.source - rng.standard_normal(case.num_cells) * case.cell_volumes
    if needs_reference_value(p):
        set_reference_value(pmat, 0, 0.0)
    out.update(_mat("op_pmat", pmat))
    psolve = ops.equation_matrix(p, pmat)
    out.update(_mat("op_pmat_solve", psolve))
    cfg = {"method": "cg", "preconditioner": "jacobi", "tolerance": 1e-9, "rel_tolerance": 0.0,
           "max_iter": 1000, "norm_type": "l_2", "max_restart": 5}
    x, st = solvers.solve(psolve, psolve.source, p.data, cfg)
    out["op_cg_x"] = x
    out["op_cg_stats"] = np.array([[s.initial_residual, s.final_residual, s.iterations, float(s.converged)] for s in st])

    umat = ops.fvm_div(phi, U) - ops.fvm_laplacian(nu_eff, U)
    umat.diag = umat.diag + case.cell_volumes / 0.01
    umat.source = umat.source + rng.standard_normal((case.num_cells, 3)) * case.cell_volumes[:, None]
    usolve = ops.equation_matrix(U, umat)
    out.update(_mat("op_umat_solve", usolve))
    cfg = dict(cfg, method="bicgstab", tolerance=1e-10)
    x, st = solvers.solve(usolve, usolve.source, U.data, cfg)
    out["op_bicg_x"] = x
    out["op_bicg_stats"] = np.array([[s.initial_residual, s.final_residual, s.iterations, float(s.converged)] for s in st])
    out["op_spmv_U"] = umat.multiply(U.data)
    out["op_H_U"] = umat.H(U.data)
    out["op_H1_U"] = umat.H1()
    out["op_flux_p"] = (-pmat).flux(p.data)
    return out, golden
