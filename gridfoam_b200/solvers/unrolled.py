"""``grad_mode="unrolled"``: the Krylov iterations themselves, differentiable.

The reference's solvers with ``grad_mode="unrolled"`` run their iterations
with autograd recording (solvers/base.py:111-115), so gradients flow through
every matrix-vector product, dot product and update of the iterations that
ran — including the Jacobi preconditioner built from the diagonal — rather
than through the converged solution's implicit adjoint.  Here the same
iterations run as device tensor algebra on the matrix's differentiable
coefficients (``FvMatrix.autograd_tensors``), one scalar component at a
time, with the reference's stopping tests and BiCGStab restarts
(solvers/cg.py:77-174, solvers/bicgstab.py:76-272, solvers/krylov.py:34-82,
solvers/preconditioners.py:76-96).  The stopping test reads each residual
norm on the host, as the reference does; this mode is for differentiation,
not for speed (the device solvers' default, ``"adjoint"``, is).
"""

from __future__ import annotations

import torch

from gridfoam_b200._lib import GF_BREAKDOWN, GF_MAX_ITER, GF_OK
from gridfoam_b200.meta.config import PreconditionerType
from gridfoam_b200.solvers.base import SolveStats, _StatsBuffer


class _HostStats(_StatsBuffer):
    """Statistics already on the host (``[ncomp, 5]`` rows)."""

    def __init__(self, rows: list[list[float]]):
        self.host = torch.tensor(rows, dtype=torch.float64)
        self._ready = True

    def ready(self) -> bool:
        return True


class _Operator:
    """``A x`` from LDU tensors (fvmatrix.py:292-323), differentiable."""

    def __init__(self, grid, diag, upper, lower):
        self.own = grid.owner
        self.nei = grid.neighbour
        self.diag, self.upper, self.lower = diag, upper, lower

    def __call__(self, x: torch.Tensor) -> torch.Tensor:
        res = self.diag * x
        res = res.index_add(0, self.own, self.upper * x[self.nei])
        return res.index_add(0, self.nei, self.lower * x[self.own])


def _jacobi(diag: torch.Tensor, kind) -> torch.Tensor | None:
    if kind != PreconditionerType.JACOBI:
        return None
    vsmall = torch.finfo(diag.dtype).eps
    return torch.where(diag.abs() < vsmall, torch.ones_like(diag), 1.0 / diag)


def _norm(r: torch.Tensor, linf: bool) -> torch.Tensor:
    return torch.linalg.vector_norm(r.detach(), ord=float("inf") if linf else 2)


def _cg(A, b, x, inv, s) -> tuple[torch.Tensor, list[float]]:
    """solvers/cg.py:77-174 for one component."""
    r = b - A(x)
    r0 = float(_norm(r, s.norm_inf))
    thresh = max(s.atol, s.rtol * r0)
    if r0 < thresh:
        return x, [r0, r0, 0, 1, GF_OK]
    z = r if inv is None else inv * r
    p = z.clone()
    rz_old = torch.sum(r * z)
    final, it = r0, 0
    for it in range(1, s.max_iter + 1):
        Ap = A(p)
        alpha = rz_old / torch.sum(p * Ap)
        x = x + alpha * p
        r = r - alpha * Ap
        final = float(_norm(r, s.norm_inf))
        if final < thresh:
            return x, [r0, final, it, 1, GF_OK]
        z = r if inv is None else inv * r
        rz_new = torch.sum(r * z)
        p = z + p * (rz_new / rz_old)
        rz_old = rz_new
    return x, [r0, final, it, 0, GF_MAX_ITER]


def _bicgstab(A, b, x, inv, s) -> tuple[torch.Tensor, list[float]]:
    """solvers/bicgstab.py:76-272 for one component (right preconditioned,
    restarts on the reference's breakdown tests)."""

    def prec(v):
        return v if inv is None else inv * v

    def tol(u=None, v=None):
        un = 1.0 if u is None else float(torch.linalg.vector_norm(u.detach()))
        vn = 1.0 if v is None else float(torch.linalg.vector_norm(v.detach()))
        return 1e-6 * un * vn

    def restart(r):
        return r.clone(), r.clone(), torch.sum(r * r)

    r = b - A(x)
    r0 = float(_norm(r, s.norm_inf))
    thresh = max(s.atol, s.rtol * r0)
    if r0 < thresh:
        return x, [r0, r0, 0, 1, GF_OK]
    restarts = 0
    r_hat, p, rho_old = restart(r)
    final, it, status = r0, 0, GF_MAX_ITER
    for it in range(1, s.max_iter + 1):
        y = prec(p)
        v = A(y)
        den = torch.sum(r_hat * v)
        if abs(float(den.detach())) <= tol(r_hat, v):
            if restarts >= s.max_restart:
                status = GF_BREAKDOWN
                break
            restarts += 1
            r_hat, p, rho_old = restart(r)
            continue
        alpha = rho_old / den
        s_vec = r - alpha * v
        final = float(_norm(s_vec, s.norm_inf))
        if final < thresh:
            return x + alpha * y, [r0, final, it, 1, GF_OK]
        z = prec(s_vec)
        t = A(z)
        den_w = torch.sum(t * t)
        if abs(float(den_w.detach())) <= tol(t, t):
            if restarts >= s.max_restart:
                status = GF_BREAKDOWN
                break
            restarts += 1
            r_hat, p, rho_old = restart(r)
            continue
        omega = torch.sum(t * s_vec) / den_w
        if abs(float(omega.detach())) <= tol():
            if restarts >= s.max_restart:
                status = GF_BREAKDOWN
                break
            restarts += 1
            r_hat, p, rho_old = restart(r)
            continue
        x = x + alpha * y + omega * z
        r = s_vec - omega * t
        final = float(_norm(r, s.norm_inf))
        if final < thresh:
            return x, [r0, final, it, 1, GF_OK]
        rho_new = torch.sum(r_hat * r)
        if abs(float(rho_new.detach())) <= tol(r_hat, r):
            if restarts >= s.max_restart:
                status = GF_BREAKDOWN
                break
            restarts += 1
            r_hat, p, rho_old = restart(r)
            continue
        beta = (rho_new / rho_old) * (alpha / omega)
        p = r + beta * (p - omega * v)
        rho_old = rho_new
    return x, [r0, final, it, 0, status]


def solve_unrolled(solver, A, rhs: torch.Tensor, x0: torch.Tensor):
    """``A x = rhs`` (``[C, *comp]``) through the differentiable iterations;
    returns ``(solution, stats)`` (solvers/krylov.py:34-82)."""
    diag, upper, lower, _ = A.autograd_tensors()
    op = _Operator(A.grid, diag, upper, lower)
    inv = _jacobi(diag, solver.precon_type)
    body = _bicgstab if solver.bicgstab else _cg
    if rhs.dim() == 1:
        x, row = body(op, rhs, x0, inv, solver)
        return x, (SolveStats(solver.solver_name, _HostStats([row]), 0),)
    cols, rows = [], []
    for k in range(rhs.shape[1]):
        x, row = body(op, rhs[:, k], x0[:, k], inv, solver)
        cols.append(x)
        rows.append(row)
    buf = _HostStats(rows)
    return torch.stack(cols, dim=1), tuple(SolveStats(solver.solver_name, buf, k) for k in range(len(rows)))
