"""Krylov solvers of the CPU oracle.

Restates ``solvers/cg.py:75-174``, ``solvers/bicgstab.py:76-272``,
``solvers/krylov.py:34-82``, ``solvers/preconditioners.py:13-96`` and
``solvers/base.py:140-162`` of the reference (paths relative to
``src/gridfoam``).
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from oracle.ops import LDU


@dataclass
class SolveStats:
    solver: str
    initial_residual: float
    final_residual: float
    iterations: int
    converged: bool


def _norm(v: np.ndarray, order: str) -> float:
    if order == "l_inf":
        return float(np.max(np.abs(v))) if v.size else 0.0
    return float(np.sqrt(np.sum(v * v)))


def jacobi_inv_diag(A: LDU, kind: str) -> np.ndarray | None:
    """preconditioners.py:76-96 (``None`` means the identity)."""
    if kind == "none":
        return None
    eps = np.finfo(np.float64).eps
    return np.where(np.abs(A.diag) < eps, 1.0, 1.0 / np.where(A.diag == 0, 1.0, A.diag))


def _apply(inv_diag, r):
    return r if inv_diag is None else inv_diag * r


def cg_single(A: LDU, b, x, inv_diag, cfg) -> tuple[np.ndarray, SolveStats]:
    """cg.py:237-336."""
    atol, rtol, order = cfg["tolerance"], cfg["rel_tolerance"], cfg["norm_type"]
    r = b - A.multiply(x)
    r0 = _norm(r, order)
    thresh = max(atol, rtol * r0)
    if r0 < thresh:
        return x, SolveStats("cg", r0, r0, 0, True)
    z = _apply(inv_diag, r)
    p = z.copy()
    rz = np.sum(r * z)
    converged = False
    final = r0
    it = 0
    for it in range(1, cfg["max_iter"] + 1):
        Ap = A.multiply(p)
        alpha = rz / np.sum(p * Ap)
        x = x + alpha * p
        r = r - alpha * Ap
        final = _norm(r, order)
        if final < thresh:
            converged = True
            break
        z = _apply(inv_diag, r)
        rz_new = np.sum(r * z)
        p = z + p * (rz_new / rz)
        rz = rz_new
    return x, SolveStats("cg", r0, final, it, converged)


def _btol(x=None, y=None, eps: float = 1e-6) -> float:
    """bicgstab.py:262-272 (always the 2-norm)."""
    xn = 1.0 if x is None else float(np.sqrt(np.sum(x * x)))
    yn = 1.0 if y is None else float(np.sqrt(np.sum(y * y)))
    return eps * xn * yn


def bicgstab_single(A: LDU, b, x, inv_diag, cfg) -> tuple[np.ndarray, SolveStats]:
    """bicgstab.py:76-236."""
    atol, rtol, order = cfg["tolerance"], cfg["rel_tolerance"], cfg["norm_type"]
    max_restart = cfg["max_restart"]
    r = b - A.multiply(x)
    r0 = _norm(r, order)
    thresh = max(atol, rtol * r0)
    if r0 < thresh:
        return x, SolveStats("bicgstab", r0, r0, 0, True)

    def restart(r):
        return r.copy(), r.copy(), np.sum(r * r)

    restarts = 0
    r_hat, p, rho_old = restart(r)
    converged = False
    final = r0
    it = 0
    for it in range(1, cfg["max_iter"] + 1):
        y = _apply(inv_diag, p)
        v = A.multiply(y)
        da = np.sum(r_hat * v)
        if abs(da) <= _btol(r_hat, v):
            if restarts >= max_restart:
                break
            restarts += 1
            r_hat, p, rho_old = restart(r)
            continue
        alpha = rho_old / da
        s = r - alpha * v
        final = _norm(s, order)
        if final < thresh:
            x = x + alpha * y
            converged = True
            break
        z = _apply(inv_diag, s)
        t = A.multiply(z)
        do = np.sum(t * t)
        if abs(do) <= _btol(t, t):
            if restarts >= max_restart:
                break
            restarts += 1
            r_hat, p, rho_old = restart(r)
            continue
        omega = np.sum(t * s) / do
        if abs(omega) <= _btol():
            if restarts >= max_restart:
                break
            restarts += 1
            r_hat, p, rho_old = restart(r)
            continue
        x = x + alpha * y + omega * z
        r = s - omega * t
        final = _norm(r, order)
        if final < thresh:
            converged = True
            break
        rho_new = np.sum(r_hat * r)
        if abs(rho_new) <= _btol(r_hat, r):
            if restarts >= max_restart:
                break
            restarts += 1
            r_hat, p, rho_old = restart(r)
            continue
        beta = (rho_new / rho_old) * (alpha / omega)
        p = r + beta * (p - omega * v)
        rho_old = rho_new
    return x, SolveStats("bicgstab", r0, final, it, converged)


# oracle.native.enable() sets this to the multi-threaded C restatement.
_NATIVE = None


def solve(A: LDU, rhs: np.ndarray, x0: np.ndarray, cfg: dict):
    """krylov.py:34-82 plus the CG/BiCGStab dispatch of solvers/factory.py."""
    if _NATIVE is not None:
        return _NATIVE(A, rhs, x0, cfg)
    method = cfg["method"]
    single = {"cg": cg_single, "bicgstab": bicgstab_single}[method]
    inv_diag = jacobi_inv_diag(A, cfg["preconditioner"])
    if rhs.ndim == 1:
        x, st = single(A, rhs, x0, inv_diag, cfg)
        return x, (st,)
    cols, stats = [], []
    for k in range(rhs.shape[1]):
        x, st = single(A, rhs[:, k], x0[:, k], inv_diag, cfg)
        cols.append(x)
        stats.append(st)
    return np.stack(cols, axis=1), tuple(stats)
