"""Implicit adjoint of the device linear solves (solvers/adjoint/*.py).

``attach_implicit_adjoint`` wraps a detached solution ``x = A^-1 b`` in a
``torch.autograd.Function`` whose backward solves the transpose system
``A^T lambda = xbar`` on the GPU (the solver's own ``solve_transpose``) and
turns ``lambda`` into coefficient gradients with the ``gf_adjoint_ldu_grads``
kernel (solvers/adjoint/ldu_grads.py:11-53):

* ``grad diag_c = -sum_k lambda_kc x_kc``,
* ``grad upper_f = -sum_k lambda_kO x_kN``, ``grad lower_f = -sum_k lambda_kN x_kO``,
* ``grad source = lambda``.

The coefficients are the matrix's differentiable tensors
(``FvMatrix.autograd_tensors``), so gradients continue into whatever built
them: torch algebra, or the hand-written reverse kernels of ``fvm.laplacian``
and ``fvm.div``.
"""

from __future__ import annotations

import ctypes

import torch

from gridfoam_b200._lib import call, ptr, stream_ptr


def _cm(t: torch.Tensor, nc: int) -> torch.Tensor:
    """Reference layout [C, *comp] -> component-major [nc][C]."""
    return t.reshape(1, -1).contiguous() if nc == 1 else t.t().contiguous()


class _ImplicitAdjoint(torch.autograd.Function):
    @staticmethod
    def forward(ctx, diag, upper, lower, source, sol, matrix, solve_transpose):  # noqa: ARG004
        ctx.matrix = matrix
        ctx.solve_transpose = solve_transpose
        ctx.save_for_backward(sol)
        return sol.clone()

    @staticmethod
    def backward(ctx, xbar):
        (x,) = ctx.saved_tensors
        A = ctx.matrix
        g = A.grid
        nc = A.num_components
        lam = ctx.solve_transpose(A.as_transpose(), xbar.detach().contiguous())
        gd = torch.empty(g.num_cells, dtype=torch.float64, device=g.device)
        gu = torch.empty(g.num_internal_faces, dtype=torch.float64, device=g.device)
        gl = torch.empty_like(gu)
        call("gf_adjoint_ldu_grads", ctypes.byref(g.cmesh), nc, ptr(_cm(lam, nc)), ptr(_cm(x, nc)), ptr(gd), ptr(gu),
             ptr(gl), stream_ptr())
        return gd, gu, gl, lam.reshape(x.shape), None, None, None


def attach_implicit_adjoint(A, solution: torch.Tensor, *, solve_transpose) -> torch.Tensor:
    """Forward returns ``solution``; backward is the implicit adjoint of
    ``A x = b`` (solvers/adjoint/attach.py:79-115)."""
    diag, upper, lower, source = A.autograd_tensors()
    return _ImplicitAdjoint.apply(diag, upper, lower, source, solution.detach(), A, solve_transpose)
