"""Implicit operators returning ``FvMatrix`` (gridfoam ``fv/fvm``).

``ddt(field)``, ``div(phi, field)`` and ``laplacian(gamma, field)`` keep the
reference signatures (``fv/fvm/ddt.py:7-40``, ``div.py:15-73``,
``laplacian.py:101-201``).  Each is one ``gf_assemble`` launch; the
algorithms fuse all three terms into a single launch instead.
"""

from __future__ import annotations

import ctypes

import torch

from gridfoam_b200 import _lib
from gridfoam_b200._lib import GfAssembly, GfBcAux, call, ptr, stream_ptr
from gridfoam_b200.core.field import CellField, FaceField
from gridfoam_b200.core.fvmatrix import FvMatrix
from gridfoam_b200.fv import schemes
from gridfoam_b200.meta.config import GradScheme


def _eval_state(field: CellField) -> None:
    aux = GfBcAux()
    phi = field.grid.get_facefield("phi")
    if phi is not None:
        aux.phi_bnd = ptr(phi.boundary_store)
    field.evaluate_bc(aux)


def _base(field: CellField, mat: FvMatrix) -> GfAssembly:
    t = field.table
    a = GfAssembly()
    a.ncomp = field.num_components
    a.psi = ptr(field.store)
    a.bc_kind = ptr(t.kind)
    a.frac = ptr(t.frac)
    a.refv = ptr(t.refv)
    a.refg = ptr(t.refg)
    a.diag = ptr(mat.diag_store)
    a.val = ptr(mat.val)
    a.source = ptr(mat.source_store)
    return a


def _lsq_grad(field: CellField) -> torch.Tensor:
    """Least-squares gradient (the hanging-face corrections always use it)."""
    grad = torch.empty((field.num_components * 3, field.grid.num_cells), dtype=torch.float64,
                       device=field.grid.device)
    t = field.table
    call("gf_lsq_grad", ctypes.byref(field.grid.cmesh), field.num_components, ptr(field.store),
         ptr(t.kind), ptr(t.psib), ptr(grad), stream_ptr())
    return grad


def _cfg_grad(field: CellField, lsq: torch.Tensor | None) -> torch.Tensor:
    """The configured gradient (the TVD limiter's, schemes/div.py:302);
    reuses ``lsq`` when the scheme is least squares."""
    if schemes.grad_scheme(field.grid.sim_config, field.name) == GradScheme.LEASTSQUARE:
        return lsq if lsq is not None else _lsq_grad(field)
    from gridfoam_b200.fv.fvc import configured_grad

    grad = torch.empty((field.num_components * 3, field.grid.num_cells), dtype=torch.float64,
                       device=field.grid.device)
    configured_grad(field, grad, lsq_buf=lsq)
    return grad


def _run(field: CellField, a: GfAssembly) -> None:
    call("gf_assemble", ctypes.byref(field.grid.cmesh), ctypes.byref(a), stream_ptr())


class _AssemblyAdjoint(torch.autograd.Function):
    """Differentiable view of an assembled term: forward returns its
    ``(diag, upper, lower, source)`` in the reference layout; backward runs
    the hand-written reverse kernel (``gf_laplacian_adjoint`` for the
    diffusivity, ``gf_div_adjoint`` for the face flux)."""

    @staticmethod
    def forward(ctx, param, mat, kernel, a, keep):  # noqa: ARG004
        ctx.mat, ctx.kernel, ctx.a, ctx.keep = mat, kernel, a, keep
        ctx.param_shape = param.shape
        upper, lower = mat._ldu()
        return mat.diag_store.clone(), upper, lower, mat._src_view(mat.source_store).clone()

    @staticmethod
    def backward(ctx, gd, gu, gl, gs):
        mat = ctx.mat
        g = mat.grid
        nc = mat.num_components
        z = lambda n: torch.zeros(n, dtype=torch.float64, device=g.device)  # noqa: E731
        gd = z(g.num_cells) if gd is None else gd.contiguous()
        gu = z(g.num_internal_faces) if gu is None else gu.contiguous()
        gl = z(g.num_internal_faces) if gl is None else gl.contiguous()
        if gs is None:
            gs = torch.zeros((nc, g.num_cells), dtype=torch.float64, device=g.device)
        else:
            gs = gs.reshape(1, -1).contiguous() if nc == 1 else gs.t().contiguous()
        out = torch.empty(ctx.param_shape, dtype=torch.float64, device=g.device)
        call(ctx.kernel, ctypes.byref(g.cmesh), ctypes.byref(ctx.a), ptr(gd), ptr(gu), ptr(gl), ptr(gs), ptr(out),
             stream_ptr())
        return out, None, None, None, None


def _frozen_state(field: CellField, a: GfAssembly) -> tuple:
    """Copies of the boundary state and field values the reverse kernels
    read, so later updates of the field do not leak into the backward."""
    t = field.table
    keep = (t.kind.clone(), t.frac.clone(), t.refv.clone(), t.refg.clone(), field.store.clone())
    a.bc_kind, a.frac, a.refv, a.refg, a.psi = (ptr(x) for x in keep)
    return keep


def _attach(mat: FvMatrix, param: torch.Tensor, kernel: str, a: GfAssembly, keep: tuple) -> FvMatrix:
    d, u, lo, src = _AssemblyAdjoint.apply(param, mat, kernel, a, keep)
    mat._ad = {"diag": d, "upper": u, "lower": lo, "source": src}
    return mat


def ddt(field: CellField) -> FvMatrix:
    """fv/fvm/ddt.py:7-40."""
    mat = FvMatrix(field)
    _eval_state(field)
    a = _base(field, mat)
    ca, cb, cc = schemes.ddt_coefficients(field)
    a.use_ddt = 1
    a.ddt_a, a.ddt_b, a.ddt_c, a.dt = ca, cb, cc, field.grid.dt
    a.psi_old = ptr(field.old_store)
    a.psi_older = ptr(field.older_store) if cc != 0.0 else None
    _run(field, a)
    return mat


def div(phi: FaceField, field: CellField) -> FvMatrix:
    """fv/fvm/div.py:15-73 with the configured scheme."""
    if phi.component_shape != ():
        raise ValueError("convection requires scalar face flux")
    mat = FvMatrix(field)
    _eval_state(field)
    scheme = schemes.div_scheme(field.grid.sim_config, phi.name, field.name)
    code = _lib.DIV_CODES[scheme.value]
    grad = lsq = None
    hanging = field.grid.num_hanging > 0
    if hanging and code == _lib.DIV_CODES["linear"]:
        # linear on hanging faces: the least-squares gradient of the offset
        # correction (schemes/div.py:134).
        lsq = _lsq_grad(field)
    if code >= _lib.DIV_CODES["vanleer"]:
        # TVD: the configured gradient, also in its hanging-face offset
        # correction (schemes/div.py:302).
        grad = _cfg_grad(field, None)
    a = _base(field, mat)
    a.div_scheme = code
    a.div_sign = 1.0
    a.phi = ptr(phi.store)
    a.grad_psi = ptr(grad)
    a.grad_lsq = ptr(lsq) if hanging else None
    _run(field, a)
    mat._keep = (grad, lsq)
    if torch.is_grad_enabled() and phi.store.requires_grad:
        # Reverse with respect to the face flux: the transpose face flux.
        keep = _frozen_state(field, a) + (grad, lsq, phi.store.detach().clone())
        a.phi = ptr(keep[-1])
        return _attach(mat, phi.store, "gf_div_adjoint", a, keep)
    return mat


def laplacian(gamma, field: CellField) -> FvMatrix:
    """fv/fvm/laplacian.py:101-201 (uniform or per-cell diffusivity)."""
    grid = field.grid
    mat = FvMatrix(field)
    _eval_state(field)
    scheme = schemes.laplacian_scheme(grid.sim_config, field.name)
    a = _base(field, mat)
    a.lap_sign = 1.0
    a.lap_harmonic = int(scheme in schemes.HARMONIC)
    g_t = None
    if isinstance(gamma, torch.Tensor) and gamma.dim() == 1:
        if gamma.shape[0] != grid.num_cells:
            raise ValueError("diffusivity must have one value per cell")
        g_t = gamma.detach().to(device=grid.device, dtype=torch.float64).contiguous()
        if a.lap_harmonic and not bool(torch.all(torch.isfinite(g_t) & (g_t >= 0))):
            raise ValueError("Harmonic diffusivity must be finite and nonnegative")
        a.gamma = ptr(g_t)
    else:
        a.gamma_scalar = float(gamma)
    grad = None
    if grid.num_hanging > 0 and scheme in schemes.CORRECTED:
        # laplacian.py:162-176: explicit hanging-face skewness correction,
        # also kept as the matrix's face-flux correction.
        grad = _lsq_grad(field)
        a.grad_lsq = ptr(grad)
        a.lap_corrected = 1
        mat._ffc = torch.zeros((field.num_components, grid.num_internal_faces), dtype=torch.float64,
                               device=grid.device)
        a.ffc = ptr(mat._ffc)
    _run(field, a)
    mat._keep = (g_t, grad)
    if torch.is_grad_enabled() and isinstance(gamma, torch.Tensor) and gamma.requires_grad:
        keep = _frozen_state(field, a) + (g_t, grad)
        return _attach(mat, gamma, "gf_laplacian_adjoint", a, keep)
    return mat
