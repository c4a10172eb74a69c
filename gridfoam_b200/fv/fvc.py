"""Explicit operators (gridfoam ``fv/fvc``): ``grad``, ``div``,
``interpolate``, ``sn_grad``.  Each wraps one library kernel."""

from __future__ import annotations

import ctypes

import torch

from gridfoam_b200._lib import GfBcAux, call, ptr, stream_ptr
from gridfoam_b200.core.field import (
    CellField,
    FaceField,
    get_or_create_cellfield,
    get_or_create_facefield,
)
from gridfoam_b200.fv import schemes
from gridfoam_b200.meta.config import GradScheme, SnGradScheme


def _eval_state(field: CellField) -> None:
    aux = GfBcAux()
    phi = field.grid.get_facefield("phi")
    if phi is not None:
        aux.phi_bnd = ptr(phi.boundary_store)
    field.evaluate_bc(aux)


def grad(field: CellField) -> CellField:
    """fv/fvc/grad.py:8-34 with the configured scheme: ``leastsquare``
    (fv/kernels/least_squares.py:29-101) or ``linear``, Green-Gauss over the
    hierarchy-aware linear face values (fv/schemes/grad.py:21-43)."""
    grid = field.grid
    _eval_state(field)
    out = get_or_create_cellfield(grid, f"grad({field.name})", field.role, field.component_shape + (3,))
    configured_grad(field, out.store)
    return out


def configured_grad(field: CellField, out: torch.Tensor, face_buf: torch.Tensor | None = None,
                    lsq_buf: torch.Tensor | None = None) -> None:
    """The configured gradient of ``field`` into ``out`` ``[ncomp*3, C]``
    (boundary state must be current).  ``linear``: ``fvc.interpolate`` into
    ``face_buf`` ``[ncomp, F + Nb]`` (its hanging-face correction takes the
    least-squares gradient, in ``lsq_buf``), then the Green-Gauss sum
    (fv/kernels/gauss_gradient.py:15-73).  The buffers are allocated when
    not given."""
    grid = field.grid
    scheme = schemes.grad_scheme(grid.sim_config, field.name)
    t = field.table
    nc = field.num_components
    s = stream_ptr()
    if scheme == GradScheme.LEASTSQUARE:
        call("gf_lsq_grad", ctypes.byref(grid.cmesh), nc, ptr(field.store), ptr(t.kind), ptr(t.psib), ptr(out), s)
        return
    if scheme != GradScheme.LINEAR:
        raise NotImplementedError(f"gradient scheme {scheme}")
    f64 = dict(dtype=torch.float64, device=grid.device)
    if face_buf is None:
        face_buf = torch.empty((nc, grid.num_internal_faces + grid.num_bnd), **f64)
    g = None
    if grid.num_hanging > 0:
        g = lsq_buf if lsq_buf is not None else torch.empty((nc * 3, grid.num_cells), **f64)
        call("gf_lsq_grad", ctypes.byref(grid.cmesh), nc, ptr(field.store), ptr(t.kind), ptr(t.psib), ptr(g), s)
    call("gf_interpolate", ctypes.byref(grid.cmesh), nc, ptr(field.store), ptr(t.kind), ptr(t.psib), ptr(g),
         ptr(face_buf), s)
    call("gf_gauss_grad", ctypes.byref(grid.cmesh), nc, ptr(face_buf), ptr(out), s)


def _hanging_grad(field: CellField) -> torch.Tensor | None:
    """Least-squares gradient for the hanging-face corrections, or None on
    meshes without hanging faces (boundary state must be current)."""
    grid = field.grid
    if grid.num_hanging == 0:
        return None
    out = torch.empty((field.num_components * 3, grid.num_cells), dtype=torch.float64, device=grid.device)
    t = field.table
    call("gf_lsq_grad", ctypes.byref(grid.cmesh), field.num_components, ptr(field.store), ptr(t.kind),
         ptr(t.psib), ptr(out), stream_ptr())
    return out


def div(phi: FaceField) -> CellField:
    """fv/fvc/div.py:15-64."""
    grid = phi.grid
    nc = phi.store.shape[0]
    out = get_or_create_cellfield(grid, f"div({phi.name})", "local", phi.component_shape)
    call("gf_fvc_div", ctypes.byref(grid.cmesh), nc, ptr(phi.store), ptr(out.store), stream_ptr())
    return out


def interpolate(field: CellField) -> FaceField:
    """fv/fvc/interpolate.py:7-26 (hierarchy-aware linear + boundary fill)."""
    grid = field.grid
    _eval_state(field)
    out = get_or_create_facefield(grid, f"{field.name}_f", "local", field.component_shape)
    t = field.table
    g = _hanging_grad(field)
    call("gf_interpolate", ctypes.byref(grid.cmesh), field.num_components, ptr(field.store), ptr(t.kind),
         ptr(t.psib), ptr(g), ptr(out.store), stream_ptr())
    return out


def sn_grad(field: CellField) -> FaceField:
    """fv/fvc/sn_grad.py:16-55."""
    grid = field.grid
    _eval_state(field)
    out = get_or_create_facefield(grid, f"snGrad({field.name})", "local", field.component_shape)
    t = field.table
    corrected = schemes.sn_grad_scheme(grid.sim_config, field.name) == SnGradScheme.CORRECTED
    g = _hanging_grad(field) if corrected else None
    call("gf_sn_grad", ctypes.byref(grid.cmesh), field.num_components, ptr(field.store), ptr(t.kind),
         ptr(t.frac), ptr(t.refv), ptr(t.refg), ptr(g), ptr(out.store), stream_ptr())
    return out


def reconstruct(phi: FaceField, U: CellField) -> torch.Tensor:
    """fv/fvc/reconstruct.py:28-117: sets and returns ``U.data`` [C, 3]."""
    if phi.component_shape != ():
        raise ValueError("phi must be a scalar face flux field.")
    if U.component_shape != (3,):
        raise ValueError("U must be a 3-component velocity field.")
    if phi.grid is not U.grid:
        raise ValueError("phi and U must share the same grid.")
    call("gf_reconstruct", ctypes.byref(U.grid.cmesh), ptr(phi.store), ptr(U.store), stream_ptr())
    return U.data


def face_flux(phi: FaceField, U: CellField) -> None:
    """fv/flux.py:132-162 ``correct_flux(phi, U, update_internal=True)``."""
    _eval_state(U)
    t = U.table
    g = _hanging_grad(U)
    call("gf_face_flux", ctypes.byref(U.grid.cmesh), 0, ptr(U.store), ptr(t.kind), ptr(t.psib), None,
         ptr(g), ptr(phi.store), stream_ptr())


def spmv_check(mat, x: torch.Tensor) -> torch.Tensor:
    return mat.multiply(x)
