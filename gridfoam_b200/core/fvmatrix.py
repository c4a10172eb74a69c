"""Finite-volume matrix stored by rows (ELL) on the device.

Public contract of gridfoam's ``FvMatrix`` (``core/fvmatrix.py:16-468``):
``diag`` ``[C]``, ``upper`` / ``lower`` ``[F]`` (LDU face order), ``source``
``[C, *component_shape]``, ``multiply``, ``H``, ``H1``, ``A``, ``flux``,
``with_fixed_values``, ``with_source``, ``as_transpose`` and ``+ - neg``.

Internally the off-diagonal part is the per-cell slot array ``val[W, C]``
(``val[k, c]`` couples row ``c`` with column ``ell_nbr[k, c]``); the LDU
``upper`` / ``lower`` arrays are produced on demand by ``gf_ell_to_ldu``.
Every operation runs on the library's kernels.
"""

from __future__ import annotations

import torch

from gridfoam_b200._lib import call, ptr, stream_ptr
from gridfoam_b200.core.field import CellField, ctypes_ref


def fixed_values_ldu(grid, diag: torch.Tensor, upper: torch.Tensor, lower: torch.Tensor, source: torch.Tensor,
                     cells: torch.Tensor, values: torch.Tensor):
    """core/fvmatrix.py:325-394 on LDU tensors (``source`` and ``values``
    ``[*, ncomp]``): the prescribed cells' couplings move to the right-hand
    side, their rows and columns are removed, each fixed row keeps its
    nonzero diagonal (a zero one becomes -1 if the diagonal sums to a
    negative value, else +1) and its right-hand side is that diagonal times
    the value.  Device tensor algebra, differentiable in every input."""
    own, nei = grid.owner.to(diag.device), grid.neighbour.to(diag.device)
    fixed = torch.zeros(grid.num_cells, dtype=torch.bool, device=diag.device)
    fixed[cells] = True
    prescribed = torch.zeros_like(source).index_copy(0, cells, values.to(source.dtype))
    unit = torch.where(diag.sum() < 0, -torch.ones_like(diag), torch.ones_like(diag))
    cdiag = torch.where(diag != 0, diag, unit)
    d2 = torch.where(fixed, cdiag, diag)
    conn = fixed[own] | fixed[nei]
    up2 = torch.where(conn, torch.zeros_like(upper), upper)
    lo2 = torch.where(conn, torch.zeros_like(lower), lower)
    pn, po = prescribed[nei], prescribed[own]
    src = source.index_add(0, own, -upper[:, None] * pn).index_add(0, nei, -lower[:, None] * po)
    src = src.index_copy(0, cells, cdiag[cells][:, None] * values.to(source.dtype))
    return d2, up2, lo2, src


class FvMatrix:
    def __init__(self, field: CellField, *, _alloc: bool = True):
        self._field = field
        self._grid = field.grid
        g = self._grid
        nc = field.num_components
        if _alloc:
            self.diag_store = torch.zeros(g.num_cells, dtype=torch.float64, device=g.device)
            self.val = torch.zeros(g.ell_width * g.num_cells, dtype=torch.float64, device=g.device)
            self.source_store = torch.zeros((nc, g.num_cells), dtype=torch.float64, device=g.device)
        # Explicit face-flux correction [nc][F] on internal faces (zero off
        # hanging faces), or None: FvMatrix.face_flux_correction.
        self._ffc: torch.Tensor | None = None
        self._ad: dict | None = None

    # ------------------------------------------------------------------
    @property
    def field(self) -> CellField:
        return self._field

    @property
    def grid(self):
        return self._grid

    @property
    def num_components(self) -> int:
        return self._field.num_components

    def _src_view(self, store: torch.Tensor) -> torch.Tensor:
        return store[0] if self._field.component_shape == () else store.t()

    # Differentiable coefficients: a tensor that requires grad, assigned
    # through a setter or produced by a differentiable operator, is kept in
    # ``_ad`` (reference layout: diag [C], upper/lower [F], source
    # [C, *comp]) while its values also go to the device stores.  The getters
    # return it, so torch algebra on the coefficients keeps its graph, and
    # the solvers' implicit adjoint takes its inputs from it.
    def _record(self, key: str, value: torch.Tensor) -> None:
        if isinstance(value, torch.Tensor) and value.requires_grad:
            if self._ad is None:
                self._ad = {}
            self._ad[key] = value
        elif self._ad is not None:
            self._ad.pop(key, None)

    @property
    def requires_grad(self) -> bool:
        return bool(self._ad) and any(t.requires_grad for t in self._ad.values())

    def autograd_tensors(self) -> tuple[torch.Tensor, torch.Tensor, torch.Tensor, torch.Tensor]:
        """``(diag, upper, lower, source)`` in the reference layout, the
        differentiable ones where recorded."""
        ad = self._ad or {}
        upper, lower = (None, None)
        if "upper" not in ad or "lower" not in ad:
            upper, lower = self._ldu()
        return (
            ad.get("diag", self.diag_store),
            ad.get("upper", upper),
            ad.get("lower", lower),
            ad.get("source", self._src_view(self.source_store)),
        )

    @property
    def diag(self) -> torch.Tensor:
        if self._ad and "diag" in self._ad:
            return self._ad["diag"]
        return self.diag_store

    @diag.setter
    def diag(self, value: torch.Tensor) -> None:
        v = torch.as_tensor(value, dtype=torch.float64, device=self._grid.device)
        self.diag_store.copy_(v.detach())
        self._record("diag", v)

    @property
    def source(self) -> torch.Tensor:
        if self._ad and "source" in self._ad:
            return self._ad["source"]
        return self._src_view(self.source_store)

    @source.setter
    def source(self, value: torch.Tensor) -> None:
        value = torch.as_tensor(value, dtype=torch.float64, device=self._grid.device)
        if self._field.component_shape == ():
            self.source_store[0].copy_(value.detach())
        else:
            self.source_store.copy_(value.detach().t())
        self._record("source", value)

    def _ldu(self) -> tuple[torch.Tensor, torch.Tensor]:
        g = self._grid
        upper = torch.empty(g.num_internal_faces, dtype=torch.float64, device=g.device)
        lower = torch.empty_like(upper)
        call("gf_ell_to_ldu", ctypes_ref(g.cmesh), ptr(self.val), ptr(upper), ptr(lower), stream_ptr())
        return upper, lower

    @property
    def upper(self) -> torch.Tensor:
        if self._ad and "upper" in self._ad:
            return self._ad["upper"]
        return self._ldu()[0]

    @upper.setter
    def upper(self, value: torch.Tensor) -> None:
        _, lower = self._ldu()
        v = torch.as_tensor(value, dtype=torch.float64, device=self._grid.device)
        self._set_ldu(v, lower)
        self._record("upper", v)

    @property
    def lower(self) -> torch.Tensor:
        if self._ad and "lower" in self._ad:
            return self._ad["lower"]
        return self._ldu()[1]

    @lower.setter
    def lower(self, value: torch.Tensor) -> None:
        upper, _ = self._ldu()
        v = torch.as_tensor(value, dtype=torch.float64, device=self._grid.device)
        self._set_ldu(upper, v)
        self._record("lower", v)

    def _set_ldu(self, upper: torch.Tensor, lower: torch.Tensor) -> None:
        g = self._grid
        up = upper.detach().contiguous()
        lo = lower.detach().contiguous()
        call("gf_ldu_to_ell", ctypes_ref(g.cmesh), ptr(up), ptr(lo), ptr(self.val), stream_ptr())

    @property
    def face_flux_correction(self):
        """core/fvmatrix.py:137-164: ``[F_single, *comp]`` or None."""
        if self._ffc is None:
            return None
        g = self._grid
        out = self._ffc if g.single_is_identity else self._ffc.index_select(1, g.single_idx)
        return out[0] if self.num_components == 1 else out.t()

    @staticmethod
    def _combine_ffc(x, y, a: float, b: float):
        """``a x + b y`` of two optional corrections (fvmatrix.py:167-180)."""
        if x is None and y is None:
            return None
        if y is None:
            return a * x
        if x is None:
            return b * y
        return a * x + b * y

    # ------------------------------------------------------------------
    def _combine(self, other: "FvMatrix", a: float, b: float) -> "FvMatrix":
        res = FvMatrix(self._field)
        s = stream_ptr()
        for x, y, out in (
            (self.diag_store, other.diag_store, res.diag_store),
            (self.val, other.val, res.val),
            (self.source_store, other.source_store, res.source_store),
        ):
            call("gf_axpby", x.numel(), a, ptr(x), b, ptr(y), ptr(out), s)
        res._ffc = self._combine_ffc(self._ffc, other._ffc, a, b)
        if self.requires_grad or other.requires_grad:
            xs, ys = self.autograd_tensors(), other.autograd_tensors()
            res._ad = {k: a * x + b * y for k, x, y in zip(("diag", "upper", "lower", "source"), xs, ys)}
        return res

    def __add__(self, other: "FvMatrix") -> "FvMatrix":
        return self._combine(other, 1.0, 1.0)

    def __sub__(self, other: "FvMatrix") -> "FvMatrix":
        return self._combine(other, 1.0, -1.0)

    def __neg__(self) -> "FvMatrix":
        return self._combine(self, -1.0, 0.0)

    def clone(self) -> "FvMatrix":
        return self._combine(self, 1.0, 0.0)

    def with_source(self, source: torch.Tensor) -> "FvMatrix":
        res = self.clone()
        res.source = source
        return res

    # ------------------------------------------------------------------
    def A(self) -> torch.Tensor:
        return self.diag_store / self._grid.cell_volumes

    def multiply(self, x: torch.Tensor) -> torch.Tensor:
        """core/fvmatrix.py:292-323 (gf_spmv)."""
        g = self._grid
        nc = self.num_components
        xs = torch.as_tensor(x, dtype=torch.float64, device=g.device)
        xs = xs.reshape(1, -1).contiguous() if nc == 1 else xs.t().contiguous()
        y = torch.empty_like(xs)
        call("gf_spmv", ctypes_ref(g.cmesh), nc, ptr(self.diag_store), ptr(self.val), ptr(xs), ptr(y), stream_ptr())
        return self._src_view(y)

    def _hbya(self, x: torch.Tensor):
        g = self._grid
        nc = self.num_components
        xs = torch.as_tensor(x, dtype=torch.float64, device=g.device)
        xs = xs.reshape(1, -1).contiguous() if nc == 1 else xs.t().contiguous()
        rau = torch.empty(g.num_cells, dtype=torch.float64, device=g.device)
        hbya = torch.empty_like(xs)
        h1 = torch.empty_like(rau)
        call(
            "gf_rau_hbya", ctypes_ref(g.cmesh), nc, ptr(self.diag_store), ptr(self.val),
            ptr(self.source_store), ptr(xs), ptr(rau), ptr(hbya), ptr(h1), stream_ptr(),
        )
        return rau, hbya, h1

    def H(self, x: torch.Tensor) -> torch.Tensor:
        """core/fvmatrix.py:266-290."""
        rau, hbya, _ = self._hbya(x)
        h = hbya / rau
        return self._src_view(h)

    def H1(self) -> torch.Tensor:
        """core/fvmatrix.py:250-264."""
        g = self._grid
        x = torch.zeros((self.num_components, g.num_cells), dtype=torch.float64, device=g.device)
        _, _, h1 = self._hbya(self._src_view(x))
        return h1

    def flux(self, psi: torch.Tensor) -> torch.Tensor:
        """core/fvmatrix.py:424-468 on single-sided faces."""
        g = self._grid
        nc = self.num_components
        ps = torch.as_tensor(psi, dtype=torch.float64, device=g.device)
        ps = ps.reshape(1, -1).contiguous() if nc == 1 else ps.t().contiguous()
        out = torch.empty((nc, g.num_internal_faces), dtype=torch.float64, device=g.device)
        call("gf_matrix_flux", ctypes_ref(g.cmesh), nc, ptr(self.val), ptr(ps), ptr(self._ffc), ptr(out),
             stream_ptr())
        if not g.single_is_identity:
            out = out.index_select(1, g.single_idx)
        return out[0] if nc == 1 else out.t()

    def with_fixed_values(self, cells: torch.Tensor, values: torch.Tensor, *, mask: torch.Tensor | None = None,
                          out: "FvMatrix | None" = None) -> "FvMatrix":
        """core/fvmatrix.py:325-394 (symmetric elimination).  With
        differentiable coefficients or values the eliminated matrix also
        carries the elimination as device tensor algebra, so gradients reach
        the coefficients and the prescribed values."""
        n = int(cells.numel())
        if n == 0:
            return self
        g = self._grid
        nc = self.num_components
        cells32 = cells.to(device=g.device, dtype=torch.int32).contiguous()
        vals = torch.as_tensor(values, dtype=torch.float64, device=g.device).reshape(n, nc).t().contiguous()
        prescribed = torch.zeros((nc, g.num_cells), dtype=torch.float64, device=g.device)
        s = stream_ptr()
        call("gf_set_cell_values", g.num_cells, nc, n, ptr(cells32), ptr(vals), n, ptr(prescribed), s)
        if mask is None:
            mask = torch.zeros(g.num_cells, dtype=torch.uint8, device=g.device)
            mask[cells32.long()] = 1
        res = out if out is not None else FvMatrix(self._field)
        scratch = torch.empty(512, dtype=torch.float64, device=g.device)
        call(
            "gf_fixed_values", ctypes_ref(g.cmesh), nc, ptr(self.diag_store), ptr(self.val), ptr(self.source_store),
            n, None, ptr(prescribed), ptr(mask), ptr(res.diag_store), ptr(res.val), ptr(res.source_store),
            ptr(scratch), s,
        )
        res._ffc = self._ffc
        values_grad = isinstance(values, torch.Tensor) and values.requires_grad
        if torch.is_grad_enabled() and (self.requires_grad or values_grad):
            diag, upper, lower, source = self.autograd_tensors()
            src = source.reshape(g.num_cells, nc)
            vals_t = torch.as_tensor(values, dtype=torch.float64, device=g.device).reshape(n, nc)
            d2, up2, lo2, src2 = fixed_values_ldu(g, diag, upper, lower, src, cells.to(g.device).long(), vals_t)
            res._ad = {"diag": d2, "upper": up2, "lower": lo2, "source": src2.reshape(source.shape)}
        return res

    def as_transpose(self) -> "FvMatrix":
        """core/fvmatrix.py:396-412 (upper and lower swapped)."""
        upper, lower = self._ldu()
        res = FvMatrix(self._field)
        res.diag_store.copy_(self.diag_store)
        res.source_store.copy_(self.source_store)
        res._set_ldu(lower, upper)
        res._ffc = self._ffc
        return res
