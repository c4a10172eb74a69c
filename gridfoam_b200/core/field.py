"""Cell and face fields stored component-major on the device.

``CellField`` / ``FaceField`` keep gridfoam's public contract
(``core/field.py:120-937``): ``data`` has shape ``[C, *component_shape]``,
face fields expose ``single_data`` / ``domain_bnd_data`` /
``immersed_upper`` / ``immersed_lower`` and ``pack()`` in the packed order
``[single | domain | immersed_upper | immersed_lower]``, and transient
fields keep ``old_data`` / ``older_data``.

Storage is component-major (``[ncomp, C]``; face fields ``[ncomp, F + Nb]``
with all internal faces first, then the boundary faces) so the kernels read
each component coalesced.  ``data`` returns a transposed view of that
storage, so reads and in-place writes through it act on the device buffer.
"""

from __future__ import annotations

from math import prod

import numpy as np
import torch

from gridfoam_b200 import _lib
from gridfoam_b200._lib import GfBc, GfBcAux, GfBcState, call, ptr, stream_ptr
from gridfoam_b200.core.boundary import (
    BoundaryCondition,
    DirichletBC,
    EmptyBC,
    InletOutletBC,
    NeumannBC,
    SlipBC,
    create_boundary_condition,
)
from gridfoam_b200.meta.config import FieldRole


class BoundaryTable:
    """Compiled per-face conditions and the evaluated state of one field."""

    def __init__(self, field: "CellField"):
        grid = field.grid
        nb = grid.num_bnd
        nc = field.num_components
        kind = np.zeros(nb, dtype=np.int8)
        value = np.zeros((nb, nc))
        bc_of_face: list[BoundaryCondition | None] = [None] * nb
        for patch, bc in field.bcs.items():
            faces = grid.patch_faces(patch)
            if isinstance(bc, EmptyBC) or faces.size == 0:
                continue
            kind[faces] = bc.kind
            vals = bc.face_values(faces.size, field.component_shape)
            value[faces] = vals.reshape(faces.size, nc)
            for b in faces:
                bc_of_face[b] = bc
        dev = grid.device
        self.kind_host = kind
        self.bc_of_face = bc_of_face
        self.kind = torch.as_tensor(kind, device=dev)
        self.value = torch.as_tensor(np.ascontiguousarray(value.T), device=dev)
        self.frac = torch.zeros(nb, dtype=torch.float64, device=dev)
        self.refv = torch.zeros((nc, nb), dtype=torch.float64, device=dev)
        self.refg = torch.zeros((nc, nb), dtype=torch.float64, device=dev)
        self.psib = torch.zeros((nc, nb), dtype=torch.float64, device=dev)
        self.cbc = GfBc()
        self.cbc.ncomp = nc
        self.cbc.kind = ptr(self.kind)
        self.cbc.value = ptr(self.value)
        self.cstate = GfBcState(ptr(self.frac), ptr(self.refv), ptr(self.refg), ptr(self.psib))
        self._constraints = None
        self._fixed_faces = None
        # Flux-dependent candidates (inletOutlet on near immersed faces):
        # (cells, distances, faces, dynamic mask, phi name) on the device.
        self._dynamic = None
        self._dynamic_fixed = None
        self.num_constraint_candidates = 0
        self._field = field

    # fv/boundary_ops.py:440-535.  Fixed-value and slip conditions select
    # their faces by geometry alone, so that selection is computed once; an
    # inletOutlet condition on near immersed faces fixes the faces that
    # currently carry inflow (fraction 1, phi < 0), so with one the
    # selection is redone from the current face flux on every call.
    @property
    def dynamic(self) -> bool:
        self.constraints()
        return self._dynamic is not None

    def constraints(self):
        """``(cells[K] int32, faces[K] int32, mask[C] uint8)`` on the device."""
        if self._constraints is None:
            self._constraints = self._build_constraints()
        if self._dynamic is not None:
            return self._select_dynamic()
        return self._constraints

    def _phi_boundary(self, name: str) -> torch.Tensor:
        phi = self._field.grid.get_facefield(name)
        if phi is None:
            raise ValueError(f"Field {name} is not found.")
        return phi.boundary_store[0]

    def _select_dynamic(self):
        """The closest constraining face per cell among the geometric
        candidates and the inflow faces of the flux-dependent ones (ties:
        candidate order, which is the reference's batch order)."""
        cell, dist, face, dyn, phi_name = self._dynamic
        grid = self._field.grid
        C = grid.num_cells
        n = int(cell.numel())
        active = ~dyn | (self._phi_boundary(phi_name)[face] < 0.0)
        inf = torch.full_like(dist, float("inf"))
        d = torch.where(active, dist, inf)
        closest = torch.full((C,), float("inf"), dtype=torch.float64, device=grid.device)
        closest = closest.scatter_reduce(0, cell, d, reduce="amin")
        idx = torch.arange(n, device=grid.device)
        cand = torch.where(active & (d == closest[cell]), idx, torch.full_like(idx, n))
        selected = torch.full((C,), n, dtype=torch.int64, device=grid.device)
        selected = selected.scatter_reduce(0, cell, cand, reduce="amin")
        unique = torch.nonzero(selected < n).reshape(-1)
        mask = torch.zeros(C, dtype=torch.uint8, device=grid.device)
        mask[unique] = 1
        return unique.to(torch.int32), face[selected[unique]].to(torch.int32), mask

    def _build_constraints(self):
        field = self._field
        grid = field.grid
        h = grid.host
        cand_cell, cand_dist, cand_face, cand_dyn = [], [], [], []
        phi_name = None
        for patch, bc in field.bcs.items():
            faces = grid.patch_faces(patch)
            if faces.size == 0 or isinstance(bc, (EmptyBC, NeumannBC)):
                continue
            imm = faces[faces >= grid.num_domain_bnd_faces]
            if imm.size == 0:
                continue
            near = h.bnd_near[imm] != 0
            dyn = False
            if isinstance(bc, DirichletBC) or (isinstance(bc, SlipBC) and field.num_components == 3):
                sel = imm[near]
            elif isinstance(bc, InletOutletBC) and near.any():
                sel = imm[near]
                dyn = True
                phi_name = bc.phi_name
            else:
                sel = imm[:0]
            cand_cell.append(h.bnd_cell[sel])
            cand_dist.append(h.bnd_mag_d[sel])
            cand_face.append(sel)
            cand_dyn.append(np.full(sel.size, dyn))
        if any(d.any() for d in cand_dyn):
            dev = grid.device
            self._dynamic = (
                torch.as_tensor(np.concatenate(cand_cell).astype(np.int64), device=dev),
                torch.as_tensor(np.concatenate(cand_dist), dtype=torch.float64, device=dev),
                torch.as_tensor(np.concatenate(cand_face).astype(np.int64), device=dev),
                torch.as_tensor(np.concatenate(cand_dyn), device=dev),
                phi_name,
            )
        self.num_constraint_candidates = int(sum(c.size for c in cand_cell))
        C = grid.num_cells
        dev = grid.device
        if cand_cell:
            cell = np.concatenate(cand_cell)
            dist = np.concatenate(cand_dist)
            face = np.concatenate(cand_face)
        else:
            cell = dist = face = np.zeros(0)
        mask = np.zeros(C, dtype=np.uint8)
        if cell.size:
            cell = cell.astype(np.int64)
            closest = np.full(C, np.inf)
            np.minimum.at(closest, cell, dist)
            idx = np.arange(cell.size)
            candidate = np.where(dist == closest[cell], idx, cell.size)
            selected = np.full(C, cell.size, dtype=np.int64)
            np.minimum.at(selected, cell, candidate)
            unique = np.nonzero(selected < cell.size)[0]
            faces_sel = face[selected[unique]]
            mask[unique] = 1
        else:
            unique = np.zeros(0, dtype=np.int64)
            faces_sel = np.zeros(0, dtype=np.int64)
        return (
            torch.as_tensor(unique.astype(np.int32), device=dev),
            torch.as_tensor(faces_sel.astype(np.int32), device=dev),
            torch.as_tensor(mask, device=dev),
        )

    def fixed_faces(self):
        """Faces flagged ``near & fraction == 1`` and their area share per cell
        (pressure_correction.py:308-335), as device tensors (recomputed from
        the current flux when an inletOutlet condition has near faces)."""
        if self._fixed_faces is None:
            field = self._field
            grid = field.grid
            h = grid.host
            faces, dyn_faces = [], []
            for patch, bc in field.bcs.items():
                fb = grid.patch_faces(patch)
                if fb.size == 0 or isinstance(bc, EmptyBC):
                    continue
                always_one = isinstance(bc, DirichletBC) or (
                    isinstance(bc, SlipBC) and field.num_components == 3
                )
                near = fb[h.bnd_near[fb] != 0]
                if isinstance(bc, InletOutletBC) and near.size:
                    dyn_faces.append((near, bc.phi_name))
                if not always_one:
                    continue
                faces.append(near)
            faces = np.concatenate(faces) if faces else np.zeros(0, dtype=np.int64)
            if dyn_faces:
                dev = grid.device
                allf = np.concatenate([faces] + [f for f, _ in dyn_faces])
                dyn = np.concatenate([np.zeros(faces.size, dtype=bool)] + [np.ones(f.size, dtype=bool)
                                                                          for f, _ in dyn_faces])
                self._dynamic_fixed = (
                    torch.as_tensor(allf.astype(np.int64), device=dev),
                    torch.as_tensor(dyn, device=dev),
                    torch.as_tensor(h.bnd_mag_sf[allf], dtype=torch.float64, device=dev),
                    torch.as_tensor(h.bnd_cell[allf].astype(np.int64), device=dev),
                    dyn_faces[0][1],
                )
            area = h.bnd_mag_sf[faces]
            cells = h.bnd_cell[faces]
            area_sum = np.bincount(cells, weights=area, minlength=grid.num_cells)
            total = area_sum[cells]
            frac = area / np.where(total > 0, total, 1.0)
            dev = grid.device
            self._fixed_faces = (
                torch.as_tensor(faces.astype(np.int32), device=dev),
                torch.as_tensor(frac, device=dev),
            )
        if self._dynamic_fixed is not None:
            faces, dyn, area, cells, phi_name = self._dynamic_fixed
            grid = self._field.grid
            active = ~dyn | (self._phi_boundary(phi_name)[faces] < 0.0)
            sel = torch.nonzero(active).reshape(-1)
            area, cells = area[sel], cells[sel]
            total = torch.zeros(grid.num_cells, dtype=torch.float64, device=grid.device).index_add(0, cells, area)
            t = total[cells]
            frac = area / torch.where(t > 0, t, torch.ones_like(t))
            return faces[sel].to(torch.int32), frac
        return self._fixed_faces


class CellField:
    """Cell-centred field (core/field.py:120-385)."""

    def __init__(self, grid, name: str, role: FieldRole | str, component_shape: tuple[int, ...], dimension=None):
        self._grid = grid
        self._name = name
        self._role = FieldRole(role)
        self._component_shape = tuple(component_shape)
        if self.num_components not in (1, 3, 9):
            raise ValueError("device fields support scalar, vector and 3x3 tensor components")
        self._store = torch.zeros(
            (self.num_components, grid.num_cells), dtype=torch.float64, device=grid.device
        )
        self._bcs: dict[str, BoundaryCondition] = {}
        self._table: BoundaryTable | None = None
        self._export = False
        self._dimension = dimension
        cond = grid.sim_config.get_field_condition(name)
        if cond is not None:
            self._export = cond.export
            self.reset_data(cond.internal)
            for bc_cfg in cond.iter_bc_configs():
                bc = create_boundary_condition(bc_cfg)
                for patch in bc_cfg.patches:
                    self._bcs[str(patch)] = bc
        grid.register_cellfield(self)
        self._old = None
        self._older = None
        self._previous_dt = None
        self.update_history(reset=True)

    # ------------------------------------------------------------------
    @property
    def grid(self):
        return self._grid

    @property
    def name(self) -> str:
        return self._name

    @property
    def role(self) -> FieldRole:
        return self._role

    @property
    def component_shape(self) -> tuple[int, ...]:
        return self._component_shape

    @property
    def num_components(self) -> int:
        return prod(self._component_shape) if self._component_shape else 1

    @property
    def dimension(self):
        return self._dimension

    @property
    def export(self) -> bool:
        return self._export

    @property
    def bcs(self) -> dict[str, BoundaryCondition]:
        return self._bcs

    def add_boundary_conditions(self, bcs: dict) -> None:
        self._bcs.update({str(k): v for k, v in bcs.items()})
        self._table = None

    @property
    def table(self) -> BoundaryTable:
        if self._table is None:
            self._table = BoundaryTable(self)
        return self._table

    # ------------------------------------------------------------------
    @property
    def store(self) -> torch.Tensor:
        """Component-major device storage ``[ncomp, C]``."""
        return self._store

    def _view(self, store: torch.Tensor) -> torch.Tensor:
        if self._component_shape == ():
            return store[0]
        if len(self._component_shape) == 1:
            return store.t()
        return store.t().reshape(store.shape[1], *self._component_shape)

    @property
    def data(self) -> torch.Tensor:
        return self._view(self._store)

    @data.setter
    def data(self, value: torch.Tensor) -> None:
        value = torch.as_tensor(value, dtype=torch.float64, device=self._grid.device)
        expected = (self._grid.num_cells, *self._component_shape)
        if tuple(value.shape) != expected:
            raise ValueError(f"{self._name}.data: expected shape {expected}, got {tuple(value.shape)}")
        if self._component_shape == ():
            self._store[0].copy_(value)
        else:
            self._store.copy_(value.reshape(value.shape[0], -1).t())

    def reset_data(self, init_value) -> None:
        v = torch.as_tensor(init_value, dtype=torch.float64)
        if tuple(v.shape) != self._component_shape:
            raise ValueError(f"Field {self._name!r} internal value shape {tuple(v.shape)}")
        self._store.copy_(v.reshape(-1, 1).to(self._grid.device).expand_as(self._store))
        if getattr(self, "_old", None) is not None:
            self.update_history(reset=True)

    # core/field.py:241-255
    def update_history(self, *, reset: bool = False) -> None:
        if self._role == FieldRole.TRANSIENT:
            if reset:
                self._older = None
                self._previous_dt = None
            else:
                if self._older is None:
                    self._older = torch.empty_like(self._store)
                self._older.copy_(self._old)
                self._previous_dt = self._grid.dt
            if self._old is None or self._old is self._store:
                self._old = torch.empty_like(self._store)
            self._old.copy_(self._store)
            return
        self._older = None
        self._previous_dt = None
        self._old = self._store

    @property
    def old_store(self) -> torch.Tensor:
        return self._old

    @property
    def older_store(self) -> torch.Tensor | None:
        return self._older

    @property
    def old_data(self) -> torch.Tensor:
        return self._view(self._old)

    @property
    def older_data(self) -> torch.Tensor | None:
        return None if self._older is None else self._view(self._older)

    @property
    def previous_dt(self) -> float | None:
        return self._previous_dt

    # ------------------------------------------------------------------
    def evaluate_bc(self, aux: GfBcAux | None = None) -> BoundaryTable:
        """Evaluate the boundary state on the device (boundary_ops.py:311-326)."""
        t = self.table
        if self._grid.num_bnd:
            call(
                "gf_bc_state",
                ctypes_ref(self._grid.cmesh),
                ctypes_ref(t.cbc),
                ptr(self._store),
                None if aux is None else ctypes_ref(aux),
                ctypes_ref(t.cstate),
                stream_ptr(),
            )
        return t


def ctypes_ref(obj):
    import ctypes

    return ctypes.byref(obj)


class FaceField:
    """Face field (core/field.py:387-799) in the extended ``[F | Nb]`` layout."""

    def __init__(self, grid, name: str, role: FieldRole | str = FieldRole.LOCAL,
                 component_shape: tuple[int, ...] = (), dimension=None, export: bool = True):
        self._grid = grid
        self._name = name
        self._role = FieldRole(role)
        self._component_shape = tuple(component_shape)
        nc = prod(self._component_shape) if self._component_shape else 1
        self._nc = nc
        rows = grid.num_internal_faces + grid.num_bnd
        self._store = torch.zeros((nc, rows), dtype=torch.float64, device=grid.device)
        self._export = export
        self._dimension = dimension
        grid.register_facefield(self)
        self._old = None
        self._older = None
        self._previous_dt = None
        self.update_history(reset=True)

    @property
    def grid(self):
        return self._grid

    @property
    def name(self) -> str:
        return self._name

    @property
    def role(self) -> FieldRole:
        return self._role

    @property
    def component_shape(self) -> tuple[int, ...]:
        return self._component_shape

    @property
    def dimension(self):
        return self._dimension

    @property
    def export(self) -> bool:
        return self._export

    @property
    def store(self) -> torch.Tensor:
        """Component-major storage ``[ncomp, F + Nb]``."""
        return self._store

    def _rows(self, start: int, stop: int) -> torch.Tensor:
        block = self._store[:, start:stop]
        return block[0] if self._component_shape == () else block.t()

    @property
    def num_single_sided(self) -> int:
        return self._grid.num_internal_faces - self._grid.num_immersed_faces

    @property
    def single_data(self) -> torch.Tensor:
        g = self._grid
        if g.single_is_identity:
            return self._rows(0, g.num_internal_faces)
        block = self._store[:, : g.num_internal_faces].index_select(1, g.single_idx)
        return block[0] if self._component_shape == () else block.t()

    @single_data.setter
    def single_data(self, value: torch.Tensor) -> None:
        g = self._grid
        value = torch.as_tensor(value, dtype=torch.float64, device=g.device)
        v = value.reshape(1, -1) if self._component_shape == () else value.t()
        self._store[:, : g.num_internal_faces].index_copy_(1, g.single_idx, v.contiguous())

    @property
    def domain_bnd_data(self) -> torch.Tensor:
        g = self._grid
        f = g.num_internal_faces
        return self._rows(f, f + g.num_domain_bnd_faces)

    @property
    def immersed_upper(self) -> torch.Tensor:
        g = self._grid
        s = g.num_internal_faces + g.num_domain_bnd_faces
        return self._rows(s, s + g.num_immersed_faces)

    @property
    def immersed_lower(self) -> torch.Tensor:
        g = self._grid
        s = g.num_internal_faces + g.num_domain_bnd_faces + g.num_immersed_faces
        return self._rows(s, s + g.num_immersed_faces)

    @property
    def boundary_store(self) -> torch.Tensor:
        """All boundary rows ``[ncomp, Nb]`` (a view)."""
        return self._store[:, self._grid.num_internal_faces :]

    def pack(self) -> torch.Tensor:
        """``[single | domain | immersed_upper | immersed_lower]`` (field.py:709-717)."""
        g = self._grid
        f = g.num_internal_faces
        single = self._store[:, :f] if g.single_is_identity else self._store[:, :f].index_select(1, g.single_idx)
        out = torch.cat([single, self._store[:, f:]], dim=1)
        return out[0] if self._component_shape == () else out.t()

    def packed_n_rows(self) -> int:
        return self.num_single_sided + self._grid.num_bnd

    def unpack(self, packed: torch.Tensor) -> None:
        g = self._grid
        packed = torch.as_tensor(packed, dtype=torch.float64, device=g.device)
        v = packed.reshape(1, -1) if self._component_shape == () else packed.t()
        ns = self.num_single_sided
        self._store[:, : g.num_internal_faces].index_copy_(1, g.single_idx, v[:, :ns].contiguous())
        self._store[:, g.num_internal_faces :].copy_(v[:, ns:])

    # core/field.py:483-495 (internal rows kept; single-sided subset read)
    def update_history(self, *, reset: bool = False) -> None:
        f = self._grid.num_internal_faces
        if reset:
            self._older = None
            self._previous_dt = None
        else:
            if self._older is None:
                self._older = torch.empty((self._nc, f), dtype=torch.float64, device=self._grid.device)
            self._older.copy_(self._old)
            self._previous_dt = self._grid.dt
        if self._old is None:
            self._old = torch.empty((self._nc, f), dtype=torch.float64, device=self._grid.device)
        self._old.copy_(self._store[:, :f])

    @property
    def old_store(self) -> torch.Tensor:
        return self._old

    @property
    def older_store(self) -> torch.Tensor | None:
        return self._older

    @property
    def old_single_data(self) -> torch.Tensor:
        g = self._grid
        b = self._old if g.single_is_identity else self._old.index_select(1, g.single_idx)
        return b[0] if self._component_shape == () else b.t()

    @property
    def older_single_data(self) -> torch.Tensor | None:
        if self._older is None:
            return None
        g = self._grid
        b = self._older if g.single_is_identity else self._older.index_select(1, g.single_idx)
        return b[0] if self._component_shape == () else b.t()

    @property
    def previous_dt(self) -> float | None:
        return self._previous_dt


def get_or_create_cellfield(grid, name: str, role, component_shape, dimension=None) -> CellField:
    """core/field.py:823-877."""
    field = grid.get_cellfield(name)
    if field is None:
        field = CellField(grid, name, role, component_shape, dimension)
    if field.role != FieldRole(role):
        raise AssertionError(f"field {name!r} exists with role {field.role}")
    if field.component_shape != tuple(component_shape):
        raise ValueError(f"Field {name!r}: component_shape {field.component_shape}, expected {component_shape}")
    return field


def get_or_create_facefield(grid, name: str, role, component_shape, dimension=None, export: bool = True) -> FaceField:
    """core/field.py:880-937."""
    field = grid.get_facefield(name)
    if field is None:
        field = FaceField(grid, name, role, component_shape, dimension, export)
    return field
