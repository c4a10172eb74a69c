"""Grid geometry, fields and boundary conditions of the CPU oracle.

Restates (paths relative to the reference's ``src/gridfoam``):

* ``core/grid/axis_projected.py:97-211, 715-811`` - topology, geometry and
  the axis-projected IBM payload;
* ``fv/kernels/face_geometry.py:107-262`` - cached face geometry, hanging
  faces and the least-squares normal-matrix inverse;
* ``core/field.py:120-820`` - cell/face fields with time history;
* ``boundaries/**`` and ``fv/boundary_ops.py:99-593`` - value-fraction
  boundary conditions, boundary batches and states, immersed Dirichlet
  constraints.
"""

from __future__ import annotations

import re
from dataclasses import dataclass

import numpy as np

DOMAIN_PATCHES = {
    "x_minus": 0,
    "x_plus": 1,
    "y_minus": 2,
    "y_plus": 3,
    "z_minus": 4,
    "z_plus": 5,
}

SOLVER_DEFAULTS = {
    "preconditioner": "none",
    "tolerance": 1e-6,
    "rel_tolerance": 1e-6,
    "max_iter": 1000,
    "norm_type": "l_2",
    "max_restart": 5,
}


# oracle.native.enable() sets this to the multi-threaded C path (same sums,
# same order).
_NATIVE_SCATTER = None


def scatter_add(n: int, index: np.ndarray, values: np.ndarray) -> np.ndarray:
    """``torch.zeros(n, *comp).index_add_(0, index, values)``."""
    if _NATIVE_SCATTER is not None:
        return _NATIVE_SCATTER(n, index, values, _scatter_add_numpy)
    return _scatter_add_numpy(n, index, values)


def _scatter_add_numpy(n: int, index: np.ndarray, values: np.ndarray) -> np.ndarray:
    values = np.asarray(values, dtype=np.float64)
    if values.ndim == 1:
        return np.bincount(index, weights=values, minlength=n)[:n]
    flat = values.reshape(values.shape[0], -1)
    out = np.empty((n, flat.shape[1]))
    for c in range(flat.shape[1]):
        out[:, c] = np.bincount(index, weights=flat[:, c], minlength=n)[:n]
    return out.reshape((n,) + values.shape[1:])


def bview(v: np.ndarray, like: np.ndarray) -> np.ndarray:
    """``core/shapes.py`` ``broadcast_entity``: append unit component axes."""
    return v.reshape(v.shape + (1,) * (like.ndim - v.ndim))


class Case:
    """Mesh + simulator configuration, the oracle's ``AxisProjectedGrid``."""

    def __init__(self, mesh, simulator: dict):
        self.sim = simulator
        self._load_topology(mesh)
        self._load_ap_payload(mesh)
        self._build_face_geometry()
        self.cellfields: dict[str, CellField] = {}
        self.facefields: dict[str, FaceField] = {}

    # ------------------------------------------------------------------
    # axis_projected.py:97-161 and 715-811
    # ------------------------------------------------------------------
    def _load_topology(self, mesh) -> None:
        self.num_cells = int(mesh.n_cells)
        self.owner = np.asarray(mesh.internal_faces_owner, dtype=np.int64)
        self.neighbour = np.asarray(mesh.internal_faces_neighbour, dtype=np.int64)
        self.axis = np.asarray(mesh.internal_faces_axis, dtype=np.int64)
        self.num_internal_faces = self.owner.shape[0]
        self.domain_bnd_owner = np.asarray(mesh.domain_bnd_faces_owner, dtype=np.int64)
        self.domain_bnd_dir_id = np.asarray(mesh.domain_bnd_faces_dir, dtype=np.int64)
        self.num_domain_bnd_faces = self.domain_bnd_owner.shape[0]
        self.patch_name_to_id = dict(mesh.patch_name_to_id)
        self.cell_centers = np.asarray(mesh.cell_centers, dtype=np.float64)
        self.cell_sizes = np.asarray(mesh.cell_sizes, dtype=np.float64)
        self.cell_volumes = np.prod(self.cell_sizes, axis=1)

        c_own = self.cell_centers[self.owner]
        c_nei = self.cell_centers[self.neighbour]
        s_own = self.cell_sizes[self.owner]
        s_nei = self.cell_sizes[self.neighbour]
        face_min = np.maximum(c_own - s_own / 2.0, c_nei - s_nei / 2.0)
        face_max = np.minimum(c_own + s_own / 2.0, c_nei + s_nei / 2.0)
        self.face_centers = (face_min + face_max) / 2.0

        min_sizes = np.minimum(s_own, s_nei)
        fidx = np.arange(self.num_internal_faces)
        area = np.prod(min_sizes, axis=1) / min_sizes[fidx, self.axis]
        self.Sf = np.zeros((self.num_internal_faces, 3))
        self.Sf[fidx, self.axis] = area

        bidx = np.arange(self.num_domain_bnd_faces)
        b_axis = self.domain_bnd_dir_id // 2
        sign = 2.0 * (self.domain_bnd_dir_id % 2) - 1.0
        normals = np.zeros((self.num_domain_bnd_faces, 3))
        normals[bidx, b_axis] = sign
        bc = self.cell_centers[self.domain_bnd_owner]
        bs = self.cell_sizes[self.domain_bnd_owner]
        self.domain_bnd_face_centers = bc + 0.5 * bs * normals
        b_area = sign * np.prod(bs, axis=1) / bs[bidx, b_axis]
        self.domain_bnd_Sf = np.zeros((self.num_domain_bnd_faces, 3))
        self.domain_bnd_Sf[bidx, b_axis] = b_area

    # axis_projected.py:163-211
    def _load_ap_payload(self, mesh) -> None:
        ap = mesh.ap
        self.ap_is_immersed_faces = np.asarray(ap.is_immersed_face, dtype=bool)
        self.num_immersed_faces = int(self.ap_is_immersed_faces.sum())
        self.ap_owner_bnd_patch_id = np.asarray(ap.owner_bnd_patch_id, dtype=np.int64)
        self.ap_neighbour_bnd_patch_id = np.asarray(ap.neighbour_bnd_patch_id, dtype=np.int64)
        self.ap_dist_owner_to_bnd = np.asarray(ap.dist_owner_to_bnd, dtype=np.float64).reshape(-1)
        self.ap_owner_near_boundary = np.asarray(ap.owner_near_boundary, dtype=bool)
        self.ap_dist_neighbour_to_bnd = np.asarray(ap.dist_neighbour_to_bnd, dtype=np.float64).reshape(-1)
        self.ap_neighbour_near_boundary = np.asarray(ap.neighbour_near_boundary, dtype=bool)

    # ------------------------------------------------------------------
    # fv/kernels/face_geometry.py:107-188
    # ------------------------------------------------------------------
    def _build_face_geometry(self) -> None:
        c = self.cell_centers
        own, nei, ax = self.owner, self.neighbour, self.axis
        fidx = np.arange(self.num_internal_faces)
        d_all = c[nei] - c[own]
        d_fN = c[nei] - self.face_centers
        d_n = np.abs(d_all[fidx, ax])
        self.w_all = np.abs(d_fN[fidx, ax]) / d_n
        self.mag_Sf_all = np.linalg.norm(self.Sf, axis=1)
        self.delta_coeffs_all = 1.0 / d_n

        self.single_mask = ~self.ap_is_immersed_faces
        self.single_idx = np.nonzero(self.single_mask)[0]
        s = self.single_idx
        self.owner_s = own[s]
        self.neighbour_s = nei[s]
        self.w_s = self.w_all[s]
        self.Sf_s = self.Sf[s]
        self.mag_Sf_s = self.mag_Sf_all[s]
        self.delta_coeffs_s = self.delta_coeffs_all[s]
        axis_s = ax[s]
        fc_s = self.face_centers[s]

        centroid = self.w_s[:, None] * c[self.owner_s] + (1.0 - self.w_s)[:, None] * c[self.neighbour_s]
        offset = fc_s - centroid
        tol = 1.0e-8 * float(self.cell_sizes.min())
        hang_mask = np.linalg.norm(offset, axis=1) > tol
        self.hang_idx = np.nonzero(hang_mask)[0]
        self.hang_offset = offset[self.hang_idx]
        h = self.hang_idx
        move_O = fc_s[h] - c[self.owner_s[h]]
        move_N = fc_s[h] - c[self.neighbour_s[h]]
        move_O[np.arange(h.shape[0]), axis_s[h]] = 0.0
        move_N[np.arange(h.shape[0]), axis_s[h]] = 0.0
        self.hang_move_O = move_O
        self.hang_move_N = move_N
        hcm = np.zeros(self.num_cells, dtype=bool)
        hcm[self.owner_s[h]] = True
        hcm[self.neighbour_s[h]] = True
        self.hang_cell_mask = hcm
        self.lsq_face_idx = np.nonzero(hcm[self.owner_s] | hcm[self.neighbour_s])[0]
        self.lsq_owner = self.owner_s[self.lsq_face_idx]
        self.lsq_neighbour = self.neighbour_s[self.lsq_face_idx]
        self.lsq_ata_inv = self._build_lsq_ata_inv()

    @property
    def num_single(self) -> int:
        return int(self.single_idx.shape[0])

    @property
    def num_hanging(self) -> int:
        return int(self.hang_idx.shape[0])

    # face_geometry.py:191-262
    @staticmethod
    def _lsq_outer(d: np.ndarray) -> np.ndarray:
        d2 = np.sum(d * d, axis=1)
        w2 = 1.0 / np.where(d2 > 0, d2, 1.0)
        return w2[:, None, None] * d[:, :, None] * d[:, None, :]

    def boundary_lsq_vectors(self) -> list[tuple[np.ndarray, np.ndarray]]:
        blocks = [
            (
                self.domain_bnd_owner,
                self.domain_bnd_face_centers - self.cell_centers[self.domain_bnd_owner],
            )
        ]
        if self.num_immersed_faces > 0:
            imm = self.ap_is_immersed_faces
            Sf = self.Sf[imm]
            n_hat = Sf / np.linalg.norm(Sf, axis=1)[:, None]
            blocks.append((self.owner[imm], self.ap_dist_owner_to_bnd[:, None] * n_hat))
            blocks.append((self.neighbour[imm], self.ap_dist_neighbour_to_bnd[:, None] * (-n_hat)))
        return blocks

    def _build_lsq_ata_inv(self) -> np.ndarray:
        c = self.cell_centers
        d = c[self.neighbour_s] - c[self.owner_s]
        outer = self._lsq_outer(d).reshape(-1, 9)
        ata = scatter_add(self.num_cells, self.owner_s, outer)
        ata += scatter_add(self.num_cells, self.neighbour_s, outer)
        for cells, d_bnd in self.boundary_lsq_vectors():
            ata += scatter_add(self.num_cells, cells, self._lsq_outer(d_bnd).reshape(-1, 9))
        return np.linalg.pinv(ata.reshape(-1, 3, 3), hermitian=True)

    # ------------------------------------------------------------------
    # configuration lookups (fv/schemes/selection.py:319-396)
    # ------------------------------------------------------------------
    @property
    def dt(self) -> float:
        return float(self.sim["control"]["deltaT"])

    def scheme(self, group: str, key: str, default: str) -> str:
        table = self.sim.get("fvSchemes", {}).get(group)
        if not table:
            return default
        table = {re.sub(r"\s*,\s*", ", ", k): v for k, v in table.items()}
        value = table.get(key, table.get("default"))
        return default if value is None else value

    def domain_bnd_mask(self, patch: str) -> np.ndarray:
        return self.domain_bnd_dir_id == DOMAIN_PATCHES[patch]

    def solver_config(self, name: str) -> dict:
        cfg = dict(SOLVER_DEFAULTS)
        cfg.update(self.sim["fvSolution"]["solvers"][name])
        return cfg


# ----------------------------------------------------------------------
# Fields (core/field.py)
# ----------------------------------------------------------------------
class CellField:
    """core/field.py:120-385 (data, old/older history, bcs)."""

    def __init__(self, case: Case, name: str, role: str, comp: tuple[int, ...]):
        self.case = case
        self.name = name
        self.role = role
        self.comp = comp
        self.data = np.zeros((case.num_cells,) + comp)
        self.bcs: dict[str, BoundaryCondition] = {}
        cond = case.sim.get("conditions", {}).get(name)
        if cond is not None:
            self.data[:] = np.asarray(cond["internal"], dtype=np.float64)
            for bc_cfg in cond["boundary"].values():
                bc = make_bc(bc_cfg)
                for patch in bc_cfg["patches"]:
                    self.bcs[patch] = bc
        case.cellfields[name] = self
        self.update_history(reset=True)

    # field.py:241-255
    def update_history(self, *, reset: bool = False) -> None:
        if self.role == "transient":
            self.older_data = None if reset else self.old_data
            self.previous_dt = None if reset else self.case.dt
            self.old_data = self.data.copy()
            return
        self.older_data = None
        self.previous_dt = None
        self.old_data = self.data


class FaceField:
    """core/field.py:387-799 packed ``[single | domain | imm_upper | imm_lower]``."""

    def __init__(self, case: Case, name: str, comp: tuple[int, ...] = ()):
        self.case = case
        self.name = name
        self.comp = comp
        self.single_data = np.zeros((case.num_single,) + comp)
        self.domain_bnd_data = np.zeros((case.num_domain_bnd_faces,) + comp)
        self.immersed_upper = np.zeros((case.num_immersed_faces,) + comp)
        self.immersed_lower = np.zeros((case.num_immersed_faces,) + comp)
        case.facefields[name] = self
        self.update_history(reset=True)

    # field.py:483-495
    def update_history(self, *, reset: bool = False) -> None:
        self.older_single_data = None if reset else self.old_single_data
        self.previous_dt = None if reset else self.case.dt
        self.old_single_data = self.single_data.copy()

    def pack(self) -> np.ndarray:
        return np.concatenate(
            [self.single_data, self.domain_bnd_data, self.immersed_upper, self.immersed_lower]
        )

    def block(self, kind: str) -> np.ndarray:
        return {
            "domain": self.domain_bnd_data,
            "upper": self.immersed_upper,
            "lower": self.immersed_lower,
        }[kind]


def get_cellfield(case: Case, name: str, role: str, comp: tuple[int, ...]) -> CellField:
    """field.py:823-877 get-or-create."""
    f = case.cellfields.get(name)
    return f if f is not None else CellField(case, name, role, comp)


def get_facefield(case: Case, name: str, comp: tuple[int, ...] = ()) -> FaceField:
    """field.py:880-937 get-or-create."""
    f = case.facefields.get(name)
    return f if f is not None else FaceField(case, name, comp)


# ----------------------------------------------------------------------
# Boundary conditions (boundaries/**), value-fraction form
# ----------------------------------------------------------------------
class BoundaryCondition:
    type = "base"
    assignable = True

    def evaluate(self, field: CellField, patch: str, side: str):
        raise NotImplementedError


def _patch_faces(case: Case, patch: str, side: str) -> np.ndarray:
    """boundaries/utils.py:495-545: mask over the patch's storage block."""
    if patch in DOMAIN_PATCHES:
        return case.domain_bnd_mask(patch)
    pid = case.patch_name_to_id.get(patch)
    if pid is None:
        return np.zeros(case.num_immersed_faces, dtype=bool)
    ids = case.ap_owner_bnd_patch_id if side == "upper" else case.ap_neighbour_bnd_patch_id
    return ids == pid


class DirichletBC(BoundaryCondition):
    """boundaries/basic/dirichlet.py:35-73 (a per-face value array is allowed)."""

    type = "dirichlet"
    assignable = False

    def __init__(self, value):
        self.value = np.asarray(value, dtype=np.float64)

    def evaluate(self, field, patch, side):
        n = int(_patch_faces(field.case, patch, side).sum())
        ref_v = np.ones((n,) + field.comp) * self.value
        return np.ones(n), ref_v, np.zeros_like(ref_v)


class NeumannBC(BoundaryCondition):
    """boundaries/basic/neumann.py:35-73."""

    type = "neumann"

    def __init__(self, grad_value):
        self.grad_value = np.asarray(grad_value, dtype=np.float64)

    def evaluate(self, field, patch, side):
        n = int(_patch_faces(field.case, patch, side).sum())
        ref_g = np.ones((n,) + field.comp) * self.grad_value
        return np.zeros(n), np.zeros((n,) + field.comp), ref_g


class EmptyBC(BoundaryCondition):
    """boundaries/basic/empty.py:20-51."""

    type = "empty"

    def evaluate(self, field, patch, side):
        n = int(_patch_faces(field.case, patch, side).sum())
        z = np.zeros((n,) + field.comp)
        return np.zeros(n), z, z.copy()


class SlipBC(BoundaryCondition):
    """boundaries/basic/slip.py:40-101."""

    type = "slip"
    assignable = False

    def evaluate(self, field, patch, side):
        case = field.case
        mask = _patch_faces(case, patch, side)
        n = int(mask.sum())
        fraction = np.ones(n)
        ref_v = np.zeros((n,) + field.comp)
        ref_g = np.zeros((n,) + field.comp)
        if field.comp == ():
            return np.zeros(n), ref_v, ref_g
        if patch in DOMAIN_PATCHES:
            cells = case.domain_bnd_owner[mask]
            Sf = case.domain_bnd_Sf[mask]
        else:
            imm = case.ap_is_immersed_faces
            if side == "upper":
                cells = case.owner[imm][mask]
                Sf = case.Sf[imm][mask]
            else:
                cells = case.neighbour[imm][mask]
                Sf = -case.Sf[imm][mask]
        n_vec = np.sign(Sf)
        psi = field.data[cells]
        normal = (psi * n_vec).sum(axis=-1)
        ref_v = psi - normal[:, None] * n_vec
        return fraction, ref_v, ref_g


class InletOutletBC(BoundaryCondition):
    """boundaries/derived/inlet_outlet.py:44-123."""

    type = "inlet_outlet"

    def __init__(self, inlet_value, phi_name: str = "phi"):
        self.inlet_value = np.asarray(inlet_value, dtype=np.float64)
        self.phi_name = phi_name

    def evaluate(self, field, patch, side):
        case = field.case
        mask = _patch_faces(case, patch, side)
        n = int(mask.sum())
        fraction = np.zeros(n)
        ref_v = np.zeros((n,) + field.comp)
        ref_g = np.zeros_like(ref_v)
        if n == 0:
            return fraction, ref_v, ref_g
        phi = case.facefields.get(self.phi_name)
        if phi is None:
            raise ValueError(f"Field {self.phi_name} is not found.")
        if patch in DOMAIN_PATCHES:
            phi_b = phi.domain_bnd_data[mask]
        else:
            phi_b = (phi.immersed_upper if side == "upper" else phi.immersed_lower)[mask]
        inflow = phi_b < 0.0
        fraction[inflow] = 1.0
        ref_v[inflow] = self.inlet_value
        return fraction, ref_v, ref_g


class FixedFluxPressureBC(BoundaryCondition):
    """boundaries/derived/fixed_flux_pressure.py:127-252."""

    type = "fixed_flux_pressure"

    def evaluate(self, field, patch, side):
        case = field.case
        mask = _patch_faces(case, patch, side)
        n = int(mask.sum())
        fraction = np.zeros(n)
        ref_v = np.zeros(n)
        ref_g = np.zeros(n)
        phi = case.facefields.get("phi")
        phi_hbya = case.facefields.get("phiHbyA")
        HbyA = case.cellfields.get("HbyA")
        coeff = case.cellfields.get("rAtU") or case.cellfields.get("rAU")
        U = case.cellfields.get("U")
        if coeff is None or (phi_hbya is None and HbyA is None):
            return fraction, ref_v, ref_g
        if patch in DOMAIN_PATCHES:
            cells = case.domain_bnd_owner[mask]
            Sf_out = case.domain_bnd_Sf[mask]
            mag_d = np.linalg.norm(
                case.domain_bnd_face_centers[mask] - case.cell_centers[cells], axis=1
            )
            block = "domain"
        else:
            imm = case.ap_is_immersed_faces
            if side == "upper":
                cells = case.owner[imm][mask]
                Sf_out = case.Sf[imm][mask]
                mag_d = case.ap_dist_owner_to_bnd[mask]
                block = "upper"
            else:
                cells = case.neighbour[imm][mask]
                Sf_out = -case.Sf[imm][mask]
                mag_d = case.ap_dist_neighbour_to_bnd[mask]
                block = "lower"
        mag_Sf = np.linalg.norm(Sf_out, axis=1)
        if phi_hbya is not None:
            flux_pred = phi_hbya.block(block)[mask]
        else:
            flux_pred = np.sum(HbyA.data[cells] * Sf_out, axis=1)
        flux_target = None
        if U is not None:
            bc = U.bcs.get(patch)
            if bc is not None:
                fr, rv, rg = bc.evaluate(U, patch, side)
                psi_O = U.data[cells]
                f = bview(fr, psi_O)
                psi_b = f * rv + (1.0 - f) * (psi_O + bview(mag_d, psi_O) * rg)
                flux_target = np.sum(psi_b * Sf_out, axis=1)
        if flux_target is None:
            if phi is None:
                return fraction, ref_v, ref_g
            flux_target = phi.block(block)[mask]
        denom = coeff.data[cells] * mag_Sf
        safe = np.where(denom > 0.0, denom, 1.0)
        ref_g = np.where(denom > 0.0, (flux_pred - flux_target) / safe, 0.0)
        return fraction, ref_v, ref_g


def make_bc(cfg: dict) -> BoundaryCondition:
    """boundaries/factory.py:25-69."""
    t = cfg["type"]
    if t == "dirichlet":
        return DirichletBC(cfg["value"])
    if t == "neumann":
        return NeumannBC(cfg["value"])
    if t == "empty":
        return EmptyBC()
    if t == "slip":
        return SlipBC()
    if t == "inlet_outlet":
        return InletOutletBC(cfg["value"])
    if t == "fixed_flux_pressure":
        return FixedFluxPressureBC()
    raise ValueError(f"Unsupported boundary condition type: {t}")


# ----------------------------------------------------------------------
# fv/boundary_ops.py
# ----------------------------------------------------------------------
@dataclass
class Batch:
    patch: str
    side: str
    kind: str  # "domain" | "upper" | "lower"
    face_mask: np.ndarray
    target_cells: np.ndarray
    d_vec: np.ndarray
    mag_d: np.ndarray
    Sf: np.ndarray
    mag_Sf: np.ndarray


def boundary_batches(field: CellField) -> list[Batch]:
    """boundary_ops.py:121-188 (cached per field and set of conditions, as
    the reference caches its batches)."""
    key = tuple((patch, id(bc), bc.type) for patch, bc in field.bcs.items())
    cached = getattr(field, "_batches", None)
    if cached is not None and cached[0] == key:
        return cached[1]
    out = _boundary_batches(field)
    field._batches = (key, out)
    return out


def _boundary_batches(field: CellField) -> list[Batch]:
    case = field.case
    out: list[Batch] = []
    for patch, bc in field.bcs.items():
        if bc.type == "empty":
            continue
        if patch in DOMAIN_PATCHES:
            mask = case.domain_bnd_mask(patch)
            if not mask.any():
                continue
            cells = case.domain_bnd_owner[mask]
            d_vec = case.domain_bnd_face_centers[mask] - case.cell_centers[cells]
            Sf = case.domain_bnd_Sf[mask]
            out.append(
                Batch(patch, "upper", "domain", mask, cells, d_vec,
                      np.linalg.norm(d_vec, axis=1), Sf, np.linalg.norm(Sf, axis=1))
            )
            continue
        pid = case.patch_name_to_id.get(patch)
        if pid is None:
            continue
        upper = case.ap_owner_bnd_patch_id == pid
        lower = case.ap_neighbour_bnd_patch_id == pid
        imm = case.ap_is_immersed_faces
        iSf = case.Sf[imm]
        mag = np.linalg.norm(iSf, axis=1)
        n_hat = iSf / mag[:, None]
        if upper.any():
            md = case.ap_dist_owner_to_bnd[upper]
            out.append(
                Batch(patch, "upper", "upper", upper, case.owner[imm][upper],
                      md[:, None] * n_hat[upper], md, iSf[upper], mag[upper])
            )
        if lower.any():
            md = case.ap_dist_neighbour_to_bnd[lower]
            out.append(
                Batch(patch, "lower", "lower", lower, case.neighbour[imm][lower],
                      md[:, None] * (-n_hat[lower]), md, -iSf[lower], mag[lower])
            )
    return out


def boundary_state(field: CellField, batch: Batch):
    """boundary_ops.py:311-326: ``(fraction, ref_v, ref_g, psi_b)``."""
    bc = field.bcs[batch.patch]
    fraction, ref_v, ref_g = bc.evaluate(field, batch.patch, batch.side)
    psi_O = field.data[batch.target_cells]
    f = bview(fraction, psi_O)
    neumann_value = psi_O + bview(batch.mag_d, psi_O) * ref_g
    return fraction, ref_v, ref_g, f * ref_v + (1.0 - f) * neumann_value


def boundary_states(field: CellField):
    """boundary_ops.py:349-365 (states of every batch, batch order)."""
    return [(b,) + boundary_state(field, b) for b in boundary_batches(field)]


def fixed_value_mask(field: CellField, batch: Batch, fraction: np.ndarray) -> np.ndarray:
    """boundary_ops.py:388-402."""
    case = field.case
    if batch.kind == "upper":
        return case.ap_owner_near_boundary[batch.face_mask] & (fraction == 1)
    if batch.kind == "lower":
        return case.ap_neighbour_near_boundary[batch.face_mask] & (fraction == 1)
    return np.zeros(fraction.shape, dtype=bool)


def value_gradient_coefficient(field, batch, fraction) -> np.ndarray:
    """boundary_ops.py:405-422."""
    active = (fraction != 0) & ~fixed_value_mask(field, batch, fraction)
    if np.any(active & (batch.mag_d == 0)):
        raise ValueError("A mixed boundary at zero distance needs a cell constraint")
    distance = np.where(active, batch.mag_d, 1.0)
    return np.where(active, fraction / distance, 0.0)


def normal_gradient(field, batch, fraction, ref_v, ref_g) -> np.ndarray:
    """boundary_ops.py:425-437."""
    coeff = value_gradient_coefficient(field, batch, fraction)
    return bview(coeff, ref_v) * (ref_v - field.data[batch.target_cells]) + bview(
        1.0 - fraction, ref_g
    ) * ref_g


def uncovered_domain_faces(field: CellField) -> np.ndarray:
    """boundary_ops.py:238-263."""
    covered = np.zeros(field.case.num_domain_bnd_faces, dtype=bool)
    for b in boundary_batches(field):
        if b.kind == "domain":
            covered |= b.face_mask
    return ~covered


def immersed_dirichlet_constraints(field: CellField):
    """boundary_ops.py:440-535: unique cells and closest-hit values."""
    batches = [
        b for b in boundary_batches(field)
        if b.kind != "domain" and type(field.bcs[b.patch]) is not NeumannBC
    ]
    cells, dists, values = [], [], []
    for b in batches:
        fraction, ref_v, _, _ = boundary_state(field, b)
        fixed = fixed_value_mask(field, b, fraction)
        if fixed.any():
            cells.append(b.target_cells[fixed])
            dists.append(b.mag_d[fixed])
            values.append(ref_v[fixed])
    if not cells:
        return np.zeros(0, dtype=np.int64), field.data[:0]
    cell = np.concatenate(cells)
    dist = np.concatenate(dists)
    n = field.case.num_cells
    closest = np.full(n, np.inf)
    np.minimum.at(closest, cell, dist)
    index = np.arange(cell.shape[0])
    candidate = np.where(dist == closest[cell], index, cell.shape[0])
    selected = np.full(n, cell.shape[0], dtype=np.int64)
    np.minimum.at(selected, cell, candidate)
    unique = np.nonzero(selected < cell.shape[0])[0]
    return unique, np.concatenate(values)[selected[unique]]


def apply_immersed_dirichlet_values(field: CellField) -> None:
    """boundary_ops.py:538-542."""
    cells, values = immersed_dirichlet_constraints(field)
    if cells.size:
        field.data = field.data.copy()
        field.data[cells] = values


def fill_boundary_face_values(field: CellField, psi_f: FaceField) -> None:
    """boundary_ops.py:545-593."""
    case = field.case
    cov_u = np.zeros(case.num_immersed_faces, dtype=bool)
    cov_l = np.zeros_like(cov_u)
    for b, _, _, _, psi_b in boundary_states(field):
        psi_f.block(b.kind)[b.face_mask] = psi_b
        if b.kind == "upper":
            cov_u |= b.face_mask
        elif b.kind == "lower":
            cov_l |= b.face_mask
    unc = uncovered_domain_faces(field)
    if unc.any():
        psi_f.domain_bnd_data[unc] = field.data[case.domain_bnd_owner[unc]]
    if case.num_immersed_faces > 0:
        imm = case.ap_is_immersed_faces
        if (~cov_u).any():
            psi_f.immersed_upper[~cov_u] = field.data[case.owner[imm][~cov_u]]
        if (~cov_l).any():
            psi_f.immersed_lower[~cov_l] = field.data[case.neighbour[imm][~cov_l]]
