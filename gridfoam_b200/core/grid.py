"""Device-resident axis-projected grid.

Mirrors gridfoam's ``AxisProjectedGrid`` (``core/grid/axis_projected.py:59-
625``): it is built from a fluxel-compatible mesh object (same attribute
contract as ``_load_topology`` / ``_load_ap_payload``) and exposes the same
topology and geometry accessors.  Set-up runs once on the host (numpy) and
uploads an SoA layout that the kernels read coalesced:

* internal-face arrays ``[F]`` in mesh face order;
* boundary faces ``[Nb] = [domain Fb | immersed upper Fi | immersed lower Fi]``;
* a cell-centric ELL adjacency ``[W][C]``: slot ``k`` of cell ``c`` holds one
  face of the cell (internal, immersed side or domain face), so per-cell
  kernels need one gather pass and no atomics.  Uniform boxes have exactly
  six slots per cell, ordered -x, +x, -y, +y, -z, +z.

Face geometry (``fv/kernels/face_geometry.py:107-262``) is computed here:
linear weights, ``|Sf|``, delta coefficients and the least-squares normal
matrix inverse.  Hanging (2:1) faces carry their offset and tangential-move
vectors for the explicit corrections of interpolation, normal gradient,
convection and Laplacian.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
import torch

from gridfoam_b200._lib import GfMesh, ptr
from gridfoam_b200.meta.config import DomainBoundaryPatch, SimulatorConfig

DOMAIN_DIRECTION = {p.value: i for i, p in enumerate(DomainBoundaryPatch)}


@dataclass
class HostGeometry:
    """Host copies of the set-up arrays (used by boundary set-up)."""

    owner: np.ndarray
    neighbour: np.ndarray
    axis: np.ndarray
    cell_centers: np.ndarray
    cell_sizes: np.ndarray
    cell_volumes: np.ndarray
    face_centers: np.ndarray
    Sf: np.ndarray
    w: np.ndarray
    mag_sf: np.ndarray
    delta: np.ndarray
    domain_owner: np.ndarray
    domain_dir: np.ndarray
    domain_face_centers: np.ndarray
    domain_Sf: np.ndarray
    immersed: np.ndarray
    imm_faces: np.ndarray
    ap_owner_patch: np.ndarray
    ap_neighbour_patch: np.ndarray
    ap_dist_owner: np.ndarray
    ap_dist_neighbour: np.ndarray
    ap_owner_near: np.ndarray
    ap_neighbour_near: np.ndarray
    bnd_cell: np.ndarray
    bnd_sf: np.ndarray
    bnd_mag_sf: np.ndarray
    bnd_d: np.ndarray
    bnd_mag_d: np.ndarray
    bnd_near: np.ndarray
    extra: dict = field(default_factory=dict)


def _lsq_outer(d: np.ndarray) -> np.ndarray:
    """``face_geometry.py:191-197``: ``w2 d d^T`` with ``w2 = 1/|d|^2``."""
    d2 = np.sum(d * d, axis=1)
    w2 = 1.0 / np.where(d2 > 0, d2, 1.0)
    return w2[:, None, None] * d[:, :, None] * d[:, None, :]


class AxisProjectedGrid:
    """Axis-projected IBM grid on one CUDA device."""

    def __init__(self, simulator_config: SimulatorConfig, fluxel_mesh, device: torch.device | str | None = None):
        self._sim_config = simulator_config
        if device is None:
            device = torch.device("cuda", torch.cuda.current_device()) if torch.cuda.is_available() else "cuda"
        self._device = torch.device(device)
        self._cellfields: dict = {}
        self._facefields: dict = {}
        self._mesh_ref = fluxel_mesh
        self.host = self._build_host(fluxel_mesh)
        self._build_ell()
        self._upload()
        self._mesh_ref = None

    def with_config(self, simulator_config: SimulatorConfig) -> "AxisProjectedGrid":
        """A grid sharing this one's topology, geometry and device arrays
        (all read-only after set-up) with its own configuration and field
        registry: many cases on one mesh pay the host set-up once."""
        g = object.__new__(AxisProjectedGrid)
        g.__dict__.update(self.__dict__)
        g._sim_config = simulator_config
        g._cellfields = {}
        g._facefields = {}
        return g

    # ------------------------------------------------------------------
    # host set-up
    # ------------------------------------------------------------------
    def _build_host(self, mesh) -> HostGeometry:
        C = int(mesh.n_cells)
        owner = np.asarray(mesh.internal_faces_owner, dtype=np.int64)
        neighbour = np.asarray(mesh.internal_faces_neighbour, dtype=np.int64)
        axis = np.asarray(mesh.internal_faces_axis, dtype=np.int64)
        F = owner.shape[0]
        centers = np.asarray(mesh.cell_centers, dtype=np.float64)
        sizes = np.asarray(mesh.cell_sizes, dtype=np.float64)
        volumes = np.prod(sizes, axis=1)
        if F and (owner.max() >= C or neighbour.max() >= C or owner.min() < 0 or neighbour.min() < 0):
            raise ValueError("face owner/neighbour index out of range")

        # axis_projected.py:715-767
        c_o, c_n, s_o, s_n = centers[owner], centers[neighbour], sizes[owner], sizes[neighbour]
        fmin = np.maximum(c_o - s_o / 2.0, c_n - s_n / 2.0)
        fmax = np.minimum(c_o + s_o / 2.0, c_n + s_n / 2.0)
        face_centers = (fmin + fmax) / 2.0
        mins = np.minimum(s_o, s_n)
        fidx = np.arange(F)
        area = np.prod(mins, axis=1) / mins[fidx, axis]
        Sf = np.zeros((F, 3))
        Sf[fidx, axis] = area

        # face_geometry.py:117-124
        d_all = c_n - c_o
        d_fN = c_n - face_centers
        d_n = np.abs(d_all[fidx, axis])
        w = np.abs(d_fN[fidx, axis]) / d_n
        mag_sf = np.linalg.norm(Sf, axis=1)
        delta = 1.0 / d_n

        # axis_projected.py:770-811
        dom_owner = np.asarray(mesh.domain_bnd_faces_owner, dtype=np.int64)
        dom_dir = np.asarray(mesh.domain_bnd_faces_dir, dtype=np.int64)
        Fb = dom_owner.shape[0]
        bidx = np.arange(Fb)
        b_axis = dom_dir // 2
        sign = 2.0 * (dom_dir % 2) - 1.0
        normals = np.zeros((Fb, 3))
        normals[bidx, b_axis] = sign
        dom_fc = centers[dom_owner] + 0.5 * sizes[dom_owner] * normals
        dom_sf = np.zeros((Fb, 3))
        dom_sf[bidx, b_axis] = sign * np.prod(sizes[dom_owner], axis=1) / sizes[dom_owner][bidx, b_axis]

        ap = mesh.ap
        immersed = np.asarray(ap.is_immersed_face, dtype=bool)
        imm_faces = np.nonzero(immersed)[0]
        Fi = imm_faces.shape[0]
        d_own = np.asarray(ap.dist_owner_to_bnd, dtype=np.float64).reshape(-1)
        d_nei = np.asarray(ap.dist_neighbour_to_bnd, dtype=np.float64).reshape(-1)

        # Hanging faces (face_geometry.py:141-162): face centre off the
        # owner-neighbour segment; offset from the linear-weight point, and
        # the tangential moves from each cell centre to the face centre.
        s_idx = np.nonzero(~immersed)[0]
        centroid = w[s_idx, None] * c_o[s_idx] + (1.0 - w[s_idx])[:, None] * c_n[s_idx]
        offset = face_centers[s_idx] - centroid
        tol = 1.0e-8 * float(sizes.min())
        hang_faces = s_idx[np.linalg.norm(offset, axis=1) > tol]
        hang_offset = offset[np.linalg.norm(offset, axis=1) > tol]
        hidx = np.arange(hang_faces.shape[0])
        move_o = face_centers[hang_faces] - c_o[hang_faces]
        move_n = face_centers[hang_faces] - c_n[hang_faces]
        move_o[hidx, axis[hang_faces]] = 0.0
        move_n[hidx, axis[hang_faces]] = 0.0

        # Boundary faces: domain | immersed upper | immersed lower
        iSf = Sf[imm_faces]
        i_mag = np.linalg.norm(iSf, axis=1) if Fi else np.zeros(0)
        n_hat = iSf / i_mag[:, None] if Fi else np.zeros((0, 3))
        dom_d = dom_fc - centers[dom_owner]
        bnd_cell = np.concatenate([dom_owner, owner[imm_faces], neighbour[imm_faces]])
        bnd_sf = np.concatenate([dom_sf, iSf, -iSf])
        bnd_mag_sf = np.concatenate([np.linalg.norm(dom_sf, axis=1), i_mag, i_mag])
        bnd_d = np.concatenate([dom_d, d_own[:, None] * n_hat, d_nei[:, None] * (-n_hat)])
        bnd_mag_d = np.concatenate([np.linalg.norm(dom_d, axis=1), d_own, d_nei])
        bnd_near = np.concatenate(
            [
                np.zeros(Fb, dtype=np.uint8),
                np.asarray(ap.owner_near_boundary, dtype=np.uint8),
                np.asarray(ap.neighbour_near_boundary, dtype=np.uint8),
            ]
        )

        # LSQ normal matrix (face_geometry.py:245-262): single faces + every
        # domain and immersed boundary vector.
        outer = _lsq_outer(d_all[s_idx]).reshape(-1, 9)
        ata = np.zeros((C, 9))
        for col in range(9):
            ata[:, col] = np.bincount(owner[s_idx], weights=outer[:, col], minlength=C) + np.bincount(
                neighbour[s_idx], weights=outer[:, col], minlength=C
            )
        b_outer = _lsq_outer(bnd_d).reshape(-1, 9)
        for col in range(9):
            ata[:, col] += np.bincount(bnd_cell, weights=b_outer[:, col], minlength=C)
        ata_inv = np.linalg.pinv(ata.reshape(C, 3, 3), hermitian=True).reshape(C, 9)

        self._num_cells = C
        self._num_internal_faces = F
        self._num_domain_bnd_faces = Fb
        self._num_immersed_faces = Fi
        self._patch_name_to_id = dict(mesh.patch_name_to_id)
        host = HostGeometry(
            owner=owner,
            neighbour=neighbour,
            axis=axis,
            cell_centers=centers,
            cell_sizes=sizes,
            cell_volumes=volumes,
            face_centers=face_centers,
            Sf=Sf,
            w=w,
            mag_sf=mag_sf,
            delta=delta,
            domain_owner=dom_owner,
            domain_dir=dom_dir,
            domain_face_centers=dom_fc,
            domain_Sf=dom_sf,
            immersed=immersed,
            imm_faces=imm_faces,
            ap_owner_patch=np.asarray(ap.owner_bnd_patch_id, dtype=np.int64),
            ap_neighbour_patch=np.asarray(ap.neighbour_bnd_patch_id, dtype=np.int64),
            ap_dist_owner=d_own,
            ap_dist_neighbour=d_nei,
            ap_owner_near=np.asarray(ap.owner_near_boundary, dtype=bool),
            ap_neighbour_near=np.asarray(ap.neighbour_near_boundary, dtype=bool),
            bnd_cell=bnd_cell,
            bnd_sf=bnd_sf,
            bnd_mag_sf=bnd_mag_sf,
            bnd_d=bnd_d,
            bnd_mag_d=bnd_mag_d,
            bnd_near=bnd_near,
        )
        host.extra["lsq_ata_inv"] = ata_inv
        normals = getattr(ap, "anchor_normal", None)
        host.extra["anchor_normal"] = (np.asarray(normals, dtype=np.float64).reshape(Fi, 3)
                                       if normals is not None else None)
        host.extra["hang_faces"] = hang_faces
        host.extra["hang_offset"] = hang_offset
        host.extra["hang_move_o"] = move_o
        host.extra["hang_move_n"] = move_n
        return host

    def _build_ell(self) -> None:
        """Cell-centric slot table sorted by (cell, direction, face).

        On meshes that are not uniform boxes the slots of a row are sorted
        internal faces first, then domain faces, so the matrix entries of a
        row lead it and ``ell_len`` (one past the last internal-face slot)
        lets the Krylov kernels stop at the row's last entry instead of
        reading the padding of the widest row.
        """
        self._build_ell_order(couplings_first=False)
        if self.box_strides is None:
            self._build_ell_order(couplings_first=True)

    def _build_ell_order(self, *, couplings_first: bool) -> None:
        h = self.host
        C, F, Fb = self._num_cells, self._num_internal_faces, self._num_domain_bnd_faces
        fidx = np.arange(F, dtype=np.int64)
        cells = np.concatenate([h.owner, h.neighbour, h.domain_owner])
        direction = np.concatenate([2 * h.axis + 1, 2 * h.axis, h.domain_dir])
        code = np.concatenate([fidx * 2, fidx * 2 + 1, (F + np.arange(Fb, dtype=np.int64)) * 2])
        nbr = np.concatenate([h.neighbour, h.owner, h.domain_owner])
        if couplings_first:
            order = np.lexsort((code, direction, code >= 2 * F, cells))
        else:
            order = np.lexsort((code, direction, cells))
        cells, code, nbr = cells[order], code[order], nbr[order]
        counts = np.bincount(cells, minlength=C)
        W = int(counts.max()) if counts.size else 1
        start = np.concatenate([[0], np.cumsum(counts)[:-1]])
        rank = np.arange(cells.shape[0]) - start[cells]
        pos = rank * C + cells
        ell_code = np.full(W * C, -1, dtype=np.int64)
        ell_nbr = np.tile(np.arange(C, dtype=np.int64), W)
        ell_code[pos] = code
        ell_nbr[pos] = nbr
        pos_owner = np.empty(F, dtype=np.int64)
        pos_neigh = np.empty(F, dtype=np.int64)
        is_int = code < 2 * F
        face_of = code[is_int] >> 1
        side_of = code[is_int] & 1
        p_int = pos[is_int]
        pos_owner[face_of[side_of == 0]] = p_int[side_of == 0]
        pos_neigh[face_of[side_of == 1]] = p_int[side_of == 1]
        # One past the last internal-face slot of each row: later slots hold
        # boundary faces or nothing, whose matrix coefficients are zero.
        ell_len = np.zeros(C, dtype=np.int64)
        np.maximum.at(ell_len, cells[is_int], rank[is_int] + 1)
        self._ell_width = W
        if not couplings_first:
            self.box_strides = self._detect_box(ell_code, ell_nbr, W)
        h.extra.update(
            ell_code=ell_code, ell_nbr=ell_nbr, face_pos_owner=pos_owner, face_pos_neigh=pos_neigh,
            ell_len=ell_len,
        )

    def _detect_box(self, ell_code: np.ndarray, ell_nbr: np.ndarray, W: int) -> tuple[int, int] | None:
        """``(stride_y, stride_z)`` when the ELL is a uniform lexicographic box.

        Slot ``2a + side`` of cell ``c`` then couples ``c -/+ stride_a``
        (``stride_x = 1``) or is a boundary slot; the Krylov kernels use the
        implicit neighbours and skip the index table.
        """
        res = getattr(self._mesh_ref, "resolution", None)
        if res is None or W != 6:
            return None
        nx, ny, nz = (int(v) for v in res)
        C = self._num_cells
        if nx * ny * nz != C:
            return None
        cells = np.arange(C, dtype=np.int64)
        strides = (1, nx, nx * ny)
        F = self._num_internal_faces
        for a, st in enumerate(strides):
            for side, sign in ((0, -1), (1, 1)):
                slot = 2 * a + side
                code = ell_code[slot * C : (slot + 1) * C]
                nbr = ell_nbr[slot * C : (slot + 1) * C]
                internal = (code >= 0) & (code < 2 * F)
                if np.any(code < 0):
                    return None
                want = np.where(internal, cells + sign * st, cells)
                if not np.array_equal(nbr, want):
                    return None
        return (nx, nx * ny)

    def _upload(self) -> None:
        h = self.host
        dev = self._device
        f64 = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device=dev)  # noqa: E731
        i32 = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.int32), device=dev)  # noqa: E731
        i64 = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.int64), device=dev)  # noqa: E731
        imm_index = np.full(self._num_internal_faces, -1, dtype=np.int64)
        imm_index[h.imm_faces] = np.arange(self._num_immersed_faces)
        t = {
            "owner": i32(h.owner),
            "neighbour": i32(h.neighbour),
            "weight": f64(h.w),
            "mag_sf": f64(h.mag_sf),
            "delta": f64(h.delta),
            "sf": f64(h.Sf.T),
            "imm_index": i32(imm_index),
            "volume": f64(h.cell_volumes),
            "center": f64(h.cell_centers.T),
            "lsq_ata_inv": f64(h.extra["lsq_ata_inv"].T),
            "ell_code": i32(h.extra["ell_code"]),
            "ell_nbr": i32(h.extra["ell_nbr"]),
            "ell_len": torch.as_tensor(np.ascontiguousarray(h.extra["ell_len"], dtype=np.uint8), device=dev),
            "bnd_cell": i32(h.bnd_cell),
            "bnd_sf": f64(h.bnd_sf.T),
            "bnd_mag_sf": f64(h.bnd_mag_sf),
            "bnd_d": f64(h.bnd_d.T),
            "bnd_mag_d": f64(h.bnd_mag_d),
            "bnd_near": torch.as_tensor(h.bnd_near.astype(np.uint8), device=dev),
            "face_pos_owner": i32(h.extra["face_pos_owner"]),
            "face_pos_neigh": i32(h.extra["face_pos_neigh"]),
            "face_axis": torch.as_tensor(np.ascontiguousarray(h.axis, dtype=np.int8), device=dev),
        }
        hf = h.extra["hang_faces"]
        face_hang = np.full(self._num_internal_faces, -1, dtype=np.int64)
        face_hang[hf] = np.arange(hf.shape[0])
        if hf.shape[0]:
            t["hang_face"] = i32(hf)
            t["face_hang"] = i32(face_hang)
            t["hang_offset"] = f64(h.extra["hang_offset"].T)
            t["hang_move_o"] = f64(h.extra["hang_move_o"].T)
            t["hang_move_n"] = f64(h.extra["hang_move_n"].T)
        self.dev = t
        m = GfMesh()
        m.n_cells = self._num_cells
        m.n_faces = self._num_internal_faces
        m.n_domain = self._num_domain_bnd_faces
        m.n_imm = self._num_immersed_faces
        m.n_bnd = self.num_bnd
        m.ell_width = self._ell_width
        m.n_hang = int(hf.shape[0])
        for name, tensor in t.items():
            setattr(m, name, ptr(tensor))
        self.cmesh = m
        # Reference-layout tensors for the public accessors.
        self._owner = i64(h.owner)
        self._neighbour = i64(h.neighbour)
        self._axis = i64(h.axis)
        self._cell_centers = f64(h.cell_centers)
        self._cell_sizes = f64(h.cell_sizes)
        self._face_centers = f64(h.face_centers)
        self._Sf = f64(h.Sf)
        self._domain_bnd_owner = i64(h.domain_owner)
        self._domain_bnd_dir_id = i64(h.domain_dir)
        self._domain_bnd_face_centers = f64(h.domain_face_centers)
        self._domain_bnd_Sf = f64(h.domain_Sf)
        self._ap_is_immersed_faces = torch.as_tensor(h.immersed, device=dev)
        self.single_idx = i64(np.nonzero(~h.immersed)[0])
        self.single_is_identity = self._num_immersed_faces == 0

    # ------------------------------------------------------------------
    # boundary patch helpers
    # ------------------------------------------------------------------
    def patch_faces(self, patch: str) -> np.ndarray:
        """Boundary-face indices (into ``[0, Nb)``) covered by ``patch``.

        Domain patches select their direction's faces; immersed patches
        select the upper side then the lower side of faces carrying the
        patch id (the reference's batch order, boundary_ops.py:150-188).
        """
        h = self.host
        name = str(patch)
        if name in DOMAIN_DIRECTION:
            return np.nonzero(h.domain_dir == DOMAIN_DIRECTION[name])[0]
        pid = self._patch_name_to_id.get(name)
        if pid is None:
            return np.zeros(0, dtype=np.int64)
        Fb, Fi = self._num_domain_bnd_faces, self._num_immersed_faces
        up = np.nonzero(h.ap_owner_patch == pid)[0] + Fb
        lo = np.nonzero(h.ap_neighbour_patch == pid)[0] + Fb + Fi
        return np.concatenate([up, lo])

    def register_cellfield(self, field) -> None:
        self._cellfields[field.name] = field

    def register_facefield(self, field) -> None:
        self._facefields[field.name] = field

    def get_cellfield(self, name: str):
        return self._cellfields.get(name)

    def get_facefield(self, name: str):
        return self._facefields.get(name)

    def cellfield_names(self):
        return self._cellfields.keys()

    def facefield_names(self):
        return self._facefields.keys()

    # ------------------------------------------------------------------
    # accessors (core/grid/base.py:19-275)
    # ------------------------------------------------------------------
    @property
    def sim_config(self) -> SimulatorConfig:
        return self._sim_config

    @sim_config.setter
    def sim_config(self, value: SimulatorConfig) -> None:
        self._sim_config = value

    @property
    def dt(self) -> float:
        return float(self._sim_config.control.deltaT)

    @property
    def dtype(self) -> torch.dtype:
        return torch.float64

    @property
    def device(self) -> torch.device:
        return self._device

    @property
    def num_cells(self) -> int:
        return self._num_cells

    @property
    def num_internal_faces(self) -> int:
        return self._num_internal_faces

    @property
    def num_domain_bnd_faces(self) -> int:
        return self._num_domain_bnd_faces

    @property
    def num_immersed_faces(self) -> int:
        return self._num_immersed_faces

    @property
    def num_bnd(self) -> int:
        return self._num_domain_bnd_faces + 2 * self._num_immersed_faces

    @property
    def num_hanging(self) -> int:
        """Hanging (coarse-fine) internal faces."""
        return int(self.cmesh.n_hang)

    @property
    def ell_width(self) -> int:
        return self._ell_width

    @property
    def patch_name_to_id(self) -> dict[str, int]:
        return self._patch_name_to_id

    @property
    def owner(self) -> torch.Tensor:
        return self._owner

    @property
    def neighbour(self) -> torch.Tensor:
        return self._neighbour

    @property
    def axis(self) -> torch.Tensor:
        return self._axis

    @property
    def domain_bnd_owner(self) -> torch.Tensor:
        return self._domain_bnd_owner

    @property
    def domain_bnd_dir_id(self) -> torch.Tensor:
        return self._domain_bnd_dir_id

    @property
    def cell_centers(self) -> torch.Tensor:
        return self._cell_centers

    @property
    def cell_sizes(self) -> torch.Tensor:
        return self._cell_sizes

    @property
    def cell_volumes(self) -> torch.Tensor:
        return self.dev["volume"]

    @property
    def face_centers(self) -> torch.Tensor:
        return self._face_centers

    @property
    def Sf(self) -> torch.Tensor:
        return self._Sf

    @property
    def domain_bnd_face_centers(self) -> torch.Tensor:
        return self._domain_bnd_face_centers

    @property
    def domain_bnd_Sf(self) -> torch.Tensor:
        return self._domain_bnd_Sf

    @property
    def ap_is_immersed_faces(self) -> torch.Tensor:
        return self._ap_is_immersed_faces
