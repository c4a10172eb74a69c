"""Fluxel-compatible synthetic mesh builder (axis-projected IBM payload).

gridfoam obtains its background mesh and the axis-projected immersed-boundary
(AP-IBM) payload from the external Rust package ``fluxel``
(``core/grid/factory.py:32-65``), which is not available here.  This module
produces an object with the same attribute contract that
``AxisProjectedGrid._load_topology`` / ``_load_ap_payload`` read
(``core/grid/axis_projected.py:97-211``), so that the reference, the CPU
oracle and the GPU path all consume the *same* mesh.

Contract followed (reference ``core/grid/axis_projected.py`` and the
"Immersed Dirichlet constraints" data contract of the reference docs):

* internal face owner is the lower-coordinate cell, so ``Sf`` points along
  ``+axis`` (``axis_projected.py:763-766``);
* domain-boundary direction ids: XMinus=0, XPlus=1, YMinus=2, YPlus=3,
  ZMinus=4, ZPlus=5 (``dir // 2`` is the axis, ``dir % 2`` the sign,
  ``axis_projected.py:781-782``);
* an internal face is *immersed* when the closed owner-to-neighbour centre
  segment meets the body surface; ``dist_*_to_bnd`` is the ray distance
  along the face axis from that cell centre to the surface;
* ``near`` is ``distance / dx <= dx / L`` with ``dx`` the cell width along
  the face axis and ``L`` the largest domain extent.

Cells of a uniform box are numbered lexicographically (x fastest), so the
six neighbours of a cell sit at constant index strides; internal faces are
grouped by axis (x, y, z) and ordered by owner inside each group.
"""

from __future__ import annotations

from dataclasses import dataclass, field
from typing import Callable

import numpy as np

SdfFn = Callable[[np.ndarray], np.ndarray]


@dataclass
class ApPayload:
    """Axis-projected IBM arrays (``mesh.ap`` in the fluxel contract)."""

    is_immersed_face: np.ndarray
    owner_bnd_patch_id: np.ndarray
    neighbour_bnd_patch_id: np.ndarray
    owner_bnd_anchor_id: np.ndarray
    neighbour_bnd_anchor_id: np.ndarray
    dist_owner_to_bnd: np.ndarray
    owner_near_boundary: np.ndarray
    dist_neighbour_to_bnd: np.ndarray
    neighbour_near_boundary: np.ndarray


@dataclass
class FluxelMesh:
    """Duck-typed stand-in for ``fluxel.CfdAxisProjectedMesh``."""

    n_cells: int
    internal_faces_owner: np.ndarray
    internal_faces_neighbour: np.ndarray
    internal_faces_axis: np.ndarray
    domain_bnd_faces_owner: np.ndarray
    domain_bnd_faces_dir: np.ndarray
    patch_name_to_id: dict[str, int]
    cell_centers: np.ndarray
    cell_sizes: np.ndarray
    ap: ApPayload
    resolution: tuple[int, int, int] | None = None
    meta: dict = field(default_factory=dict)


@dataclass
class Body:
    """An immersed body given by a level-set ``sdf`` (surface at zero)."""

    sdf: SdfFn
    patch: str = "body"


def cylinder_sdf(
    center: tuple[float, float], radius: float, axis: int = 2
) -> SdfFn:
    """Signed distance to an infinite circular cylinder along ``axis``."""
    a, b = [i for i in range(3) if i != axis]

    def sdf(x: np.ndarray) -> np.ndarray:
        return (
            np.sqrt((x[..., a] - center[0]) ** 2 + (x[..., b] - center[1]) ** 2)
            - radius
        )

    return sdf


def plane_sdf(point: float, axis: int = 0) -> SdfFn:
    """Signed distance to the plane ``x[axis] = point``."""

    def sdf(x: np.ndarray) -> np.ndarray:
        return x[..., axis] - point

    return sdf


def _segment_roots(
    sdf: SdfFn, p0: np.ndarray, p1: np.ndarray, n_bisect: int = 80
) -> np.ndarray:
    """Parameter ``t`` in [0, 1] of the surface crossing on each segment.

    ``p0`` / ``p1`` are ``[N, 3]`` end points whose ``sdf`` values have
    opposite signs or where one end value is zero.  Plain bisection on the
    level set converges to the crossing to round-off.
    """
    f0 = sdf(p0)
    lo = np.zeros(len(p0))
    hi = np.ones(len(p0))
    zero0 = f0 == 0.0
    for _ in range(n_bisect):
        mid = 0.5 * (lo + hi)
        fm = sdf(p0 + mid[:, None] * (p1 - p0))
        same = np.sign(fm) == np.sign(f0)
        lo = np.where(same, mid, lo)
        hi = np.where(same, hi, mid)
    t = 0.5 * (lo + hi)
    t = np.where(zero0, 0.0, t)
    f1 = sdf(p1)
    t = np.where((f1 == 0.0) & ~zero0, 1.0, t)
    return t


def build_uniform_mesh(
    lower: tuple[float, float, float],
    upper: tuple[float, float, float],
    resolution: tuple[int, int, int],
    *,
    bodies: list[Body] | None = None,
) -> FluxelMesh:
    """Uniform Cartesian box with optional axis-projected immersed bodies.

    Parameters
    ----------
    lower, upper : tuple of float
        Domain corners.
    resolution : tuple of int
        Cells per axis ``(nx, ny, nz)``.
    bodies : list of Body, optional
        Immersed bodies; each gets its own patch id in body order.
    """
    nx, ny, nz = (int(v) for v in resolution)
    lo = np.asarray(lower, dtype=np.float64)
    hi = np.asarray(upper, dtype=np.float64)
    h = (hi - lo) / np.array([nx, ny, nz], dtype=np.float64)
    n_cells = nx * ny * nz

    idx = np.arange(n_cells, dtype=np.int64)
    i = idx % nx
    j = (idx // nx) % ny
    k = idx // (nx * ny)
    centers = np.stack(
        [lo[0] + (i + 0.5) * h[0], lo[1] + (j + 0.5) * h[1], lo[2] + (k + 0.5) * h[2]],
        axis=1,
    )
    sizes = np.broadcast_to(h, (n_cells, 3)).copy()

    owners, neighbours, axes = [], [], []
    strides = (1, nx, nx * ny)
    coords = (i, j, k)
    counts = (nx, ny, nz)
    for axis in range(3):
        sel = coords[axis] < counts[axis] - 1
        own = idx[sel]
        owners.append(own)
        neighbours.append(own + strides[axis])
        axes.append(np.full(own.shape, axis, dtype=np.int64))
    owner = np.concatenate(owners)
    neighbour = np.concatenate(neighbours)
    axis_arr = np.concatenate(axes)

    bnd_owner, bnd_dir = [], []
    for direction in range(6):
        axis = direction // 2
        side_max = direction % 2 == 1
        target = counts[axis] - 1 if side_max else 0
        cells = idx[coords[axis] == target]
        bnd_owner.append(cells)
        bnd_dir.append(np.full(cells.shape, direction, dtype=np.int64))
    domain_owner = np.concatenate(bnd_owner)
    domain_dir = np.concatenate(bnd_dir)

    extent = float(np.max(hi - lo))
    ap, patches = _axis_projected_payload(
        centers, sizes, owner, neighbour, axis_arr, bodies or [], extent
    )
    return FluxelMesh(
        n_cells=n_cells,
        internal_faces_owner=owner,
        internal_faces_neighbour=neighbour,
        internal_faces_axis=axis_arr,
        domain_bnd_faces_owner=domain_owner,
        domain_bnd_faces_dir=domain_dir,
        patch_name_to_id=patches,
        cell_centers=centers,
        cell_sizes=sizes,
        ap=ap,
        resolution=(nx, ny, nz),
        meta={"lower": tuple(lo), "upper": tuple(hi)},
    )


def _axis_projected_payload(
    centers: np.ndarray,
    sizes: np.ndarray,
    owner: np.ndarray,
    neighbour: np.ndarray,
    axis: np.ndarray,
    bodies: list[Body],
    extent: float,
) -> tuple[ApPayload, dict[str, int]]:
    """Immersed-face mask, ray distances and near flags for ``bodies``."""
    n_faces = owner.shape[0]
    patches: dict[str, int] = {}
    immersed = np.zeros(n_faces, dtype=bool)
    patch_of = np.full(n_faces, -1, dtype=np.int64)
    t_own = np.zeros(n_faces)
    p0 = centers[owner]
    p1 = centers[neighbour]
    for body in bodies:
        pid = patches.setdefault(body.patch, len(patches))
        f0 = body.sdf(p0)
        f1 = body.sdf(p1)
        hit = ((np.sign(f0) != np.sign(f1)) | (f0 == 0.0) | (f1 == 0.0)) & ~immersed
        if not np.any(hit):
            continue
        t = _segment_roots(body.sdf, p0[hit], p1[hit])
        immersed[hit] = True
        patch_of[hit] = pid
        t_own[hit] = t
    faces = np.nonzero(immersed)[0]
    seg = np.abs(p1[faces, axis[faces]] - p0[faces, axis[faces]])
    d_own = t_own[faces] * seg
    d_nei = (1.0 - t_own[faces]) * seg
    dx_own = sizes[owner[faces], axis[faces]]
    dx_nei = sizes[neighbour[faces], axis[faces]]
    ap = ApPayload(
        is_immersed_face=immersed,
        owner_bnd_patch_id=patch_of[faces].copy(),
        neighbour_bnd_patch_id=patch_of[faces].copy(),
        owner_bnd_anchor_id=np.arange(faces.shape[0], dtype=np.int64),
        neighbour_bnd_anchor_id=np.arange(faces.shape[0], dtype=np.int64),
        dist_owner_to_bnd=d_own,
        owner_near_boundary=(d_own / dx_own) <= (dx_own / extent),
        dist_neighbour_to_bnd=d_nei,
        neighbour_near_boundary=(d_nei / dx_nei) <= (dx_nei / extent),
    )
    return ap, patches
