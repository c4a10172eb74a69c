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
    # [Fi, 3] body-outward unit surface normal per anchor (one anchor per
    # immersed face); stands in for the surface mesh's face area vectors.
    anchor_normal: np.ndarray | None = None


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


# Shape parameters of the slanted bluff body, in this order: length, width,
# height, front rounding radius in plan view (vertical front edges), front
# rounding radius in side view (horizontal front edges), rear slant angle
# (degrees), slant length along x, ground clearance.
BLUFF_PARAMS = ("length", "width", "height", "r_plan", "r_side", "slant_deg", "slant_len", "clearance")
BLUFF_DEFAULT = (1.0, 0.39, 0.29, 0.1, 0.1, 25.0, 0.222, 0.05)


def _rounded_front_rect(u: np.ndarray, v: np.ndarray, u0: float, u1: float, v0: float, v1: float,
                        r: float) -> np.ndarray:
    """Signed distance to the rectangle [u0, u1] x [v0, v1] whose two corners
    at u = u0 are rounded with radius r (the rear corners stay sharp)."""
    cu, cv = 0.5 * (u0 + u1), 0.5 * (v0 + v1)
    bu, bv = 0.5 * (u1 - u0), 0.5 * (v1 - v0)
    rr = np.where(u < cu, r, 0.0)
    qu = np.abs(u - cu) - bu + rr
    qv = np.abs(v - cv) - bv + rr
    outside = np.sqrt(np.maximum(qu, 0.0) ** 2 + np.maximum(qv, 0.0) ** 2)
    return outside + np.minimum(np.maximum(qu, qv), 0.0) - rr


def bluff_body_sdf(x0: float = 0.0, params=BLUFF_DEFAULT) -> SdfFn:
    """Level set of a slanted bluff body (an Ahmed-type car body): a box
    from x = x0 to x0 + length, centred on y = 0, from z = clearance to
    clearance + height, its front edges rounded in plan and side view, its
    top rear edge cut by a plane at ``slant_deg`` to the horizontal over
    ``slant_len``.  Negative inside.  The zero set is exact; away from it the
    value is a bound (intersections by max)."""
    L, Wd, H, r_plan, r_side, slant, ls, g = (float(v) for v in params)
    th = np.deg2rad(slant)
    nx, nz = np.sin(th), np.cos(th)
    xs, zs = x0 + L - ls, g + H

    def sdf(x: np.ndarray) -> np.ndarray:
        px, py, pz = x[..., 0], x[..., 1], x[..., 2]
        plan = _rounded_front_rect(px, py, x0, x0 + L, -0.5 * Wd, 0.5 * Wd, r_plan)
        side = _rounded_front_rect(px, pz, x0, x0 + L, g, g + H, r_side)
        cut = nx * (px - xs) + nz * (pz - zs)
        return np.maximum(np.maximum(plan, side), cut)

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
    # Body-outward unit normal at each crossing (the SDF gradient by central
    # differences; outward for a body occupying sdf < 0): the surface normal
    # the force integral orients its samples by.
    normals = np.zeros((faces.shape[0], 3))
    if faces.shape[0]:
        pts = p0[faces] + t_own[faces][:, None] * (p1[faces] - p0[faces])
        h = 1e-6 * extent
        body_of = patch_of[faces]
        for body in bodies:
            sel = body_of == patches.get(body.patch, -1)
            if not np.any(sel):
                continue
            for ax in range(3):
                e = np.zeros(3)
                e[ax] = h
                normals[sel, ax] = (body.sdf(pts[sel] + e) - body.sdf(pts[sel] - e)) / (2 * h)
        nrm = np.linalg.norm(normals, axis=1)
        normals = normals / np.where(nrm > 0, nrm, 1.0)[:, None]
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
        anchor_normal=normals,
    )
    return ap, patches


# ----------------------------------------------------------------------
# Octree meshes (2:1 balanced, hanging faces)
# ----------------------------------------------------------------------
@dataclass
class BoxRegion:
    """Refine every leaf that holds a finest-level cell centre inside the
    box ``[lo, hi]`` to at least ``level``."""

    lo: tuple[float, float, float]
    hi: tuple[float, float, float]
    level: int


@dataclass
class SdfRegion:
    """Refine to ``level`` where the body's signed distance is below
    ``distance`` (a band around and inside the body)."""

    sdf: SdfFn
    distance: float
    level: int


def _block_max(a: np.ndarray, s: int) -> np.ndarray:
    """Max over aligned ``s^3`` blocks of a 3-D array (sizes divisible by s)."""
    X, Y, Z = a.shape
    return a.reshape(X // s, s, Y // s, s, Z // s, s).max(axis=(1, 3, 5))


def _morton(i: np.ndarray, j: np.ndarray, k: np.ndarray, bits: int) -> np.ndarray:
    code = np.zeros(i.shape, dtype=np.int64)
    for b in range(bits):
        code |= ((i >> b) & 1) << (3 * b)
        code |= ((j >> b) & 1) << (3 * b + 1)
        code |= ((k >> b) & 1) << (3 * b + 2)
    return code


def build_octree_mesh(
    lower: tuple[float, float, float],
    upper: tuple[float, float, float],
    root_resolution: tuple[int, int, int],
    regions: list | None = None,
    *,
    bodies: list[Body] | None = None,
) -> FluxelMesh:
    """Octree refinement of a root Cartesian grid, 2:1 balanced across faces.

    Leaves are refined to the highest level any region asks for, then leaves
    with a face neighbour more than one level finer are refined until the
    2:1 rule holds.  The result follows the fluxel mesh contract:

    * one internal face per fine sub-face at a coarse-fine interface, owner
      the lower-coordinate cell (the reference derives the face centre as
      the centre of the two cells' overlap and the area from the finer cell,
      ``core/grid/axis_projected.py:715-767``);
    * one domain-boundary face per leaf face on the domain boundary;
    * cells sorted by refinement level, then Morton order of their
      finest-level lower corner; internal faces sorted by (axis, owner,
      neighbour), domain faces by (direction, owner).

    Immersed bodies must lie inside uniformly refined regions: an immersed
    face between cells of different levels raises ``ValueError``.
    """
    regions = list(regions or [])
    rx, ry, rz = (int(v) for v in root_resolution)
    lo = np.asarray(lower, dtype=np.float64)
    hi = np.asarray(upper, dtype=np.float64)
    L = max([r.level for r in regions], default=0)
    f = 1 << L
    FX, FY, FZ = rx * f, ry * f, rz * f
    hf = (hi - lo) / np.array([FX, FY, FZ], dtype=np.float64)

    req = _required_levels(lo, hf, (FX, FY, FZ), regions)

    # Level of the leaf covering each finest cell; refine level by level.
    lev = np.zeros((FX, FY, FZ), dtype=np.int8)
    for _ in range(64):
        changed = False
        # 2:1 balance: highest level among each finest cell's face neighbours.
        nb = lev.copy()
        for ax in range(3):
            sl_a = [slice(None)] * 3
            sl_b = [slice(None)] * 3
            sl_a[ax], sl_b[ax] = slice(1, None), slice(None, -1)
            np.maximum(nb[tuple(sl_b)], lev[tuple(sl_a)], out=nb[tuple(sl_b)])
            np.maximum(nb[tuple(sl_a)], lev[tuple(sl_b)], out=nb[tuple(sl_a)])
        for level in range(L):
            s = 1 << (L - level)
            at = _block_max(lev, s) == level  # leaves of this level (uniform blocks)
            at &= -_block_max(-lev, s) == level
            want = (_block_max(req, s) > level) | (_block_max(nb, s) > level + 1)
            grow = at & want
            if np.any(grow):
                changed = True
                g = np.repeat(np.repeat(np.repeat(grow, s, 0), s, 1), s, 2)
                lev[g] = level + 1
        if not changed:
            break
    else:
        raise RuntimeError("octree refinement did not settle")

    # Leaves: one per aligned block of its level.
    li, lj, lk, ll = [], [], [], []
    for level in range(L + 1):
        s = 1 << (L - level)
        blk = (_block_max(lev, s) == level) & (-_block_max(-lev, s) == level)
        I, J, K = np.nonzero(blk)
        li.append(I * s)
        lj.append(J * s)
        lk.append(K * s)
        ll.append(np.full(I.shape, level, dtype=np.int64))
    li, lj, lk, ll = (np.concatenate(a).astype(np.int64) for a in (li, lj, lk, ll))
    bits = int(np.ceil(np.log2(max(FX, FY, FZ, 2))))
    order = np.lexsort((_morton(li, lj, lk, bits), ll))
    li, lj, lk, ll = li[order], lj[order], lk[order], ll[order]

    ids = np.empty((FX, FY, FZ), dtype=np.int64)
    for level in range(L + 1):
        s = 1 << (L - level)
        sel = np.nonzero(ll == level)[0]
        if sel.size == 0:
            continue
        blk = np.full((FX // s, FY // s, FZ // s), -1, dtype=np.int64)
        blk[li[sel] // s, lj[sel] // s, lk[sel] // s] = sel
        full = np.repeat(np.repeat(np.repeat(blk, s, 0), s, 1), s, 2)
        m = full >= 0
        ids[m] = full[m]

    owners, neighbours, axes = [], [], []
    for ax in range(3):
        sl_a = [slice(None)] * 3
        sl_b = [slice(None)] * 3
        sl_a[ax], sl_b[ax] = slice(None, -1), slice(1, None)
        a = ids[tuple(sl_a)].ravel()
        b = ids[tuple(sl_b)].ravel()
        d = a != b
        pairs = np.unique(np.stack([a[d], b[d]], axis=1), axis=0)
        owners.append(pairs[:, 0])
        neighbours.append(pairs[:, 1])
        axes.append(np.full(pairs.shape[0], ax, dtype=np.int64))
    owner = np.concatenate(owners)
    neighbour = np.concatenate(neighbours)
    axis_arr = np.concatenate(axes)

    bnd_owner, bnd_dir = [], []
    for direction in range(6):
        ax, side_max = direction // 2, direction % 2 == 1
        sl = [slice(None)] * 3
        sl[ax] = -1 if side_max else 0
        cells = np.unique(ids[tuple(sl)].ravel())
        bnd_owner.append(cells)
        bnd_dir.append(np.full(cells.shape, direction, dtype=np.int64))
    domain_owner = np.concatenate(bnd_owner)
    domain_dir = np.concatenate(bnd_dir)
    return _octree_mesh(lo, hi, hf, L, (rx, ry, rz), (li, lj, lk, ll), (owner, neighbour, axis_arr),
                        (domain_owner, domain_dir), bodies)


def _required_levels(lo: np.ndarray, hf: np.ndarray, shape: tuple[int, int, int], regions: list,
                     slab: int = 32) -> np.ndarray:
    """Required level per finest cell (max over the refinement regions).

    Signed-distance regions are evaluated on slabs of ``slab`` finest x
    planes (the same per-point expressions as one whole-grid evaluation, in
    bounded memory)."""
    FX, FY, FZ = shape
    req = np.zeros((FX, FY, FZ), dtype=np.int8)
    if not regions:
        return req
    xs = lo[0] + (np.arange(FX) + 0.5) * hf[0]
    ys = lo[1] + (np.arange(FY) + 0.5) * hf[1]
    zs = lo[2] + (np.arange(FZ) + 0.5) * hf[2]
    for r in regions:
        if isinstance(r, BoxRegion):
            mx = (xs >= r.lo[0]) & (xs <= r.hi[0])
            my = (ys >= r.lo[1]) & (ys <= r.hi[1])
            mz = (zs >= r.lo[2]) & (zs <= r.hi[2])
            m = mx[:, None, None] & my[None, :, None] & mz[None, None, :]
            req = np.maximum(req, np.where(m, np.int8(r.level), np.int8(0)))
        elif isinstance(r, SdfRegion):
            for x0 in range(0, FX, slab):
                P = np.stack(np.meshgrid(xs[x0:x0 + slab], ys, zs, indexing="ij"), axis=-1)
                m = r.sdf(P) <= r.distance
                req[x0:x0 + slab] = np.maximum(req[x0:x0 + slab], np.where(m, np.int8(r.level), np.int8(0)))
        else:
            raise TypeError(f"unknown refinement region {r!r}")
    return req


def _octree_mesh(lo, hi, hf, L, root, leaves, faces, domain, bodies) -> FluxelMesh:
    """The fluxel mesh from the leaves (finest-level lower corners and
    levels, in cell order) and the face lists: cell geometry and the AP-IBM
    payload."""
    li, lj, lk, ll = leaves
    owner, neighbour, axis_arr = faces
    domain_owner, domain_dir = domain
    size_f = (1 << (L - ll)).astype(np.int64)  # leaf edge in finest cells
    centers = np.stack(
        [lo[0] + (li + 0.5 * size_f) * hf[0], lo[1] + (lj + 0.5 * size_f) * hf[1],
         lo[2] + (lk + 0.5 * size_f) * hf[2]], axis=1)
    sizes = size_f[:, None] * hf[None, :]
    extent = float(np.max(hi - lo))
    ap, patches = _axis_projected_payload(centers, sizes, owner, neighbour, axis_arr, bodies or [], extent)
    imm = np.nonzero(ap.is_immersed_face)[0]
    if imm.size and np.any(ll[owner[imm]] != ll[neighbour[imm]]):
        raise ValueError("an immersed face lies on a coarse-fine interface; refine around the body")
    return FluxelMesh(
        n_cells=int(li.shape[0]),
        internal_faces_owner=owner,
        internal_faces_neighbour=neighbour,
        internal_faces_axis=axis_arr,
        domain_bnd_faces_owner=domain_owner,
        domain_bnd_faces_dir=domain_dir,
        patch_name_to_id=patches,
        cell_centers=centers,
        cell_sizes=sizes,
        ap=ap,
        resolution=None if L > 0 else root,
        meta={"lower": tuple(lo), "upper": tuple(hi), "levels": ll, "root_resolution": root},
    )


def build_octree_mesh_device(
    lower: tuple[float, float, float],
    upper: tuple[float, float, float],
    root_resolution: tuple[int, int, int],
    regions: list | None = None,
    *,
    bodies: list[Body] | None = None,
    device: str = "cuda",
) -> FluxelMesh:
    """``build_octree_mesh`` with the finest-level work on the GPU; the same
    mesh, array for array.

    The required levels come from the same host expressions.  The 2:1
    refinement, the leaves, their level-then-Morton order, the finest-level
    leaf ids and the domain-boundary cells are integer tensor work on
    ``device``.  The internal faces come from ``gf_octree_face_keys``: each
    owner/neighbour pair is emitted once as ``owner * n_cells +
    neighbour``, and a device sort gives the (owner, neighbour) order of the
    host builder's ``np.unique``.  Cell geometry and the immersed-boundary
    payload are then computed on the host from the same integer arrays with
    the same expressions as the host builder.
    """
    import torch

    from gridfoam_b200._lib import call, ptr, stream_ptr

    dev = torch.device(device)
    regions = list(regions or [])
    rx, ry, rz = (int(v) for v in root_resolution)
    lo = np.asarray(lower, dtype=np.float64)
    hi = np.asarray(upper, dtype=np.float64)
    L = max([r.level for r in regions], default=0)
    f = 1 << L
    FX, FY, FZ = rx * f, ry * f, rz * f
    hf = (hi - lo) / np.array([FX, FY, FZ], dtype=np.float64)
    req = torch.from_numpy(_required_levels(lo, hf, (FX, FY, FZ), regions)).to(dev)

    def bmax(a, s):
        return a.reshape(FX // s, s, FY // s, s, FZ // s, s).amax(dim=(1, 3, 5))

    def expand(a, s):
        return a.repeat_interleave(s, 0).repeat_interleave(s, 1).repeat_interleave(s, 2)

    lev = torch.zeros((FX, FY, FZ), dtype=torch.int8, device=dev)
    for _ in range(64):
        changed = False
        nb = lev.clone()
        for ax in range(3):
            lo_sl = [slice(None)] * 3
            hi_sl = [slice(None)] * 3
            lo_sl[ax], hi_sl[ax] = slice(None, -1), slice(1, None)
            v = nb[tuple(lo_sl)]
            v.copy_(torch.maximum(v, lev[tuple(hi_sl)]))
            v = nb[tuple(hi_sl)]
            v.copy_(torch.maximum(v, lev[tuple(lo_sl)]))
        for level in range(L):
            s = 1 << (L - level)
            at = (bmax(lev, s) == level) & (-bmax(-lev, s) == level)
            want = (bmax(req, s) > level) | (bmax(nb, s) > level + 1)
            grow = at & want
            if bool(grow.any()):
                changed = True
                lev.masked_fill_(expand(grow, s), level + 1)
        if not changed:
            break
    else:
        raise RuntimeError("octree refinement did not settle")

    li, lj, lk, ll = [], [], [], []
    for level in range(L + 1):
        s = 1 << (L - level)
        blk = (bmax(lev, s) == level) & (-bmax(-lev, s) == level)
        I, J, K = torch.nonzero(blk, as_tuple=True)
        li.append(I * s)
        lj.append(J * s)
        lk.append(K * s)
        ll.append(torch.full_like(I, level))
    li, lj, lk, ll = (torch.cat(a) for a in (li, lj, lk, ll))
    bits = int(np.ceil(np.log2(max(FX, FY, FZ, 2))))
    code = torch.zeros_like(li)
    for b in range(bits):
        code |= ((li >> b) & 1) << (3 * b)
        code |= ((lj >> b) & 1) << (3 * b + 1)
        code |= ((lk >> b) & 1) << (3 * b + 2)
    # np.lexsort((code, ll)): level first, then Morton code (unique per level).
    o1 = torch.argsort(code, stable=True)
    order = o1[torch.argsort(ll[o1], stable=True)]
    li, lj, lk, ll = li[order], lj[order], lk[order], ll[order]
    n = int(li.shape[0])

    ids = torch.full((FX, FY, FZ), -1, dtype=torch.int64, device=dev)
    for level in range(L + 1):
        s = 1 << (L - level)
        sel = torch.nonzero(ll == level, as_tuple=True)[0]
        if sel.numel() == 0:
            continue
        blk = torch.full((FX // s, FY // s, FZ // s), -1, dtype=torch.int64, device=dev)
        blk[li[sel] // s, lj[sel] // s, lk[sel] // s] = sel
        full = expand(blk, s)
        ids = torch.where(full >= 0, full, ids)

    corner = torch.stack([li, lj, lk]).contiguous()
    owners, neighbours, axes = [], [], []
    for ax in range(3):
        shape = [FX, FY, FZ]
        shape[ax] -= 1
        keys = torch.empty(int(np.prod(shape)), dtype=torch.int64, device=dev)
        call("gf_octree_face_keys", ptr(ids), FX, FY, FZ, ptr(corner), n, ax, ptr(keys), stream_ptr())
        if bool((keys == -2).any()):
            raise RuntimeError("gf_octree_face_keys: a finest cell is not covered by a leaf")
        keys = torch.sort(keys[keys >= 0]).values
        owners.append(keys // n)
        neighbours.append(keys % n)
        axes.append(torch.full_like(keys, ax))
    bnd_owner, bnd_dir = [], []
    for direction in range(6):
        ax, side_max = direction // 2, direction % 2 == 1
        cells = torch.unique(ids.select(ax, -1 if side_max else 0))
        bnd_owner.append(cells)
        bnd_dir.append(torch.full_like(cells, direction))

    def host(parts):
        return torch.cat(parts).cpu().numpy()

    leaves = tuple(t.cpu().numpy() for t in (li, lj, lk, ll))
    faces = (host(owners), host(neighbours), host(axes))
    domain = (host(bnd_owner), host(bnd_dir))
    return _octree_mesh(lo, hi, hf, L, (rx, ry, rz), leaves, faces, domain, bodies)
