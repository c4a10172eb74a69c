"""Immersed-surface forces and coefficients (gridfoam ``post/forces``).

``patch_force`` integrates one immersed patch with the ``gf_force_integral``
kernel: axis-projected boundary samples whose outward direction points into
the body contribute ``rho p_b Sf`` and ``-rho nu (gradU + gradU^T) Sf``
(post/forces/sampling.py:69-168, integration.py:76-187).  The reference
orients samples by its STL surface mesh; here the mesh builder supplies the
body-outward normal of each anchor (immersed face) from the body's signed
distance, so no surface mesh is read.  ``ForceEvaluator`` and ``ForceCoeffs``
follow post/forces/evaluator.py and coeffs.py.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from gridfoam_b200._lib import GfBcAux, call, ptr, stream_ptr


@dataclass
class PatchForce:
    force: np.ndarray            # [3]
    moment: np.ndarray           # [3] about the centre of rotation
    pressure_force: np.ndarray   # [n_anchor, 3] per surface anchor
    viscous_force: np.ndarray    # [n_anchor, 3]


def _anchor_normals(grid) -> torch.Tensor:
    cache = grid.__dict__.setdefault("_post_cache", {})
    t = cache.get("anchor_normal")
    if t is None:
        normals = grid.host.extra.get("anchor_normal")
        if normals is None:
            raise ValueError("the mesh carries no anchor normals for the force integral")
        t = torch.as_tensor(np.ascontiguousarray(normals.T), dtype=torch.float64, device=grid.device)
        cache["anchor_normal"] = t
    return t


def _eval(field) -> None:
    aux = GfBcAux()
    phi = field.grid.get_facefield("phi")
    if phi is not None:
        aux.phi_bnd = ptr(phi.boundary_store)
    field.evaluate_bc(aux)


def patch_force(grid, p, U, nu_eff, patch_name: str, rho: float, center_of_rotation) -> PatchForce:
    """integration.py:125-187 on the device for one immersed patch."""
    if grid.num_immersed_faces == 0:
        raise ValueError("the grid has no immersed faces")
    faces = torch.as_tensor(grid.patch_faces(patch_name), dtype=torch.int32, device=grid.device)
    faces = faces[faces >= grid.num_domain_bnd_faces].contiguous()
    n = int(faces.numel())
    _eval(p)
    _eval(U)
    normals = _anchor_normals(grid)
    samples = torch.zeros((12, max(n, 1)), dtype=torch.float64, device=grid.device)
    total = torch.zeros(6, dtype=torch.float64, device=grid.device)
    nu_t = nu_eff if isinstance(nu_eff, torch.Tensor) else None
    if nu_t is not None:
        nu_t = nu_t.to(device=grid.device, dtype=torch.float64).contiguous()
    cofr = [float(v) for v in np.asarray(center_of_rotation, dtype=np.float64).reshape(3)]
    pt, ut = p.table, U.table
    call("gf_force_integral", ctypes.byref(grid.cmesh), n, ptr(faces), ptr(normals), ptr(pt.kind),
         ctypes.byref(pt.cstate), ptr(p.store), ptr(ut.kind), ctypes.byref(ut.cstate), ptr(U.store), ptr(nu_t),
         0.0 if nu_t is not None else float(nu_eff), float(rho), *cofr, ptr(samples), ptr(total), stream_ptr())
    # Per-anchor accumulation (integration.py:37-73): an anchor has at most
    # one sample per side, so the two-term sums are order independent.
    Fb, Fi = grid.num_domain_bnd_faces, grid.num_immersed_faces
    anchor = (faces.long() - Fb) % Fi
    pf = torch.zeros((Fi, 3), dtype=torch.float64, device=grid.device)
    vf = torch.zeros_like(pf)
    if n:
        pf.index_add_(0, anchor, samples[0:3, :n].t())
        vf.index_add_(0, anchor, samples[3:6, :n].t())
    tot = total.cpu().numpy()
    return PatchForce(tot[:3].copy(), tot[3:].copy(), pf.cpu().numpy(), vf.cpu().numpy())


@dataclass(frozen=True)
class ForceCoeffs:
    """post/forces/coeffs.py:11-74."""

    time: float
    Cd: float
    Cd_f: float
    Cd_r: float
    Cl: float
    Cl_f: float
    Cl_r: float
    CmPitch: float
    CmRoll: float
    CmYaw: float
    Cs: float
    Cs_f: float
    Cs_r: float

    @classmethod
    def from_force_moment(cls, *, time, force, moment, e1, e2, e3, force_scale, moment_scale):
        Cd = float(force @ e1) / force_scale
        Cs = float(force @ e2) / force_scale
        Cl = float(force @ e3) / force_scale
        CmRoll = float(moment @ e1) / moment_scale
        CmPitch = float(moment @ e2) / moment_scale
        CmYaw = float(moment @ e3) / moment_scale
        return cls(time, Cd, 0.5 * Cd + CmRoll, 0.5 * Cd - CmRoll, Cl, 0.5 * Cl + CmPitch, 0.5 * Cl - CmPitch,
                   CmPitch, CmRoll, CmYaw, Cs, 0.5 * Cs + CmYaw, 0.5 * Cs - CmYaw)


def _unit(v) -> np.ndarray:
    v = np.asarray(v, dtype=np.float64)
    return v / np.linalg.norm(v)


def local_axes(local_coord: dict) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """post/forces/coord.py:40-60: drag/lift or drag/pitch orthonormal axes."""
    e1 = _unit(local_coord["drag_dir"])
    if "lift_dir" in local_coord:
        lift = np.asarray(local_coord["lift_dir"], dtype=np.float64)
        e3 = _unit(lift - e1 * (lift @ e1))
        e2 = np.cross(e3, e1)
    else:
        pitch = np.asarray(local_coord["pitch_axis"], dtype=np.float64)
        e2 = _unit(pitch - e1 * (pitch @ e1))
        e3 = np.cross(e1, e2)
    return e1, e2, e3


class ForceEvaluator:
    """post/forces/evaluator.py:22-180, configured by the simulator's
    ``post_processing.forceCoeff`` section (patches, rho, magU_ref, A_ref,
    L_ref, local_coord)."""

    def __init__(self, grid, U, p):
        cfg = (grid.sim_config.post_processing or {}).get("forceCoeff")
        if cfg is None:
            raise ValueError("post_processing.forceCoeff is not configured")
        self.grid, self.U, self.p = grid, U, p
        self.patches = list(cfg["patches"])
        self.rho = float(cfg["rho"])
        q = 0.5 * self.rho * float(cfg["magU_ref"]) ** 2
        self.force_scale = q * float(cfg["A_ref"])
        self.moment_scale = self.force_scale * float(cfg["L_ref"])
        if self.force_scale == 0.0 or self.moment_scale == 0.0:
            raise ValueError("force coefficient reference scale is zero")
        lc = cfg["local_coord"]
        self.e1, self.e2, self.e3 = local_axes(lc)
        self.cofr = np.asarray(lc["center_of_rotation"], dtype=np.float64)
        self.history: list[ForceCoeffs] = []

    def evaluate(self, time: float, nu_eff) -> ForceCoeffs:
        force = np.zeros(3)
        moment = np.zeros(3)
        for patch in self.patches:
            r = patch_force(self.grid, self.p, self.U, nu_eff, patch, self.rho, self.cofr)
            force += r.force
            moment += r.moment
        c = ForceCoeffs.from_force_moment(time=time, force=force, moment=moment, e1=self.e1, e2=self.e2,
                                          e3=self.e3, force_scale=self.force_scale,
                                          moment_scale=self.moment_scale)
        self.history.append(c)
        return c
