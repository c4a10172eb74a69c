"""OpenFOAM ``adjustPhi`` on the device (gridfoam ``fv/adjust_phi.py``)."""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from gridfoam_b200._lib import call, ptr, stream_ptr
from gridfoam_b200.core.boundary import DirichletBC, InletOutletBC


def adjust_classes(U) -> torch.Tensor:
    """adjust_phi.py:14-41, per domain face: 0 no condition on its patch,
    1 fixed value (Dirichlet, not inletOutlet), 2 adjustable."""
    g = U.grid
    cls = np.zeros(g.num_domain_bnd_faces, dtype=np.int8)
    for patch, bc in U.bcs.items():
        faces = g.patch_faces(patch)
        faces = faces[faces < g.num_domain_bnd_faces]
        fixes = isinstance(bc, DirichletBC) and not isinstance(bc, InletOutletBC)
        cls[faces] = 1 if fixes else 2
    return torch.as_tensor(cls, device=g.device)


def adjust_phi(phi, U, p=None, classes: torch.Tensor | None = None) -> bool:
    """adjust_phi.py:44-127: scale adjustable outflow on domain faces to
    balance inflow (one-block kernel, no host round trip).  A no-op when
    ``p`` has a Dirichlet condition.  Returns whether the kernel ran."""
    if p is not None and any(isinstance(bc, DirichletBC) for bc in p.bcs.values()):
        return False
    if U.grid.num_domain_bnd_faces == 0:
        return False
    cls = adjust_classes(U) if classes is None else classes
    call("gf_adjust_phi", ctypes.byref(U.grid.cmesh), ptr(cls), ptr(phi.store), stream_ptr())
    return True
