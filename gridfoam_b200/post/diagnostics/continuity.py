"""Continuity error of a face flux (gridfoam ``post/diagnostics/continuity.py``).

``compute_continuity_error`` keeps the reference's signature and host
result.  The sums behind it come from one device reduction
(``gf_continuity_sums``: fixed-order block partials, the same bits on every
launch), and ``continuity_sums_async`` leaves them on the device so a
caller can copy them to the host off the critical path.
"""

from __future__ import annotations

import torch

from gridfoam_b200._lib import call, load, ptr, stream_ptr
from gridfoam_b200.fv import fvc


def scratch_doubles() -> int:
    return int(load().gf_continuity_scratch_doubles())


def continuity_sums_async(phi, cell_volumes: torch.Tensor, out: torch.Tensor, scratch: torch.Tensor) -> None:
    """Enqueue ``out[0:3] = (sum |div phi| V, sum div phi V, sum V)`` on the
    current stream; ``div phi = fvc.div(phi)`` as in the reference."""
    div = fvc.div(phi).store
    n = div.shape[-1]
    vol = cell_volumes.contiguous()
    if out.numel() < 3 or scratch.numel() < scratch_doubles():
        raise ValueError("continuity sums need a 3-double output and gf_continuity_scratch_doubles() scratch")
    call("gf_continuity_sums", n, ptr(div), ptr(vol), ptr(scratch), ptr(out), stream_ptr())


def compute_continuity_error(phi, cell_volumes: torch.Tensor, delta_t: float) -> tuple[float, float]:
    """post/diagnostics/continuity.py:11-49: ``(local, global)`` continuity
    errors, ``dt * sum(|div phi| V) / sum(V)`` and ``dt * sum(div phi V) /
    sum(V)``.  Returns host floats (one synchronisation, as the reference's
    ``.item()``)."""
    dev = cell_volumes.device
    out = torch.empty(3, dtype=torch.float64, device=dev)
    scratch = torch.empty(scratch_doubles(), dtype=torch.float64, device=dev)
    continuity_sums_async(phi, cell_volumes, out, scratch)
    a, g, v = out.tolist()
    return delta_t * (a / v), delta_t * (g / v)
