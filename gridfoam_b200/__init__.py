"""gridfoam_b200: gridfoam's per-iteration hot path on NVIDIA B200 (sm_100a).

Finite-volume assembly, the pressure/momentum Krylov solves and the SIMPLE,
PISO and PIMPLE loops of gridfoam, behind the same Python solver/operator/
YAML API, with every numerical step in hand-written CUDA kernels loaded
from the in-tree C-ABI library ``gridfoam_b200/_lib/libgridfoam_b200.so``.
"""

__version__ = "0.1.0"
