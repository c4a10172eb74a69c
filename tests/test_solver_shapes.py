"""Host logic of the CG launch-shape choice (no GPU): the size bands of
``default_variant`` and the autotuner's variant table."""

from __future__ import annotations

import pytest

from gridfoam_b200.solvers.autotune import N_VARIANTS, VARIANTS
from gridfoam_b200.solvers.krylov import default_variant


@pytest.mark.parametrize(
    "n, mixed, symmetric, box, want",
    [
        (512, False, True, True, 10),         # tiny FP64: halo form (falls back to 8 below its flag space)
        (262144, False, True, True, 10),      # 64^3
        (400000, False, True, True, 10),
        (400001, False, True, True, 8),       # q-recurrence band
        (1048576, False, True, True, 8),      # the IB pipe
        (1300001, False, True, True, 5),      # symmetric box beyond shared memory: staged tiles
        (1300001, False, False, True, 29),
        (1300001, False, True, False, 29),    # ELL beyond shared memory: split CG
        (4096, True, True, True, 0),          # FP32-inner below ~32K: register blocks
        (32767, True, True, True, 0),
        (32768, True, True, True, 10),        # FP32-inner halo form
        (1048576, True, True, False, 10),
        (1300001, True, True, True, 2),
    ],
)
def test_default_variant_bands(n, mixed, symmetric, box, want):
    assert default_variant(n, mixed, symmetric, box) == want


def test_variant_table_covers_every_launch_shape():
    assert sorted(VARIANTS) == list(range(N_VARIANTS))
    assert N_VARIANTS == 32
