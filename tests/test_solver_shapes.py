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


def test_split_and_persistent_variant_sets():
    """Every launch shape is either a split CG (graph-loop) form or a
    single-launch form; the headline octree's pressure CG takes a split one."""
    from gridfoam_b200.solvers.autotune import PERSISTENT_VARIANTS, SPLIT_VARIANTS

    assert not set(SPLIT_VARIANTS) & set(PERSISTENT_VARIANTS)
    assert set(SPLIT_VARIANTS) | set(PERSISTENT_VARIANTS) == set(range(N_VARIANTS))
    assert default_variant(4_079_808, False, True, False) in SPLIT_VARIANTS


def test_bench_traffic_table_holds_the_default_variant():
    """The bench's measured DRAM bytes per cell-iteration (its roofline's
    ``traffic``) exist for the variant the 4.08M-cell wake runs by default."""
    import bench

    v = default_variant(4_079_808, False, True, False)
    assert v in bench.PCG_DRAM_BYTES_PER_CELL_ITER
    assert 0.9 < bench.PCG_DRAM_BYTES_PER_CELL_ITER[v] / (14 * 8 + 3 * 16) < 1.2
