"""The octree mesh built on the GPU (``build_octree_mesh_device``) against
the host builder: the same mesh, array for array.

CPU: the slab-wise evaluation of signed-distance refinement regions against
one whole-grid evaluation.  GPU: the golden octree meshes, the cylinder
wake at a reduced base, a root grid without regions, and two overlapping
regions of different levels.
"""

from __future__ import annotations

import numpy as np
import pytest

from gridfoam_b200.mesh.builder import (
    Body,
    BoxRegion,
    SdfRegion,
    _required_levels,
    build_octree_mesh,
    cylinder_sdf,
)
from tests.golden.cases import ALL_CASES, build_mesh, cylinder_wake_case

MESH_ARRAYS = ("internal_faces_owner", "internal_faces_neighbour", "internal_faces_axis",
               "domain_bnd_faces_owner", "domain_bnd_faces_dir", "cell_centers", "cell_sizes")


def test_required_levels_slabs_match_whole_grid():
    lo = np.array([0.0, 0.0, 0.0])
    hf = np.array([0.25, 0.25, 0.5])
    shape = (70, 40, 6)
    sdf = cylinder_sdf((6.0, 5.0), 1.3)
    regions = [SdfRegion(sdf, 2.0, 2), BoxRegion((1.0, 1.0, 0.0), (3.0, 9.0, 3.0), 1)]
    got = _required_levels(lo, hf, shape, regions, slab=16)
    xs = lo[0] + (np.arange(shape[0]) + 0.5) * hf[0]
    ys = lo[1] + (np.arange(shape[1]) + 0.5) * hf[1]
    zs = lo[2] + (np.arange(shape[2]) + 0.5) * hf[2]
    P = np.stack(np.meshgrid(xs, ys, zs, indexing="ij"), axis=-1)
    want = np.where(sdf(P) <= 2.0, 2, 0).astype(np.int8)
    box = ((xs >= 1.0) & (xs <= 3.0))[:, None, None] & ((ys >= 1.0) & (ys <= 9.0))[None, :, None] \
        & ((zs >= 0.0) & (zs <= 3.0))[None, None, :]
    want = np.maximum(want, np.where(box, 1, 0).astype(np.int8))
    np.testing.assert_array_equal(got, want)


def _assert_same_mesh(a, b):
    assert a.n_cells == b.n_cells
    for k in MESH_ARRAYS:
        np.testing.assert_array_equal(getattr(a, k), getattr(b, k), err_msg=k)
    np.testing.assert_array_equal(a.meta["levels"], b.meta["levels"])
    assert a.patch_name_to_id == b.patch_name_to_id
    assert a.resolution == b.resolution
    for k, v in vars(a.ap).items():
        w = getattr(b.ap, k)
        if v is None:
            assert w is None, k
        else:
            np.testing.assert_array_equal(v, w, err_msg=k)


torch = pytest.importorskip("torch")


def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["cavity_oct", "duct_oct", "ibcyl_oct"])
def test_device_builder_matches_host_on_golden_octrees(name):
    _cuda()
    spec = ALL_CASES[name]()["mesh"]
    _assert_same_mesh(build_mesh(spec, device="cuda"), build_mesh(spec))


@pytest.mark.gpu
def test_device_builder_matches_host_on_cylinder_wake():
    _cuda()
    spec = cylinder_wake_case(base=(48, 32, 6), levels=2)["mesh"]
    _assert_same_mesh(build_mesh(spec, device="cuda"), build_mesh(spec))


@pytest.mark.gpu
def test_device_builder_without_regions_and_with_nested_levels():
    from gridfoam_b200.mesh.builder import build_octree_mesh_device

    _cuda()
    args = ((0.0, 0.0, 0.0), (3.0, 2.0, 1.0), (6, 4, 2))
    _assert_same_mesh(build_octree_mesh_device(*args, device="cuda"), build_octree_mesh(*args))
    body = Body(sdf=cylinder_sdf((1.5, 1.0), 0.3), patch="cyl")
    regions = [BoxRegion((0.2, 0.2, 0.0), (2.8, 1.8, 1.0), 1), SdfRegion(body.sdf, 0.4, 3)]
    _assert_same_mesh(build_octree_mesh_device(*args, regions, bodies=[body], device="cuda"),
                      build_octree_mesh(*args, regions, bodies=[body]))
