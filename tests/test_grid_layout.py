"""Host-side grid set-up: ELL adjacency, boundary-face layout and the
uniform-box detection that lets CG skip the neighbour table (no GPU)."""

from __future__ import annotations

import numpy as np
import pytest

from gridfoam_b200.core.grid import AxisProjectedGrid
from gridfoam_b200.meta.config import SimulatorConfig
from tests.golden.cases import ALL_CASES, build_mesh


def _grid(name: str):
    case = ALL_CASES[name]()
    mesh = build_mesh(case["mesh"])
    return mesh, AxisProjectedGrid(SimulatorConfig.model_validate(case["simulator"]), mesh, device="cpu")


@pytest.mark.parametrize("name", ["cavity8", "pipe10x20", "channel", "ibplane"])
def test_ell_covers_every_face_once(name):
    mesh, g = _grid(name)
    h = g.host
    C, F, W = g.num_cells, g.num_internal_faces, g.ell_width
    code = h.extra["ell_code"].reshape(W, C)
    nbr = h.extra["ell_nbr"].reshape(W, C)
    internal = code[(code >= 0) & (code < 2 * F)]
    # every internal face appears once from each side
    assert np.array_equal(np.sort(internal), np.arange(2 * F))
    domain = code[code >= 2 * F] // 2 - F
    assert np.array_equal(np.sort(domain), np.arange(g.num_domain_bnd_faces))
    # the owner-side slot of face f couples owner -> neighbour
    pos_o, pos_n = h.extra["face_pos_owner"], h.extra["face_pos_neigh"]
    assert np.array_equal(nbr.reshape(-1)[pos_o], h.neighbour)
    assert np.array_equal(nbr.reshape(-1)[pos_n], h.owner)
    assert np.array_equal(pos_o % C, h.owner) and np.array_equal(pos_n % C, h.neighbour)


def test_boundary_faces_follow_packed_order():
    mesh, g = _grid("pipe10x20")
    h = g.host
    Fb, Fi = g.num_domain_bnd_faces, g.num_immersed_faces
    assert Fi > 0 and g.num_bnd == Fb + 2 * Fi
    imm = np.nonzero(mesh.ap.is_immersed_face)[0]
    assert np.array_equal(h.bnd_cell[Fb : Fb + Fi], mesh.internal_faces_owner[imm])
    assert np.array_equal(h.bnd_cell[Fb + Fi :], mesh.internal_faces_neighbour[imm])
    np.testing.assert_allclose(h.bnd_mag_d[Fb : Fb + Fi], mesh.ap.dist_owner_to_bnd)
    # outward normals: upper side along +Sf, lower side along -Sf
    assert np.all(h.bnd_sf[Fb : Fb + Fi].sum(axis=1) > 0)
    assert np.all(h.bnd_sf[Fb + Fi :].sum(axis=1) < 0)


@pytest.mark.parametrize("name,strides", [("cavity8", (8, 64)), ("pipe10x20", (10, 100)), ("channel", (16, 128))])
def test_uniform_box_is_detected(name, strides):
    _, g = _grid(name)
    assert g.ell_width == 6
    assert g.box_strides == strides


def test_permuted_mesh_is_not_a_box():
    case = ALL_CASES["cavity8"]()
    mesh = build_mesh(case["mesh"])
    perm = np.random.default_rng(0).permutation(mesh.n_cells)
    inv = np.argsort(perm)
    mesh.cell_centers = mesh.cell_centers[perm]
    mesh.cell_sizes = mesh.cell_sizes[perm]
    mesh.internal_faces_owner = inv[mesh.internal_faces_owner]
    mesh.internal_faces_neighbour = inv[mesh.internal_faces_neighbour]
    mesh.domain_bnd_faces_owner = inv[mesh.domain_bnd_faces_owner]
    g = AxisProjectedGrid(SimulatorConfig.model_validate(case["simulator"]), mesh, device="cpu")
    assert g.box_strides is None


@pytest.mark.parametrize("name", ["cavity_oct", "duct_oct", "ibcyl_oct", "ibplane"])
def test_ell_rows_are_packed_with_at_least_six_slots(name):
    """The octree gradient and assembly kernels (6 < W <= 12) stage a row's
    first six slots unconditionally and read slot 6 on to the row's first
    empty slot: every row holds one or more faces in each of its six
    directions, its used slots come first, and its internal-face slots (the
    matrix couplings, up to ell_len) lead it."""
    _, g = _grid(name)
    h = g.host
    C, F, W = g.num_cells, g.num_internal_faces, g.ell_width
    code = h.extra["ell_code"].reshape(W, C)
    used = code >= 0
    count = used.sum(0)
    assert count.min() >= 6
    # packed: slot s used exactly when s < count
    assert np.array_equal(used, np.arange(W)[:, None] < count[None, :])
    # couplings first: internal-face slots exactly below ell_len
    internal = used & (code < 2 * F)
    ell_len = np.asarray(h.extra["ell_len"])
    if g.box_strides is None:
        assert np.array_equal(internal, np.arange(W)[:, None] < ell_len[None, :])
    if name != "ibplane":
        assert 6 < W <= 12
