"""Immersed-surface force integral against the reference.

The reference's own ``integrate_patch_on_surface_mesh`` ran on the
immersed-cylinder octree case (``tests/golden/forces_*.npz``, written by
``make_golden.py --forces``) with the mesh builder's body normals standing in
for its surface mesh.  The oracle restatement is pinned to it on CPU and the
device kernel (``gf_force_integral``) on the GPU.
"""

from __future__ import annotations

import pathlib

import numpy as np
import pytest

HERE = pathlib.Path(__file__).resolve().parent / "golden"


def _golden():
    with np.load(HERE / "forces_ibcyl_oct.npz") as d:
        return {k: d[k] for k in d.files}


def _close(a, b, scale, tol=1e-12):
    assert np.abs(np.asarray(a) - np.asarray(b)).max() <= tol * scale, (a, b)


def test_oracle_force_integral_matches_reference():
    from oracle.forces import patch_force
    from tests.golden.oracle_harness import oracle_case

    g = _golden()
    _, mesh, _, algo = oracle_case("ibcyl_oct")
    algo.U.data = g["U"].copy()
    algo.p.data = g["p"].copy()
    f, m, pf, vf = patch_force(algo.p, algo.U, g["nu_eff"], "cylinder", float(g["rho"]), g["cofr"],
                               mesh.ap.anchor_normal)
    scale = np.abs(g["force"]).max()
    _close(f, g["force"], scale)
    _close(m, g["moment"], scale)
    _close(pf, g["pressure_force"], np.abs(g["pressure_force"]).max())
    _close(vf, g["viscous_force"], np.abs(g["viscous_force"]).max())


@pytest.mark.gpu
def test_device_force_integral_matches_reference():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    from gridfoam_b200.post.forces import patch_force
    from tests.golden.device_harness import device_case

    g = _golden()
    _, _, grid, algo = device_case("ibcyl_oct")
    algo.U.data = torch.as_tensor(g["U"], device="cuda")
    algo.p.data = torch.as_tensor(g["p"], device="cuda")
    algo.phi.unpack(torch.as_tensor(g["phi"], device="cuda"))
    nu = torch.as_tensor(np.broadcast_to(g["nu_eff"], (grid.num_cells,)).copy(), device="cuda")
    res = patch_force(grid, algo.p, algo.U, nu, "cylinder", float(g["rho"]), g["cofr"])
    scale = np.abs(g["force"]).max()
    _close(res.force, g["force"], scale)
    _close(res.moment, g["moment"], scale)
    _close(res.pressure_force, g["pressure_force"], np.abs(g["pressure_force"]).max())
    _close(res.viscous_force, g["viscous_force"], np.abs(g["viscous_force"]).max())


def test_force_coefficients_and_axes():
    """coeffs.py:52-74 / coord.py:40-60: drag-lift axes are orthonormal and
    the coefficients split into front and rear parts as in the reference."""
    from gridfoam_b200.post.forces import ForceCoeffs, local_axes

    e1, e2, e3 = local_axes({"drag_dir": [2.0, 0.0, 0.0], "lift_dir": [0.3, 0.0, 1.0],
                             "center_of_rotation": [0, 0, 0]})
    np.testing.assert_allclose([e1 @ e1, e2 @ e2, e3 @ e3, e1 @ e2, e1 @ e3, e2 @ e3], [1, 1, 1, 0, 0, 0],
                               atol=1e-15)
    np.testing.assert_allclose(e3, [0, 0, 1], atol=1e-15)
    c = ForceCoeffs.from_force_moment(time=0.0, force=np.array([2.0, 1.0, 4.0]), moment=np.array([0.5, 1.0, 2.0]),
                                      e1=e1, e2=e2, e3=e3, force_scale=2.0, moment_scale=4.0)
    assert c.Cd == pytest.approx(1.0) and c.Cl == pytest.approx(2.0)
    assert c.Cd_f == pytest.approx(0.5 * c.Cd + c.CmRoll) and c.Cl_r == pytest.approx(0.5 * c.Cl - c.CmPitch)
