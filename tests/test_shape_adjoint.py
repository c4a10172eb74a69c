"""Shape gradient of the bluff body's drag (steady SIMPLE, fixed-point
adjoint) against central finite differences of the device solver, on a
uniform channel and on a 3-level octree (hanging faces).

The body (8 shape parameters: length, width, height, the two front
rounding radii, slant angle in degrees, slant length, ground clearance) sits
in a uniform 60x18x12 channel over [-1, 3] x [-0.6, 0.6] x [0, 0.8]; its
steady state is converged with exact solves so that it is the discrete
solution.  Every perturbed mesh (h up to 1e-3) keeps the immersed faces and
near flags of the base mesh, so the finite differences see the smooth
dependence the adjoint differentiates.

Central differences at h = 1e-3 carry their own truncation error: second
order (3e-4 relative at h = 1e-3) for six parameters, first order for the
two front rounding radii (5e-3), whose perturbation moves the front
stagnation region where face fluxes change sign (upwind is not twice
differentiable there).  The test therefore checks the differences at
h = 1e-3, 5e-4 and 2.5e-4: their error against the adjoint shrinks as h
does, and the Richardson extrapolation with the order estimated from the
three of them matches the adjoint to 1e-4.
"""

from __future__ import annotations

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

RES, LO, HI = (60, 18, 12), (-1.0, -0.6, 0.0), (3.0, 0.6, 0.8)
STEPS = (1e-3, 5e-4, 2.5e-4)


@pytest.fixture(autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")


def _make(params):
    from gridfoam_b200.cases import bluff_body_case, create_case

    return create_case(bluff_body_case(RES, params=params, uniform=True, lower=LO, upper=HI), device="cuda")


def _drag(grid, algo) -> float:
    from gridfoam_b200.post.forces import patch_force

    return float(patch_force(grid, algo.p, algo.U, algo.nu, "body", 1.0, np.zeros(3)).force[0])


def _make_octree(params):
    from gridfoam_b200.cases import bluff_body_case, create_case

    case = bluff_body_case(OCT_RES, levels=2, params=params, lower=OCT_LO, upper=OCT_HI)
    return create_case(case, device="cuda")


# 3-level octree channel (levels 0-2, 28,146 cells, 6,016 hanging faces):
# no perturbation up to 1e-3 changes the immersed faces, near flags or the
# refinement.  Central differences there are far from their limit at
# h = 1e-3 (1e-2 to 1e-1) and converge to the adjoint as h shrinks, so the
# check uses h = 5e-4, 2.5e-4, 1.25e-4.
OCT_RES, OCT_LO, OCT_HI = (30, 10, 8), (-1.03, -0.61, 0.0), (3.0, 0.61, 0.8)
OCT_STEPS = (5e-4, 2.5e-4, 1.25e-4)


@pytest.mark.parametrize("make", ["uniform", "octree"])
def test_differentiable_iteration_matches_library_step(make):
    """One evaluation of the differentiable SIMPLE iteration against the
    library's step from the same state, both with exact solves."""
    from gridfoam_b200.solvers import shape_adjoint as sa

    from gridfoam_b200.mesh.builder import BLUFF_DEFAULT

    _, grid, algo = (_make if make == "uniform" else _make_octree)(BLUFF_DEFAULT)
    for _ in range(20):
        algo.step()
    it = sa.DifferentiableSimpleIteration(algo)
    U, p, phi = it.state()
    trace = {}
    with sa.exact_solves(algo, rtol=1e-13), torch.no_grad():
        U1, p1, phi1 = it.step(U, p, phi, it.distances(), trace=trace)
        algo.step()

    def rel(a, b):
        return float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))

    assert rel(trace["rAtU"], algo.rAtU.store[0]) < 1e-13
    assert rel(trace["HbyA"], algo.HbyA.data) < 1e-12
    assert rel(trace["phiHbyA"], algo.phi_hbya.store[0]) < 1e-12
    assert rel(phi1, algo.phi.store[0]) < 1e-10
    # outside the body (its enclosed cells hold a pressure fixed only up to
    # a constant)
    from gridfoam_b200.mesh.builder import bluff_body_sdf

    c = grid.host.cell_centers
    ext = torch.as_tensor(np.nonzero(bluff_body_sdf(0.0, BLUFF_DEFAULT)(np.asarray(c)) > 0)[0], device="cuda")
    assert rel(U1[ext], algo.U.data[ext]) < 1e-10
    assert rel(p1[ext], algo.p.data[ext]) < 1e-10


def _check_against_differences(make, theta, steps, extent):
    """Adjoint gradient and central differences at ``steps``; returns the
    relative errors of the differences ``[len(steps), P]`` and the
    differences themselves."""
    from gridfoam_b200.mesh.builder import bluff_body_sdf
    from gridfoam_b200.solvers import shape_adjoint as sa

    mesh, grid, algo = make(tuple(theta))
    sdf = bluff_body_sdf(0.0, theta)
    ext = torch.as_tensor(np.nonzero(sdf(np.asarray(mesh.cell_centers)) > 0)[0], device="cuda")
    sa.converge_exact(algo, cells=ext)
    it = sa.DifferentiableSimpleIteration(algo)
    U, p, phi = it.state()
    with torch.no_grad():
        U1, p1, _ = it.step(U, p, phi, it.distances())
    assert float(torch.linalg.vector_norm(U1[ext] - U[ext]) / torch.linalg.vector_norm(U[ext])) < 1e-10
    J0 = _drag(grid, algo)
    g = sa.shape_gradient(algo, lambda t: bluff_body_sdf(0.0, t), theta, patch="body", extent=extent)
    assert abs(g.objective - J0) < 1e-12 * abs(J0)
    assert g.adjoint_change < 1e-10
    base = it.state()
    imm0 = np.asarray(grid.host.imm_faces)
    near0 = np.asarray(grid.host.bnd_near)
    fd = np.zeros((len(steps), theta.size))
    for k, h in enumerate(steps):
        for j in range(theta.size):
            J = []
            for sign in (1.0, -1.0):
                th = theta.copy()
                th[j] += sign * h
                _, gj, aj = make(tuple(th))
                assert gj.num_cells == grid.num_cells
                assert np.array_equal(np.asarray(gj.host.imm_faces), imm0)
                assert np.array_equal(np.asarray(gj.host.bnd_near), near0)
                with torch.no_grad():
                    aj.U.store.copy_(base[0].t())
                    aj.p.store.copy_(base[1].reshape(1, -1))
                    aj.phi.store[0].copy_(base[2])
                sa.converge_exact(aj, cells=ext)
                J.append(_drag(gj, aj))
                del aj, gj
            fd[k, j] = (J[0] - J[1]) / (2 * h)
    err = np.abs(fd - g.grad) / np.abs(g.grad)
    return err, fd, g.grad


def test_bluff_drag_shape_gradient_matches_finite_differences_octree():
    """On the octree the differences approach the adjoint as h shrinks
    (second order for most parameters, with an irregular first step where
    face fluxes change sign); at h = 1.25e-4 every parameter is within
    1e-3 of the adjoint."""
    from gridfoam_b200.mesh.builder import BLUFF_DEFAULT

    err, fd, grad = _check_against_differences(_make_octree, np.array(BLUFF_DEFAULT), OCT_STEPS,
                                               extent=max(h - l for h, l in zip(OCT_HI, OCT_LO)))
    assert np.all((err[2] < err[0]) | (err[2] < 1e-5)), err
    assert np.all(err[2] < 1e-3), err


def test_bluff_drag_shape_gradient_matches_finite_differences():
    from gridfoam_b200.mesh.builder import BLUFF_DEFAULT

    err, fd, grad = _check_against_differences(_make, np.array(BLUFF_DEFAULT), STEPS, extent=4.0)
    assert np.all(err[0] < 1e-2), err
    assert np.all((err[2] < err[0]) | (err[2] < 1e-5)), err
    # Richardson extrapolation with the observed order of each parameter
    d1, d2 = fd[0] - fd[1], fd[1] - fd[2]
    order = np.clip(np.log2(np.abs(d1 / np.where(d2 != 0, d2, 1e-300))), 0.5, 3.0)
    rich = fd[2] + (fd[2] - fd[1]) / (2.0**order - 1.0)
    rel = np.abs(rich - grad) / np.abs(grad)
    assert np.all(rel < 1e-4), (rel, order)
