"""fvc.reconstruct and the potential-flow initialisation against the
reference (``tests/golden/potential_*.npz``, written by
``make_golden.py --potential``): the oracle on CPU, the device path on GPU,
on an octree duct and an immersed cylinder in a refined band."""

from __future__ import annotations

import pathlib

import numpy as np
import pytest

from tests.golden.cases import POTENTIAL_CASES, build_mesh, potential_case

HERE = pathlib.Path(__file__).resolve().parent / "golden"


def _golden(name):
    with np.load(HERE / f"potential_{name}.npz") as d:
        return {k: d[k] for k in d.files}


def _rel(a, b):
    return float(np.abs(np.asarray(a) - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("name", POTENTIAL_CASES)
def test_oracle_potential_flow_matches_reference(name):
    from oracle.case import Case, CellField, FaceField
    from oracle.potential import fvc_reconstruct, potential_flow

    g = _golden(name)
    case_def = potential_case(name)
    case = Case(build_mesh(case_def["mesh"]), case_def["simulator"])
    U = CellField(case, "U", "local", (3,))
    p = CellField(case, "p", "local", ())
    phi = FaceField(case, "phi")
    Phi = potential_flow(case, U, p, phi)
    assert Phi is not None
    assert _rel(U.data, g["U"]) < 1e-9
    assert _rel(phi.pack(), g["phi"]) < 1e-9
    # reconstruct on the reference's initial flux
    U2 = CellField(case, "U_rec", "local", (3,))
    phi2 = FaceField(case, "phi_init")
    n = [phi2.single_data.size, phi2.domain_bnd_data.size, phi2.immersed_upper.size]
    parts = np.split(g["init_phi"], np.cumsum(n))
    phi2.single_data, phi2.domain_bnd_data, phi2.immersed_upper, phi2.immersed_lower = (x.copy() for x in parts)
    assert _rel(fvc_reconstruct(phi2, U2), g["reconstruct_init"]) < 1e-13


@pytest.mark.gpu
@pytest.mark.parametrize("name", POTENTIAL_CASES)
def test_device_potential_flow_matches_reference(name):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    from gridfoam_b200.core.grid import AxisProjectedGrid
    from gridfoam_b200.fv import fvc
    from gridfoam_b200.meta.config import SimulatorConfig
    from gridfoam_b200.pre.potential_flow import PotentialFlow

    g = _golden(name)
    case_def = potential_case(name)
    grid = AxisProjectedGrid(SimulatorConfig.model_validate(case_def["simulator"]), build_mesh(case_def["mesh"]),
                             device="cuda")
    pf = PotentialFlow(grid)
    pf.solve()
    assert _rel(pf.U.data.cpu().numpy(), g["U"]) < 1e-8
    assert _rel(pf.phi.pack().cpu().numpy(), g["phi"]) < 1e-8
    phi0 = pf.phi
    phi0.unpack(torch.as_tensor(g["init_phi"], device="cuda"))
    rec = fvc.reconstruct(phi0, pf.U)
    assert _rel(rec.cpu().numpy(), g["reconstruct_init"]) < 1e-13
