"""Case files and gridfoam YAML configs (CPU only).

* The reference's own example configs (``examples/*/gridfoam/data/config.yaml``)
  validate against ``gridfoam_b200.meta.config.GridfoamConfig`` unchanged;
  this runs where ``GRIDFOAM_REF`` names the reference's ``src`` directory
  and is skipped elsewhere.
* Every synthetic case of ``gridfoam_b200.cases`` round-trips through a YAML
  file and ``load_case``, and ``load_case`` rejects a file without a mesh.
"""

from __future__ import annotations

import os
import pathlib

import pytest
import yaml

from gridfoam_b200 import cases
from gridfoam_b200.meta.config import GridfoamConfig, SimulatorConfig


def _reference_examples() -> list[pathlib.Path]:
    src = os.environ.get("GRIDFOAM_REF")
    if not src:
        return []
    root = pathlib.Path(src).resolve().parent / "examples"
    return sorted(root.glob("*/gridfoam/data/config.yaml"))


@pytest.mark.skipif(not _reference_examples(), reason="GRIDFOAM_REF is not set to the reference's src directory")
@pytest.mark.parametrize("path", _reference_examples() or [None], ids=lambda p: p and p.parts[-4])
def test_reference_example_configs_validate(path):
    data = yaml.safe_load(path.read_text())
    cfg = GridfoamConfig.model_validate(data)
    assert cfg.simulator.fvSolution.solvers
    assert cfg.fluxel.root_resolution


CASE_BUILDERS = {
    "cavity32": lambda: cases.cavity_case(32),
    "pipe64": lambda: cases.pipe_case(64, 256, 4.0),
    "channel": cases.channel_case,
    "channel_ffp": cases.ffp_case,
    "ibplane": cases.ibplane_case,
    "cavity_oct": cases.cavity_oct_case,
    "duct_oct": cases.duct_oct_case,
    "ibcyl_oct": cases.ibcyl_oct_case,
    "cylinder_wake": lambda: cases.cylinder_wake_case((256, 160, 32)),
}


@pytest.mark.parametrize("name", sorted(CASE_BUILDERS))
def test_case_yaml_round_trip(name, tmp_path):
    case = CASE_BUILDERS[name]()
    path = tmp_path / f"{name}.yaml"
    path.write_text(yaml.safe_dump(case))
    loaded = cases.load_case(path)
    assert loaded["mesh"] == case["mesh"]
    assert loaded["inlet_profile"] == case["inlet_profile"]
    a = SimulatorConfig.model_validate(loaded["simulator"])
    b = SimulatorConfig.model_validate(case["simulator"])
    assert a == b


def test_load_case_requires_mesh(tmp_path):
    case = cases.cavity_case(8)
    del case["mesh"]
    path = tmp_path / "bad.yaml"
    path.write_text(yaml.safe_dump(case))
    with pytest.raises(ValueError, match="mesh"):
        cases.load_case(path)
