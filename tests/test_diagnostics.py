"""Per-step diagnostics and VTU export against the reference's own output.

The fixtures ``tests/golden/diagnostics_<case>.npz`` come from the
reference's ``DiagnosticsCollector`` attached to its algorithm
(``make_golden.py --diagnostics``: continuity every step, solver statistics
every third step and the last) and from its ``io/vtu.py`` export of the final
state through a pyvista stand-in that records points, cells and cell data.

CPU: the continuity oracle on the reference's own fluxes, the collector's
solverInfo rows from the reference's statistics (formatting, columns and
the record rule), the hexahedron points and connectivity, and the VTU file
round trip.  GPU: the device continuity sums on the reference's fluxes, a
whole run with the collector attached, and the synchronous and asynchronous
VTU exports.
"""

from __future__ import annotations

import csv
import pathlib

import numpy as np
import pytest

from oracle.diagnostics import continuity_rows
from tests.golden.cases import STEPS
from tests.golden.oracle_harness import oracle_case

HERE = pathlib.Path(__file__).resolve().parent / "golden"
CASES = ("cavity8", "pipe10x20")
SOLVER_INTERVAL = 3


def _golden(name):
    with np.load(HERE / f"diagnostics_{name}.npz") as d:
        return {k: d[k] for k in d.files}


def _read_csv(path):
    with open(path) as fh:
        return list(csv.reader(fh))


@pytest.mark.parametrize("name", CASES)
def test_continuity_oracle_matches_reference(name):
    g = _golden(name)
    _, _, case, _ = oracle_case(name)
    phis = [g[f"step{k}_phi"] for k in range(int(g["n_steps"]))]
    rows = continuity_rows(case, phis, float(g["delta_t"]))
    ref = g["continuity"]
    assert rows.shape == ref.shape
    np.testing.assert_array_equal(rows[:, 0], ref[:, 0])
    # A cell's net flux cancels face fluxes up to ~1e6 times larger (the
    # pipe), so summation order alone moves it by ~1e-10 relative.
    np.testing.assert_allclose(rows[:, 1], ref[:, 1], rtol=1e-9, atol=0)
    # the signed sums cancel to rounding level: compare against the local scale
    scale = np.abs(ref[:, 1]).max()
    assert np.abs(rows[:, 2] - ref[:, 2]).max() <= 1e-9 * scale
    assert np.abs(rows[:, 3] - ref[:, 3]).max() <= 1e-9 * scale


class _Stats:
    """A solve statistic with the SolveStats attributes the collector reads."""

    def __init__(self, solver, initial, final, iters, converged):
        self.solver = solver
        self.initial_residual = float(initial)
        self.final_residual = float(final)
        self.iterations = int(iters)
        self.converged = bool(int(converged))

    def ready(self) -> bool:
        return True


class _Field:
    def __init__(self, nc):
        self.num_components = nc


class _Grid:
    """What the collector reads of a grid when only solverInfo is enabled."""

    device = "cpu"

    def __init__(self, fields):
        self._fields = fields
        self.sim_config = type("S", (), {"conditions": {}})()

    def get_cellfield(self, name):
        return self._fields.get(name)


@pytest.mark.parametrize("name", CASES)
def test_solver_info_rows_match_reference_format(name, tmp_path):
    """The reference's statistics fed through this collector reproduce its
    solver_info.csv text: header, columns, number formatting, and the record
    rule (every third step and the last)."""
    from gridfoam_b200.post.diagnostics import DiagnosticsCollector

    g = _golden(name)
    n_steps = int(g["n_steps"])
    dt = float(g["delta_t"])
    ref_rows = [list(r) for r in g["solver_info"]]
    by_time = {float(r[0]): r for r in ref_rows}
    grid = _Grid({"U": _Field(3), "p": _Field(1)})
    cfg = {"solverInfo": {"writeInterval": SOLVER_INTERVAL}}
    with DiagnosticsCollector.from_config(grid, cfg, tmp_path, n_steps=n_steps, delta_t=dt) as diag:
        for step in range(1, n_steps + 1):
            row = by_time.get(step * dt)
            if row is None:  # not a recorded step: the stats are never read
                stats = {"U": (None, None, None), "p": (None,)}
            else:
                vals = [row[1 + 5 * k:6 + 5 * k] for k in range(4)]
                stats = {"U": tuple(_Stats(*v) for v in vals[:3]), "p": (_Stats(*vals[3]),)}
            diag.record_step(step, None, stats)
    out = _read_csv(tmp_path / "solver_info.csv")
    assert out[0] == list(g["solver_info_header"])
    assert out[1:] == ref_rows
    assert not (tmp_path / "continuity_error.csv").exists()


@pytest.mark.parametrize("name", CASES)
def test_vtu_points_and_cells_match_reference(name):
    from gridfoam_b200.io.vtu import VTK_HEXAHEDRON, hex_points

    g = _golden(name)
    _, _, case, _ = oracle_case(name)
    n = case.num_cells
    np.testing.assert_array_equal(hex_points(case.cell_centers, case.cell_sizes), g["vtu_points"])
    cells = g["vtu_cells"].reshape(n, 9)
    assert np.all(cells[:, 0] == 8)
    np.testing.assert_array_equal(cells[:, 1:], np.arange(8 * n).reshape(n, 8))
    assert np.all(g["vtu_cell_types"] == VTK_HEXAHEDRON)


def test_vtu_file_round_trip(tmp_path):
    from gridfoam_b200.io.vtu import UnstructuredGrid, hex_points, read_vtu

    g = _golden("cavity8")
    n = g["vtu_data_p"].shape[0]
    centers = g["vtu_points"].reshape(n, 8, 3).mean(axis=1)
    sizes = np.ptp(g["vtu_points"].reshape(n, 8, 3), axis=1)
    ug = UnstructuredGrid(hex_points(centers, sizes), np.arange(8 * n).reshape(n, 8),
                          np.full(n, 12, dtype=np.uint8),
                          {"U": g["vtu_data_U"], "p": g["vtu_data_p"]})
    path = tmp_path / "cavity.vtu"
    ug.save(path)
    text = path.read_bytes()[:600].decode(errors="replace")
    assert 'type="UnstructuredGrid"' in text and f'NumberOfCells="{n}"' in text
    back = read_vtu(path)
    np.testing.assert_array_equal(back.points, ug.points)
    np.testing.assert_array_equal(back.connectivity, ug.connectivity)
    np.testing.assert_array_equal(back.cell_types, ug.cell_types)
    assert sorted(back.cell_data) == ["U", "p"]
    np.testing.assert_array_equal(back.cell_data["U"], g["vtu_data_U"])
    np.testing.assert_array_equal(back.cell_data["p"], g["vtu_data_p"])


# ---------------------------------------------------------------------------
# GPU

torch = pytest.importorskip("torch")

# Tolerances of a whole run against the reference's run: cavity8 converges its
# solves tightly; the pipe's pressure solves stop loosely (rel 0.01), so its
# continuity error (a solver-residual-level quantity) and final residuals
# agree only in magnitude.
RUN_TOL = {"cavity8": dict(local=1e-6, initial=1e-8, final=1e-4, slack=0),
           "pipe10x20": dict(local=0.5, initial=1e-3, final=0.5, slack=1)}


def _device(name):
    from tests.golden.device_harness import device_case

    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    return device_case(name)


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_device_continuity_error_on_reference_flux(name):
    from gridfoam_b200.post.diagnostics import compute_continuity_error

    g = _golden(name)
    _, _, grid, algo = _device(name)
    dt = float(g["delta_t"])
    scale = np.abs(g["continuity"][:, 1]).max()
    for k in range(int(g["n_steps"])):
        algo.phi.unpack(torch.as_tensor(g[f"step{k}_phi"], device="cuda"))
        loc, glo = compute_continuity_error(algo.phi, grid.cell_volumes, dt)
        assert loc == pytest.approx(g["continuity"][k, 1], rel=1e-9)
        assert abs(glo - g["continuity"][k, 2]) <= 1e-9 * scale


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_collector_run_matches_reference(name, tmp_path):
    from gridfoam_b200.post.diagnostics import DiagnosticsCollector

    g = _golden(name)
    _, _, grid, algo = _device(name)
    tol = RUN_TOL[name]
    n_steps = STEPS[name]
    cfg = {"continuityError": {"writeInterval": 1}, "solverInfo": {"writeInterval": SOLVER_INTERVAL}}
    diag = DiagnosticsCollector.from_config(grid, cfg, tmp_path, n_steps=n_steps, delta_t=float(g["delta_t"]))
    algo.attach_diagnostics(diag)
    for _ in range(n_steps):
        algo.step()
    diag.close()

    cont = _read_csv(tmp_path / "continuity_error.csv")
    assert cont[0] == list(g["continuity_header"])
    vals = np.array(cont[1:], dtype=np.float64)
    ref = g["continuity"]
    assert vals.shape == ref.shape
    np.testing.assert_array_equal(vals[:, 0], ref[:, 0])
    np.testing.assert_allclose(vals[:, 1], ref[:, 1], rtol=tol["local"])
    np.testing.assert_allclose(vals[:, 3], np.cumsum(vals[:, 2]), rtol=1e-12, atol=1e-300)

    info = _read_csv(tmp_path / "solver_info.csv")
    assert info[0] == list(g["solver_info_header"])
    assert len(info) - 1 == len(g["solver_info"])
    for row, ref_row in zip(info[1:], g["solver_info"]):
        assert row[0] == ref_row[0]
        for k in range(4):
            s, r = row[1 + 5 * k:6 + 5 * k], list(ref_row[1 + 5 * k:6 + 5 * k])
            assert s[0] == r[0] and s[4] == r[4], (k, s, r)
            assert abs(int(s[3]) - int(r[3])) <= tol["slack"], (k, s, r)
            assert float(s[1]) == pytest.approx(float(r[1]), rel=tol["initial"])
            assert float(s[2]) == pytest.approx(float(r[2]), rel=tol["final"])


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_vtu_export_matches_reference_state(name, tmp_path):
    """Synchronous export after the golden steps: the reference's exported
    fields, points and cells; the asynchronous exporter writes the same
    bytes as the synchronous one at every step."""
    from gridfoam_b200.io.vtu import AsyncVtuExporter, read_vtu, save_export_fields_as_vtu

    g = _golden(name)
    _, _, grid, algo = _device(name)
    with AsyncVtuExporter(grid) as exp:
        for k in range(STEPS[name]):
            algo.step()
            exp.snapshot(tmp_path / f"async_{k}.vtu")
            save_export_fields_as_vtu(grid, str(tmp_path / f"sync_{k}.vtu"))
    for k in range(STEPS[name]):
        assert (tmp_path / f"async_{k}.vtu").read_bytes() == (tmp_path / f"sync_{k}.vtu").read_bytes()
    back = read_vtu(tmp_path / f"sync_{STEPS[name] - 1}.vtu")
    assert sorted(back.cell_data) == list(g["vtu_fields"])
    np.testing.assert_array_equal(back.points, g["vtu_points"])
    step_tol = 1e-10 if name == "cavity8" else 1e-4
    for key in g["vtu_fields"]:
        ref = g[f"vtu_data_{key}"]
        err = np.linalg.norm(back.cell_data[key] - ref) / np.linalg.norm(ref)
        assert err < (10 if key == "p" else 1) * step_tol, (key, err)
