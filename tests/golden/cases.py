"""Case tables of the golden fixtures and the tests.

The case definitions themselves live in ``gridfoam_b200.cases`` (the
product's case loader); this module adds the per-case step counts and
scheme lists the fixture generator and the tests share.
"""

from __future__ import annotations

import copy

from gridfoam_b200.cases import (  # noqa: F401
    TRANSIENT,
    WALL0,
    bluff_body_case,
    build_mesh,
    cavity_case,
    cavity_oct_case,
    channel_case,
    create_case,
    cylinder_wake_case,
    duct_oct_case,
    ffp_case,
    ibcyl_oct_case,
    ibplane_case,
    inlet_profile_values,
    pipe_analytic_uz,
    pipe_case,
)


def potential_case(name: str) -> dict:
    """A case definition with the potential-flow initialisation configured
    (fvSolution.potentialFlow and a ``Phi`` solver): one non-orthogonal
    corrector, Jacobi-CG to 1e-11."""
    case = copy.deepcopy(ALL_CASES[name]())
    sol = case["simulator"]["fvSolution"]
    sol["potentialFlow"] = {"nNonOrthogonalCorrectors": 1, "phiRefCell": 0, "phiRefValue": 0.0}
    sol["solvers"]["Phi"] = {"method": "cg", "preconditioner": "jacobi", "tolerance": 1e-11,
                             "rel_tolerance": 0.0, "max_iter": 5000}
    case["name"] = name + "_potential"
    return case



def ibplane_io_case() -> dict:
    """The immersed plate with an inletOutlet velocity condition on the
    plate: its near faces (zero ray distance) constrain their cells only
    while they carry inflow, so the Gibou constraints and the fixed-cell
    flux closure follow the flux (boundary_ops.py:440-535)."""
    case = copy.deepcopy(ibplane_case())
    bnd = case["simulator"]["conditions"]["U"]["boundary"]
    bnd["wall"]["patches"] = [p for p in bnd["wall"]["patches"] if p != "plate"]
    bnd["plate"] = {"type": "inlet_outlet", "patches": ["plate"], "value": [0.0, 0.0, 0.0]}
    case["name"] = "ibplane_io"
    return case


ALL_CASES = {
    "cavity8": lambda: cavity_case(8),
    "pipe10x20": lambda: pipe_case(10, 20),
    "channel": channel_case,
    "channel_ffp": ffp_case,
    "ibplane": ibplane_case,
    "ibplane_io": ibplane_io_case,
    "cavity_oct": cavity_oct_case,
    "duct_oct": duct_oct_case,
    "ibcyl_oct": ibcyl_oct_case,
}
# Cases on octree meshes (hanging faces).
OCTREE_CASES = ("cavity_oct", "duct_oct", "ibcyl_oct")
# Cases whose potential-flow initialisation is pinned to the reference.
POTENTIAL_CASES = ("duct_oct", "ibcyl_oct")


# Steps stored per golden case and the convection schemes dumped per case.
STEPS = {"cavity8": 4, "pipe10x20": 3, "channel": 3, "channel_ffp": 3, "ibplane": 3, "ibplane_io": 3,
         "cavity_oct": 4, "duct_oct": 3, "ibcyl_oct": 3}
DIV_SCHEMES = [
    "upwind",
    "linear",
    "vanleer",
    "minmod",
    "superbee",
    "monotonized_central",
    "limitedlinear",
    "koren",
]


# Cases whose whole steps and gradients are also pinned with the Green-Gauss
# ('linear') gradient scheme: SIMPLE on a box, PIMPLE with a TVD scheme (the
# configured gradient enters the limiter), an octree with TVD (and its
# hanging-face offset correction) and an immersed octree case.
GRAD_LINEAR_CASES = ("cavity8", "channel", "duct_oct", "ibcyl_oct")


def grad_linear_case(name: str) -> dict:
    case = copy.deepcopy(ALL_CASES[name]())
    schemes = case["simulator"].setdefault("fvSchemes", {})
    schemes["gradSchemes"] = {"default": "linear"}
    case["name"] = name + "_gradlinear"
    return case
