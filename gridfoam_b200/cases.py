"""Synthetic case definitions and the case loader of the product path.

A case is a plain dictionary: a ``simulator`` entry in gridfoam's YAML
schema (``meta/config.py:812-868`` of the reference), a ``mesh`` recipe for
``gridfoam_b200.mesh.builder`` (standing in for the reference's ``fluxel``
section, whose STL bodies are replaced by signed-distance bodies) and an
optional parabolic ``inlet_profile``.  ``create_case`` turns one into a mesh,
a device grid and an algorithm (the reference's ``runner.py`` path from a
config to ``create_algorithm(grid)``); ``load_case`` reads one from a YAML
file.  The workloads of the benchmark are here with their full sizes: the
lid-driven cavity, the immersed Hagen-Poiseuille pipe, the octree cylinder
wake and the bluff body.
"""


from __future__ import annotations

import copy

import numpy as np

from gridfoam_b200.mesh.builder import (
    BLUFF_DEFAULT,
    bluff_body_sdf,
    Body,
    BoxRegion,
    SdfRegion,
    build_octree_mesh,
    build_octree_mesh_device,
    build_uniform_mesh,
    cylinder_sdf,
    plane_sdf,
)

WALL0 = [0.0, 0.0, 0.0]


def _control(dt: float, end: float) -> dict:
    return {
        "deltaT": dt,
        "endTime": end,
        "writeInterval": 1000,
        "output": {"output_dir": "/tmp/gf_golden", "base_name": "golden"},
        "precision": "float64",
    }


def _props(nu: float) -> dict:
    return {
        "transport": {"type": "newtonian", "nu": nu},
        "turbulence": {"type": "laminar"},
    }


def cavity_case(n: int = 8, div: str = "linear") -> dict:
    """Lid-driven cubic cavity, SIMPLE (the CPU-runnable cavity config)."""
    sim = {
        "control": _control(1.0, 300.0),
        "fvSchemes": {
            "divSchemes": {"default": div},
            "gradSchemes": {"default": "leastsquare"},
            "laplacianSchemes": {"default": "corrected"},
        },
        "fvSolution": {
            "adjustPhi": True,
            "algorithm": {
                "type": "simple",
                "nNonOrthogonalCorrectors": 0,
                "relaxationFactors": {"equations": {"U": 0.7, "p": 0.3}},
                "pRefCell": 0,
                "pRefValue": 0.0,
            },
            "solvers": {
                "U": {
                    "method": "bicgstab",
                    "preconditioner": "jacobi",
                    "tolerance": 1e-8,
                    "rel_tolerance": 0.1,
                    "max_iter": 1000,
                },
                "p": {
                    "method": "cg",
                    "preconditioner": "jacobi",
                    "tolerance": 1e-6,
                    "rel_tolerance": 0.0,
                    "max_iter": 2000,
                },
            },
        },
        "conditions": {
            "U": {
                "internal": [0.0, 0.0, 0.0],
                "boundary": {
                    "wall": {
                        "type": "dirichlet",
                        "patches": [
                            "x_minus",
                            "x_plus",
                            "y_minus",
                            "z_minus",
                            "z_plus",
                        ],
                        "value": WALL0,
                    },
                    "lid": {
                        "type": "dirichlet",
                        "patches": ["y_plus"],
                        "value": [1.0, 0.0, 0.0],
                    },
                },
            },
            "p": {
                "internal": 0.0,
                "boundary": {
                    "wall": {
                        "type": "neumann",
                        "patches": [
                            "x_minus",
                            "x_plus",
                            "y_minus",
                            "y_plus",
                            "z_minus",
                            "z_plus",
                        ],
                        "value": 0.0,
                    }
                },
            },
        },
        "properties": _props(0.01),
        "device": "cpu",
    }
    return {
        "name": f"cavity{n}",
        "mesh": {"kind": "uniform", "lower": [0, 0, 0], "upper": [1, 1, 1], "res": [n, n, n]},
        "simulator": sim,
        "inlet_profile": None,
    }


def pipe_case(n: int = 12, nz: int = 24, length: float = 2.0) -> dict:
    """Hagen-Poiseuille pipe through an immersed cylinder, PISO.

    The inlet velocity ``u_z = 2 (1 - r^2 / R^2)`` (mean 1) is a per-face
    Dirichlet value, zero outside the pipe.
    """
    sim = {
        "control": _control(1e-3, 2.0),
        "fvSchemes": {"divSchemes": {"default": "upwind"}},
        "fvSolution": {
            "adjustPhi": True,
            "algorithm": {"type": "piso", "nCorrectors": 2, "nNonOrthogonalCorrectors": 0},
            "solvers": {
                "U": {
                    "method": "bicgstab",
                    "preconditioner": "jacobi",
                    "tolerance": 1e-8,
                    "rel_tolerance": 0.1,
                    "max_iter": 1000,
                },
                "p": {
                    "method": "cg",
                    "preconditioner": "jacobi",
                    "tolerance": 1e-7,
                    "rel_tolerance": 0.01,
                    "max_iter": 2000,
                },
                "pFinal": {
                    "method": "cg",
                    "preconditioner": "jacobi",
                    "tolerance": 1e-7,
                    "rel_tolerance": 0.0,
                    "max_iter": 2000,
                },
            },
        },
        "conditions": {
            "U": {
                "internal": [0.0, 0.0, 0.0],
                "boundary": {
                    "walls": {
                        "type": "dirichlet",
                        "patches": ["x_minus", "x_plus", "y_minus", "y_plus", "pipe"],
                        "value": WALL0,
                    },
                    "inlet": {
                        "type": "dirichlet",
                        "patches": ["z_minus"],
                        "value": WALL0,
                    },
                    "outlet": {
                        "type": "neumann",
                        "patches": ["z_plus"],
                        "value": WALL0,
                    },
                },
            },
            "p": {
                "internal": 0.0,
                "boundary": {
                    "walls": {
                        "type": "neumann",
                        "patches": [
                            "x_minus",
                            "x_plus",
                            "y_minus",
                            "y_plus",
                            "z_minus",
                            "pipe",
                        ],
                        "value": 0.0,
                    },
                    "outlet": {"type": "dirichlet", "patches": ["z_plus"], "value": 0.0},
                },
            },
        },
        "properties": _props(0.02),
        "device": "cpu",
    }
    return {
        "name": f"pipe{n}x{nz}",
        "mesh": {
            "kind": "uniform",
            "lower": [0, 0, 0],
            "upper": [1, 1, length],
            "res": [n, n, nz],
            "bodies": [{"kind": "cylinder", "center": [0.5, 0.5], "radius": 0.4, "axis": 2, "patch": "pipe"}],
        },
        "simulator": sim,
        "inlet_profile": {"patch": "z_minus", "center": [0.5, 0.5], "radius": 0.4, "umax": 2.0},
    }


def channel_case() -> dict:
    """Quasi-2-D channel: empty z patches, inletOutlet, slip, PIMPLE, SIMPLEC,
    backward ddt and a TVD (vanLeer) convection scheme."""
    sim = {
        "control": _control(0.02, 1.0),
        "fvSchemes": {
            "divSchemes": {"default": "vanleer"},
            "ddtSchemes": {"default": "backward"},
        },
        "fvSolution": {
            "adjustPhi": True,
            "algorithm": {
                "type": "pimple",
                "nOuterCorrectors": 2,
                "nCorrectors": 2,
                "consistent": True,
                "pRefCell": 0,
                "pRefValue": 0.0,
            },
            "solvers": {
                "U": {"method": "bicgstab", "preconditioner": "jacobi", "tolerance": 1e-9, "rel_tolerance": 0.0},
                "p": {"method": "cg", "preconditioner": "jacobi", "tolerance": 1e-8, "rel_tolerance": 0.0},
                "pFinal": {"method": "cg", "preconditioner": "jacobi", "tolerance": 1e-9, "rel_tolerance": 0.0},
            },
        },
        "conditions": {
            "U": {
                "internal": [0.5, 0.0, 0.0],
                "boundary": {
                    "inlet": {"type": "dirichlet", "patches": ["x_minus"], "value": [1.0, 0.0, 0.0]},
                    "outlet": {"type": "inlet_outlet", "patches": ["x_plus"], "value": WALL0},
                    "bottom": {"type": "dirichlet", "patches": ["y_minus"], "value": WALL0},
                    "top": {"type": "slip", "patches": ["y_plus"]},
                    "empty": {"type": "empty", "patches": ["z_minus", "z_plus"]},
                },
            },
            "p": {
                "internal": 0.0,
                "boundary": {
                    "inlet": {"type": "neumann", "patches": ["x_minus"], "value": 0.0},
                    "outlet": {"type": "dirichlet", "patches": ["x_plus"], "value": 0.0},
                    "walls": {"type": "neumann", "patches": ["y_minus", "y_plus"], "value": 0.0},
                    "empty": {"type": "empty", "patches": ["z_minus", "z_plus"]},
                },
            },
        },
        "properties": _props(0.02),
        "device": "cpu",
    }
    return {
        "name": "channel",
        "mesh": {"kind": "uniform", "lower": [0, 0, 0], "upper": [2.0, 1.0, 0.1], "res": [16, 8, 1]},
        "simulator": sim,
        "inlet_profile": None,
    }


def ffp_case() -> dict:
    """Channel with fixedFluxPressure at the inlet, PISO, linear convection."""
    case = copy.deepcopy(channel_case())
    sim = case["simulator"]
    sim["fvSchemes"] = {"divSchemes": {"default": "linear"}}
    sim["fvSolution"]["algorithm"] = {"type": "piso", "nCorrectors": 2}
    sim["conditions"]["p"]["boundary"]["inlet"] = {
        "type": "fixed_flux_pressure",
        "patches": ["x_minus"],
    }
    case["name"] = "channel_ffp"
    return case


def ibplane_case() -> dict:
    """Box cut by an immersed plane through a row of cell centres.

    A surface through a cell centre gives zero ray distance, so the Gibou
    near-boundary constraint (``with_fixed_values``) and the fixed-cell flux
    closure of ``correct_phi`` are exercised.  PISO, minmod convection.
    """
    n = 12
    x_plane = (6 + 0.5) / n
    sim = {
        "control": _control(5e-3, 1.0),
        "fvSchemes": {"divSchemes": {"default": "minmod"}},
        "fvSolution": {
            "adjustPhi": True,
            "algorithm": {"type": "piso", "nCorrectors": 2, "pRefCell": 0, "pRefValue": 0.0},
            "solvers": {
                "U": {"method": "bicgstab", "preconditioner": "jacobi", "tolerance": 1e-9, "rel_tolerance": 0.0},
                "p": {"method": "cg", "preconditioner": "jacobi", "tolerance": 1e-8, "rel_tolerance": 0.0},
            },
        },
        "conditions": {
            "U": {
                "internal": WALL0,
                "boundary": {
                    "wall": {
                        "type": "dirichlet",
                        "patches": ["x_minus", "x_plus", "y_minus", "z_minus", "z_plus", "plate"],
                        "value": WALL0,
                    },
                    "lid": {"type": "dirichlet", "patches": ["y_plus"], "value": [1.0, 0.0, 0.5]},
                },
            },
            "p": {
                "internal": 0.0,
                "boundary": {
                    "wall": {
                        "type": "neumann",
                        "patches": ["x_minus", "x_plus", "y_minus", "y_plus", "z_minus", "z_plus"],
                        "value": 0.0,
                    },
                    "plate": {"type": "dirichlet", "patches": ["plate"], "value": 0.0},
                },
            },
        },
        "properties": _props(0.05),
        "device": "cpu",
    }
    return {
        "name": "ibplane",
        "mesh": {
            "kind": "uniform",
            "lower": [0, 0, 0],
            "upper": [1, 0.5, 0.5],
            "res": [n, 6, 6],
            "bodies": [{"kind": "plane", "point": x_plane, "axis": 0, "patch": "plate"}],
        },
        "simulator": sim,
        "inlet_profile": None,
    }


def _sdf(b: dict):
    if b["kind"] == "cylinder":
        return cylinder_sdf(tuple(b["center"]), b["radius"], b["axis"])
    if b["kind"] == "plane":
        return plane_sdf(b["point"], b["axis"])
    if b["kind"] == "bluff":
        return bluff_body_sdf(b.get("x0", 0.0), tuple(b.get("params", BLUFF_DEFAULT)))
    raise ValueError(b["kind"])


def build_mesh(spec: dict, device: str | None = None):
    """Build the mesh described by a case's ``mesh`` entry (octrees on
    ``device`` when it is a CUDA device: the same mesh, built on the GPU)."""
    bodies = [Body(sdf=_sdf(b), patch=b["patch"]) for b in spec.get("bodies", [])]
    if spec["kind"] == "octree":
        regions = []
        for r in spec.get("regions", []):
            if r["kind"] == "box":
                regions.append(BoxRegion(tuple(r["lo"]), tuple(r["hi"]), r["level"]))
            else:
                regions.append(SdfRegion(_sdf(r["body"]), r["distance"], r["level"]))
        args = (tuple(spec["lower"]), tuple(spec["upper"]), tuple(spec["res"]), regions)
        if device is not None and str(device).startswith("cuda"):
            return build_octree_mesh_device(*args, bodies=bodies, device=device)
        return build_octree_mesh(*args, bodies=bodies)
    return build_uniform_mesh(
        tuple(spec["lower"]), tuple(spec["upper"]), tuple(spec["res"]), bodies=bodies
    )


def inlet_profile_values(mesh, profile: dict) -> np.ndarray:
    """Per-face parabolic inlet velocity ``[F_patch, 3]`` on ``profile['patch']``."""
    direction = {"x_minus": 0, "x_plus": 1, "y_minus": 2, "y_plus": 3, "z_minus": 4, "z_plus": 5}[
        profile["patch"]
    ]
    sel = mesh.domain_bnd_faces_dir == direction
    cells = mesh.domain_bnd_faces_owner[sel]
    c = mesh.cell_centers[cells]
    r2 = (c[:, 0] - profile["center"][0]) ** 2 + (c[:, 1] - profile["center"][1]) ** 2
    uz = profile["umax"] * np.clip(1.0 - r2 / profile["radius"] ** 2, 0.0, None)
    out = np.zeros((cells.shape[0], 3))
    out[:, 2] = uz
    return out


def cavity_oct_case() -> dict:
    """Cavity on a two-level octree: refined under the lid and again near
    its centre, so hanging faces meet the lid, the walls and each other.
    SIMPLE, linear convection, corrected Laplacian."""
    case = cavity_case(6)
    case["name"] = "cavity_oct"
    case["mesh"] = {
        "kind": "octree", "lower": [0, 0, 0], "upper": [1, 1, 1], "res": [6, 6, 6],
        "regions": [
            {"kind": "box", "lo": [0.2, 0.55, 0.2], "hi": [0.8, 1.0, 0.8], "level": 1},
            {"kind": "box", "lo": [0.4, 0.8, 0.4], "hi": [0.6, 1.0, 0.6], "level": 2},
        ],
    }
    return case


def duct_oct_case() -> dict:
    """Duct flow on an octree refined in the middle: PISO, vanLeer TVD
    convection (the hanging-face offset correction of the linear value),
    inletOutlet outlet."""
    sim = {
        "control": _control(0.01, 1.0),
        "fvSchemes": {"divSchemes": {"default": "vanleer"}},
        "fvSolution": {
            "adjustPhi": True,
            "algorithm": {"type": "piso", "nCorrectors": 2, "pRefCell": 0, "pRefValue": 0.0},
            "solvers": {
                "U": {"method": "bicgstab", "preconditioner": "jacobi", "tolerance": 1e-10, "rel_tolerance": 0.0},
                "p": {"method": "cg", "preconditioner": "jacobi", "tolerance": 1e-9, "rel_tolerance": 0.0},
            },
        },
        "conditions": {
            "U": {
                "internal": [0.2, 0.0, 0.0],
                "boundary": {
                    "inlet": {"type": "dirichlet", "patches": ["x_minus"], "value": [1.0, 0.0, 0.0]},
                    "outlet": {"type": "inlet_outlet", "patches": ["x_plus"], "value": WALL0},
                    "walls": {"type": "dirichlet", "patches": ["y_minus", "y_plus", "z_minus", "z_plus"],
                              "value": WALL0},
                },
            },
            "p": {
                "internal": 0.0,
                "boundary": {
                    "inlet": {"type": "neumann", "patches": ["x_minus"], "value": 0.0},
                    "outlet": {"type": "dirichlet", "patches": ["x_plus"], "value": 0.0},
                    "walls": {"type": "neumann", "patches": ["y_minus", "y_plus", "z_minus", "z_plus"],
                              "value": 0.0},
                },
            },
        },
        "properties": _props(0.02),
        "device": "cpu",
    }
    return {
        "name": "duct_oct",
        "mesh": {
            "kind": "octree", "lower": [0, 0, 0], "upper": [2.0, 1.0, 1.0], "res": [8, 4, 4],
            "regions": [{"kind": "box", "lo": [0.6, 0.2, 0.2], "hi": [1.4, 0.8, 0.8], "level": 1}],
        },
        "simulator": sim,
        "inlet_profile": None,
    }


def ibcyl_oct_case() -> dict:
    """Immersed cylinder inside a refined band (octree), PISO, upwind: IB
    faces on the fine level, hanging faces around the band."""
    cyl = {"kind": "cylinder", "center": [0.5, 0.5], "radius": 0.2, "axis": 2, "patch": "cylinder"}
    sim = {
        "control": _control(5e-3, 1.0),
        "fvSchemes": {"divSchemes": {"default": "upwind"}},
        "fvSolution": {
            "adjustPhi": True,
            "algorithm": {"type": "piso", "nCorrectors": 2, "pRefCell": 0, "pRefValue": 0.0},
            "solvers": {
                "U": {"method": "bicgstab", "preconditioner": "jacobi", "tolerance": 1e-10, "rel_tolerance": 0.0},
                "p": {"method": "cg", "preconditioner": "jacobi", "tolerance": 1e-9, "rel_tolerance": 0.0},
            },
        },
        "conditions": {
            "U": {
                "internal": [0.5, 0.0, 0.0],
                "boundary": {
                    "inlet": {"type": "dirichlet", "patches": ["x_minus"], "value": [1.0, 0.0, 0.0]},
                    "outlet": {"type": "neumann", "patches": ["x_plus"], "value": WALL0},
                    "side": {"type": "slip", "patches": ["y_minus", "y_plus"]},
                    "ends": {"type": "neumann", "patches": ["z_minus", "z_plus"], "value": WALL0},
                    "cyl": {"type": "dirichlet", "patches": ["cylinder"], "value": WALL0},
                },
            },
            "p": {
                "internal": 0.0,
                "boundary": {
                    "outlet": {"type": "dirichlet", "patches": ["x_plus"], "value": 0.0},
                    # Dirichlet on the body also pins the (disconnected) interior.
                    "cyl": {"type": "dirichlet", "patches": ["cylinder"], "value": 0.0},
                    "rest": {"type": "neumann",
                             "patches": ["x_minus", "y_minus", "y_plus", "z_minus", "z_plus"],
                             "value": 0.0},
                },
            },
        },
        "properties": _props(0.05),
        "device": "cpu",
    }
    return {
        "name": "ibcyl_oct",
        "mesh": {
            "kind": "octree", "lower": [0, 0, 0], "upper": [1.0, 1.0, 0.5], "res": [8, 8, 4],
            "regions": [{"kind": "sdf", "body": cyl, "distance": 0.12, "level": 1}],
            "bodies": [cyl],
        },
        "simulator": sim,
        "inlet_profile": None,
    }


def cylinder_wake_case(base: tuple[int, int, int] = (96, 64, 12), levels: int = 2) -> dict:
    """Cylinder wake on a 3-level octree (the cylinder-wake config, scaled
    by its base resolution): domain 30D x 20D x 4D, cylinder D = 1 at
    (10, 10) spanning z, refined ``levels`` levels within 2D of its surface;
    inflow 1, nu 0.01 (Re 100), PISO at CFL 0.5 on the finest cell."""
    cyl = {"kind": "cylinder", "center": [10.0, 10.0], "radius": 0.5, "axis": 2, "patch": "cylinder"}
    dx_fine = 30.0 / base[0] / 2**levels
    sim = {
        "control": _control(0.5 * dx_fine / 1.0, 1.0e3),
        "fvSchemes": {"divSchemes": {"default": "upwind"}},
        "fvSolution": {
            "adjustPhi": True,
            "algorithm": {"type": "piso", "nCorrectors": 2, "pRefCell": 0, "pRefValue": 0.0},
            "solvers": {
                "U": {"method": "bicgstab", "preconditioner": "jacobi", "tolerance": 1e-8, "rel_tolerance": 0.1},
                "p": {"method": "cg", "preconditioner": "jacobi", "tolerance": 1e-7, "rel_tolerance": 0.01},
                "pFinal": {"method": "cg", "preconditioner": "jacobi", "tolerance": 1e-7, "rel_tolerance": 0.0},
            },
        },
        "conditions": {
            "U": {
                "internal": [1.0, 0.0, 0.0],
                "boundary": {
                    "inlet": {"type": "dirichlet", "patches": ["x_minus"], "value": [1.0, 0.0, 0.0]},
                    "outlet": {"type": "inlet_outlet", "patches": ["x_plus"], "value": WALL0},
                    "sides": {"type": "slip", "patches": ["y_minus", "y_plus", "z_minus", "z_plus"]},
                    "cyl": {"type": "dirichlet", "patches": ["cylinder"], "value": WALL0},
                },
            },
            "p": {
                "internal": 0.0,
                "boundary": {
                    "outlet": {"type": "dirichlet", "patches": ["x_plus"], "value": 0.0},
                    "cyl": {"type": "dirichlet", "patches": ["cylinder"], "value": 0.0},
                    "rest": {"type": "neumann", "patches": ["x_minus", "y_minus", "y_plus", "z_minus", "z_plus"],
                             "value": 0.0},
                },
            },
        },
        "properties": _props(0.01),
        "device": "cpu",
    }
    return {
        "name": f"cylinder_wake_{base[0]}x{base[1]}x{base[2]}",
        "mesh": {
            "kind": "octree", "lower": [0, 0, 0], "upper": [30.0, 20.0, 4.0], "res": list(base),
            "regions": [{"kind": "sdf", "body": cyl, "distance": 2.0, "level": levels}],
            "bodies": [cyl],
        },
        "simulator": sim,
        "inlet_profile": None,
    }




TRANSIENT = {"piso", "pimple"}


def create_case(case_def: dict, device: str = "cuda"):
    """Build ``(mesh, grid, algorithm)`` for a case on ``device``.

    The reference's ``runner.py`` path: mesh generation (here the
    fluxel-compatible builder; octrees are built on the GPU when ``device``
    is a CUDA device), ``AxisProjectedGrid(simulator, mesh)``, the velocity
    field with its per-face inlet profile, then ``create_algorithm(grid)``.
    """
    from gridfoam_b200.algorithms.pressure_velocity import create_algorithm
    from gridfoam_b200.core.boundary import DirichletBC
    from gridfoam_b200.core.field import CellField
    from gridfoam_b200.core.grid import AxisProjectedGrid
    from gridfoam_b200.meta.config import FieldRole, SimulatorConfig

    case_def = copy.deepcopy(case_def)
    mesh = build_mesh(case_def["mesh"], device=device)
    sim = SimulatorConfig.model_validate(case_def["simulator"])
    grid = AxisProjectedGrid(sim, mesh, device=device)
    kind = case_def["simulator"]["fvSolution"]["algorithm"]["type"]
    role = FieldRole.TRANSIENT if kind in TRANSIENT else FieldRole.LOCAL
    U = CellField(grid, "U", role, (3,))
    profile = case_def.get("inlet_profile")
    if profile is not None:
        U.add_boundary_conditions({profile["patch"]: DirichletBC(inlet_profile_values(mesh, profile))})
    algo = create_algorithm(grid)
    return mesh, grid, algo


def load_case(path) -> dict:
    """Read a case from a YAML file: ``simulator`` (gridfoam's schema, checked
    by ``SimulatorConfig``), ``mesh`` (a builder recipe as above) and an
    optional ``inlet_profile``.  Raises ``ValueError`` on a missing section."""
    import pathlib

    import yaml

    from gridfoam_b200.meta.config import SimulatorConfig

    data = yaml.safe_load(pathlib.Path(path).read_text())
    for key in ("simulator", "mesh"):
        if key not in data:
            raise ValueError(f"case file {path} has no '{key}' section")
    SimulatorConfig.model_validate(data["simulator"])
    data.setdefault("inlet_profile", None)
    data.setdefault("name", pathlib.Path(path).stem)
    return data


def pipe_analytic_uz(mesh, profile: dict) -> np.ndarray:
    """Hagen-Poiseuille axial velocity ``umax (1 - r^2 / R^2)`` at every cell
    centre (0 outside the pipe), the fully developed solution of the pipe."""
    c = mesh.cell_centers
    r2 = (c[:, 0] - profile["center"][0]) ** 2 + (c[:, 1] - profile["center"][1]) ** 2
    return profile["umax"] * np.clip(1.0 - r2 / profile["radius"] ** 2, 0.0, None)


def bluff_body_case(base: tuple[int, int, int] = (128, 32, 24), levels: int = 3, params=BLUFF_DEFAULT,
                    iterations: int = 500, nu: float = 0.0024, uniform: bool = False,
                    lower=(-2.0, -1.0, 0.0), upper=(6.0, 1.0, 1.2)) -> dict:
    """Slanted bluff body in a channel on a 4-level octree (levels 0-3):
    domain [-2, 6] x [-1, 1] x [0, 1.2], the body (length 1, front at x = 0,
    shape ``params``) on the floor side with its clearance; refined to level
    1 in the box around body and near wake, 2 closer, 3 within 0.04 of the
    surface.  Inflow 1, laminar, steady SIMPLE (SIMPLEC), upwind
    convection; floor and body no-slip, top and sides slip.

    ``nu`` defaults to 0.0024, Re = 418 on the body length: the Reynolds
    number of the reference's own Ahmed-body example (inflow 40, nu 0.1,
    length 1.044).  At nu = 2e-6 steady SIMPLE has no usable fixed point on
    these grids: the cells enclosed by the body carry almost no flux, so
    their momentum diagonal (outflow plus nu terms, no time derivative)
    nearly vanishes and 1/A blows up in the first iterations, in the
    reference's own run of this case as here.

    ``uniform``: one level of ``base`` cells over [``lower``, ``upper``]
    (no refinement, no hanging faces)."""
    body = {"kind": "bluff", "x0": 0.0, "params": list(params), "patch": "body"}
    sim = {
        "control": {"deltaT": 1.0, "endTime": float(iterations), "writeInterval": 100000,
                    "output": {"output_dir": "/tmp/gf_bluff", "base_name": "bluff"}, "precision": "float64"},
        "fvSchemes": {"divSchemes": {"default": "upwind"}, "gradSchemes": {"default": "leastsquare"},
                      "laplacianSchemes": {"default": "corrected"}},
        "fvSolution": {
            "adjustPhi": True,
            "algorithm": {"type": "simple", "nNonOrthogonalCorrectors": 0, "consistent": True,
                          "relaxationFactors": {"equations": {"U": 0.7, "p": 0.3}},
                          "pRefCell": 0, "pRefValue": 0.0},
            "solvers": {
                "U": {"method": "bicgstab", "preconditioner": "jacobi", "tolerance": 1e-8,
                      "rel_tolerance": 0.1, "max_iter": 2000},
                "p": {"method": "cg", "preconditioner": "jacobi", "tolerance": 1e-7,
                      "rel_tolerance": 0.01, "max_iter": 2000},
            },
        },
        "conditions": {
            "U": {
                "internal": [1.0, 0.0, 0.0],
                "boundary": {
                    "inlet": {"type": "dirichlet", "patches": ["x_minus"], "value": [1.0, 0.0, 0.0]},
                    "outlet": {"type": "inlet_outlet", "patches": ["x_plus"], "value": WALL0},
                    "sides": {"type": "slip", "patches": ["y_minus", "y_plus", "z_plus"]},
                    "floor": {"type": "dirichlet", "patches": ["z_minus"], "value": WALL0},
                    "body": {"type": "dirichlet", "patches": ["body"], "value": WALL0},
                },
            },
            "p": {
                "internal": 0.0,
                "boundary": {
                    "outlet": {"type": "dirichlet", "patches": ["x_plus"], "value": 0.0},
                    "rest": {"type": "neumann",
                             "patches": ["x_minus", "y_minus", "y_plus", "z_minus", "z_plus", "body"],
                             "value": 0.0},
                },
            },
        },
        "properties": _props(nu),
        "device": "cpu",
    }
    if uniform:
        return {
            "name": f"bluff_body_{base[0]}x{base[1]}x{base[2]}_uniform",
            "mesh": {"kind": "uniform", "lower": list(lower), "upper": list(upper), "res": list(base),
                     "bodies": [body]},
            "simulator": sim,
            "inlet_profile": None,
        }
    return {
        "name": f"bluff_body_{base[0]}x{base[1]}x{base[2]}_l{levels}",
        "mesh": {
            "kind": "octree", "lower": list(lower), "upper": list(upper), "res": list(base),
            "regions": [
                {"kind": "box", "lo": [-0.5, -0.45, 0.0], "hi": [3.0, 0.45, 0.6], "level": 1},
                {"kind": "box", "lo": [-0.2, -0.3, 0.0], "hi": [1.6, 0.3, 0.45], "level": 2},
                {"kind": "sdf", "body": body, "distance": 0.04, "level": levels},
            ],
            "bodies": [body],
        },
        "simulator": sim,
        "inlet_profile": None,
    }
