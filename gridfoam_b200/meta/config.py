"""YAML configuration schema, compatible with gridfoam's ``GridfoamConfig``.

The field names, defaults and validation follow the reference schema
(``meta/config.py:34-882`` and ``meta/enums.py``) so that a gridfoam YAML
case file loads unchanged.  Sections outside the hot path (post-processing,
potential flow) are accepted and carried as plain data.
"""

from __future__ import annotations

import pathlib
import re
from enum import StrEnum
from typing import Annotated, Any, Literal, Self

from pydantic import BaseModel, Field, field_validator, model_validator

type TensorValue = float | list[TensorValue]


class IbmType(StrEnum):
    NONE = "none"
    AXIS_PROJECTED = "axis_projected"
    GHOST_CELL = "ghost_cell"


class MeshMotion(StrEnum):
    STATIC = "static"
    DYNAMIC = "dynamic"


class DeviceType(StrEnum):
    CPU = "cpu"
    CUDA = "cuda"


class DomainBoundaryPatch(StrEnum):
    X_MINUS = "x_minus"
    X_PLUS = "x_plus"
    Y_MINUS = "y_minus"
    Y_PLUS = "y_plus"
    Z_MINUS = "z_minus"
    Z_PLUS = "z_plus"

    def direction(self) -> int:
        """fluxel ``Direction`` id: XMinus=0 ... ZPlus=5."""
        return list(DomainBoundaryPatch).index(self)


class FieldRole(StrEnum):
    TRANSIENT = "transient"
    LOCAL = "local"
    MONITOR = "monitor"


class DdtScheme(StrEnum):
    EULER = "euler"
    BACKWARD = "backward"


class GradScheme(StrEnum):
    LINEAR = "linear"
    LEASTSQUARE = "leastsquare"


class DivScheme(StrEnum):
    UPWIND = "upwind"
    LINEAR = "linear"
    VANLEER = "vanleer"
    MINMOD = "minmod"
    SUPERBEE = "superbee"
    MONOTONIZED_CENTRAL = "monotonized_central"
    LIMITEDLINEAR = "limitedlinear"
    KOREN = "koren"


class SnGradScheme(StrEnum):
    UNCORRECTED = "uncorrected"
    CORRECTED = "corrected"


class LaplacianScheme(StrEnum):
    LINEAR = "linear"
    CORRECTED = "corrected"
    UNCORRECTED = "uncorrected"
    GAUSS_LINEAR_CORRECTED = "Gauss linear corrected"
    GAUSS_LINEAR_UNCORRECTED = "Gauss linear uncorrected"
    GAUSS_HARMONIC_CORRECTED = "Gauss harmonic corrected"
    GAUSS_HARMONIC_UNCORRECTED = "Gauss harmonic uncorrected"


class SolverType(StrEnum):
    CG = "cg"
    BiCGSTAB = "bicgstab"
    PyAMG = "pyamg"


class NormType(StrEnum):
    L_inf = "l_inf"
    L_2 = "l_2"


class PreconditionerType(StrEnum):
    NONE = "none"
    JACOBI = "jacobi"


class PrecisionType(StrEnum):
    FLOAT32 = "float32"
    FLOAT64 = "float64"


class FaceSide(StrEnum):
    UPPER = "upper"
    LOWER = "lower"


class BoundaryConditionType(StrEnum):
    DIRICHLET = "dirichlet"
    NEUMANN = "neumann"
    EMPTY = "empty"
    SLIP = "slip"
    INLET_OUTLET = "inlet_outlet"
    FIXED_FLUX_PRESSURE = "fixed_flux_pressure"


class AlgorithmType(StrEnum):
    SIMPLE = "simple"
    PISO = "piso"
    PIMPLE = "pimple"
    MANUAL = "manual"


class TransportModelType(StrEnum):
    NEWTONIAN = "newtonian"


class TurbulenceType(StrEnum):
    LAMINAR = "laminar"


class DomainConfig(BaseModel, frozen=True):
    lower: list[float]
    upper: list[float]


class RefinementRegionConfig(BaseModel, frozen=True):
    name: str | None = None
    min: list[float]
    max: list[float]
    level: int = Field(ge=0)


class FluxelConfig(BaseModel, frozen=True):
    domain: DomainConfig
    root_resolution: list[int]
    target_level: int = 0
    n_leaf_refinement: int = 0
    refinement_regions: list[RefinementRegionConfig] = Field(default_factory=list)
    mesh_path: pathlib.Path | None = None
    ibm_type: IbmType = IbmType.AXIS_PROJECTED
    motion: MeshMotion = MeshMotion.STATIC


class OutputConfig(BaseModel, frozen=True):
    output_dir: pathlib.Path
    base_name: str
    overwrite_file: bool = True


class ControlConfig(BaseModel, frozen=True):
    deltaT: float
    endTime: float
    writeInterval: int
    output: OutputConfig
    precision: PrecisionType


def _regularize(d: dict | None) -> dict | None:
    if d is None:
        return None
    return {re.sub(r"\s*,\s*", ", ", k): v for k, v in d.items()}


class fvSchemesConfig(BaseModel, frozen=True):
    ddtSchemes: dict[str, DdtScheme] | None = None
    gradSchemes: dict[str, GradScheme] | None = None
    divSchemes: dict[str, DivScheme] | None = None
    laplacianSchemes: dict[str, LaplacianScheme] | None = None
    snGradSchemes: dict[str, SnGradScheme] | None = None

    @field_validator(
        "ddtSchemes", "divSchemes", "laplacianSchemes", "gradSchemes", "snGradSchemes", mode="before"
    )
    @classmethod
    def regularize_keys(cls, d):
        return _regularize(d)


class SolverConfig(BaseModel, frozen=True):
    method: SolverType
    preconditioner: PreconditionerType = PreconditionerType.NONE
    tolerance: float = 1e-6
    rel_tolerance: float = 1e-6
    max_iter: int = 1000
    norm_type: NormType = NormType.L_2
    max_restart: int = 5
    log_interval: int = 25
    # Extension (not in the reference schema; defaults keep its behaviour):
    # ``inner_precision: float32`` runs CG's inner iterations in FP32 inside
    # FP64 iterative refinement; the stopping test stays the FP64 true
    # residual.  ``max_outer`` bounds the refinement cycles,
    # ``inner_eta`` is the relative reduction of one FP32 cycle, and a cycle
    # also ends once its FP32 residual is below ``inner_margin`` times the
    # stopping threshold (margin for the FP32 rounding of that residual).
    inner_precision: PrecisionType = PrecisionType.FLOAT64
    max_outer: int = Field(default=10, ge=1)
    inner_eta: float = Field(default=1e-4, gt=0.0, lt=1.0)
    inner_margin: float = Field(default=0.9, gt=0.0, le=1.0)


class PotentialFlowConfig(BaseModel, frozen=True):
    nNonOrthogonalCorrectors: int = Field(default=0, ge=0)
    phiRefCell: int | None = Field(default=None, ge=0)
    phiRefValue: float | None = None


class RelaxationFactorsConfig(BaseModel, frozen=True):
    equations: dict[str, float] = Field(default_factory=dict)


class ResidualControlEntry(BaseModel, frozen=True):
    tolerance: float
    rel_tolerance: float = 0.0


ResidualControlValue = ResidualControlEntry | float


def normalize_residual_control(value: dict) -> dict[str, ResidualControlEntry]:
    out: dict[str, ResidualControlEntry] = {}
    for name, entry in value.items():
        out[name] = (
            ResidualControlEntry(tolerance=float(entry)) if isinstance(entry, (int, float)) else entry
        )
    return out


class SIMPLEAlgorithm(BaseModel, frozen=True):
    type: Literal[AlgorithmType.SIMPLE]
    nNonOrthogonalCorrectors: int = Field(default=0, ge=0)
    residualControl: dict[str, ResidualControlValue] = Field(default_factory=dict)
    consistent: bool = False
    relaxationFactors: RelaxationFactorsConfig = Field(default_factory=RelaxationFactorsConfig)
    pRefCell: int | None = Field(default=None, ge=0)
    pRefValue: float | None = None


class PISOAlgorithm(BaseModel, frozen=True):
    type: Literal[AlgorithmType.PISO]
    nNonOrthogonalCorrectors: int = Field(default=0, ge=0)
    nCorrectors: int = Field(default=2, ge=1)
    pRefCell: int | None = Field(default=None, ge=0)
    pRefValue: float | None = None


class PIMPLEAlgorithm(BaseModel, frozen=True):
    type: Literal[AlgorithmType.PIMPLE]
    nNonOrthogonalCorrectors: int = Field(default=0, ge=0)
    nCorrectors: int = Field(default=2, ge=1)
    nOuterCorrectors: int = Field(default=1, ge=1)
    residualControl: dict[str, ResidualControlValue] = Field(default_factory=dict)
    consistent: bool = False
    pRefCell: int | None = Field(default=None, ge=0)
    pRefValue: float | None = None


class ManualAlgorithm(BaseModel, frozen=True):
    type: Literal[AlgorithmType.MANUAL]


Algorithm = Annotated[
    SIMPLEAlgorithm | PISOAlgorithm | PIMPLEAlgorithm | ManualAlgorithm,
    Field(discriminator="type"),
]


class fvSolutionConfig(BaseModel, frozen=True):
    algorithm: Algorithm
    solvers: dict[str, SolverConfig]
    potentialFlow: PotentialFlowConfig | None = None
    adjustPhi: bool = True


class BoundaryConditionConfig(BaseModel, frozen=True):
    type: BoundaryConditionType
    patches: list[str]
    value: TensorValue | None = None
    phase: str | None = None

    @field_validator("patches", mode="before")
    @classmethod
    def regularize_patches(cls, patches):
        out = []
        for p in patches:
            if not isinstance(p, str):
                raise TypeError("patch names must be strings")
            try:
                out.append(DomainBoundaryPatch(p))
            except ValueError:
                out.append(p)
        return out


class NewtonianTransportConfig(BaseModel, frozen=True):
    type: Literal[TransportModelType.NEWTONIAN]
    nu: float


class LaminarConfig(BaseModel, frozen=True):
    type: Literal[TurbulenceType.LAMINAR]


class PropertiesConfig(BaseModel, frozen=True):
    transport: Annotated[NewtonianTransportConfig, Field(discriminator="type")]
    turbulence: Annotated[LaminarConfig, Field(discriminator="type")]


class ConditionConfig(BaseModel, frozen=True):
    dimension: dict[str, float | int] | None = None
    internal: TensorValue
    boundary: dict[str, BoundaryConditionConfig]
    export: bool = True

    def iter_bc_configs(self):
        yield from self.boundary.values()


class ContinuityErrorConfig(BaseModel, frozen=True):
    """meta/config.py:768-778: the flux field and the record interval."""

    phi: str = "phi"
    writeInterval: int = Field(default=1, ge=1)


class SolverInfoConfig(BaseModel, frozen=True):
    """meta/config.py:781-791: fields (default U and p) and the interval."""

    fields: list[str] | None = None
    writeInterval: int = Field(default=1, ge=1)


class PostProcessingConfig(BaseModel, frozen=True):
    """meta/config.py:794-811.  ``forceCoeff`` stays the raw mapping that
    ``post.forces.ForceEvaluator`` reads."""

    forceCoeff: dict[str, Any] | None = None
    continuityError: ContinuityErrorConfig | None = None
    solverInfo: SolverInfoConfig | None = None


class SimulatorConfig(BaseModel, frozen=True):
    control: ControlConfig
    fvSchemes: fvSchemesConfig
    fvSolution: fvSolutionConfig
    conditions: dict[str, ConditionConfig]
    properties: PropertiesConfig
    post_processing: dict[str, Any] | None = None
    device: DeviceType

    @model_validator(mode="after")
    def check_algorithm_time_compatibility(self) -> Self:
        if self.fvSolution.algorithm.type == AlgorithmType.SIMPLE:
            if self.control.deltaT != 1.0 or not float(self.control.endTime).is_integer():
                raise ValueError("SIMPLE requires deltaT=1.0 and endTime to be an integer")
        return self

    def get_field_condition(self, name: str) -> ConditionConfig | None:
        return self.conditions.get(name)


class GridfoamConfig(BaseModel, frozen=True):
    simulator: SimulatorConfig
    fluxel: FluxelConfig
