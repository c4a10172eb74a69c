"""SIMPLE, PISO and PIMPLE on the device.

Each class keeps gridfoam's algorithm API (``algorithms/simple.py``,
``piso.py``, ``pimple.py``): fields ``U``, ``p``, ``phi``, ``phi_hbya``,
``rAU``, ``rAtU``, ``HbyA``; ``solvers``; ``step()``; ``has_converged()``;
``set_grad_mode()``.  A step is a fixed sequence of library kernels on
preallocated buffers — boundary states, least-squares gradients, one fused
assembly pass per matrix, persistent Krylov solves, flux and velocity
corrections — with no host synchronisation (solver statistics and residuals
are copied back asynchronously and read lazily).
"""

from __future__ import annotations

import ctypes
import logging

import torch

from gridfoam_b200 import _lib
from gridfoam_b200._lib import GfAssembly, GfBcAux, GfDdtCorr, call, ptr, stream_ptr
from gridfoam_b200.core.boundary import DirichletBC
from gridfoam_b200.core.field import (
    CellField,
    FaceField,
    get_or_create_cellfield,
    get_or_create_facefield,
)
from gridfoam_b200.core.fvmatrix import FvMatrix
from gridfoam_b200.fv import schemes
from gridfoam_b200.fv.adjust_phi import adjust_classes
from gridfoam_b200.meta.config import (
    AlgorithmType,
    FieldRole,
    GradScheme,
    PIMPLEAlgorithm,
    PISOAlgorithm,
    SIMPLEAlgorithm,
    normalize_residual_control,
)
from gridfoam_b200.solvers.factory import create_solver, resolve_solver

logger = logging.getLogger(__name__)

byref = ctypes.byref


def _name(base: str, phase: str | None) -> str:
    return base if phase is None else f"{base}.{phase}"


class _LazyScalar:
    """A device scalar copied to pinned host memory, read on first use."""

    def __init__(self, dev: torch.Tensor):
        self.host = torch.empty(1, dtype=torch.float64, pin_memory=True)
        self.host.copy_(dev.reshape(1), non_blocking=True)
        self.event = torch.cuda.Event()
        self.event.record()

    def value(self) -> float:
        self.event.synchronize()
        return float(self.host[0])


class _PressureVelocity:
    """Shared device state and stages of the three algorithms."""

    transient = False

    def __init__(self, grid, phase: str | None = None):
        self._grid = grid
        g = grid
        role = FieldRole.TRANSIENT if self.transient else FieldRole.LOCAL
        self.U = get_or_create_cellfield(g, _name("U", phase), role, (3,))
        self.p = get_or_create_cellfield(g, _name("p", phase), FieldRole.LOCAL, ())
        self.phi = get_or_create_facefield(g, _name("phi", phase), FieldRole.LOCAL, ())
        self.phi_hbya = get_or_create_facefield(g, _name("phiHbyA", phase), FieldRole.LOCAL, (), export=False)
        self.rAU = get_or_create_cellfield(g, _name("rAU", phase), FieldRole.LOCAL, ())
        self.rAtU = get_or_create_cellfield(g, _name("rAtU", phase), FieldRole.LOCAL, ())
        self.HbyA = get_or_create_cellfield(g, _name("HbyA", phase), FieldRole.LOCAL, (3,))
        self.nu_t = get_or_create_cellfield(g, "nu_t", FieldRole.LOCAL, ())
        sim = g.sim_config
        self._solvers = {name: create_solver(cfg) for name, cfg in sim.fvSolution.solvers.items()}
        # False: a step makes no pinned host copies (solver statistics,
        # residual scalars), so it can be captured into a CUDA graph; the
        # residuals stay in ``res_buf`` on the device.
        self.host_readback = True
        self.nu = float(sim.properties.transport.nu)
        alg = sim.fvSolution.algorithm
        self._alg = alg
        self.n_non_orthogonal_correctors = int(getattr(alg, "nNonOrthogonalCorrectors", 0))
        self.adjust_phi_enabled = bool(sim.fvSolution.adjustPhi)
        self.p_needs_ref = not any(isinstance(bc, DirichletBC) for bc in self.p.bcs.values())
        self.p_ref_cell = -1
        self.p_ref_value = 0.0
        if self.p_needs_ref:
            if alg.pRefCell is None:
                raise ValueError("pRefCell is required when p_needs_ref is True")
            if alg.pRefValue is None:
                raise ValueError("pRefValue is required when p_needs_ref is True")
            self.p_ref_cell = int(alg.pRefCell)
            self.p_ref_value = float(alg.pRefValue)
        self._u_harmonic = int(schemes.laplacian_scheme(sim, self.U.name) in schemes.HARMONIC)
        self._p_harmonic = int(schemes.laplacian_scheme(sim, self.p.name) in schemes.HARMONIC)
        self._u_corrected = int(schemes.laplacian_scheme(sim, self.U.name) in schemes.CORRECTED)
        self._p_corrected = int(schemes.laplacian_scheme(sim, self.p.name) in schemes.CORRECTED)
        # Octree meshes: explicit hanging-face corrections need least-squares
        # gradients of U, p and HbyA (fv/kernels/face_interpolation.py).
        self._hanging = g.num_hanging > 0
        self._div_code = _lib.DIV_CODES[schemes.div_scheme(sim, self.phi.name, self.U.name).value]
        # Configured gradient scheme per field (fvc.grad, the TVD limiter);
        # the hanging-face corrections always take the least-squares one.
        self._gg = {fld.name: schemes.grad_scheme(sim, fld.name) == GradScheme.LINEAR for fld in (self.U, self.p)}
        self._alloc()
        self._adjust_classes = self._build_adjust_classes()
        self._p_ffp = any(bc.kind == _lib.BC_FIXED_FLUX_P for bc in self.p.bcs.values())
        self.last_stats: dict = {}
        # Not None: Krylov solves are recorded here as (solver, descriptor)
        # instead of launched, and the step generator pauses after each one
        # (the solve server launches the same-phase solves of many cases at
        # once, then resumes every case).
        self._deferred: list | None = None
        self._diagnostics = None
        self._diagnostics_step = 0
        # flux.py:132-162 correct_flux(phi, U, update_internal=True)
        self._eval_U()
        if self._hanging:
            self._grad(self.U, self.grad_U)
        call("gf_face_flux", byref(g.cmesh), 0, ptr(self.U.store), ptr(self.U.table.kind),
             ptr(self.U.table.psib), None, ptr(self.grad_U) if self._hanging else None, ptr(self.phi.store),
             stream_ptr())
        if self.transient:
            self.U.update_history(reset=True)
            self.phi.update_history(reset=True)

    # ------------------------------------------------------------------
    @property
    def grid(self):
        return self._grid

    @property
    def solvers(self) -> dict:
        return self._solvers

    def attach_diagnostics(self, diagnostics) -> None:
        """algorithms/base.py:66-75: record continuity and solver statistics
        after every step (``post.diagnostics.DiagnosticsCollector``)."""
        self._diagnostics = diagnostics

    def _finalize_diagnostics(self, phi, solve_stats: dict) -> None:
        """algorithms/base.py:77-100 (enqueues only: no host round trip)."""
        if self._diagnostics is None:
            return
        self._diagnostics_step += 1
        self._diagnostics.record_step(self._diagnostics_step, phi, solve_stats)

    def set_host_readback(self, enabled: bool) -> None:
        """Switch the per-step pinned host copies on or off (see ``host_readback``)."""
        self.host_readback = bool(enabled)
        for s in self._solvers.values():
            s.host_stats = bool(enabled)

    @property
    def p_residual(self) -> torch.Tensor:
        """Device scalar: the last recorded pressure-equation residual."""
        return self.res_buf[0:1]

    def set_grad_mode(self, grad_mode: str) -> None:
        for solver in self._solvers.values():
            solver.grad_mode = grad_mode

    def has_simulation_converged(self) -> bool:
        return False

    # ------------------------------------------------------------------
    def _alloc(self) -> None:
        g = self._grid
        C, dev = g.num_cells, g.device
        f64 = dict(dtype=torch.float64, device=dev)
        self.UEqn = FvMatrix(self.U)
        self.USolve = FvMatrix(self.U)
        self.pEqn = FvMatrix(self.p)
        self.pSolve = FvMatrix(self.p)
        self.pred_source = torch.zeros((3, C), **f64)
        # grad_p / grad_U_cfg: the configured gradients; grad_p_lsq / grad_U:
        # the least-squares ones of the hanging-face corrections (the same
        # buffers when the configured scheme is least squares).
        self.grad_p = torch.zeros((3, C), **f64)
        self.grad_U = torch.zeros((9, C), **f64)
        gg_u, gg_p = self._gg[self.U.name], self._gg[self.p.name]
        self.grad_U_cfg = torch.zeros((9, C), **f64) if gg_u else self.grad_U
        self.grad_p_lsq = torch.zeros((3, C), **f64) if gg_p else self.grad_p
        rows = g.num_internal_faces + g.num_bnd
        self._gg_faces = {self.U.name: torch.zeros((3, rows), **f64) if gg_u else None,
                          self.p.name: torch.zeros((1, rows), **f64) if gg_p else None}
        # Hanging faces: HbyA gradient and the pressure Laplacian's face flux
        # correction (zero off hanging faces).
        self.grad_H = torch.zeros((9, C) if self._hanging else (9, 1), **f64)
        self.p_ffc = torch.zeros(max(1, g.num_internal_faces) if self._hanging else 1, **f64)
        self.div_buf = torch.zeros(C, **f64)
        self.p_old = torch.zeros(C, **f64)
        self.h1 = torch.zeros(C, **f64)
        self.d_r = torch.zeros(C, **f64)
        self.prescribed_U = torch.zeros((3, C), **f64)
        self.prescribed_p = torch.zeros((1, C), **f64)
        self.scratch = torch.zeros(1024, **f64)
        self.res_buf = torch.zeros(8, **f64)
        self.u_cells, self.u_faces, self.u_mask = self.U.table.constraints()
        self.p_cells, self.p_faces, self.p_mask = self.p.table.constraints()
        self.p_fixed_faces, self.p_fixed_frac = self.p.table.fixed_faces()
        # inletOutlet on near immersed faces: selections follow the flux
        self._u_dynamic = self.U.table.dynamic
        self._p_dynamic = self.p.table.dynamic or self.p.table._dynamic_fixed is not None
        self.u_vals = torch.zeros((3, max(1, self.U.table.num_constraint_candidates)), **f64)
        self.p_vals = torch.zeros((1, max(1, self.p.table.num_constraint_candidates)), **f64)
        n_fix = g.num_bnd if self._p_dynamic else self.p_fixed_faces.numel()
        self.fix_scratch = torch.zeros(max(1, n_fix), **f64)

    def _refresh_constraints(self, *, u: bool = False, p: bool = False) -> None:
        """Re-select the flux-dependent immersed constraints (inletOutlet on
        near immersed faces fixes the faces carrying inflow) from the
        current face flux, as the reference evaluates them at each use."""
        if u and self._u_dynamic:
            self.u_cells, self.u_faces, self.u_mask = self.U.table.constraints()
        if p and self._p_dynamic:
            self.p_cells, self.p_faces, self.p_mask = self.p.table.constraints()
            self.p_fixed_faces, self.p_fixed_frac = self.p.table.fixed_faces()

    def _build_adjust_classes(self) -> torch.Tensor:
        """adjust_phi.py:21-41 classes per domain face: 0 skip, 1 fixed, 2 adjustable."""
        return adjust_classes(self.U)

    # ------------------------------------------------------------------
    # boundary states
    # ------------------------------------------------------------------
    def _eval_U(self) -> None:
        aux = GfBcAux()
        aux.phi_bnd = ptr(self.phi.boundary_store)
        self.U.evaluate_bc(aux)

    def _eval_p(self) -> None:
        aux = GfBcAux()
        aux.phi_bnd = ptr(self.phi.boundary_store)
        if self._p_ffp:
            self._eval_U()
            aux.ffp_phi_pred = ptr(self.phi_hbya.boundary_store)
            aux.ffp_u_kind = ptr(self.U.table.kind)
            aux.ffp_u_psib = ptr(self.U.table.psib)
            aux.ffp_coeff = ptr(self.rAtU.store)
        self.p.evaluate_bc(aux)

    def _grad(self, field: CellField, out: torch.Tensor) -> None:
        """least_squares.py:29-101 (boundary state must be current)."""
        t = field.table
        call("gf_lsq_grad", byref(self._grid.cmesh), field.num_components, ptr(field.store),
             ptr(t.kind), ptr(t.psib), ptr(out), stream_ptr())

    def _grad_cfg(self, field: CellField, out: torch.Tensor, lsq: torch.Tensor) -> None:
        """The configured gradient into ``out`` (fv/schemes/grad.py): least
        squares, or Green-Gauss over the linear face values, whose hanging
        correction needs the least-squares gradient (written to ``lsq``;
        ``out`` is ``lsq`` itself when the scheme is least squares)."""
        if not self._gg[field.name]:
            self._grad(field, out)
            return
        from gridfoam_b200.fv.fvc import configured_grad

        configured_grad(field, out, self._gg_faces[field.name], lsq)

    # ------------------------------------------------------------------
    # momentum predictor
    # ------------------------------------------------------------------
    def _assemble_momentum(self, relax: float) -> None:
        g = self._grid
        self._refresh_constraints(u=True)
        self._eval_U()
        tvd = self._div_code >= _lib.DIV_CODES["vanleer"]
        if tvd:
            # also fills grad_U (the hanging corrections') on a hanging mesh
            self._grad_cfg(self.U, self.grad_U_cfg, self.grad_U)
        elif self._hanging:
            self._grad(self.U, self.grad_U)
        a = GfAssembly()
        a.ncomp = 3
        a.div_scheme = self._div_code
        a.lap_harmonic = self._u_harmonic
        a.div_sign = 1.0
        a.lap_sign = -1.0
        a.gamma_scalar = self.nu
        a.gamma = None
        a.phi = ptr(self.phi.store)
        a.psi = ptr(self.U.store)
        a.grad_psi = ptr(self.grad_U_cfg)
        if self.transient:
            ca, cb, cc = schemes.ddt_coefficients(self.U)
            a.use_ddt = 1
            a.ddt_a, a.ddt_b, a.ddt_c, a.dt = ca, cb, cc, g.dt
            a.psi_old = ptr(self.U.old_store)
            a.psi_older = ptr(self.U.older_store) if cc != 0.0 else None
        t = self.U.table
        a.bc_kind = ptr(t.kind)
        a.frac = ptr(t.frac)
        a.refv = ptr(t.refv)
        a.refg = ptr(t.refg)
        a.diag = ptr(self.UEqn.diag_store)
        a.val = ptr(self.UEqn.val)
        a.source = ptr(self.UEqn.source_store)
        if self._hanging:
            a.grad_lsq = ptr(self.grad_U)
            a.lap_corrected = self._u_corrected
        s = stream_ptr()
        call("gf_assemble", byref(g.cmesh), byref(a), s)
        if relax > 0.0:
            call("gf_momentum_finalize", byref(g.cmesh), 3, relax, ptr(self.U.store), None,
                 ptr(self.UEqn.diag_store), ptr(self.UEqn.source_store), None, s)
        # predictor source b - V grad(p)
        self._eval_p()
        self._grad_cfg(self.p, self.grad_p, self.grad_p_lsq)
        call("gf_momentum_finalize", byref(g.cmesh), 3, 0.0, None, ptr(self.grad_p),
             ptr(self.UEqn.diag_store), ptr(self.UEqn.source_store), ptr(self.pred_source), s)

    def _constrain(self, field: CellField, mat_diag, mat_val, mat_src, out: FvMatrix, cells, faces, mask,
                   vals, prescribed) -> tuple:
        """core/equation.py:42-47 + fvmatrix.py:325-394 on the device."""
        n = int(cells.numel())
        if n == 0:
            return mat_diag, mat_val, mat_src
        g = self._grid
        nc = field.num_components
        s = stream_ptr()
        call("gf_gather_bnd", g.num_bnd, nc, n, ptr(faces), ptr(field.table.refv), ptr(vals), s)
        call("gf_set_cell_values", g.num_cells, nc, n, ptr(cells), ptr(vals), n, ptr(prescribed), s)
        call("gf_fixed_values", byref(g.cmesh), nc, ptr(mat_diag), ptr(mat_val), ptr(mat_src), n, None,
             ptr(prescribed), ptr(mask), ptr(out.diag_store), ptr(out.val), ptr(out.source_store),
             ptr(self.scratch), s)
        return out.diag_store, out.val, out.source_store

    def _apply_fixed(self, field: CellField, cells, faces, vals) -> None:
        """boundary_ops.py:538-542 (state of ``field`` must be current)."""
        n = int(cells.numel())
        if n == 0:
            return
        g = self._grid
        nc = field.num_components
        s = stream_ptr()
        call("gf_gather_bnd", g.num_bnd, nc, n, ptr(faces), ptr(field.table.refv), ptr(vals), s)
        call("gf_set_cell_values", g.num_cells, nc, n, ptr(cells), ptr(vals), n, ptr(field.store), s)

    def _solve(self, solver, d, v, src, x, *, symmetric: bool = False):
        """A Krylov solve (generator): launched at once, or recorded and
        paused on when solves are deferred."""
        if self._deferred is None:
            return solver.solve_arrays(self._grid, d, v, src, x, symmetric=symmetric)
        k, _ = solver.describe(self._grid, d, v, src, x, symmetric=symmetric)
        self._deferred.append((solver, k))
        yield
        return ()

    def _momentum_solve(self, residual_key: str | None = None):
        d, v, src = self._constrain(self.U, self.UEqn.diag_store, self.UEqn.val, self.pred_source, self.USolve,
                                    self.u_cells, self.u_faces, self.u_mask, self.u_vals, self.prescribed_U)
        if residual_key is not None:
            self._record_residual_dev(residual_key, d, v, src, self.U)
        stats = yield from self._solve(self._solvers[self.U.name], d, v, src, self.U.store)
        # UEqn for H/A: constraints of the updated velocity
        if self.u_cells.numel():
            self._eval_U()
        self._Ud, self._Uv, self._Us = self._constrain(
            self.U, self.UEqn.diag_store, self.UEqn.val, self.UEqn.source_store, self.USolve,
            self.u_cells, self.u_faces, self.u_mask, self.u_vals, self.prescribed_U)
        return stats

    # ------------------------------------------------------------------
    # pressure stage
    # ------------------------------------------------------------------
    def _hbya(self, *, ddt: bool, consistent: bool) -> None:
        g = self._grid
        s = stream_ptr()
        call("gf_rau_hbya", byref(g.cmesh), 3, ptr(self._Ud), ptr(self._Uv), ptr(self._Us), ptr(self.U.store),
             ptr(self.rAU.store), ptr(self.HbyA.store), ptr(self.h1), s)
        self._eval_U()
        d = None
        if ddt:
            _, cb, cc = schemes.ddt_coefficients(self.U)
            if cc != 0.0 and self.phi.previous_dt != self.U.previous_dt:
                raise ValueError("backward ddtCorr requires synchronized U and phi histories")
            d = GfDdtCorr()
            d.rau = ptr(self.rAU.store)
            d.u_old = ptr(self.U.old_store)
            d.u_older = ptr(self.U.older_store) if cc != 0.0 else None
            d.phi_old = ptr(self.phi.old_store)
            d.phi_older = ptr(self.phi.older_store) if cc != 0.0 else None
            d.b, d.c, d.dt = cb, cc, g.dt
        grad_h = None
        if self._hanging:
            # fvc.interpolate(HbyA): HbyA carries no boundary conditions, so
            # its least-squares gradient has internal equations only.
            t = self.HbyA.table
            call("gf_lsq_grad", byref(g.cmesh), 3, ptr(self.HbyA.store), ptr(t.kind), ptr(t.psib),
                 ptr(self.grad_H), s)
            grad_h = ptr(self.grad_H)
        call("gf_face_flux", byref(g.cmesh), 1, ptr(self.HbyA.store), ptr(self.U.table.kind),
             ptr(self.U.table.psib), None if d is None else byref(d), grad_h, ptr(self.phi_hbya.store), s)
        if self.adjust_phi_enabled and self.p_needs_ref:
            call("gf_adjust_phi", byref(g.cmesh), ptr(self._adjust_classes), ptr(self.phi_hbya.store), s)
        if consistent:
            # pressure_correction.py:163-267 (bounded SIMPLEC)
            call("gf_simplec_rAtU", byref(g.cmesh), ptr(self.rAU.store), ptr(self.h1), ptr(self.rAtU.store), s)
            call("gf_axpby", g.num_cells, 1.0, ptr(self.rAtU.store), -1.0, ptr(self.rAU.store), ptr(self.d_r), s)
            self._eval_p()
            t = self.p.table
            # (with Green-Gauss on a hanging mesh this also leaves the
            # least-squares gradient of the correction in grad_p_lsq)
            self._grad_cfg(self.p, self.grad_p, self.grad_p_lsq)
            call("gf_correct_phi", byref(g.cmesh), ptr(self.phi_hbya.store), ptr(self.d_r), ptr(self.p.store),
                 ptr(t.kind), ptr(t.frac), ptr(t.refv), ptr(t.refg), 1.0, 1,
                 ptr(self.grad_p_lsq) if self._hanging else None, None, ptr(self.phi_hbya.store), s)
            call("gf_axpby", g.num_cells, 1.0, ptr(self.rAU.store), -1.0, ptr(self.rAtU.store), ptr(self.d_r), s)
            call("gf_correct_velocity", byref(g.cmesh), ptr(self.HbyA.store), ptr(self.d_r), ptr(self.grad_p),
                 ptr(self.HbyA.store), s)
        else:
            self.rAtU.store.copy_(self.rAU.store)

    def _pressure_solve(self, *, final_solver=None, record: bool = False):
        """pressure_correction.py:68-160."""
        g = self._grid
        s = stream_ptr()
        stats = None
        first_res = last_res = None
        self._refresh_constraints(p=True)
        for corr in range(self.n_non_orthogonal_correctors + 1):
            self._eval_p()
            t = self.p.table
            a = GfAssembly()
            a.ncomp = 1
            a.div_scheme = 0
            a.lap_harmonic = self._p_harmonic
            a.lap_sign = -1.0
            a.gamma = ptr(self.rAtU.store)
            a.bc_kind = ptr(t.kind)
            a.frac = ptr(t.frac)
            a.refv = ptr(t.refv)
            a.refg = ptr(t.refg)
            a.diag = ptr(self.pEqn.diag_store)
            a.val = ptr(self.pEqn.val)
            a.source = ptr(self.pEqn.source_store)
            if self._hanging:
                self._grad(self.p, self.grad_p_lsq)
                a.grad_lsq = ptr(self.grad_p_lsq)
                a.lap_corrected = self._p_corrected
                a.ffc = ptr(self.p_ffc)
            call("gf_assemble", byref(g.cmesh), byref(a), s)
            call("gf_pressure_finalize", byref(g.cmesh), ptr(self.phi_hbya.store), ptr(self.pEqn.diag_store),
                 ptr(self.pEqn.source_store), ptr(self.div_buf), self.p_ref_cell, self.p_ref_value, s)
            d, v, src = self._constrain(self.p, self.pEqn.diag_store, self.pEqn.val, self.pEqn.source_store,
                                        self.pSolve, self.p_cells, self.p_faces, self.p_mask, self.p_vals,
                                        self.prescribed_p)
            if record:
                call("gf_field_residual", byref(g.cmesh), 1, ptr(d), ptr(v), ptr(src), ptr(self.p.store),
                     ptr(self.scratch), ptr(self.res_buf), s)
                last_res = _LazyScalar(self.res_buf[0]) if self.host_readback else None
                if first_res is None:
                    first_res = last_res
            solver = self._solvers[self.p.name]
            if final_solver is not None and corr == self.n_non_orthogonal_correctors:
                solver = final_solver
            stats = yield from self._solve(solver, d, v, src, self.p.store, symmetric=True)
        return stats, first_res, last_res

    def _correct_phi(self) -> None:
        """pressure_correction.py:270-335."""
        g = self._grid
        s = stream_ptr()
        self._refresh_constraints(p=True)
        self._eval_p()
        t = self.p.table
        call("gf_correct_phi", byref(g.cmesh), ptr(self.phi_hbya.store), ptr(self.rAtU.store), ptr(self.p.store),
             ptr(t.kind), ptr(t.frac), ptr(t.refv), ptr(t.refg), -1.0, 0, None,
             ptr(self.p_ffc) if self._hanging else None, ptr(self.phi.store), s)
        n = int(self.p_fixed_faces.numel())
        if n:
            call("gf_close_fixed_flux", byref(g.cmesh), n, ptr(self.p_fixed_faces), ptr(self.p_fixed_frac),
                 ptr(self.phi.store), ptr(self.fix_scratch), s)

    def _correct_velocity(self) -> None:
        """pressure_correction.py:338-363."""
        g = self._grid
        self._refresh_constraints(u=True, p=True)
        self._eval_p()
        self._grad_cfg(self.p, self.grad_p, self.grad_p_lsq)
        call("gf_correct_velocity", byref(g.cmesh), ptr(self.HbyA.store), ptr(self.rAtU.store), ptr(self.grad_p),
             ptr(self.U.store), stream_ptr())
        if self.u_cells.numel():
            self._eval_U()
            self._apply_fixed(self.U, self.u_cells, self.u_faces, self.u_vals)

    # residual helpers (algorithms/utils/residual.py)
    def _record_residual_dev(self, key, d, v, src, field) -> None:
        g = self._grid
        call("gf_field_residual", byref(g.cmesh), field.num_components, ptr(d), ptr(v), ptr(src),
             ptr(field.store), ptr(self.scratch), ptr(self.res_buf[1:]), stream_ptr())
        self._pending_residual = (key, _LazyScalar(self.res_buf[1]) if self.host_readback else None)

    def continuity_residual(self) -> float:
        """residual.py:39-53: |div(phi)|_2."""
        g = self._grid
        call("gf_fvc_div", byref(g.cmesh), 1, ptr(self.phi.store), ptr(self.div_buf), stream_ptr())
        return float(torch.linalg.vector_norm(self.div_buf).item())


class SIMPLE(_PressureVelocity):
    """Steady SIMPLE / SIMPLEC (algorithms/simple.py:48-408)."""

    transient = False

    def __init__(self, grid, phase: str | None = None):
        super().__init__(grid, phase)
        alg = self._alg
        assert isinstance(alg, SIMPLEAlgorithm)
        self.alpha_U = float(alg.relaxationFactors.equations[self.U.name])
        self.alpha_p = float(alg.relaxationFactors.equations[self.p.name])
        self.consistent = bool(alg.consistent)
        self._residual_control = normalize_residual_control(alg.residualControl)
        self._initial_residuals: dict = {}
        self._current_residuals: dict = {}

    def _record(self, name: str, value) -> None:
        if name not in self._initial_residuals:
            self._initial_residuals[name] = value
        self._current_residuals[name] = value

    def has_converged(self) -> bool:
        """simple.py:245-271 (absolute tolerances only)."""
        if not self._residual_control:
            return False
        for name, entry in self._residual_control.items():
            cur = self._current_residuals.get(name)
            if cur is None or self._initial_residuals.get(name) is None:
                return False
            cur = cur.value() if isinstance(cur, _LazyScalar) else cur
            if not cur < entry.tolerance:
                return False
        return True

    def has_simulation_converged(self) -> bool:
        return self.has_converged()

    def step(self) -> None:
        """simple.py:287-408."""
        for _ in self.step_phases():
            pass

    def step_phases(self):
        """One step as a generator that pauses after each deferred Krylov
        solve (see ``_deferred``); without deferral it runs straight through."""
        g = self._grid
        self._assemble_momentum(self.alpha_U)
        key = self.U.name if self.U.name in self._residual_control else None
        st_u = yield from self._momentum_solve(residual_key=key)
        if key is not None:
            self._record(*self._pending_residual)
        self._hbya(ddt=False, consistent=self.consistent)
        self.p_old.copy_(self.p.store[0])
        record = self.p.name in self._residual_control
        st_p, first, _ = yield from self._pressure_solve(record=record)
        if record:
            self._record(self.p.name, first)
        self._correct_phi()
        call("gf_relax_field", g.num_cells, self.alpha_p, ptr(self.p_old), ptr(self.p.store), stream_ptr())
        self._refresh_constraints(p=True)
        if self.p_cells.numel():
            self._eval_p()
            self._apply_fixed(self.p, self.p_cells, self.p_faces, self.p_vals)
        self._correct_velocity()
        if "phi" in self._residual_control:
            self._record("phi", self.continuity_residual())
        self.last_stats = {self.U.name: st_u, self.p.name: st_p}
        self._finalize_diagnostics(self.phi, self.last_stats)


class PISO(_PressureVelocity):
    """Transient PISO (algorithms/piso.py:44-326)."""

    transient = True

    def __init__(self, grid, phase: str | None = None):
        super().__init__(grid, phase)
        alg = self._alg
        assert isinstance(alg, PISOAlgorithm)
        self.n_correctors = int(alg.nCorrectors)
        self.consistent = False

    def has_converged(self) -> bool:
        return False

    def step(self) -> None:
        """piso.py:227-326."""
        for _ in self.step_phases():
            pass

    def step_phases(self):
        """One step as a generator that pauses after each deferred solve."""
        self._assemble_momentum(0.0)
        st_u = yield from self._momentum_solve()
        st_p = None
        for i in range(self.n_correctors):
            self._hbya(ddt=True, consistent=False)
            final = resolve_solver(self._solvers, self.p.name, is_final=(i == self.n_correctors - 1))
            st_p, _, _ = yield from self._pressure_solve(final_solver=final)
            self._correct_phi()
            self._correct_velocity()
        self.U.update_history()
        self.phi.update_history()
        self.last_stats = {self.U.name: st_u, self.p.name: st_p}
        self._finalize_diagnostics(self.phi, self.last_stats)


class PIMPLE(_PressureVelocity):
    """PIMPLE outer loop with residual control (algorithms/pimple.py:50-454)."""

    transient = True

    def __init__(self, grid, phase: str | None = None):
        super().__init__(grid, phase)
        alg = self._alg
        assert isinstance(alg, PIMPLEAlgorithm)
        self.n_outer_correctors = int(alg.nOuterCorrectors)
        self.n_correctors = int(alg.nCorrectors)
        self.consistent = bool(alg.consistent)
        self._residual_control = normalize_residual_control(alg.residualControl)
        self._initial_residuals: dict = {}
        self._current_residuals: dict = {}
        self._outer_converged = False

    def has_converged(self) -> bool:
        return self._outer_converged

    def _value(self, v):
        return v.value() if isinstance(v, _LazyScalar) else v

    def _check_outer_convergence(self, *, allow_relative: bool = True) -> bool:
        """pimple.py:271-288."""
        if not self._residual_control:
            return False
        for name, entry in self._residual_control.items():
            cur = self._current_residuals.get(name)
            ini = self._initial_residuals.get(name)
            if cur is None or ini is None:
                return False
            cur, ini = self._value(cur), self._value(ini)
            rel = entry.rel_tolerance if allow_relative else 0.0
            if not (cur < entry.tolerance or (rel > 0.0 and cur < rel * ini)):
                return False
        return True

    def _record(self, name: str, value) -> None:
        if name not in self._initial_residuals:
            self._initial_residuals[name] = value
        self._current_residuals[name] = value

    def step(self) -> None:
        """pimple.py:290-454."""
        for _ in self.step_phases():
            pass

    def step_phases(self):
        """One step as a generator that pauses after each deferred solve."""
        self._outer_converged = False
        self._initial_residuals.clear()
        self._current_residuals.clear()
        st_u = st_p = None
        for outer in range(self.n_outer_correctors):
            final_after = 0 < outer < self.n_outer_correctors - 1 and self._check_outer_convergence(
                allow_relative=outer > 1
            )
            if final_after:
                self._outer_converged = True
            self._assemble_momentum(0.0)
            key = self.U.name if self.U.name in self._residual_control else None
            st_u = yield from self._momentum_solve(residual_key=key)
            if key is not None:
                self._record(*self._pending_residual)
            for inner in range(self.n_correctors):
                self._hbya(ddt=True, consistent=self.consistent)
                final = resolve_solver(self._solvers, self.p.name, is_final=(inner == self.n_correctors - 1))
                record = self.p.name in self._residual_control
                st_p, first, last = yield from self._pressure_solve(final_solver=final, record=record)
                if record:
                    if inner == 0:
                        self._record(self.p.name, first)
                    self._current_residuals[self.p.name] = last
                self._correct_phi()
                self._correct_velocity()
            if "phi" in self._residual_control:
                self._record("phi", self.continuity_residual())
            if final_after:
                break
        self.U.update_history()
        self.phi.update_history()
        self.last_stats = {self.U.name: st_u, self.p.name: st_p}
        self._finalize_diagnostics(self.phi, self.last_stats)


def create_algorithm(grid, phase: str | None = None):
    """algorithms/factory.py:9-38."""
    match grid.sim_config.fvSolution.algorithm.type:
        case AlgorithmType.SIMPLE:
            return SIMPLE(grid, phase=phase)
        case AlgorithmType.PIMPLE:
            return PIMPLE(grid, phase=phase)
        case AlgorithmType.PISO:
            return PISO(grid, phase=phase)
        case AlgorithmType.MANUAL:
            raise ValueError("Manual algorithm has no step sequence")
