"""Shape gradients of an immersed body's drag at a steady SIMPLE solution.

The body is the zero set of a signed-distance function ``sdf(x; theta)`` of
shape parameters ``theta``; the mesh's immersed faces carry the distance
from each side's cell centre to the crossing of the owner-neighbour segment
(``dist_owner_to_bnd`` / ``dist_neighbour_to_bnd``) and the body-outward
surface normal there (the force integral's sample orientation).  For fixed
discrete structure (the same immersed faces, near flags and cell
constraints) the steady solution and its drag are smooth functions of those
distances and normals, and the gradient is

    dJ/dtheta = (dJ/dg) (dg/dtheta),  g = (distances, normals),

with ``dJ/dg`` from the discrete adjoint of the steady solution and
``dg/dtheta`` from the geometry:

* the crossing parameter ``t`` of a segment ``x0 + t (x1 - x0)`` moves by
  ``dt/dtheta = -(d sdf/d theta) / (grad sdf . (x1 - x0))`` (implicit
  differentiation of ``sdf(x(t); theta) = 0``), the distances by
  ``+-|x1 - x0| dt/dtheta``; the normals are re-evaluated at the moved
  crossing (central differences in ``theta``);
* the steady state ``x* = Phi(x*, g)`` is the fixed point of one SIMPLE
  iteration ``Phi``; the adjoint is its reverse accumulation (Christianson's
  fixed-point adjoint): ``lambda <- dJ/dx + lambda dPhi/dx`` until it stops
  changing, then ``dJ/dg = dJ/dg|_x + lambda dPhi/dg``.  Each sweep is one
  reverse pass through ``Phi`` at ``x*``: the momentum and pressure solves
  run backwards as transpose solves on the GPU (``solvers/adjoint.py``,
  ``gf_adjoint_ldu_grads``), the remaining algebra of the iteration is
  device tensor algebra whose derivatives autograd forms.

The reference differentiates through torch autograd but holds no shape
derivative (its immersed geometry is discrete); the reverse sweep follows
its SIMPLE iteration (algorithms/simple.py:287-408,
algorithms/utils/pressure_correction.py:68-363) term by term, and
``DifferentiableSimpleIteration.check`` compares one forward evaluation with
the library's own SIMPLE step.

Scope: uniform and octree grids (hanging-face offset and skewness terms)
with immersed bodies, steady SIMPLE or SIMPLEC, upwind convection, least-squares gradients, velocity conditions
dirichlet / neumann / slip / inlet_outlet, pressure conditions dirichlet /
neumann, a pressure outlet (no adjustPhi, no reference cell) and no
pressure constraints at immersed faces.
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
import torch

from gridfoam_b200 import _lib
from gridfoam_b200.meta.config import PreconditionerType, SolverConfig
from gridfoam_b200.solvers.adjoint import attach_implicit_adjoint

_EPS = float(np.finfo(np.float64).eps)


def _bc_codes() -> dict:
    return {"none": _lib.BC_NONE, "dirichlet": _lib.BC_DIRICHLET, "neumann": _lib.BC_NEUMANN,
            "slip": _lib.BC_SLIP, "inlet_outlet": _lib.BC_INLET_OUTLET}


def _check_supported(algo) -> None:
    from gridfoam_b200.algorithms.pressure_velocity import SIMPLE
    from gridfoam_b200.fv import schemes

    g = algo.grid
    if not isinstance(algo, SIMPLE):
        raise NotImplementedError("the shape adjoint differentiates steady SIMPLE solutions")
    sim = g.sim_config
    if schemes.div_scheme(sim, algo.phi.name, algo.U.name).value != "upwind":
        raise NotImplementedError("the shape adjoint covers upwind convection")
    if algo._gg[algo.U.name] or algo._gg[algo.p.name]:
        raise NotImplementedError("the shape adjoint covers least-squares gradients")
    if algo.n_non_orthogonal_correctors:
        raise NotImplementedError("the shape adjoint covers nNonOrthogonalCorrectors 0")
    if algo.p_needs_ref:
        raise NotImplementedError("the shape adjoint needs a pressure outlet (no reference cell, no adjustPhi)")
    codes = _bc_codes()
    allowed_u = {codes["none"], codes["dirichlet"], codes["neumann"], codes["slip"], codes["inlet_outlet"]}
    allowed_p = {codes["none"], codes["dirichlet"], codes["neumann"]}
    if not set(np.unique(algo.U.table.kind_host)) <= allowed_u:
        raise NotImplementedError("velocity conditions other than dirichlet/neumann/slip/inlet_outlet")
    if not set(np.unique(algo.p.table.kind_host)) <= allowed_p:
        raise NotImplementedError("pressure conditions other than dirichlet/neumann")
    if algo.p_cells.numel() or algo.p_fixed_faces.numel():
        raise NotImplementedError("pressure constraints at immersed faces")
    if algo.U.table.dynamic:
        raise NotImplementedError("flux-dependent velocity constraints (inletOutlet on near immersed faces)")
    if algo._u_harmonic or algo._p_harmonic:
        raise NotImplementedError("harmonic diffusivity interpolation")


def _tight(method: str) -> SolverConfig:
    return SolverConfig(method=method, preconditioner=PreconditionerType.JACOBI, tolerance=0.0,
                        rel_tolerance=1e-13, max_iter=50000)


class DifferentiableSimpleIteration:
    """One SIMPLE(C) iteration of ``algo``'s case as a differentiable map

        (U [C,3], p [C], phi [F+Nb], dist [2 Fi]) -> (U', p', phi')

    on the device, with exact (tightly converged) solves: at a fixed point
    the iteration's Jacobian is that of the discrete steady equations, which
    do not depend on how accurately the primal iterations solved."""

    def __init__(self, algo):
        _check_supported(algo)
        from gridfoam_b200.solvers.krylov import BiCGSTABSolver, CGSolver

        self.algo = algo
        g = algo.grid
        h = g.host
        dev = g.device
        f64 = dict(dtype=torch.float64, device=dev)
        self.grid = g
        self.C, self.F = g.num_cells, g.num_internal_faces
        self.Fb, self.Fi, self.Nb = g.num_domain_bnd_faces, g.num_immersed_faces, g.num_bnd
        imm = np.asarray(h.immersed, dtype=bool)
        s = np.nonzero(~imm)[0]
        self.single = torch.as_tensor(s, device=dev)
        self.own_s = torch.as_tensor(h.owner[s], device=dev)
        self.nei_s = torch.as_tensor(h.neighbour[s], device=dev)
        self.w_s = torch.as_tensor(h.w[s], **f64)
        self.Sf_s = torch.as_tensor(h.Sf[s], **f64)
        self.magSf_s = torch.as_tensor(h.mag_sf[s], **f64)
        self.delta_s = torch.as_tensor(h.delta[s], **f64)
        c = np.asarray(h.cell_centers)
        d = c[h.neighbour[s]] - c[h.owner[s]]
        self.d_s = torch.as_tensor(d, **f64)
        self.w2_s = torch.as_tensor(1.0 / np.where((d * d).sum(1) > 0, (d * d).sum(1), 1.0), **f64)
        self.own = torch.as_tensor(h.owner, device=dev)
        self.nei = torch.as_tensor(h.neighbour, device=dev)
        self.V = torch.as_tensor(h.cell_volumes, **f64)
        self.bcell = torch.as_tensor(h.bnd_cell, device=dev)
        self.bsf = torch.as_tensor(h.bnd_sf, **f64)
        self.bmagsf = torch.as_tensor(h.bnd_mag_sf, **f64)
        self.bmagd = torch.as_tensor(h.bnd_mag_d, **f64)
        bd = np.asarray(h.bnd_d, dtype=np.float64)
        mag = np.linalg.norm(bd, axis=1)
        self.bdir = torch.as_tensor(bd / np.where(mag > 0, mag, 1.0)[:, None], **f64)  # unit d_b
        self.bnear = torch.as_tensor(np.asarray(h.bnd_near) != 0, device=dev)
        self.is_imm_b = torch.arange(self.Nb, device=dev) >= self.Fb
        self.ata_inv = torch.as_tensor(np.asarray(h.extra["lsq_ata_inv"]).reshape(-1, 3, 3), **f64)
        self.n_sign = torch.sign(self.bsf)  # slip: axis-aligned face normal
        self.nu = float(algo.nu)
        self.alpha_U, self.alpha_p = float(algo.alpha_U), float(algo.alpha_p)
        self.consistent = bool(algo.consistent)
        codes = _bc_codes()
        self.codes = codes
        self.ukind = torch.as_tensor(algo.U.table.kind_host.astype(np.int64), device=dev)
        self.pkind = torch.as_tensor(algo.p.table.kind_host.astype(np.int64), device=dev)
        self.uval = algo.U.table.value.t().contiguous()  # [Nb, 3]
        self.pval = algo.p.table.value.t().contiguous()  # [Nb, 1]
        # non-assignable velocity conditions fix the predicted flux (flux.py:74-87)
        self.u_fixed_flux = (self.ukind == codes["dirichlet"]) | (self.ukind == codes["slip"])
        uncov = np.asarray(algo.U.table.kind_host) == codes["none"]
        self.u_uncovered = torch.as_tensor(uncov, device=dev)
        self.u_cells = algo.u_cells.long()
        self.u_faces = algo.u_faces.long()
        # Hanging (coarse-fine) faces, as positions among the single faces:
        # offset of the face centre from the linear-weight point and the
        # tangential moves from each cell centre (face_geometry.py:141-162).
        hf = np.asarray(h.extra["hang_faces"], dtype=np.int64)
        self.H = int(hf.size)
        if self.H:
            pos = np.full(self.F, -1, dtype=np.int64)
            pos[s] = np.arange(s.size)
            self.hpos = torch.as_tensor(pos[hf], device=dev)
            self.hoff = torch.as_tensor(np.asarray(h.extra["hang_offset"]), **f64)
            self.hmo = torch.as_tensor(np.asarray(h.extra["hang_move_o"]), **f64)
            self.hmn = torch.as_tensor(np.asarray(h.extra["hang_move_n"]), **f64)
            self.u_corrected = bool(algo._u_corrected)
            self.p_corrected = bool(algo._p_corrected)
        self.u_solver = BiCGSTABSolver(_tight("bicgstab"))
        self.p_solver = CGSolver(_tight("cg"))

    # ------------------------------------------------------------------
    def _scatter(self, idx: torch.Tensor, val: torch.Tensor) -> torch.Tensor:
        out = torch.zeros((self.C,) + tuple(val.shape[1:]), dtype=val.dtype, device=val.device)
        return out.index_add(0, idx, val)

    def bc_state(self, kind, value, psi_c, phi_b, dist_b):
        """boundary_ops.py:311-437 per boundary face: fraction, ref_v, ref_g,
        the face value and the value-gradient coefficient (near faces with
        fraction 1 impose a cell constraint and get none)."""
        codes = self.codes
        nc = psi_c.shape[1]
        zero = torch.zeros_like(psi_c)
        frac = torch.zeros(self.Nb, dtype=torch.float64, device=psi_c.device)
        refv, refg = zero, zero
        dmask = kind == codes["dirichlet"]
        frac = torch.where(dmask, 1.0, frac)
        refv = torch.where(dmask[:, None], value, refv)
        nmask = kind == codes["neumann"]
        refg = torch.where(nmask[:, None], value, refg)
        if nc == 3:
            smask = kind == codes["slip"]
            normal = (psi_c * self.n_sign).sum(1, keepdim=True)
            tang = psi_c - normal * self.n_sign
            frac = torch.where(smask, 1.0, frac)
            refv = torch.where(smask[:, None], tang, refv)
            io = (kind == codes["inlet_outlet"]) & (phi_b.detach() < 0.0)
            frac = torch.where(io, 1.0, frac)
            refv = torch.where(io[:, None], value, refv)
        fv = frac[:, None]
        psib = fv * refv + (1.0 - fv) * (psi_c + dist_b[:, None] * refg)
        fixed = self.is_imm_b & self.bnear & (frac == 1.0)
        active = (frac != 0.0) & ~fixed & (kind != codes["none"])
        safe = torch.where(active, dist_b, torch.ones_like(dist_b))
        vgc = torch.where(active, frac / safe, torch.zeros_like(frac))
        covered = kind != codes["none"]
        return frac, refv, refg, psib, vgc, covered

    def _hang_sn(self, grad):
        """face_interpolation.py:99-145 on the hanging faces:
        delta (grad_N . move_N - grad_O . move_O), ``grad [C, nc, 3]``."""
        hp = self.hpos
        o, n = self.own_s[hp], self.nei_s[hp]
        gn = torch.einsum("hkj,hj->hk", grad[n], self.hmn)
        go = torch.einsum("hkj,hj->hk", grad[o], self.hmo)
        return self.delta_s[hp][:, None] * (gn - go)

    def _hang_value(self, grad):
        """face_interpolation.py:45-96: offset . (w grad_O + (1 - w) grad_N)."""
        hp = self.hpos
        w = self.w_s[hp][:, None, None]
        gf = w * grad[self.own_s[hp]] + (1.0 - w) * grad[self.nei_s[hp]]
        return torch.einsum("hkj,hj->hk", gf, self.hoff)

    def lsq_grad(self, psi, psib, covered, dist_b):
        """least_squares.py:29-101: single faces plus every conditioned
        boundary face, normal matrix from the grid."""
        dpsi = psi[self.nei_s] - psi[self.own_s]
        t = (self.w2_s[:, None] * dpsi)[:, :, None] * self.d_s[:, None, :]  # [Fs, nc, 3]
        atb = self._scatter(self.own_s, t) + self._scatter(self.nei_s, t)
        db = dist_b[:, None] * self.bdir
        d2 = (db * db).sum(1)
        w2b = 1.0 / torch.where(d2 > 0, d2, torch.ones_like(d2))
        dpb = torch.where(covered[:, None], psib - psi[self.bcell], torch.zeros_like(psib))
        tb = (w2b[:, None] * dpb)[:, :, None] * db[:, None, :]
        atb = atb + self._scatter(self.bcell, tb)
        return torch.einsum("cij,ckj->cki", self.ata_inv, atb)  # [C, nc, 3]

    def _fixed(self, diag, upper, lower, source, cells, values):
        """fvmatrix.py:325-394 (symmetric elimination) on LDU tensors."""
        if cells.numel() == 0:
            return diag, upper, lower, source
        from gridfoam_b200.core.fvmatrix import fixed_values_ldu

        return fixed_values_ldu(self.grid, diag, upper, lower, source, cells, values)

    def _solve(self, solver, field, diag, upper, lower, source, x0, symmetric):
        from gridfoam_b200.core.fvmatrix import FvMatrix

        M = FvMatrix(field)
        M.diag = diag
        M.upper = upper
        M.lower = lower
        src = source[:, 0] if source.shape[1] == 1 else source
        M.source = src
        with torch.no_grad():
            # a copy: the solve writes its solution into x, and the guess
            # must stay the caller's (the scalar case would be a view)
            x = (x0.detach().t() if x0.shape[1] > 1 else x0.detach().reshape(1, -1)).clone(
                memory_format=torch.contiguous_format)
            solver.solve_arrays(self.grid, M.diag_store, M.val, M.source_store, x, symmetric=symmetric)
        sol = x[0] if source.shape[1] == 1 else x.t()
        if not torch.is_grad_enabled():
            return sol.reshape(source.shape)
        out = attach_implicit_adjoint(M, sol, solve_transpose=solver.solve_transpose)
        return out.reshape(source.shape)

    def _off(self, upper, lower, x):
        """sum of off-diagonal couplings times x, per cell."""
        return self._scatter(self.own, upper[:, None] * x[self.nei]) + self._scatter(self.nei, lower[:, None] * x[self.own])

    # ------------------------------------------------------------------
    def step(self, U, p, phi, dist, trace: dict | None = None):
        """One SIMPLE iteration (simple.py:287-408) from (U, p, phi);
        ``trace`` receives the intermediate fields (rAU, rAtU, HbyA,
        phiHbyA) when given."""
        algo = self.algo
        C, F, Fb = self.C, self.F, self.Fb
        V = self.V
        dist_b = torch.cat([self.bmagd[:Fb], dist])
        phi_b = phi[F:]
        phi_s = phi[:F][self.single]
        p2 = p[:, None]
        # --- momentum: div(phi, U) - laplacian(nu, U), upwind (div.py:36-80, laplacian.py:101-201)
        f, refv, refg, psib, vgc, cov = self.bc_state(self.ukind, self.uval, U[self.bcell], phi_b, dist_b)
        pos, neg = torch.clamp(phi_s, min=0.0), torch.clamp(phi_s, max=0.0)
        coeff = self.nu * self.magSf_s * self.delta_s
        upper = torch.zeros(F, dtype=torch.float64, device=U.device)
        lower = torch.zeros_like(upper)
        upper = upper.index_copy(0, self.single, neg - coeff)
        lower = lower.index_copy(0, self.single, -pos - coeff)
        diag = self._scatter(self.own_s, pos + coeff) + self._scatter(self.nei_s, -neg + coeff)
        fcov = torch.where(cov, 1.0 - f, torch.zeros_like(f))
        bsrc = f[:, None] * refv + (1.0 - f)[:, None] * dist_b[:, None] * refg
        bsrc = torch.where(cov[:, None], bsrc, torch.zeros_like(bsrc))
        diag = diag + self._scatter(self.bcell, phi_b * fcov)
        source = -self._scatter(self.bcell, phi_b[:, None] * bsrc)
        cond = self.nu * self.bmagsf
        cv = cond * vgc
        cg = torch.where(cov, cond * (1.0 - f), torch.zeros_like(f))
        diag = diag + self._scatter(self.bcell, cv)
        source = source + self._scatter(self.bcell, cv[:, None] * refv + cg[:, None] * refg)
        if self.H and self.u_corrected:
            # laplacian.py:162-176: the explicit skewness source on hanging
            # faces from the velocity's least-squares gradient
            gU = self.lsq_grad(U, psib, cov, dist_b)
            hp = self.hpos
            hsrc = (self.nu * self.magSf_s[hp])[:, None] * self._hang_sn(gU)
            source = source + self._scatter(self.own_s[hp], hsrc) - self._scatter(self.nei_s[hp], hsrc)
        # relaxation (fvmatrix relax): A/alpha, b + (1 - alpha)/alpha A U
        a = self.alpha_U
        source = source + ((1.0 - a) / a * diag)[:, None] * U
        diag = diag / a
        # predictor source b - V grad(p)
        pf, prefv, prefg, ppsib, pvgc, pcov = self.bc_state(self.pkind, self.pval, p2[self.bcell], phi_b, dist_b)
        gp = self.lsq_grad(p2, ppsib, pcov, dist_b)[:, 0, :]
        pred = source - V[:, None] * gp
        # velocity constraints at near immersed faces (their values: ref_v)
        ucells = self.u_cells
        uvals = refv[self.u_faces]
        d_c, up_c, lo_c, src_c = self._fixed(diag, upper, lower, pred, ucells, uvals)
        Us = self._solve(self.u_solver, algo.U, d_c, up_c, lo_c, src_c, U, symmetric=False)
        # constrained UEqn (relaxed source) for H/A with the solved velocity
        f2, refv2, _, _, _, _ = self.bc_state(self.ukind, self.uval, Us[self.bcell], phi_b, dist_b)
        d_h, up_h, lo_h, src_h = self._fixed(diag, upper, lower, source, ucells, refv2[self.u_faces])
        rAU = V / d_h
        HbyA = (src_h - self._off(up_h, lo_h, Us)) / d_h[:, None]
        h1 = -(self._scatter(self.own, up_h) + self._scatter(self.nei, lo_h)) / V
        # phiHbyA (flux.py:32-129): linear interpolation on single faces; the
        # boundary carries HbyA's cell value, U's value on non-assignable faces
        Hf = self.w_s[:, None] * HbyA[self.own_s] + (1.0 - self.w_s)[:, None] * HbyA[self.nei_s]
        if self.H:
            # fvc.interpolate(HbyA): HbyA carries no boundary conditions, so
            # its least-squares gradient has internal equations only
            none = torch.zeros(self.Nb, dtype=torch.bool, device=U.device)
            gH = self.lsq_grad(HbyA, torch.zeros_like(HbyA[self.bcell]), none, dist_b)
            Hf = Hf.index_add(0, self.hpos, self._hang_value(gH))
        phiH_s = (Hf * self.Sf_s).sum(1)
        _, _, _, Ub, _, _ = self.bc_state(self.ukind, self.uval, Us[self.bcell], phi_b, dist_b)
        flux_h = (HbyA[self.bcell] * self.bsf).sum(1)
        flux_h = torch.where(self.u_uncovered & ~self.is_imm_b, torch.zeros_like(flux_h), flux_h)
        flux_u = (Ub * self.bsf).sum(1)
        phiH_b = torch.where(self.u_fixed_flux, flux_u, flux_h)
        if self.consistent:
            # pressure_correction.py:163-267 (bounded SIMPLEC)
            inv = torch.maximum(1.0 / rAU - h1, 0.1 / rAU)
            rAtU = 1.0 / inv
            d_r = rAtU - rAU
            drf = self.w_s * d_r[self.own_s] + (1.0 - self.w_s) * d_r[self.nei_s]
            sn = self.delta_s * (p[self.nei_s] - p[self.own_s])
            if self.H:
                gp3 = self.lsq_grad(p2, ppsib, pcov, dist_b)
                sn = sn.index_add(0, self.hpos, self._hang_sn(gp3)[:, 0])
            phiH_s = phiH_s + drf * self.magSf_s * sn
            ng = pvgc * (prefv[:, 0] - p[self.bcell]) + (1.0 - pf) * prefg[:, 0]
            ng = torch.where(pcov, ng, torch.zeros_like(ng))
            phiH_b = phiH_b + d_r[self.bcell] * self.bmagsf * ng
            HbyA = HbyA - (rAU - rAtU)[:, None] * gp
        else:
            rAtU = rAU
        if trace is not None:
            phiH = torch.zeros(F + self.Nb, dtype=torch.float64, device=U.device).index_copy(0, self.single, phiH_s)
            trace.update(rAU=rAU, rAtU=rAtU, HbyA=HbyA, phiHbyA=torch.cat([phiH[:F], phiH_b]), U_star=Us)
        # pressure: -laplacian(rAtU, p) = -div(phiHbyA)   (pressure_correction.py:68-160)
        gam_f = self.w_s * rAtU[self.own_s] + (1.0 - self.w_s) * rAtU[self.nei_s]
        pc = gam_f * self.magSf_s * self.delta_s
        p_up = torch.zeros(F, dtype=torch.float64, device=U.device).index_copy(0, self.single, pc)
        p_diag = self._scatter(self.own_s, pc) + self._scatter(self.nei_s, pc)
        pcond = rAtU[self.bcell] * self.bmagsf
        pcv = pcond * pvgc
        pcg = torch.where(pcov, pcond * (1.0 - pf), torch.zeros_like(pf))
        p_diag = p_diag + self._scatter(self.bcell, pcv)
        p_src = self._scatter(self.bcell, pcv * prefv[:, 0] + pcg * prefg[:, 0])
        ffc = None
        if self.H and self.p_corrected:
            # the Laplacian's hanging skewness source from the pressure's
            # least-squares gradient, also the matrix's face-flux correction
            hp = self.hpos
            gpl = self.lsq_grad(p2, ppsib, pcov, dist_b)
            ffc = gam_f[hp] * self.magSf_s[hp] * self._hang_sn(gpl)[:, 0]
            p_src = p_src + self._scatter(self.own_s[hp], ffc) - self._scatter(self.nei_s[hp], ffc)
        div = self._scatter(self.own_s, phiH_s) - self._scatter(self.nei_s, phiH_s) + self._scatter(self.bcell, phiH_b)
        p_src = p_src - div
        p_new = self._solve(self.p_solver, algo.p, p_diag, -p_up, -p_up, p_src[:, None], p2, symmetric=True)[:, 0]
        # flux correction (pressure_correction.py:270-305)
        phi_s_new = phiH_s - pc * (p_new[self.nei_s] - p_new[self.own_s])
        if ffc is not None:
            phi_s_new = phi_s_new.index_add(0, self.hpos, -ffc)
        pf2, prefv2, prefg2, _, pvgc2, pcov2 = self.bc_state(self.pkind, self.pval, p_new[:, None][self.bcell], phi_b,
                                                             dist_b)
        ng2 = pvgc2 * (prefv2[:, 0] - p_new[self.bcell]) + (1.0 - pf2) * prefg2[:, 0]
        ng2 = torch.where(pcov2, ng2, torch.zeros_like(ng2))
        phi_b_new = phiH_b - rAtU[self.bcell] * self.bmagsf * ng2
        phi_new = torch.zeros(F + self.Nb, dtype=torch.float64, device=U.device)
        phi_new = phi_new.index_copy(0, self.single, phi_s_new)
        phi_new = torch.cat([phi_new[:F], phi_b_new])
        # pressure relaxation, velocity correction (pressure_correction.py:338-363)
        p_rel = p + self.alpha_p * (p_new - p)
        pf3, _, _, ppsib3, _, pcov3 = self.bc_state(self.pkind, self.pval, p_rel[:, None][self.bcell], phi_b, dist_b)
        gp3 = self.lsq_grad(p_rel[:, None], ppsib3, pcov3, dist_b)[:, 0, :]
        U_new = HbyA - rAtU[:, None] * gp3
        if ucells.numel():
            f4, refv4, _, _, _, _ = self.bc_state(self.ukind, self.uval, U_new[self.bcell], phi_new[F:], dist_b)
            U_new = U_new.index_copy(0, ucells, refv4[self.u_faces])
        return U_new, p_rel, phi_new

    # ------------------------------------------------------------------
    def state(self):
        a = self.algo
        return (a.U.data.detach().clone(), a.p.data.detach().clone(), a.phi.store[0].detach().clone())

    def distances(self) -> torch.Tensor:
        return self.bmagd[self.Fb:].clone()

    def check(self) -> dict:
        """Relative differences between this map and the library's SIMPLE
        step from the current state (the library step's solves stop at its
        own tolerances, so agreement is to those)."""
        U, p, phi = self.state()
        with torch.no_grad():
            U1, p1, phi1 = self.step(U, p, phi, self.distances())
        self.algo.step()
        U2, p2, phi2 = self.state()

        def rel(a, b):
            return float(torch.linalg.vector_norm(a - b) / max(float(torch.linalg.vector_norm(b)), 1e-300))

        return {"U": rel(U1, U2), "p": rel(p1, p2), "phi": rel(phi1, phi2)}


def drag_force(it: DifferentiableSimpleIteration, U, p, phi, dist, normals, patch: str, rho: float = 1.0,
               direction=(1.0, 0.0, 0.0)) -> torch.Tensor:
    """The force integral of ``gf_force_integral`` (post/forces/integration.py
    :125-187) on ``patch`` as device tensor algebra, projected on
    ``direction``: samples whose outward direction points into the body
    contribute ``rho p_b Sf - rho nu (dU/dn n + n dU/dn) Sf`` with
    ``dU/dn = (U_b - U_P) / (|d| n_hat . n_s)``."""
    g = it.grid
    F, Fb, Fi = it.F, it.Fb, it.Fi
    faces = torch.as_tensor(g.patch_faces(patch), device=U.device)
    faces = faces[faces >= Fb]
    dist_b = torch.cat([it.bmagd[:Fb], dist])
    phi_b = phi[F:]
    _, _, _, Ub, _, _ = it.bc_state(it.ukind, it.uval, U[it.bcell], phi_b, dist_b)
    _, _, _, pb, _, _ = it.bc_state(it.pkind, it.pval, p[:, None][it.bcell], phi_b, dist_b)
    uk = it.ukind[faces]
    pk = it.pkind[faces]
    cells = it.bcell[faces]
    Ub_f = torch.where((uk == it.codes["none"])[:, None], U[cells], Ub[faces])
    pb_f = torch.where(pk == it.codes["none"], p[cells], pb[faces, 0])
    anchor = (faces - Fb) % Fi
    sf = it.bsf[faces]
    nh = sf / it.bmagsf[faces][:, None]
    sb = -normals[anchor]
    align = (nh * sb).sum(1)
    keep = align.detach() > 0.0
    area = torch.sqrt((sb * sb).sum(1))
    ns = sb / area[:, None]
    nal = (nh * ns).sum(1)
    wall = dist_b[faces] * torch.clamp(nal, min=1e-12)
    dudn = (Ub_f - U[cells]) / wall[:, None]
    pforce = rho * pb_f[:, None] * sf
    sym = dudn[:, :, None] * ns[:, None, :] + dudn[:, None, :] * ns[:, :, None]
    vforce = -rho * it.nu * torch.einsum("nik,nk->ni", sym, sf)
    tot = torch.where(keep[:, None], pforce + vforce, torch.zeros_like(pforce))
    e = torch.as_tensor(direction, dtype=torch.float64, device=U.device)
    return (tot.sum(0) * e).sum()


# ----------------------------------------------------------------------
# geometry sensitivities (host)
# ----------------------------------------------------------------------
@dataclass
class ImmersedGeometry:
    """Crossing geometry of the immersed faces (grid order)."""

    p0: np.ndarray  # [Fi, 3] owner centres
    p1: np.ndarray  # [Fi, 3] neighbour centres
    t: np.ndarray  # [Fi] crossing parameter from the owner side
    seg: np.ndarray  # [Fi] |p1 - p0|


def immersed_geometry(grid) -> ImmersedGeometry:
    h = grid.host
    f = np.asarray(h.imm_faces)
    c = np.asarray(h.cell_centers)
    p0, p1 = c[h.owner[f]], c[h.neighbour[f]]
    seg = np.linalg.norm(p1 - p0, axis=1)
    t = np.asarray(h.ap_dist_owner) / seg
    return ImmersedGeometry(p0, p1, t, seg)


def _normals(sdf, pts: np.ndarray, h: float) -> np.ndarray:
    n = np.zeros_like(pts)
    for ax in range(3):
        e = np.zeros(3)
        e[ax] = h
        n[:, ax] = (sdf(pts + e) - sdf(pts - e)) / (2 * h)
    nrm = np.linalg.norm(n, axis=1)
    return n / np.where(nrm > 0, nrm, 1.0)[:, None]


def geometry_jacobian(grid, sdf_of, theta, *, extent: float, steps=None):
    """``(d dist / d theta [2 Fi, P], d normals / d theta [Fi, 3, P])`` of
    the immersed faces for the level set ``sdf_of(theta)``.

    Distances by implicit differentiation of the crossing; the builder's
    normal (central differences of the SDF, step ``1e-6 * extent``) at the
    moved crossing by central differences in ``theta`` (``steps``, default
    ``1e-6 max(1, |theta_j|)``)."""
    theta = np.asarray(theta, dtype=np.float64)
    P = theta.shape[0]
    geo = immersed_geometry(grid)
    sdf = sdf_of(theta)
    u = geo.p1 - geo.p0
    x = geo.p0 + geo.t[:, None] * u
    dt_ = 1e-7
    g_seg = (sdf(x + dt_ * u) - sdf(x - dt_ * u)) / (2 * dt_)
    hn = 1e-6 * extent
    Fi = x.shape[0]
    ddist = np.zeros((2 * Fi, P))
    dnorm = np.zeros((Fi, 3, P))
    for j in range(P):
        eps = (steps[j] if steps is not None else 1e-6 * max(1.0, abs(theta[j])))
        tp, tm = theta.copy(), theta.copy()
        tp[j] += eps
        tm[j] -= eps
        sp, sm = sdf_of(tp), sdf_of(tm)
        ds = (sp(x) - sm(x)) / (2 * eps)
        dtdth = -ds / np.where(g_seg != 0, g_seg, np.inf)
        ddist[:Fi, j] = geo.seg * dtdth
        ddist[Fi:, j] = -geo.seg * dtdth
        xp = x + (eps * dtdth)[:, None] * u
        xm = x - (eps * dtdth)[:, None] * u
        dnorm[:, :, j] = (_normals(sp, xp, hn) - _normals(sm, xm, hn)) / (2 * eps)
    return ddist, dnorm


# ----------------------------------------------------------------------
# the steady adjoint
# ----------------------------------------------------------------------
@dataclass
class ShapeGradient:
    objective: float
    grad: np.ndarray  # [P]
    grad_dist: np.ndarray  # [2 Fi]
    grad_normals: np.ndarray  # [Fi, 3]
    adjoint_sweeps: int
    adjoint_change: float
    map_check: dict


class exact_solves:
    """Context: ``algo``'s Krylov solves reduce their residual by ``rtol``
    with no absolute tolerance, instead of their configured tolerances.  A
    SIMPLE fixed point reached with the configured ones satisfies the
    discrete steady equations only to those tolerances (a solve whose
    initial residual is below its absolute tolerance returns at once), which
    is not sharp enough to difference; without an absolute tolerance every
    solve keeps reducing the residual, so the fixed point is the discrete
    solution (a relative reduction per solve is enough, and cheaper than
    solving each system to round-off; round-off-level tolerances also let
    the pressure CG wander in the body's enclosed cells, whose block of the
    system is singular)."""

    def __init__(self, algo, rtol: float = 1e-6):
        self.solvers = list(algo.solvers.values())
        self.rtol = rtol

    def __enter__(self):
        self.saved = [(s.atol, s.rtol, s.max_iter) for s in self.solvers]
        for s in self.solvers:
            s.atol, s.rtol, s.max_iter = 0.0, self.rtol, max(s.max_iter, 20000)
        return self

    def __exit__(self, *exc):
        for s, (a, r, m) in zip(self.solvers, self.saved):
            s.atol, s.rtol, s.max_iter = a, r, m
        return False


def converge(algo, *, tol: float = 1e-13, max_iterations: int = 20000, check_every: int = 20,
             cells: torch.Tensor | None = None) -> int:
    """Run SIMPLE iterations until the relative change of (U, p) over
    ``check_every`` iterations falls below ``tol`` (on ``cells`` only when
    given: cells enclosed by a body carry a pressure fixed only up to a
    constant); returns the iterations."""
    prev = None
    for k in range(1, max_iterations + 1):
        algo.step()
        if k % check_every == 0:
            U, p = algo.U.data, algo.p.data
            if cells is not None:
                U, p = U[cells], p[cells]
            cur = torch.cat([U.reshape(-1), p.reshape(-1)])
            if prev is not None:
                ch = float(torch.linalg.vector_norm(cur - prev) / torch.linalg.vector_norm(cur))
                if not math.isfinite(ch):
                    raise FloatingPointError("SIMPLE diverged")
                if ch < tol:
                    return k
            prev = cur.clone()
    return max_iterations


def converge_exact(algo, *, tol: float = 1e-12, cells: torch.Tensor | None = None, loose_tol: float = 1e-7,
                   max_iterations: int = 20000) -> tuple[int, int]:
    """SIMPLE with the configured solves until the state moves less than
    ``loose_tol``, then with exact solves (``exact_solves``) until it moves
    less than ``tol``; returns the iterations of both phases."""
    n1 = converge(algo, tol=loose_tol, cells=cells, max_iterations=max_iterations)
    with exact_solves(algo):
        n2 = converge(algo, tol=tol, cells=cells, max_iterations=max_iterations, check_every=5)
    return n1, n2


def shape_gradient(algo, sdf_of, theta, *, patch: str, extent: float, direction=(1.0, 0.0, 0.0),
                   scale: float = 1.0, tol: float = 1e-10, max_sweeps: int = 5000) -> ShapeGradient:
    """``d (scale * force . direction) / d theta`` at ``algo``'s (converged)
    steady state by the fixed-point adjoint (see the module doc)."""
    it = DifferentiableSimpleIteration(algo)
    g = algo.grid
    U0, p0, phi0 = it.state()
    dist0 = it.distances()
    nrm0 = torch.as_tensor(np.asarray(g.host.extra["anchor_normal"]), dtype=torch.float64, device=g.device)
    U = U0.clone().requires_grad_(True)
    p = p0.clone().requires_grad_(True)
    phi = phi0.clone().requires_grad_(True)
    dist = dist0.clone().requires_grad_(True)
    nrm = nrm0.clone().requires_grad_(True)
    J = scale * drag_force(it, U, p, phi, dist, nrm, patch, direction=direction)
    jU, jp, jphi, jd, jn = torch.autograd.grad(J, (U, p, phi, dist, nrm), allow_unused=True)
    zeros = (torch.zeros_like(U0), torch.zeros_like(p0), torch.zeros_like(phi0))
    jx = tuple(z if v is None else v for v, z in zip((jU, jp, jphi), zeros))
    jd = torch.zeros_like(dist0) if jd is None else jd
    jn = torch.zeros_like(nrm0) if jn is None else jn
    outs = it.step(U, p, phi, dist)
    mismatch = {"U": float(torch.linalg.vector_norm(outs[0].detach() - U0) / torch.linalg.vector_norm(U0)),
                "p": float(torch.linalg.vector_norm(outs[1].detach() - p0) / max(float(torch.linalg.vector_norm(p0)),
                                                                                 1e-300))}
    lam = jx
    change = float("inf")
    sweeps = 0
    for sweeps in range(1, max_sweeps + 1):
        vjp = torch.autograd.grad(outs, (U, p, phi), grad_outputs=lam, retain_graph=True, allow_unused=True)
        new = tuple(j + (torch.zeros_like(j) if v is None else v) for j, v in zip(jx, vjp))
        num = sum(float(torch.linalg.vector_norm(a - b) ** 2) for a, b in zip(new, lam))
        den = sum(float(torch.linalg.vector_norm(a) ** 2) for a in new)
        change = math.sqrt(num / max(den, 1e-300))
        lam = new
        if not math.isfinite(change):
            raise FloatingPointError("the adjoint iteration diverged")
        if change < tol:
            break
    (gd,) = torch.autograd.grad(outs, (dist,), grad_outputs=lam, allow_unused=True)
    gd = jd + (torch.zeros_like(jd) if gd is None else gd)
    ddist, dnorm = geometry_jacobian(g, sdf_of, theta, extent=extent)
    grad = gd.detach().cpu().numpy() @ ddist + np.einsum("ik,ikp->p", jn.detach().cpu().numpy(), dnorm)
    return ShapeGradient(float(J.detach()), grad, gd.detach().cpu().numpy(), jn.detach().cpu().numpy(), sweeps,
                         change, mismatch)
