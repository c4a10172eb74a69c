"""Reverse mode through PISO time steps, with time-step checkpointing.

The reference differentiates whole algorithm steps through torch autograd
(``solvers/adjoint/attach.py:21-115``; the step history of
``algorithms/piso.py:323-324``).  Here the forward run is the device
algorithm (``PISO.step``, library kernels, no autograd graph), and the
reverse sweep re-executes one step at a time in differentiable form from a
stored state:

* the assembly terms run the library kernels with their hand-written reverse
  kernels (``fvm.div`` with respect to the face flux, ``fvm.laplacian`` with
  respect to the per-cell diffusivity);
* the momentum and pressure solves run the device BiCGStab / CG with the
  implicit adjoint (a transpose solve on the GPU, ``solvers/adjoint.py``);
* the remaining algebra of the step (the Euler time derivative, the
  least-squares pressure gradient, H / A, the face interpolation, ddtCorr,
  the flux divergence, the flux and velocity corrections) is torch tensor
  algebra on the device, whose derivatives autograd forms.

``piso_gradient`` runs N steps, keeps the state ``(U, phi, p)`` every
``checkpoint_every`` steps, and in the reverse sweep recomputes each
segment's states from its checkpoint with the device algorithm before
differentiating its steps in reverse order; the memory held is the
checkpoints plus one segment's states plus one step's autograd graph.

Scope: uniform or octree-free grids without immersed faces (cell
constraints), Euler time derivative, upwind or linear convection, velocity
boundary conditions with no normal flow (Dirichlet walls and lids) and
zero-gradient pressure walls -- the closed lid-driven cavity in PISO form.
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import torch

from gridfoam_b200.core.equation import equation
from gridfoam_b200.core.field import FaceField
from gridfoam_b200.fv import fvm, schemes

_TINY = torch.finfo(torch.float64).tiny


def _check_supported(algo) -> None:
    from gridfoam_b200.algorithms.pressure_velocity import PISO

    g = algo.grid
    if not isinstance(algo, PISO):
        raise NotImplementedError("the step adjoint differentiates PISO steps")
    if g.num_hanging or g.num_immersed_faces:
        raise NotImplementedError("the step adjoint covers grids without hanging or immersed faces")
    sim = g.sim_config
    if schemes.ddt_coefficients(algo.U) != (1.0, 1.0, 0.0):
        raise NotImplementedError("the step adjoint covers the Euler time derivative")
    div = schemes.div_scheme(sim, algo.phi.name, algo.U.name).value
    if div not in ("upwind", "linear"):
        raise NotImplementedError("the step adjoint covers upwind and linear convection")
    if algo.n_non_orthogonal_correctors:
        raise NotImplementedError("the step adjoint covers nNonOrthogonalCorrectors 0")
    if not algo.p_needs_ref:
        raise NotImplementedError("the step adjoint covers zero-gradient pressure walls (closed domains)")
    if float(algo.phi.boundary_store.abs().max()) != 0.0:
        raise NotImplementedError("the step adjoint covers boundaries without normal flow")


class DifferentiablePisoStep:
    """One PISO step of ``algo``'s case as a differentiable function
    ``(U_old [C,3], phi [F+Nb], p_old [C], nu) -> (U, phi, p)``."""

    def __init__(self, algo):
        _check_supported(algo)
        self.algo = algo
        g = algo.grid
        self.grid = g
        d = g.dev
        self.own = d["owner"].long()
        self.nei = d["neighbour"].long()
        self.w = d["weight"]
        self.Sf = d["sf"].t().contiguous()
        self.V = g.cell_volumes
        self.dt = g.dt
        c = d["center"].t()
        self.d_int = (c[self.nei] - c[self.own]).contiguous()
        self.w2 = 1.0 / (self.d_int * self.d_int).sum(1)
        self.ata_inv = d["lsq_ata_inv"].t().reshape(-1, 3, 3)
        self.F = g.num_internal_faces
        self.C = g.num_cells
        self.phi_field = FaceField(g, "phi_step_adjoint", "local", (), export=False)
        self.ref_cell = algo.p_ref_cell
        self.ref_value = algo.p_ref_value
        sol = algo.solvers
        self.u_solver = sol[algo.U.name]
        self.p_solver = sol[algo.p.name]
        from gridfoam_b200.solvers.factory import resolve_solver

        self.p_final = resolve_solver(sol, algo.p.name, is_final=True)

    # ------------------------------------------------------------------
    def _lsq_grad(self, psi: torch.Tensor) -> torch.Tensor:
        """Least-squares gradient (fv/kernels/least_squares.py:29-101) of a
        cell scalar with zero-gradient boundaries: the boundary equations
        add nothing to the right-hand side."""
        t = (self.w2 * (psi[self.nei] - psi[self.own]))[:, None] * self.d_int
        atb = torch.zeros((self.C, 3), dtype=psi.dtype, device=psi.device)
        atb = atb.index_add(0, self.own, t).index_add(0, self.nei, t)
        return torch.einsum("cji,ci->cj", self.ata_inv, atb)

    def _face(self, x: torch.Tensor) -> torch.Tensor:
        """Linear interpolation to internal faces (w x_O + (1 - w) x_N)."""
        if x.dim() == 1:
            return self.w * x[self.own] + (1.0 - self.w) * x[self.nei]
        return self.w[:, None] * x[self.own] + (1.0 - self.w)[:, None] * x[self.nei]

    def step(self, U_old: torch.Tensor, phi: torch.Tensor, p_old: torch.Tensor, nu: torch.Tensor):
        algo, g = self.algo, self.grid
        own, nei, V, F = self.own, self.nei, self.V, self.F
        # momentum: ddt + div(phi, U) - laplacian(nu, U)   (piso.py:240-260)
        self.phi_field._store = phi.reshape(1, -1)
        with torch.no_grad():
            algo.U.store.copy_(U_old.detach().t())
            algo.p.store.copy_(p_old.detach().reshape(1, -1))
        nu_cells = nu * torch.ones(self.C, dtype=torch.float64, device=g.device)
        UEqn = fvm.div(self.phi_field, algo.U) - fvm.laplacian(nu_cells, algo.U)
        UEqn.diag = UEqn.diag + V / self.dt
        UEqn.source = UEqn.source + (V / self.dt)[:, None] * U_old
        # predictor: b - V grad(p)
        pred = UEqn.with_source(UEqn.source - V[:, None] * self._lsq_grad(p_old))
        U = self.u_solver.solve(equation(algo.U, pred)).solution
        diag, up, lo, src = UEqn.autograd_tensors()
        rAU = V / diag
        U0f = self._face(U_old)
        phi0 = phi[:F]
        corr = phi0 - (U0f * self.Sf).sum(1)
        coupling = 1.0 - torch.clamp(corr.abs() / (phi0.abs() + _TINY), max=1.0)
        ddt_corr = self._face(rAU) * coupling * corr / self.dt
        p = p_old
        n_corr = algo.n_correctors
        for i in range(n_corr):
            # HbyA = rAU H(U)   (fvmatrix.py:266-290)
            off = torch.zeros((self.C, 3), dtype=torch.float64, device=g.device)
            off = off.index_add(0, own, up[:, None] * U[nei]).index_add(0, nei, lo[:, None] * U[own])
            HbyA = rAU[:, None] * ((src - off) / V[:, None])
            phi_h = (self._face(HbyA) * self.Sf).sum(1) + ddt_corr
            # pressure: -laplacian(rAU, p) = -div(phiHbyA)   (pressure_correction.py:68-160)
            with torch.no_grad():
                algo.p.store.copy_(p.detach().reshape(1, -1))
            lap = fvm.laplacian(rAU, algo.p)
            pmat = -lap
            div_sum = torch.zeros(self.C, dtype=torch.float64, device=g.device)
            div_sum = div_sum.index_add(0, own, phi_h).index_add(0, nei, -phi_h)
            psrc = pmat.source - div_sum
            pdiag = pmat.diag
            if self.ref_cell is not None and self.ref_cell >= 0:
                # reference_value.py:33-51
                onehot = torch.zeros(self.C, dtype=torch.float64, device=g.device)
                onehot[self.ref_cell] = 1.0
                psrc = psrc + onehot * pdiag * self.ref_value
                pdiag = pdiag + onehot * pdiag
            pmat.diag = pdiag
            pmat.source = psrc
            solver = self.p_final if i == n_corr - 1 else self.p_solver
            p = solver.solve(equation(algo.p, pmat)).solution
            # phi = phiHbyA - flux(p); U = HbyA - rAU grad(p)   (pressure_correction.py:270-363)
            _, lup, llo, _ = lap.autograd_tensors()
            phi_int = phi_h - (lup * p[nei] - llo * p[own])
            U = HbyA - rAU[:, None] * self._lsq_grad(p)
        phi_new = torch.cat([phi_int, torch.zeros(phi.shape[0] - F, dtype=torch.float64, device=g.device)])
        return U, phi_new, p


@dataclass
class StepGradient:
    """Result of ``piso_gradient``: the objective, its derivative with
    respect to nu, and the checkpoint accounting (states held at most:
    ``peak_states`` states of ``3 C + F + Nb + C`` doubles each, plus one
    step's autograd graph)."""

    objective: float
    grad_nu: float
    steps: int
    checkpoints: int
    recomputed_steps: int
    peak_states: int


def _state(algo):
    return (algo.U.data.detach().clone(), algo.phi.store[0].detach().clone(), algo.p.data.detach().clone())


def _restore(algo, state) -> None:
    U, phi, p = state
    with torch.no_grad():
        algo.U.store.copy_(U.t())
        algo.phi.store[0].copy_(phi)
        algo.p.store.copy_(p.reshape(1, -1))
    algo.U.update_history(reset=True)
    algo.phi.update_history(reset=True)


def piso_gradient(algo, n_steps: int, objective, *, checkpoint_every: int | None = None) -> StepGradient:
    """``d objective(U_N) / d nu`` through ``n_steps`` PISO steps of ``algo``
    (its state on entry is step 0).  ``objective`` maps the final velocity
    ``[C, 3]`` to a scalar tensor.  States are kept every
    ``checkpoint_every`` steps (default: about sqrt(n_steps)) and each
    segment is recomputed with the device algorithm in the reverse sweep."""
    _check_supported(algo)
    k = checkpoint_every or max(1, int(math.isqrt(max(1, n_steps))))
    dstep = DifferentiablePisoStep(algo)
    nu0 = float(algo.nu)
    checkpoints = {0: _state(algo)}
    for n in range(n_steps):
        algo.step()
        if (n + 1) % k == 0 and n + 1 < n_steps:
            checkpoints[n + 1] = _state(algo)
    U_N = algo.U.data.detach().clone().requires_grad_(True)
    J = objective(U_N)
    (Ubar,) = torch.autograd.grad(J, U_N)
    adj = (Ubar, torch.zeros_like(checkpoints[0][1]), torch.zeros_like(checkpoints[0][2]))
    nu_bar = 0.0
    recomputed, peak = 0, 0
    for start in sorted(checkpoints, reverse=True):
        stop = min(start + k, n_steps)
        # recompute the segment's states with the device algorithm
        _restore(algo, checkpoints[start])
        states = [checkpoints[start]]
        for _ in range(start, stop - 1):
            algo.step()
            states.append(_state(algo))
            recomputed += 1
        peak = max(peak, len(checkpoints) + len(states))
        for s in reversed(states):
            _restore(algo, s)
            U_in = s[0].clone().requires_grad_(True)
            phi_in = s[1].clone().requires_grad_(True)
            p_in = s[2].clone().requires_grad_(True)
            nu_t = torch.tensor(nu0, dtype=torch.float64, device=U_in.device, requires_grad=True)
            outs = dstep.step(U_in, phi_in, p_in, nu_t)
            grads = torch.autograd.grad(outs, (U_in, phi_in, p_in, nu_t), grad_outputs=adj, allow_unused=True)
            adj = tuple(torch.zeros_like(x) if g_ is None else g_ for g_, x in zip(grads[:3], (U_in, phi_in, p_in)))
            nu_bar += 0.0 if grads[3] is None else float(grads[3])
    return StepGradient(float(J.detach()), nu_bar, n_steps, len(checkpoints), recomputed, peak)
