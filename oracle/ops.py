"""LDU matrix and finite-volume operators of the CPU oracle.

Restates (paths relative to the reference's ``src/gridfoam``):

* ``core/fvmatrix.py:16-468`` - LDU algebra, SpMV, H/H1/A, flux and the
  symmetric elimination of prescribed cells;
* ``fv/kernels/{face_interpolation,least_squares,gauss_gradient}.py``;
* ``fv/schemes/{div,grad,sn_grad,ddt,interpolate}.py``;
* ``fv/fvm/{laplacian,div,ddt}.py`` and ``fv/fvc/*.py``;
* ``fv/flux.py`` and ``fv/adjust_phi.py``.
"""

from __future__ import annotations

import numpy as np

from oracle.case import (
    DOMAIN_PATCHES,
    Case,
    CellField,
    DirichletBC,
    FaceField,
    InletOutletBC,
    boundary_batches,
    boundary_state,
    boundary_states,
    bview,
    fill_boundary_face_values,
    get_facefield,
    immersed_dirichlet_constraints,
    normal_gradient,
    scatter_add,
    uncovered_domain_faces,
    value_gradient_coefficient,
)


class LDU:
    """core/fvmatrix.py:16-468."""

    def __init__(self, field: CellField):
        case = field.case
        self.field = field
        self.case = case
        self.diag = np.zeros(case.num_cells)
        self.upper = np.zeros(case.num_internal_faces)
        self.lower = np.zeros(case.num_internal_faces)
        self.source = np.zeros((case.num_cells,) + field.comp)
        self.ffc: np.ndarray | None = None

    def copy(self) -> "LDU":
        m = LDU(self.field)
        m.diag, m.upper, m.lower = self.diag.copy(), self.upper.copy(), self.lower.copy()
        m.source = self.source.copy()
        m.ffc = None if self.ffc is None else self.ffc.copy()
        return m

    @staticmethod
    def _comb(a, b, sign):
        if a is None:
            return None if b is None else sign * b
        if b is None:
            return a.copy()
        return a + sign * b

    def __add__(self, o: "LDU") -> "LDU":
        m = LDU(self.field)
        m.diag, m.upper, m.lower = self.diag + o.diag, self.upper + o.upper, self.lower + o.lower
        m.source = self.source + o.source
        m.ffc = self._comb(self.ffc, o.ffc, 1.0)
        return m

    def __sub__(self, o: "LDU") -> "LDU":
        m = LDU(self.field)
        m.diag, m.upper, m.lower = self.diag - o.diag, self.upper - o.upper, self.lower - o.lower
        m.source = self.source - o.source
        m.ffc = self._comb(self.ffc, o.ffc, -1.0)
        return m

    def __neg__(self) -> "LDU":
        m = LDU(self.field)
        m.diag, m.upper, m.lower, m.source = -self.diag, -self.upper, -self.lower, -self.source
        m.ffc = None if self.ffc is None else -self.ffc
        return m

    def with_source(self, source: np.ndarray) -> "LDU":
        m = self.copy()
        m.source = source.copy()
        return m

    def A(self) -> np.ndarray:
        return self.diag / self.case.cell_volumes

    def H1(self) -> np.ndarray:
        c = self.case
        h1 = scatter_add(c.num_cells, c.owner, -self.upper) + scatter_add(
            c.num_cells, c.neighbour, -self.lower
        )
        return h1 / c.cell_volumes

    def multiply(self, x: np.ndarray) -> np.ndarray:
        """fvmatrix.py:292-323."""
        c = self.case
        xo, xn = x[c.owner], x[c.neighbour]
        res = bview(self.diag, x) * x
        res = res + scatter_add(c.num_cells, c.owner, bview(self.upper, xn) * xn)
        res = res + scatter_add(c.num_cells, c.neighbour, bview(self.lower, xo) * xo)
        return res

    def H(self, x: np.ndarray) -> np.ndarray:
        """fvmatrix.py:266-290."""
        return (self.source - self.multiply(x) + bview(self.diag, x) * x) / bview(
            self.case.cell_volumes, x
        )

    def with_fixed_values(self, cells: np.ndarray, values: np.ndarray) -> "LDU":
        """fvmatrix.py:325-394."""
        if cells.size == 0:
            return self
        c = self.case
        fixed = np.zeros(c.num_cells, dtype=bool)
        fixed[cells] = True
        prescribed = np.zeros_like(self.source)
        prescribed[cells] = values
        unit = -1.0 if self.diag.sum() < 0 else 1.0
        cdiag = np.where(self.diag != 0, self.diag, unit)
        m = LDU(self.field)
        m.diag = np.where(fixed, cdiag, self.diag)
        conn = fixed[c.owner] | fixed[c.neighbour]
        m.upper = np.where(conn, 0.0, self.upper)
        m.lower = np.where(conn, 0.0, self.lower)
        pn, po = prescribed[c.neighbour], prescribed[c.owner]
        src = self.source + scatter_add(c.num_cells, c.owner, -bview(self.upper, pn) * pn)
        src = src + scatter_add(c.num_cells, c.neighbour, -bview(self.lower, po) * po)
        src[cells] = bview(cdiag[cells], values) * values
        m.source = src
        return m

    def as_transpose(self) -> "LDU":
        m = LDU(self.field)
        m.diag, m.upper, m.lower, m.source, m.ffc = self.diag, self.lower, self.upper, self.source, self.ffc
        return m

    def flux(self, psi: np.ndarray) -> np.ndarray:
        """fvmatrix.py:424-468 (single-sided faces)."""
        c = self.case
        s = c.single_idx
        po, pn = psi[c.owner[s]], psi[c.neighbour[s]]
        out = bview(self.upper[s], pn) * pn - bview(self.lower[s], po) * po
        if self.ffc is not None:
            out = out + self.ffc
        return out


# ----------------------------------------------------------------------
# fv/kernels
# ----------------------------------------------------------------------
def linear_internal_face_values(field: CellField) -> np.ndarray:
    """face_interpolation.py:13-42."""
    c = field.case
    po, pn = field.data[c.owner_s], field.data[c.neighbour_s]
    w = bview(c.w_s, po)
    return w * po + (1.0 - w) * pn


def correct_internal_values(field: CellField, base: np.ndarray, grad: np.ndarray) -> np.ndarray:
    """face_interpolation.py:45-96."""
    c = field.case
    if c.num_hanging == 0:
        return base
    h = c.hang_idx
    go, gn = grad[c.owner_s[h]], grad[c.neighbour_s[h]]
    w = bview(c.w_s[h], go)
    gf = w * go + (1.0 - w) * gn
    corr = np.einsum("n...j,nj->n...", gf, c.hang_offset)
    out = base.copy()
    out[h] += corr
    return out


def sn_grad_hanging_correction(field: CellField, grad: np.ndarray) -> np.ndarray:
    """face_interpolation.py:99-145."""
    c = field.case
    h = c.hang_idx
    cn = np.einsum("n...j,nj->n...", grad[c.neighbour_s[h]], c.hang_move_N)
    co = np.einsum("n...j,nj->n...", grad[c.owner_s[h]], c.hang_move_O)
    diff = cn - co
    return bview(c.delta_coeffs_s[h], diff) * diff


def _accumulate_atb(atb, cells, d, dpsi):
    d2 = np.sum(d * d, axis=1)
    w2 = 1.0 / np.where(d2 > 0, d2, 1.0)
    atb += scatter_add(atb.shape[0], cells, np.einsum("n...,nj->n...j", dpsi, w2[:, None] * d))


def least_squares_gradient(field: CellField, *, hanging_cells_only: bool = False) -> np.ndarray:
    """least_squares.py:29-101."""
    c = field.case
    psi = field.data
    atb = np.zeros((c.num_cells,) + field.comp + (3,))
    if hanging_cells_only:
        own, nei = c.lsq_owner, c.lsq_neighbour
    else:
        own, nei = c.owner_s, c.neighbour_s
    d = c.cell_centers[nei] - c.cell_centers[own]
    dpsi = psi[nei] - psi[own]
    d2 = np.sum(d * d, axis=1)
    w2 = 1.0 / np.where(d2 > 0, d2, 1.0)
    atb_face = np.einsum("n...,nj->n...j", dpsi, w2[:, None] * d)
    atb += scatter_add(c.num_cells, own, atb_face)
    atb += scatter_add(c.num_cells, nei, atb_face)
    for b, _, _, _, psi_b in boundary_states(field):
        cells, d_b = b.target_cells, b.d_vec
        if hanging_cells_only:
            sel = c.hang_cell_mask[cells]
            if not sel.any():
                continue
            cells, d_b, psi_b = cells[sel], d_b[sel], psi_b[sel]
        _accumulate_atb(atb, cells, d_b, psi_b - psi[cells])
    return np.einsum("nij,n...j->n...i", c.lsq_ata_inv, atb)


def gauss_gradient(case: Case, psi_f: FaceField) -> np.ndarray:
    """gauss_gradient.py:15-73."""
    c = case
    g = np.zeros((c.num_cells,) + psi_f.comp + (3,))
    flux = np.einsum("n...,nj->n...j", psi_f.single_data, c.Sf_s)
    g += scatter_add(c.num_cells, c.owner_s, flux)
    g -= scatter_add(c.num_cells, c.neighbour_s, flux)
    g += scatter_add(
        c.num_cells, c.domain_bnd_owner,
        np.einsum("n...,nj->n...j", psi_f.domain_bnd_data, c.domain_bnd_Sf),
    )
    if c.num_immersed_faces > 0:
        imm = c.ap_is_immersed_faces
        iSf = c.Sf[imm]
        g += scatter_add(c.num_cells, c.owner[imm], np.einsum("n...,nj->n...j", psi_f.immersed_upper, iSf))
        g += scatter_add(c.num_cells, c.neighbour[imm], np.einsum("n...,nj->n...j", psi_f.immersed_lower, -iSf))
    return g / bview(c.cell_volumes, g)


# ----------------------------------------------------------------------
# schemes
# ----------------------------------------------------------------------
def interpolate_linear(field: CellField) -> FaceField:
    """schemes/interpolate.py:20-63 (``fvc.interpolate``)."""
    c = field.case
    psi_f = get_facefield(c, f"{field.name}_f", field.comp)
    base = linear_internal_face_values(field)
    fill_boundary_face_values(field, psi_f)
    if c.num_hanging > 0:
        grad_h = least_squares_gradient(field, hanging_cells_only=True)
        psi_f.single_data = correct_internal_values(field, base, grad_h)
    else:
        psi_f.single_data = base
    return psi_f


def eval_grad(field: CellField) -> np.ndarray:
    """schemes/grad.py:257-275."""
    scheme = field.case.scheme("gradSchemes", f"grad({field.name})", "leastsquare")
    if scheme == "linear":
        return gauss_gradient(field.case, interpolate_linear(field))
    return least_squares_gradient(field)


def grad(field: CellField) -> np.ndarray:
    """fvc/grad.py:8-34 (tensor only)."""
    return eval_grad(field)


LIMITERS = {
    "vanleer": lambda r: (r + np.abs(r)) / (1.0 + np.abs(r)),
    "minmod": lambda r: np.clip(np.minimum(1.0, r), 0.0, None),
    "superbee": lambda r: np.clip(np.maximum(np.minimum(2.0 * r, 1.0), np.minimum(r, 2.0)), 0.0, None),
    "monotonized_central": lambda r: np.clip(np.minimum(np.minimum(2.0 * r, 0.5 * r + 0.5), 2.0), 0.0, None),
    "limitedlinear": lambda r: np.clip(np.minimum(2.0 * r, 1.0), 0.0, None),
    "koren": lambda r: np.clip(np.minimum(np.minimum(2.0 * r, (2.0 + r) / 3.0), 2.0), 0.0, None),
}


def _div_upwind(phi: FaceField, field: CellField):
    """schemes/div.py:36-80."""
    pos = np.clip(phi.single_data, 0.0, None)
    neg = np.clip(phi.single_data, None, 0.0)
    src = np.zeros((phi.single_data.shape[0],) + field.comp)
    return neg, -pos, pos, -neg, src


def _div_linear(phi: FaceField, field: CellField):
    """schemes/div.py:83-139."""
    c = field.case
    w = c.w_s
    f = phi.single_data
    src = np.zeros((f.shape[0],) + field.comp)
    if c.num_hanging > 0:
        base = linear_internal_face_values(field)
        grad_h = least_squares_gradient(field, hanging_cells_only=True)
        corr = correct_internal_values(field, base, grad_h)
        src = -bview(f, base) * (corr - base)
    return f * (1.0 - w), -f * w, f * w, -f * (1.0 - w), src


def _div_tvd(phi: FaceField, field: CellField, limiter):
    """schemes/div.py:240-351."""
    c = field.case
    own, nei, w = c.owner_s, c.neighbour_s, c.w_s
    d_on = c.cell_centers[nei] - c.cell_centers[own]
    f = phi.single_data
    pos = np.clip(f, 0.0, None)
    neg = np.clip(f, None, 0.0)
    po, pn = field.data[own], field.data[nei]
    fmask = f > 0
    p_up = np.where(bview(fmask, po), po, pn)
    gt = eval_grad(field)
    wv = bview(w, po)
    base = wv * po + (1.0 - wv) * pn
    p_lin = correct_internal_values(field, base, gt)
    if field.comp == ():
        g_u = np.where(fmask[:, None], gt[own], gt[nei])
        gradcf = np.sum(g_u * d_on, axis=1)
        gradf = pn - po
    else:
        g_u = np.where(bview(fmask, gt[own]), gt[own], gt[nei])
        gv = pn - po
        gradf = np.sum((gv * gv).reshape(gv.shape[0], -1), axis=1)
        dg = np.einsum("n...j,nj->n...", g_u, d_on)
        gradcf = np.sum((gv * dg).reshape(gv.shape[0], -1), axis=1)
    steep = np.abs(gradcf) >= 1000.0 * np.abs(gradf)
    safe = np.where(steep, 1.0, gradf)
    r = np.where(steep, 2.0 * 1000.0 * np.sign(gradcf) * np.sign(gradf) - 1.0, 2.0 * gradcf / safe - 1.0)
    lim = limiter(r)
    src = -bview(f * lim, p_lin) * (p_lin - p_up)
    return neg, -pos, pos, -neg, src


def div_scheme_terms(phi: FaceField, field: CellField):
    scheme = field.case.scheme("divSchemes", f"div({phi.name}, {field.name})", "upwind")
    if scheme == "upwind":
        return _div_upwind(phi, field)
    if scheme == "linear":
        return _div_linear(phi, field)
    return _div_tvd(phi, field, LIMITERS[scheme])


def ddt_coefficients(field: CellField) -> tuple[float, float, float]:
    """schemes/ddt.py:13-58."""
    case = field.case
    dt = case.dt
    scheme = case.scheme("ddtSchemes", f"ddt({field.name})", "euler")
    if scheme == "euler":
        return 1.0, 1.0, 0.0
    if field.older_data is None:
        return 1.0, 1.0, 0.0
    dt0 = field.previous_dt
    ratio = dt / dt0
    a = 1.0 + dt / (dt + dt0)
    cc = ratio * dt / (dt + dt0)
    return a, a + cc, cc


# ----------------------------------------------------------------------
# fvm
# ----------------------------------------------------------------------
def fvm_ddt(field: CellField) -> LDU:
    """fvm/ddt.py:7-40."""
    case = field.case
    m = LDU(field)
    vdt = case.cell_volumes / case.dt
    a, b, cc = ddt_coefficients(field)
    m.diag = m.diag + a * vdt
    hist = b * field.old_data
    if cc != 0.0:
        hist = hist - cc * field.older_data
    m.source = m.source + bview(vdt, hist) * hist
    return m


def fvm_div(phi: FaceField, field: CellField) -> LDU:
    """fvm/div.py:15-73."""
    c = field.case
    m = LDU(field)
    upper, lower, dO, dN, src_f = div_scheme_terms(phi, field)
    m.upper[c.single_idx] = upper
    m.lower[c.single_idx] = lower
    m.diag += scatter_add(c.num_cells, c.owner_s, dO) + scatter_add(c.num_cells, c.neighbour_s, dN)
    m.source = m.source + scatter_add(c.num_cells, c.owner_s, src_f) - scatter_add(
        c.num_cells, c.neighbour_s, src_f
    )
    for b in boundary_batches(field):
        f, ref_v, ref_g, _ = boundary_state(field, b)
        fv = bview(f, ref_v)
        bsrc = fv * ref_v + (1.0 - fv) * bview(b.mag_d, ref_g) * ref_g
        flux = phi.block(b.kind)[b.face_mask]
        m.diag += scatter_add(c.num_cells, b.target_cells, flux * (1.0 - f))
        m.source = m.source - scatter_add(c.num_cells, b.target_cells, bview(flux, bsrc) * bsrc)
    return m


def _interpolate_gamma(case: Case, gamma, harmonic: bool):
    """fvm/laplacian.py:38-73."""
    if harmonic:
        g = np.asarray(gamma)
        if not np.all(np.isfinite(g) & (g >= 0)):
            raise ValueError("Harmonic diffusivity must be finite and nonnegative")
    if np.ndim(gamma) == 0:
        return float(gamma)
    go, gn = gamma[case.owner], gamma[case.neighbour]
    w = case.w_all
    if not harmonic:
        return w * go + (1.0 - w) * gn
    scale = np.maximum(go, gn)
    safe = np.where(scale > 0, scale, 1.0)
    den = w * (go / safe) + (1.0 - w) * (gn / safe)
    sden = np.where(den > 0, den, 1.0)
    return np.minimum(go, gn) / sden


LAPLACIAN_POLICY = {
    "corrected": (False, True),
    "uncorrected": (False, False),
    "linear": (False, True),
    "Gauss linear corrected": (False, True),
    "Gauss linear uncorrected": (False, False),
    "Gauss harmonic corrected": (True, True),
    "Gauss harmonic uncorrected": (True, False),
}


def fvm_laplacian(gamma, field: CellField) -> LDU:
    """fvm/laplacian.py:101-201."""
    c = field.case
    m = LDU(field)
    harmonic, corrected = LAPLACIAN_POLICY[
        c.scheme("laplacianSchemes", f"laplacian({field.name})", "corrected")
    ]
    gamma_f = _interpolate_gamma(c, gamma, harmonic)
    coeff = gamma_f * c.mag_Sf_all * c.delta_coeffs_all
    if c.num_immersed_faces > 0:
        coeff = np.where(c.ap_is_immersed_faces, 0.0, coeff)
    m.upper = coeff.copy()
    m.lower = coeff.copy()
    m.diag = m.diag - scatter_add(c.num_cells, c.owner, coeff) - scatter_add(c.num_cells, c.neighbour, coeff)
    if corrected and c.num_hanging > 0:
        grad_h = least_squares_gradient(field, hanging_cells_only=True)
        corr = sn_grad_hanging_correction(field, grad_h)
        hang_faces = c.single_idx[c.hang_idx]
        g_h = gamma_f[hang_faces] if np.ndim(gamma_f) else gamma_f
        src = bview(g_h * c.mag_Sf_s[c.hang_idx], corr) * corr
        h = c.hang_idx
        m.source = m.source - scatter_add(c.num_cells, c.owner_s[h], src) + scatter_add(
            c.num_cells, c.neighbour_s[h], src
        )
        m.ffc = scatter_add(c.num_single, h, src)
    for b in boundary_batches(field):
        f, ref_v, ref_g, _ = boundary_state(field, b)
        gb = gamma[b.target_cells] if np.ndim(gamma) else gamma
        cond = gb * b.mag_Sf
        cv = cond * value_gradient_coefficient(field, b, f)
        cg = cond * (1.0 - f)
        src = bview(cv, ref_v) * ref_v + bview(cg, ref_g) * ref_g
        m.diag = m.diag - scatter_add(c.num_cells, b.target_cells, cv)
        m.source = m.source - scatter_add(c.num_cells, b.target_cells, src)
    return m


# ----------------------------------------------------------------------
# fvc
# ----------------------------------------------------------------------
def fvc_div(phi: FaceField) -> np.ndarray:
    """fvc/div.py:15-64 (data only)."""
    c = phi.case
    data = scatter_add(c.num_cells, c.owner_s, phi.single_data) - scatter_add(
        c.num_cells, c.neighbour_s, phi.single_data
    )
    data = data + scatter_add(c.num_cells, c.domain_bnd_owner, phi.domain_bnd_data)
    if c.num_immersed_faces > 0:
        imm = c.ap_is_immersed_faces
        data = data + scatter_add(c.num_cells, c.owner[imm], phi.immersed_upper)
        data = data + scatter_add(c.num_cells, c.neighbour[imm], phi.immersed_lower)
    return data / bview(c.cell_volumes, data)


def sn_grad_single(field: CellField) -> np.ndarray:
    """schemes/sn_grad.py:82-154."""
    c = field.case
    diff = field.data[c.neighbour_s] - field.data[c.owner_s]
    base = bview(c.delta_coeffs_s, diff) * diff
    scheme = c.scheme("snGradSchemes", f"snGrad({field.name})", "corrected")
    if scheme == "uncorrected" or c.num_hanging == 0:
        return base
    grad_h = least_squares_gradient(field, hanging_cells_only=True)
    out = base.copy()
    out[c.hang_idx] += sn_grad_hanging_correction(field, grad_h)
    return out


def fvc_sn_grad(field: CellField) -> FaceField:
    """fvc/sn_grad.py:16-55."""
    c = field.case
    out = get_facefield(c, f"snGrad({field.name})", field.comp)
    out.single_data = sn_grad_single(field)
    for b, f, ref_v, ref_g, _ in boundary_states(field):
        out.block(b.kind)[b.face_mask] = normal_gradient(field, b, f, ref_v, ref_g)
    return out


def fvc_ddt_corr(U: CellField, phi: FaceField) -> np.ndarray:
    """fvc/ddt_corr.py:13-78."""
    c = U.case
    U0 = U.old_data
    U0f = c.w_s[:, None] * U0[c.owner_s] + (1.0 - c.w_s)[:, None] * U0[c.neighbour_s]
    phi0 = phi.old_single_data
    corr = phi0 - np.sum(U0f * c.Sf_s, axis=1)
    _, b, cc = ddt_coefficients(U)
    hist = b * corr
    if cc != 0.0:
        if phi.older_single_data is None or phi.previous_dt != U.previous_dt:
            raise ValueError("backward ddtCorr requires synchronized U and phi histories")
        U00 = U.older_data
        U00f = c.w_s[:, None] * U00[c.owner_s] + (1.0 - c.w_s)[:, None] * U00[c.neighbour_s]
        hist = hist - cc * (phi.older_single_data - np.sum(U00f * c.Sf_s, axis=1))
    eps = np.finfo(np.float64).tiny
    coupling = 1.0 - np.minimum(np.abs(corr) / (np.abs(phi0) + eps), 1.0)
    return coupling * hist / c.dt


# ----------------------------------------------------------------------
# fv/flux.py and fv/adjust_phi.py
# ----------------------------------------------------------------------
def flux_from_face_velocity(phi: FaceField, U_f: FaceField, U: CellField) -> None:
    """flux.py:32-71."""
    c = phi.case
    phi.single_data = np.sum(U_f.single_data * c.Sf_s, axis=1)
    dom = np.sum(U_f.domain_bnd_data * c.domain_bnd_Sf, axis=1)
    phi.domain_bnd_data = np.where(uncovered_domain_faces(U), 0.0, dom)
    if c.num_immersed_faces > 0:
        iSf = c.Sf[c.ap_is_immersed_faces]
        phi.immersed_upper = np.sum(U_f.immersed_upper * iSf, axis=1)
        phi.immersed_lower = np.sum(U_f.immersed_lower * (-iSf), axis=1)


def _constrain_hbya_boundary_flux(phi_hbya: FaceField, U: CellField) -> None:
    """flux.py:74-87."""
    for b, _, _, _, psi_b in boundary_states(U):
        if U.bcs[b.patch].assignable:
            continue
        phi_hbya.block(b.kind)[b.face_mask] = np.sum(psi_b * b.Sf, axis=1)


def compute_phi_hbya(phi_hbya: FaceField, HbyA: CellField, U: CellField, ddt_corr=None) -> None:
    """flux.py:90-129."""
    HbyA_f = interpolate_linear(HbyA)
    flux_from_face_velocity(phi_hbya, HbyA_f, U)
    if ddt_corr is not None:
        phi_hbya.single_data = phi_hbya.single_data + ddt_corr
    _constrain_hbya_boundary_flux(phi_hbya, U)


def correct_flux(phi: FaceField, U: CellField, update_internal: bool = False) -> None:
    """flux.py:132-162."""
    if update_internal:
        flux_from_face_velocity(phi, interpolate_linear(U), U)
    for b, _, _, _, psi_b in boundary_states(U):
        phi.block(b.kind)[b.face_mask] = np.sum(psi_b * b.Sf, axis=1)


def adjust_phi(phi: FaceField, U: CellField, p: CellField | None = None) -> bool:
    """adjust_phi.py:44-127."""
    if p is not None and any(isinstance(bc, DirichletBC) for bc in p.bcs.values()):
        return False
    c = phi.case

    def fixes(patch):
        bc = U.bcs.get(patch)
        if bc is None or isinstance(bc, InletOutletBC):
            return False
        return isinstance(bc, DirichletBC)

    mass_in = fixed_out = adj_out = 0.0
    for patch in U.bcs:
        if patch not in DOMAIN_PATCHES:
            continue
        mask = c.domain_bnd_mask(patch)
        if not mask.any():
            continue
        pp = phi.domain_bnd_data[mask]
        mass_in -= pp[pp < 0.0].sum()
        if fixes(patch):
            fixed_out += pp[pp > 0.0].sum()
        else:
            adj_out += pp[pp > 0.0].sum()
    if adj_out <= 0.0:
        return False
    corr = (mass_in - fixed_out) / adj_out
    for patch in U.bcs:
        if patch not in DOMAIN_PATCHES or fixes(patch):
            continue
        mask = c.domain_bnd_mask(patch)
        if not mask.any():
            continue
        pp = phi.domain_bnd_data[mask]
        out = pp > 0.0
        if out.any():
            phi.domain_bnd_data[mask] = np.where(out, pp * corr, pp)
    return True


def equation_matrix(field: CellField, mat: LDU) -> LDU:
    """core/equation.py:6-68."""
    cells, values = immersed_dirichlet_constraints(field)
    return mat.with_fixed_values(cells, values)
