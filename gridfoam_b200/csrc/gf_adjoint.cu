// Hand-written adjoint (reverse-mode) kernels (sm_100a).
//
// * gf_adjoint_ldu_grads: gradients of x = A^-1 b with respect to the LDU
//   coefficients, from the adjoint lambda = A^-T xbar
//   (solvers/adjoint/ldu_grads.py:11-53).
// * gf_laplacian_adjoint: reverse of fvm.laplacian(gamma, psi) with respect
//   to the per-cell diffusivity gamma (fv/fvm/laplacian.py:101-201): the
//   face conductances, the hanging-face skewness source and the boundary
//   conductances each scatter their cotangents back to the cells.
// * gf_div_adjoint: reverse of fvm.div(phi, psi) with respect to the face
//   flux phi (the transpose of the face-flux -> coefficient map,
//   fv/fvm/div.py:15-73, fv/schemes/div.py upwind / linear / TVD).
//
// Per-cell results are gathers over the cell's ELL slots and per-face
// results are independent, so no kernel uses atomics and every result is
// bitwise reproducible.
#include "gf_common.cuh"

namespace gf {

static bool adj_valid(const gf_mesh_t* m, int nc, const char* what) {
    if (m == nullptr || m->n_cells <= 0 || m->ell_code == nullptr || m->ell_nbr == nullptr ||
        m->owner == nullptr || m->neighbour == nullptr || (nc != 1 && nc != 3)) {
        set_error("%s: invalid arguments", what);
        return false;
    }
    if (m->n_hang > 0 && (m->face_hang == nullptr || m->hang_move_o == nullptr || m->hang_move_n == nullptr)) {
        set_error("%s: hanging-face arrays missing", what);
        return false;
    }
    return true;
}

// grad_diag_c = -sum_k lambda_kc x_kc
__global__ void k_ldu_grad_diag(int64_t C, int nc, const double* __restrict__ lam, const double* __restrict__ x,
                                double* __restrict__ gd) {
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < C; c += (int64_t)gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int k = 0; k < nc; ++k) s += lam[k * C + c] * x[k * C + c];
        gd[c] = -s;
    }
}

// grad_upper_f = -sum_k lambda_kO x_kN, grad_lower_f = -sum_k lambda_kN x_kO
__global__ void k_ldu_grad_faces(gf_mesh_t m, int nc, const double* __restrict__ lam, const double* __restrict__ x,
                                 double* __restrict__ gu, double* __restrict__ gl) {
    const int64_t C = m.n_cells, F = m.n_faces;
    for (int64_t f = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; f < F; f += (int64_t)gridDim.x * blockDim.x) {
        const int o = __ldg(m.owner + f), n = __ldg(m.neighbour + f);
        double su = 0.0, sl = 0.0;
        for (int k = 0; k < nc; ++k) {
            su += lam[k * C + o] * x[k * C + n];
            sl += lam[k * C + n] * x[k * C + o];
        }
        gu[f] = -su;
        gl[f] = -sl;
    }
}

// d gamma_f / d gamma of the owner (side 0) or neighbour (side 1) cell.
// Linear: w, 1 - w.  Harmonic (fv/fvm/laplacian.py:38-73): the forward's
// min(go, gn) / (w go / s + (1 - w) gn / s), s = max(go, gn), equals
// go gn / D with D = w go + (1 - w) gn, so the derivatives are
// (1 - w) gn^2 / D^2 and w go^2 / D^2 (also at go = gn, where torch's
// min/max split the cotangent evenly and give the same values); with both
// zero the forward is min(go, gn) and each side gets half.
__device__ __forceinline__ double gamma_face_weight(const gf_assembly_t& a, double w, int o, int n, int side) {
    if (!a.lap_harmonic || a.gamma == nullptr) return side ? (1.0 - w) : w;
    const double go = a.gamma[o], gn = a.gamma[n];
    const double D = w * go + (1.0 - w) * gn;
    if (!(D > 0.0)) return 0.5;
    return side ? (w * go * go) / (D * D) : ((1.0 - w) * gn * gn) / (D * D);
}

// Reverse of the Laplacian assembly with respect to gamma (face
// interpolation gamma_f linear or harmonic, gamma_face_weight).  The cotangent of a
// face conductance is |Sf| delta (gu + gl - gd_O - gd_N) plus, on hanging
// faces, |Sf| sum_k corr_k (gs_kN - gs_kO); each cell gathers w (owner) or
// 1 - w (neighbour) of it, and its boundary conductances add
// |Sf_b| (-vgc gd_c - sum_k (vgc refv_k + (1 - f) refg_k) gs_kc).
__global__ void k_laplacian_adjoint(gf_mesh_t m, gf_assembly_t a, const double* __restrict__ gd,
                                    const double* __restrict__ gu, const double* __restrict__ gl,
                                    const double* __restrict__ gs, double* __restrict__ ggamma) {
    const int64_t C = m.n_cells, nb = m.n_bnd;
    const int W = m.ell_width;
    const int nc = a.ncomp;
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < C; c += (int64_t)gridDim.x * blockDim.x) {
        double acc = 0.0;
        for (int s = 0; s < W; ++s) {
            const int32_t code = __ldg(m.ell_code + s * C + c);
            const Slot sl = decode_slot(m, code);
            if (sl.kind == kInternal) {
                const int f = sl.face;
                const int nbr = __ldg(m.ell_nbr + s * C + c);
                const int o = sl.side ? nbr : (int)c;
                const int n = sl.side ? (int)c : nbr;
                const double w = __ldg(m.weight + f);
                const double msf = __ldg(m.mag_sf + f), dl = __ldg(m.delta + f);
                double gf = msf * dl * (gu[f] + gl[f] - gd[o] - gd[n]);
                const int h = hang_of(m, f);
                if (h >= 0 && a.lap_corrected && a.grad_lsq != nullptr) {
                    for (int k = 0; k < nc; ++k) {
                        const double corr = hang_sn_corr(m, a.grad_lsq, k, o, n, dl, h);
                        gf += msf * corr * (gs[k * C + n] - gs[k * C + o]);
                    }
                }
                acc += gamma_face_weight(a, w, o, n, sl.side) * gf;
            } else if (sl.kind == kBoundary) {
                const int b = sl.bnd;
                if (a.bc_kind[b] == GF_BC_NONE) continue;
                const double fr = a.frac[b];
                const double msf = __ldg(m.bnd_mag_sf + b);
                const double vg = value_grad_coeff(m, b, fr);
                double t = -vg * gd[c];
                for (int k = 0; k < nc; ++k)
                    t -= (vg * a.refv[k * nb + b] + (1.0 - fr) * a.refg[k * nb + b]) * gs[k * C + c];
                acc += msf * t;
            }
        }
        ggamma[c] = acc;
    }
}

// Reverse of the convection assembly with respect to the extended face flux
// [F internal | Nb boundary].  Upwind/TVD use torch.clamp's convention: the
// positive and negative parts both pass the cotangent at phi = 0.
__global__ void k_div_adjoint(gf_mesh_t m, gf_assembly_t a, const double* __restrict__ gd,
                              const double* __restrict__ gu, const double* __restrict__ gl,
                              const double* __restrict__ gs, double* __restrict__ gphi) {
    const int64_t C = m.n_cells, F = m.n_faces, nb = m.n_bnd;
    const int nc = a.ncomp;
    const bool tvd = a.div_scheme >= GF_DIV_VANLEER;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < F + nb;
         i += (int64_t)gridDim.x * blockDim.x) {
        if (i < F) {
            const int f = (int)i;
            if (m.imm_index && __ldg(m.imm_index + f) >= 0) {
                gphi[f] = 0.0;  // immersed faces act through their boundary sides
                continue;
            }
            const int o = __ldg(m.owner + f), n = __ldg(m.neighbour + f);
            const double w = __ldg(m.weight + f);
            const double flux = a.phi[f];
            double g;
            if (a.div_scheme == GF_DIV_LINEAR) {
                g = gu[f] * (1.0 - w) - gl[f] * w + gd[o] * w - gd[n] * (1.0 - w);
                const int h = hang_of(m, f);
                if (h >= 0 && a.grad_lsq != nullptr) {
                    for (int k = 0; k < nc; ++k) {
                        const double base = w * a.psi[k * C + o] + (1.0 - w) * a.psi[k * C + n];
                        const double corrected = base + hang_value_corr(m, a.grad_lsq, k, o, n, w, h);
                        g += -(corrected - base) * (gs[k * C + o] - gs[k * C + n]);
                    }
                }
            } else {
                const double dpos = flux >= 0.0 ? 1.0 : 0.0;  // d max(phi, 0)
                const double dneg = flux <= 0.0 ? 1.0 : 0.0;  // d min(phi, 0)
                g = gu[f] * dneg - gl[f] * dpos + gd[o] * dpos - gd[n] * dneg;
                if (tvd) {
                    // sf_k = -phi lim (plin_k - pup_k); lim and the upwind
                    // choice are constant in |phi|.
                    const bool up_o = flux > 0.0;
                    const int u = up_o ? o : n;
                    const double d0 = __ldg(m.center + n) - __ldg(m.center + o);
                    const double d1 = __ldg(m.center + C + n) - __ldg(m.center + C + o);
                    const double d2 = __ldg(m.center + 2 * C + n) - __ldg(m.center + 2 * C + o);
                    double gradf = 0.0, gradcf = 0.0;
                    double plin[3], pup[3];
                    const int h = hang_of(m, f);
                    for (int k = 0; k < nc; ++k) {
                        const double po = a.psi[k * C + o], pn = a.psi[k * C + n];
                        pup[k] = up_o ? po : pn;
                        plin[k] = w * po + (1.0 - w) * pn;
                        if (h >= 0) plin[k] = plin[k] + hang_value_corr(m, a.grad_psi, k, o, n, w, h);
                        const double dg = a.grad_psi[(k * 3 + 0) * C + u] * d0 +
                                          a.grad_psi[(k * 3 + 1) * C + u] * d1 +
                                          a.grad_psi[(k * 3 + 2) * C + u] * d2;
                        const double gv = pn - po;
                        if (nc == 1) {
                            gradf = gv;
                            gradcf = dg;
                        } else {
                            gradf += gv * gv;
                            gradcf += gv * dg;
                        }
                    }
                    const bool steep = fabs(gradcf) >= 1000.0 * fabs(gradf);
                    const double r = steep ? 2.0 * 1000.0 * sgn(gradcf) * sgn(gradf) - 1.0
                                           : 2.0 * gradcf / gradf - 1.0;
                    double lim;
                    switch (a.div_scheme) {
                        case GF_DIV_VANLEER: lim = (r + fabs(r)) / (1.0 + fabs(r)); break;
                        case GF_DIV_MINMOD: lim = fmax(fmin(1.0, r), 0.0); break;
                        case GF_DIV_SUPERBEE: lim = fmax(fmax(fmin(2.0 * r, 1.0), fmin(r, 2.0)), 0.0); break;
                        case GF_DIV_MC: lim = fmax(fmin(fmin(2.0 * r, 0.5 * r + 0.5), 2.0), 0.0); break;
                        case GF_DIV_LIMITEDLINEAR: lim = fmax(fmin(2.0 * r, 1.0), 0.0); break;
                        case GF_DIV_KOREN: lim = fmax(fmin(fmin(2.0 * r, (2.0 + r) / 3.0), 2.0), 0.0); break;
                        default: lim = 0.0;
                    }
                    for (int k = 0; k < nc; ++k) g += -lim * (plin[k] - pup[k]) * (gs[k * C + o] - gs[k * C + n]);
                }
            }
            gphi[f] = a.div_sign * g;
        } else {
            const int b = (int)(i - F);
            double g = 0.0;
            if (a.bc_kind[b] != GF_BC_NONE) {
                const int c = __ldg(m.bnd_cell + b);
                const double fr = a.frac[b];
                const double mag_d = __ldg(m.bnd_mag_d + b);
                g = gd[c] * (1.0 - fr);
                for (int k = 0; k < nc; ++k) {
                    const double bsrc = fr * a.refv[k * nb + b] + (1.0 - fr) * mag_d * a.refg[k * nb + b];
                    g -= bsrc * gs[k * C + c];
                }
            }
            gphi[i] = a.div_sign * g;
        }
    }
}

}  // namespace gf

using namespace gf;

extern "C" {

int gf_adjoint_ldu_grads(const gf_mesh_t* m, int32_t ncomp, const double* lambda, const double* x,
                         double* grad_diag, double* grad_upper, double* grad_lower, void* stream) {
    if (!adj_valid(m, ncomp, "gf_adjoint_ldu_grads") || lambda == nullptr || x == nullptr ||
        grad_diag == nullptr || grad_upper == nullptr || grad_lower == nullptr) {
        set_error("gf_adjoint_ldu_grads: invalid arguments");
        return GF_ERR_INVALID;
    }
    k_ldu_grad_diag<<<grid_for(m->n_cells), kThreads, 0, GF_STREAM(stream)>>>(m->n_cells, ncomp, lambda, x,
                                                                              grad_diag);
    if (m->n_faces > 0)
        k_ldu_grad_faces<<<grid_for(m->n_faces), kThreads, 0, GF_STREAM(stream)>>>(*m, ncomp, lambda, x, grad_upper,
                                                                                   grad_lower);
    return check_launch("gf_adjoint_ldu_grads");
}

int gf_laplacian_adjoint(const gf_mesh_t* m, const gf_assembly_t* a, const double* g_diag, const double* g_upper,
                         const double* g_lower, const double* g_source, double* g_gamma, void* stream) {
    if (a == nullptr || !adj_valid(m, a->ncomp, "gf_laplacian_adjoint") || a->bc_kind == nullptr ||
        a->frac == nullptr || a->refv == nullptr || a->refg == nullptr || g_diag == nullptr ||
        g_upper == nullptr || g_lower == nullptr || g_source == nullptr || g_gamma == nullptr) {
        set_error("gf_laplacian_adjoint: invalid arguments");
        return GF_ERR_INVALID;
    }
    k_laplacian_adjoint<<<grid_for(m->n_cells), kThreads, 0, GF_STREAM(stream)>>>(*m, *a, g_diag, g_upper, g_lower,
                                                                                  g_source, g_gamma);
    return check_launch("gf_laplacian_adjoint");
}

int gf_div_adjoint(const gf_mesh_t* m, const gf_assembly_t* a, const double* g_diag, const double* g_upper,
                   const double* g_lower, const double* g_source, double* g_phi, void* stream) {
    if (a == nullptr || !adj_valid(m, a->ncomp, "gf_div_adjoint") || a->phi == nullptr || a->psi == nullptr ||
        a->bc_kind == nullptr || a->frac == nullptr || a->refv == nullptr || a->refg == nullptr ||
        g_diag == nullptr || g_upper == nullptr || g_lower == nullptr || g_source == nullptr || g_phi == nullptr ||
        a->div_scheme == GF_DIV_NONE || (a->div_scheme >= GF_DIV_VANLEER && a->grad_psi == nullptr)) {
        set_error("gf_div_adjoint: invalid arguments");
        return GF_ERR_INVALID;
    }
    k_div_adjoint<<<grid_for(m->n_faces + m->n_bnd), kThreads, 0, GF_STREAM(stream)>>>(*m, *a, g_diag, g_upper,
                                                                                       g_lower, g_source, g_phi);
    return check_launch("gf_div_adjoint");
}

}  // extern "C"
