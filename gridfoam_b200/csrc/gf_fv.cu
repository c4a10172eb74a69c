// Finite-volume operator kernels (sm_100a): boundary states, least-squares
// gradient, matrix assembly, fluxes, divergence and pressure-velocity
// corrections of gridfoam's SIMPLE/PISO/PIMPLE step.
//
// Every per-cell kernel is a single gather pass over the cell's ELL slots
// (internal faces, immersed face sides and domain faces alike), so results
// are written once, without atomics, and are bitwise reproducible.
#include "gf_common.cuh"

#include <mutex>

namespace gf {

static thread_local std::string g_last_error;

void set_error(const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
}

// ---------------------------------------------------------------------------
// Boundary states (fv/boundary_ops.py:311-326, boundaries/**)
// ---------------------------------------------------------------------------
__global__ void k_bc_state(gf_mesh_t m, gf_bc_t bc, const double* __restrict__ psi,
                           gf_bc_aux_t aux, gf_bc_state_t out) {
    const int64_t nb = m.n_bnd;
    const int64_t C = m.n_cells;
    for (int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; b < nb;
         b += (int64_t)gridDim.x * blockDim.x) {
        const int c = __ldg(m.bnd_cell + b);
        const int kind = bc.kind[b];
        const int nc = bc.ncomp;
        const double mag_d = __ldg(m.bnd_mag_d + b);
        double psiP[3], refv[3] = {0, 0, 0}, refg[3] = {0, 0, 0};
        for (int k = 0; k < nc; ++k) psiP[k] = psi[k * C + c];
        double frac = 0.0;
        switch (kind) {
            case GF_BC_DIRICHLET:
                frac = 1.0;
                for (int k = 0; k < nc; ++k) refv[k] = bc.value[k * nb + b];
                break;
            case GF_BC_NEUMANN:
                for (int k = 0; k < nc; ++k) refg[k] = bc.value[k * nb + b];
                break;
            case GF_BC_SLIP:
                if (nc == 3) {
                    frac = 1.0;
                    double n[3], normal = 0.0;
                    for (int k = 0; k < 3; ++k) {
                        n[k] = sgn(__ldg(m.bnd_sf + k * nb + b));
                        normal += psiP[k] * n[k];
                    }
                    for (int k = 0; k < 3; ++k) refv[k] = psiP[k] - normal * n[k];
                }
                break;
            case GF_BC_INLET_OUTLET:
                if (aux.phi_bnd != nullptr && aux.phi_bnd[b] < 0.0) {
                    frac = 1.0;
                    for (int k = 0; k < nc; ++k) refv[k] = bc.value[k * nb + b];
                }
                break;
            case GF_BC_FIXED_FLUX_P:
                if (aux.ffp_coeff != nullptr && aux.ffp_phi_pred != nullptr) {
                    const double mag_sf = __ldg(m.bnd_mag_sf + b);
                    double target = 0.0;
                    bool have_target = false;
                    if (aux.ffp_u_kind != nullptr && aux.ffp_u_kind[b] != GF_BC_NONE &&
                        aux.ffp_u_psib != nullptr) {
                        for (int k = 0; k < 3; ++k)
                            target += aux.ffp_u_psib[k * nb + b] * __ldg(m.bnd_sf + k * nb + b);
                        have_target = true;
                    } else if (aux.phi_bnd != nullptr) {
                        target = aux.phi_bnd[b];
                        have_target = true;
                    }
                    if (have_target) {
                        const double denom = aux.ffp_coeff[c] * mag_sf;
                        refg[0] = denom > 0.0 ? (aux.ffp_phi_pred[b] - target) / denom : 0.0;
                    }
                }
                break;
            default:
                break;
        }
        out.frac[b] = frac;
        for (int k = 0; k < nc; ++k) {
            out.refv[k * nb + b] = refv[k];
            out.refg[k * nb + b] = refg[k];
            out.psib[k * nb + b] =
                (kind == GF_BC_NONE) ? psiP[k]
                                     : frac * refv[k] + (1.0 - frac) * (psiP[k] + mag_d * refg[k]);
        }
    }
}

// ---------------------------------------------------------------------------
// Least-squares gradient (fv/kernels/least_squares.py:29-101)
// ---------------------------------------------------------------------------
template <int NC>
__global__ void k_lsq_grad(gf_mesh_t m, const double* __restrict__ psi,
                           const int8_t* __restrict__ kind, const double* __restrict__ psib,
                           double* __restrict__ grad) {
    const int64_t C = m.n_cells;
    const int64_t nb = m.n_bnd;
    const int W = m.ell_width;
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < C;
         c += (int64_t)gridDim.x * blockDim.x) {
        double atb[NC][3];
#pragma unroll
        for (int k = 0; k < NC; ++k) atb[k][0] = atb[k][1] = atb[k][2] = 0.0;
        const double cx = __ldg(m.center + c), cy = __ldg(m.center + C + c),
                     cz = __ldg(m.center + 2 * C + c);
        double pc[NC];
#pragma unroll
        for (int k = 0; k < NC; ++k) pc[k] = psi[k * C + c];
        for (int s = 0; s < W; ++s) {
            const int32_t code = __ldg(m.ell_code + s * C + c);
            const Slot sl = decode_slot(m, code);
            if (sl.kind == kInternal) {
                const int n = __ldg(m.ell_nbr + s * C + c);
                double d0 = __ldg(m.center + n) - cx, d1 = __ldg(m.center + C + n) - cy,
                       d2 = __ldg(m.center + 2 * C + n) - cz;
                if (sl.side == 1) {
                    d0 = -d0;
                    d1 = -d1;
                    d2 = -d2;
                }
                const double dd = d0 * d0 + d1 * d1 + d2 * d2;
                const double w2 = 1.0 / (dd > 0.0 ? dd : 1.0);
                const double wd0 = w2 * d0, wd1 = w2 * d1, wd2 = w2 * d2;
#pragma unroll
                for (int k = 0; k < NC; ++k) {
                    double dpsi = psi[k * C + n] - pc[k];
                    if (sl.side == 1) dpsi = -dpsi;
                    atb[k][0] += dpsi * wd0;
                    atb[k][1] += dpsi * wd1;
                    atb[k][2] += dpsi * wd2;
                }
            } else if (sl.kind == kBoundary) {
                const int b = sl.bnd;
                if (kind[b] == GF_BC_NONE) continue;
                const double d0 = __ldg(m.bnd_d + b), d1 = __ldg(m.bnd_d + nb + b),
                             d2 = __ldg(m.bnd_d + 2 * nb + b);
                const double dd = d0 * d0 + d1 * d1 + d2 * d2;
                const double w2 = 1.0 / (dd > 0.0 ? dd : 1.0);
                const double wd0 = w2 * d0, wd1 = w2 * d1, wd2 = w2 * d2;
#pragma unroll
                for (int k = 0; k < NC; ++k) {
                    const double dpsi = psib[k * nb + b] - pc[k];
                    atb[k][0] += dpsi * wd0;
                    atb[k][1] += dpsi * wd1;
                    atb[k][2] += dpsi * wd2;
                }
            }
        }
        double inv[9];
#pragma unroll
        for (int i = 0; i < 9; ++i) inv[i] = __ldg(m.lsq_ata_inv + i * C + c);
#pragma unroll
        for (int k = 0; k < NC; ++k) {
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                grad[(k * 3 + i) * C + c] =
                    inv[i * 3 + 0] * atb[k][0] + inv[i * 3 + 1] * atb[k][1] + inv[i * 3 + 2] * atb[k][2];
            }
        }
    }
}

// k_lsq_grad for six-slot rows: the slot codes and neighbours, then the
// immersed ordinals and the neighbours' centres and values (at the slot's
// own neighbour index, valid for every slot) are loaded for all six slots
// before any is used; the slots are then accumulated in order with the
// arithmetic of k_lsq_grad (same bits).  Boundary slots take its branch.
template <int NC>
__global__ void __launch_bounds__(256, 2) k_lsq_grad6(gf_mesh_t m, const double* __restrict__ psi,
                                                      const int8_t* __restrict__ kind,
                                                      const double* __restrict__ psib, double* __restrict__ grad) {
    constexpr int W = 6;
    const int64_t C = m.n_cells;
    const int64_t nb = m.n_bnd;
    const int F = (int)m.n_faces;
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < C;
         c += (int64_t)gridDim.x * blockDim.x) {
        int code[W], nbr[W], imm[W];
#pragma unroll
        for (int s = 0; s < W; ++s) {
            code[s] = __ldg(m.ell_code + s * C + c);
            nbr[s] = __ldg(m.ell_nbr + s * C + c);
        }
        double cn[W][3], pn[W][NC];
#pragma unroll
        for (int s = 0; s < W; ++s) {
            const int f = code[s] >> 1;
            const int fc = (code[s] >= 0 && f < F) ? f : 0;
            imm[s] = m.imm_index ? __ldg(m.imm_index + fc) : -1;
#pragma unroll
            for (int j = 0; j < 3; ++j) cn[s][j] = __ldg(m.center + j * C + nbr[s]);
#pragma unroll
            for (int k = 0; k < NC; ++k) pn[s][k] = psi[k * C + nbr[s]];
        }
        double atb[NC][3];
#pragma unroll
        for (int k = 0; k < NC; ++k) atb[k][0] = atb[k][1] = atb[k][2] = 0.0;
        const double cx = __ldg(m.center + c), cy = __ldg(m.center + C + c), cz = __ldg(m.center + 2 * C + c);
        double pc[NC];
#pragma unroll
        for (int k = 0; k < NC; ++k) pc[k] = psi[k * C + c];
#pragma unroll
        for (int s = 0; s < W; ++s) {
            const int f = code[s] >> 1;
            const int side = code[s] & 1;
            if (code[s] < 0) continue;
            if (f < F && imm[s] < 0) {
                double d0 = cn[s][0] - cx, d1 = cn[s][1] - cy, d2 = cn[s][2] - cz;
                if (side == 1) {
                    d0 = -d0;
                    d1 = -d1;
                    d2 = -d2;
                }
                const double dd = d0 * d0 + d1 * d1 + d2 * d2;
                const double w2 = 1.0 / (dd > 0.0 ? dd : 1.0);
                const double wd0 = w2 * d0, wd1 = w2 * d1, wd2 = w2 * d2;
#pragma unroll
                for (int k = 0; k < NC; ++k) {
                    double dpsi = pn[s][k] - pc[k];
                    if (side == 1) dpsi = -dpsi;
                    atb[k][0] += dpsi * wd0;
                    atb[k][1] += dpsi * wd1;
                    atb[k][2] += dpsi * wd2;
                }
            } else {
                const int b = f >= F ? f - F : (int)m.n_domain + (side ? (int)m.n_imm : 0) + imm[s];
                if (kind[b] == GF_BC_NONE) continue;
                const double d0 = __ldg(m.bnd_d + b), d1 = __ldg(m.bnd_d + nb + b),
                             d2 = __ldg(m.bnd_d + 2 * nb + b);
                const double dd = d0 * d0 + d1 * d1 + d2 * d2;
                const double w2 = 1.0 / (dd > 0.0 ? dd : 1.0);
                const double wd0 = w2 * d0, wd1 = w2 * d1, wd2 = w2 * d2;
#pragma unroll
                for (int k = 0; k < NC; ++k) {
                    const double dpsi = psib[k * nb + b] - pc[k];
                    atb[k][0] += dpsi * wd0;
                    atb[k][1] += dpsi * wd1;
                    atb[k][2] += dpsi * wd2;
                }
            }
        }
        double inv[9];
#pragma unroll
        for (int i = 0; i < 9; ++i) inv[i] = __ldg(m.lsq_ata_inv + i * C + c);
#pragma unroll
        for (int k = 0; k < NC; ++k) {
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                grad[(k * 3 + i) * C + c] =
                    inv[i * 3 + 0] * atb[k][0] + inv[i * 3 + 1] * atb[k][1] + inv[i * 3 + 2] * atb[k][2];
            }
        }
    }
}

// G ELL slots [s0, s0 + G) of row c for the least-squares gradient, staged
// as in k_lsq_grad6 (slot codes and neighbours, then immersed ordinals and
// the neighbours' centres and values, all before any is used; slots at or
// past W count as empty and load nothing), then accumulated into atb in slot
// order with the arithmetic of k_lsq_grad.
template <int NC, int G>
__device__ __forceinline__ void lsq_slots(const gf_mesh_t& m, int64_t c, int s0, int W,
                                           const double* __restrict__ psi, const int8_t* __restrict__ kind,
                                           const double* __restrict__ psib, const double (&cc)[3],
                                           const double (&pc)[NC], double (&atb)[NC][3]) {
    const int64_t C = m.n_cells;
    const int64_t nb = m.n_bnd;
    const int F = (int)m.n_faces;
    int code[G], nbr[G], imm[G];
#pragma unroll
    for (int s = 0; s < G; ++s) {
        const bool in = s0 + s < W;
        code[s] = in ? __ldg(m.ell_code + (s0 + s) * C + c) : -1;
        nbr[s] = in ? __ldg(m.ell_nbr + (s0 + s) * C + c) : (int)c;
    }
    double cn[G][3], pn[G][NC];
#pragma unroll
    for (int s = 0; s < G; ++s) {
        const int f = code[s] >> 1;
        const int fc = (code[s] >= 0 && f < F) ? f : 0;
        imm[s] = m.imm_index ? __ldg(m.imm_index + fc) : -1;
#pragma unroll
        for (int j = 0; j < 3; ++j) cn[s][j] = __ldg(m.center + j * C + nbr[s]);
#pragma unroll
        for (int k = 0; k < NC; ++k) pn[s][k] = psi[k * C + nbr[s]];
    }
#pragma unroll
    for (int s = 0; s < G; ++s) {
        const int f = code[s] >> 1;
        const int side = code[s] & 1;
        if (code[s] < 0) continue;
        if (f < F && imm[s] < 0) {
            double d0 = cn[s][0] - cc[0], d1 = cn[s][1] - cc[1], d2 = cn[s][2] - cc[2];
            if (side == 1) {
                d0 = -d0;
                d1 = -d1;
                d2 = -d2;
            }
            const double dd = d0 * d0 + d1 * d1 + d2 * d2;
            const double w2 = 1.0 / (dd > 0.0 ? dd : 1.0);
            const double wd0 = w2 * d0, wd1 = w2 * d1, wd2 = w2 * d2;
#pragma unroll
            for (int k = 0; k < NC; ++k) {
                double dpsi = pn[s][k] - pc[k];
                if (side == 1) dpsi = -dpsi;
                atb[k][0] += dpsi * wd0;
                atb[k][1] += dpsi * wd1;
                atb[k][2] += dpsi * wd2;
            }
        } else {
            const int b = f >= F ? f - F : (int)m.n_domain + (side ? (int)m.n_imm : 0) + imm[s];
            if (kind[b] == GF_BC_NONE) continue;
            const double d0 = __ldg(m.bnd_d + b), d1 = __ldg(m.bnd_d + nb + b), d2 = __ldg(m.bnd_d + 2 * nb + b);
            const double dd = d0 * d0 + d1 * d1 + d2 * d2;
            const double w2 = 1.0 / (dd > 0.0 ? dd : 1.0);
            const double wd0 = w2 * d0, wd1 = w2 * d1, wd2 = w2 * d2;
#pragma unroll
            for (int k = 0; k < NC; ++k) {
                const double dpsi = psib[k * nb + b] - pc[k];
                atb[k][0] += dpsi * wd0;
                atb[k][1] += dpsi * wd1;
                atb[k][2] += dpsi * wd2;
            }
        }
    }
}

// k_lsq_grad for octree rows (6 < W <= 12): a row's slots in staged groups
// of three (one component: 80 registers, three blocks an SM; three
// components: 110 registers, two blocks, and groups of six would spill), the
// groups from slot 6 on only where their first slot is used (cells with
// hanging faces; a row's used slots come first, and a row of the
// axis-projected grid holds at least six, one or more faces in each
// direction).  Same sums in the same order as k_lsq_grad (same bits); a row
// reads only its own slots instead of all W.
template <int NC>
__global__ void __launch_bounds__(256, NC == 1 ? 3 : 2) k_lsq_grad12(gf_mesh_t m, const double* __restrict__ psi,
                                                       const int8_t* __restrict__ kind,
                                                       const double* __restrict__ psib, double* __restrict__ grad) {
    const int64_t C = m.n_cells;
    const int W = m.ell_width;
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < C;
         c += (int64_t)gridDim.x * blockDim.x) {
        double atb[NC][3];
#pragma unroll
        for (int k = 0; k < NC; ++k) atb[k][0] = atb[k][1] = atb[k][2] = 0.0;
        const double cc[3] = {__ldg(m.center + c), __ldg(m.center + C + c), __ldg(m.center + 2 * C + c)};
        double pc[NC];
#pragma unroll
        for (int k = 0; k < NC; ++k) pc[k] = psi[k * C + c];
        constexpr int G = 3;
        for (int s0 = 0; s0 < W; s0 += G) {
            if (s0 >= 6 && __ldg(m.ell_code + s0 * C + c) < 0) break;
            lsq_slots<NC, G>(m, c, s0, W, psi, kind, psib, cc, pc, atb);
        }
        double inv[9];
#pragma unroll
        for (int i = 0; i < 9; ++i) inv[i] = __ldg(m.lsq_ata_inv + i * C + c);
#pragma unroll
        for (int k = 0; k < NC; ++k) {
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                grad[(k * 3 + i) * C + c] =
                    inv[i * 3 + 0] * atb[k][0] + inv[i * 3 + 1] * atb[k][1] + inv[i * 3 + 2] * atb[k][2];
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Matrix assembly: ddt + div_sign div(phi, psi) + lap_sign laplacian(gamma, psi)
// (fv/fvm/ddt.py:7-40, fv/fvm/div.py:15-73, fv/schemes/div.py:36-351,
//  fv/fvm/laplacian.py:38-201)
// ---------------------------------------------------------------------------
__device__ __forceinline__ double limiter(int scheme, double r) {
    switch (scheme) {
        case GF_DIV_VANLEER:
            return (r + fabs(r)) / (1.0 + fabs(r));
        case GF_DIV_MINMOD:
            return fmax(fmin(1.0, r), 0.0);
        case GF_DIV_SUPERBEE:
            return fmax(fmax(fmin(2.0 * r, 1.0), fmin(r, 2.0)), 0.0);
        case GF_DIV_MC:
            return fmax(fmin(fmin(2.0 * r, 0.5 * r + 0.5), 2.0), 0.0);
        case GF_DIV_LIMITEDLINEAR:
            return fmax(fmin(2.0 * r, 1.0), 0.0);
        case GF_DIV_KOREN:
            return fmax(fmin(fmin(2.0 * r, (2.0 + r) / 3.0), 2.0), 0.0);
        default:
            return 0.0;
    }
}

__device__ __forceinline__ double gamma_face(const gf_assembly_t& a, double w, int o, int n) {
    if (a.gamma == nullptr) return a.gamma_scalar;
    const double go = a.gamma[o], gn = a.gamma[n];
    if (!a.lap_harmonic) return w * go + (1.0 - w) * gn;
    const double scale = fmax(go, gn);
    const double safe = scale > 0.0 ? scale : 1.0;
    const double den = w * (go / safe) + (1.0 - w) * (gn / safe);
    return fmin(go, gn) / (den > 0.0 ? den : 1.0);
}

template <int NC>
__global__ void k_assemble(gf_mesh_t m, gf_assembly_t a) {
    const int64_t C = m.n_cells;
    const int64_t F = m.n_faces;
    const int64_t nb = m.n_bnd;
    const int W = m.ell_width;
    const bool conv = a.div_scheme != GF_DIV_NONE;
    const bool lap = a.lap_sign != 0.0;
    const bool tvd = a.div_scheme >= GF_DIV_VANLEER;
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < C;
         c += (int64_t)gridDim.x * blockDim.x) {
        double diag = 0.0;
        double src[NC];
#pragma unroll
        for (int k = 0; k < NC; ++k) src[k] = 0.0;
        if (a.use_ddt) {
            const double vdt = __ldg(m.volume + c) / a.dt;
            diag += a.ddt_a * vdt;
#pragma unroll
            for (int k = 0; k < NC; ++k) {
                double hist = a.ddt_b * a.psi_old[k * C + c];
                if (a.ddt_c != 0.0) hist = hist - a.ddt_c * a.psi_older[k * C + c];
                src[k] += vdt * hist;
            }
        }
        for (int s = 0; s < W; ++s) {
            const int32_t code = __ldg(m.ell_code + s * C + c);
            const Slot sl = decode_slot(m, code);
            double val = 0.0;
            if (sl.kind == kInternal) {
                const int f = sl.face;
                const int nbr = __ldg(m.ell_nbr + s * C + c);
                const int o = sl.side ? nbr : (int)c;
                const int n = sl.side ? (int)c : nbr;
                const double w = __ldg(m.weight + f);
                const int h = hang_of(m, f);
                if (conv) {
                    const double flux = a.phi[f];
                    double upper, lower, dO, dN;
                    if (a.div_scheme == GF_DIV_LINEAR) {
                        upper = flux * (1.0 - w);
                        lower = -flux * w;
                        dO = flux * w;
                        dN = -flux * (1.0 - w);
                    } else {
                        const double pos = fmax(flux, 0.0), neg = fmin(flux, 0.0);
                        upper = neg;
                        lower = -pos;
                        dO = pos;
                        dN = -neg;
                    }
                    if (sl.side == 0) {
                        val += a.div_sign * upper;
                        diag += a.div_sign * dO;
                    } else {
                        val += a.div_sign * lower;
                        diag += a.div_sign * dN;
                    }
                    if (a.div_scheme == GF_DIV_LINEAR && h >= 0 && a.grad_lsq != nullptr) {
                        // schemes/div.py:126-137: face-centre offset as an
                        // explicit deferred source.
#pragma unroll
                        for (int k = 0; k < NC; ++k) {
                            const double base = w * a.psi[k * C + o] + (1.0 - w) * a.psi[k * C + n];
                            const double corrected = base + hang_value_corr(m, a.grad_lsq, k, o, n, w, h);
                            const double sf = -flux * (corrected - base);
                            src[k] += (sl.side == 0 ? a.div_sign : -a.div_sign) * sf;
                        }
                    }
                    if (tvd) {
                        // schemes/div.py:240-351 deferred correction.
                        const bool up_o = flux > 0.0;
                        const int u = up_o ? o : n;
                        const double d0 = __ldg(m.center + n) - __ldg(m.center + o);
                        const double d1 = __ldg(m.center + C + n) - __ldg(m.center + C + o);
                        const double d2 = __ldg(m.center + 2 * C + n) - __ldg(m.center + 2 * C + o);
                        double gradf = 0.0, gradcf = 0.0;
                        double plin[NC], pup[NC];
#pragma unroll
                        for (int k = 0; k < NC; ++k) {
                            const double po = a.psi[k * C + o], pn = a.psi[k * C + n];
                            pup[k] = up_o ? po : pn;
                            plin[k] = w * po + (1.0 - w) * pn;
                            // schemes/div.py:300-305: hanging offset with the
                            // configured gradient.
                            if (h >= 0) plin[k] = plin[k] + hang_value_corr(m, a.grad_psi, k, o, n, w, h);
                            const double dg = a.grad_psi[(k * 3 + 0) * C + u] * d0 +
                                              a.grad_psi[(k * 3 + 1) * C + u] * d1 +
                                              a.grad_psi[(k * 3 + 2) * C + u] * d2;
                            const double gv = pn - po;
                            if (NC == 1) {
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
                        const double lim = limiter(a.div_scheme, r);
                        const double lf = flux * lim;
#pragma unroll
                        for (int k = 0; k < NC; ++k) {
                            const double sf = -lf * (plin[k] - pup[k]);
                            src[k] += (sl.side == 0 ? a.div_sign : -a.div_sign) * sf;
                        }
                    }
                }
                double ffc_k[NC];
#pragma unroll
                for (int k = 0; k < NC; ++k) ffc_k[k] = 0.0;
                if (lap) {
                    const double gf = gamma_face(a, w, o, n);
                    const double coeff = gf * __ldg(m.mag_sf + f) * __ldg(m.delta + f);
                    val += a.lap_sign * coeff;
                    diag += a.lap_sign * (-coeff);
                    if (h >= 0 && a.lap_corrected && a.grad_lsq != nullptr) {
                        // laplacian.py:162-176: explicit skewness source,
                        // owner -= corr, neighbour += corr.
#pragma unroll
                        for (int k = 0; k < NC; ++k) {
                            const double corr = hang_sn_corr(m, a.grad_lsq, k, o, n, __ldg(m.delta + f), h);
                            const double cs = (gf * __ldg(m.mag_sf + f)) * corr;
                            src[k] += a.lap_sign * (sl.side == 0 ? -cs : cs);
                            ffc_k[k] = cs;
                        }
                    }
                }
                if (a.ffc != nullptr && sl.side == 0) {
#pragma unroll
                    for (int k = 0; k < NC; ++k) a.ffc[k * F + f] = ffc_k[k];
                }
            } else if (sl.kind == kBoundary) {
                const int b = sl.bnd;
                if (a.bc_kind[b] != GF_BC_NONE) {
                    const double fr = a.frac[b];
                    const double mag_d = __ldg(m.bnd_mag_d + b);
                    if (conv) {
                        const double flux = a.phi[F + b];
                        diag += a.div_sign * (flux * (1.0 - fr));
#pragma unroll
                        for (int k = 0; k < NC; ++k) {
                            const double bsrc = fr * a.refv[k * nb + b] + (1.0 - fr) * mag_d * a.refg[k * nb + b];
                            src[k] += -a.div_sign * (flux * bsrc);
                        }
                    }
                    if (lap) {
                        const double g = a.gamma ? a.gamma[c] : a.gamma_scalar;
                        const double cond = g * __ldg(m.bnd_mag_sf + b);
                        const double cv = cond * value_grad_coeff(m, b, fr);
                        const double cg = cond * (1.0 - fr);
                        diag += a.lap_sign * (-cv);
#pragma unroll
                        for (int k = 0; k < NC; ++k) {
                            const double ls = cv * a.refv[k * nb + b] + cg * a.refg[k * nb + b];
                            src[k] += a.lap_sign * (-ls);
                        }
                    }
                }
            }
            a.val[s * C + c] = val;
        }
        a.diag[c] = diag;
#pragma unroll
        for (int k = 0; k < NC; ++k) a.source[k * C + c] = src[k];
    }
}

// k_assemble for the common case: six slots a row, no hanging faces, no
// TVD correction and no face-flux correction output.  The loads of all six
// slots are staged (slot codes and neighbours, then immersed ordinals, then
// the face data at clamped indices) before any of them is used, so a row's
// gathers are in flight together; the slots' contributions are then added
// in slot order with the arithmetic of k_assemble, so the matrix is the
// same bits.  Boundary slots (rare) take the branchy path of k_assemble.
// CONV / LAP: whether the convection / Laplacian term is assembled (fixed at
// compile time so a row's staged face data holds only what is used).
template <int NC, bool CONV, bool LAP>
__global__ void __launch_bounds__(256, 2) k_assemble6(gf_mesh_t m, gf_assembly_t a) {
    constexpr int W = 6;
    const int64_t C = m.n_cells;
    const int F = (int)m.n_faces;
    const int64_t nb = m.n_bnd;
    constexpr bool conv = CONV;
    constexpr bool lap = LAP;
    const bool linear = a.div_scheme == GF_DIV_LINEAR;
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < C;
         c += (int64_t)gridDim.x * blockDim.x) {
        int code[W], nbr[W], fc[W], imm[W];
#pragma unroll
        for (int s = 0; s < W; ++s) {
            code[s] = __ldg(m.ell_code + s * C + c);
            nbr[s] = __ldg(m.ell_nbr + s * C + c);
        }
#pragma unroll
        for (int s = 0; s < W; ++s) {
            const int f = code[s] >> 1;
            fc[s] = (code[s] >= 0 && f < F) ? f : 0;
            imm[s] = m.imm_index ? __ldg(m.imm_index + fc[s]) : -1;
        }
        double w[W], phi[W], msf[W], dl[W], go[W], gn[W];
#pragma unroll
        for (int s = 0; s < W; ++s) {
            const int side = code[s] & 1;
            const int o = side ? nbr[s] : (int)c;
            const int n = side ? (int)c : nbr[s];
            w[s] = __ldg(m.weight + fc[s]);
            if (CONV) phi[s] = __ldg(a.phi + fc[s]);
            if (LAP) {
                msf[s] = __ldg(m.mag_sf + fc[s]);
                dl[s] = __ldg(m.delta + fc[s]);
                go[s] = a.gamma ? __ldg(a.gamma + o) : 0.0;
                gn[s] = a.gamma ? __ldg(a.gamma + n) : 0.0;
            }
        }
        double diag = 0.0;
        double src[NC];
#pragma unroll
        for (int k = 0; k < NC; ++k) src[k] = 0.0;
        if (a.use_ddt) {
            const double vdt = __ldg(m.volume + c) / a.dt;
            diag += a.ddt_a * vdt;
#pragma unroll
            for (int k = 0; k < NC; ++k) {
                double hist = a.ddt_b * a.psi_old[k * C + c];
                if (a.ddt_c != 0.0) hist = hist - a.ddt_c * a.psi_older[k * C + c];
                src[k] += vdt * hist;
            }
        }
        double vals[W];
#pragma unroll
        for (int s = 0; s < W; ++s) {
            double val = 0.0;
            const int f = code[s] >> 1;
            const int side = code[s] & 1;
            const bool empty = code[s] < 0;
            const bool internal = !empty && f < F && imm[s] < 0;
            if (internal) {
                if (conv) {
                    const double flux = phi[s], ww = w[s];
                    double upper, lower, dO, dN;
                    if (linear) {
                        upper = flux * (1.0 - ww);
                        lower = -flux * ww;
                        dO = flux * ww;
                        dN = -flux * (1.0 - ww);
                    } else {
                        const double pos = fmax(flux, 0.0), neg = fmin(flux, 0.0);
                        upper = neg;
                        lower = -pos;
                        dO = pos;
                        dN = -neg;
                    }
                    if (side == 0) {
                        val += a.div_sign * upper;
                        diag += a.div_sign * dO;
                    } else {
                        val += a.div_sign * lower;
                        diag += a.div_sign * dN;
                    }
                }
                if (lap) {
                    double gf;
                    if (a.gamma == nullptr) {
                        gf = a.gamma_scalar;
                    } else if (!a.lap_harmonic) {
                        gf = w[s] * go[s] + (1.0 - w[s]) * gn[s];
                    } else {
                        const double scale = fmax(go[s], gn[s]);
                        const double safe = scale > 0.0 ? scale : 1.0;
                        const double den = w[s] * (go[s] / safe) + (1.0 - w[s]) * (gn[s] / safe);
                        gf = fmin(go[s], gn[s]) / (den > 0.0 ? den : 1.0);
                    }
                    const double coeff = gf * msf[s] * dl[s];
                    val += a.lap_sign * coeff;
                    diag += a.lap_sign * (-coeff);
                }
            } else if (!empty) {
                const int b = f >= F ? f - F : (int)m.n_domain + (side ? (int)m.n_imm : 0) + imm[s];
                if (a.bc_kind[b] != GF_BC_NONE) {
                    const double fr = a.frac[b];
                    const double mag_d = __ldg(m.bnd_mag_d + b);
                    if (conv) {
                        const double flux = a.phi[F + b];
                        diag += a.div_sign * (flux * (1.0 - fr));
#pragma unroll
                        for (int k = 0; k < NC; ++k) {
                            const double bsrc = fr * a.refv[k * nb + b] + (1.0 - fr) * mag_d * a.refg[k * nb + b];
                            src[k] += -a.div_sign * (flux * bsrc);
                        }
                    }
                    if (lap) {
                        const double g = a.gamma ? a.gamma[c] : a.gamma_scalar;
                        const double cond = g * __ldg(m.bnd_mag_sf + b);
                        const double cv = cond * value_grad_coeff(m, b, fr);
                        const double cg = cond * (1.0 - fr);
                        diag += a.lap_sign * (-cv);
#pragma unroll
                        for (int k = 0; k < NC; ++k) {
                            const double ls = cv * a.refv[k * nb + b] + cg * a.refg[k * nb + b];
                            src[k] += a.lap_sign * (-ls);
                        }
                    }
                }
            }
            vals[s] = val;
        }
#pragma unroll
        for (int s = 0; s < W; ++s) a.val[s * C + c] = vals[s];
        a.diag[c] = diag;
#pragma unroll
        for (int k = 0; k < NC; ++k) a.source[k * C + c] = src[k];
    }
}

// G ELL slots [s0, s0 + G) of row c for the assembly (no TVD scheme): the
// slot codes and neighbours, then the immersed and hanging ordinals, then
// the face data (at clamped indices) are loaded for all G before any is
// used; the contributions are then added to diag / src in slot order with
// the arithmetic of k_assemble, and the slots' coefficients (and face flux
// corrections) written.  Slots at or past W are skipped.
template <int NC, bool CONV, bool LAP, int G>
__device__ __forceinline__ void assemble_slots(const gf_mesh_t& m, const gf_assembly_t& a, int64_t c, int s0,
                                               int W, double& diag, double (&src)[NC]) {
    const int64_t C = m.n_cells;
    const int F = (int)m.n_faces;
    const int64_t nb = m.n_bnd;
    const bool linear = a.div_scheme == GF_DIV_LINEAR;
    int code[G], nbr[G], fc[G], imm[G], hg[G];
#pragma unroll
    for (int s = 0; s < G; ++s) {
        const bool in = s0 + s < W;
        code[s] = in ? __ldg(m.ell_code + (s0 + s) * C + c) : -1;
        nbr[s] = in ? __ldg(m.ell_nbr + (s0 + s) * C + c) : (int)c;
    }
#pragma unroll
    for (int s = 0; s < G; ++s) {
        const int f = code[s] >> 1;
        fc[s] = (code[s] >= 0 && f < F) ? f : 0;
        imm[s] = m.imm_index ? __ldg(m.imm_index + fc[s]) : -1;
        hg[s] = hang_of(m, fc[s]);
    }
    double w[G], phi[G], msf[G], dl[G], go[G], gn[G];
#pragma unroll
    for (int s = 0; s < G; ++s) {
        const int side = code[s] & 1;
        const int o = side ? nbr[s] : (int)c;
        const int n = side ? (int)c : nbr[s];
        w[s] = __ldg(m.weight + fc[s]);
        if (CONV) phi[s] = __ldg(a.phi + fc[s]);
        if (LAP) {
            msf[s] = __ldg(m.mag_sf + fc[s]);
            dl[s] = __ldg(m.delta + fc[s]);
            go[s] = a.gamma ? __ldg(a.gamma + o) : 0.0;
            gn[s] = a.gamma ? __ldg(a.gamma + n) : 0.0;
        }
    }
#pragma unroll
    for (int s = 0; s < G; ++s) {
        if (s0 + s >= W) break;
        double val = 0.0;
        const int f = code[s] >> 1;
        const int side = code[s] & 1;
        const bool empty = code[s] < 0;
        if (!empty && f < F && imm[s] < 0) {
            const int o = side ? nbr[s] : (int)c;
            const int n = side ? (int)c : nbr[s];
            const int h = hg[s];
            if (CONV) {
                const double flux = phi[s], ww = w[s];
                double upper, lower, dO, dN;
                if (linear) {
                    upper = flux * (1.0 - ww);
                    lower = -flux * ww;
                    dO = flux * ww;
                    dN = -flux * (1.0 - ww);
                } else {
                    const double pos = fmax(flux, 0.0), neg = fmin(flux, 0.0);
                    upper = neg;
                    lower = -pos;
                    dO = pos;
                    dN = -neg;
                }
                if (side == 0) {
                    val += a.div_sign * upper;
                    diag += a.div_sign * dO;
                } else {
                    val += a.div_sign * lower;
                    diag += a.div_sign * dN;
                }
                if (linear && h >= 0 && a.grad_lsq != nullptr) {
#pragma unroll
                    for (int k = 0; k < NC; ++k) {
                        const double base = ww * a.psi[k * C + o] + (1.0 - ww) * a.psi[k * C + n];
                        const double corrected = base + hang_value_corr(m, a.grad_lsq, k, o, n, ww, h);
                        const double sf = -flux * (corrected - base);
                        src[k] += (side == 0 ? a.div_sign : -a.div_sign) * sf;
                    }
                }
            }
            double ffc_k[NC];
#pragma unroll
            for (int k = 0; k < NC; ++k) ffc_k[k] = 0.0;
            if (LAP) {
                double gf;
                if (a.gamma == nullptr) {
                    gf = a.gamma_scalar;
                } else if (!a.lap_harmonic) {
                    gf = w[s] * go[s] + (1.0 - w[s]) * gn[s];
                } else {
                    const double scale = fmax(go[s], gn[s]);
                    const double safe = scale > 0.0 ? scale : 1.0;
                    const double den = w[s] * (go[s] / safe) + (1.0 - w[s]) * (gn[s] / safe);
                    gf = fmin(go[s], gn[s]) / (den > 0.0 ? den : 1.0);
                }
                const double coeff = gf * msf[s] * dl[s];
                val += a.lap_sign * coeff;
                diag += a.lap_sign * (-coeff);
                if (h >= 0 && a.lap_corrected && a.grad_lsq != nullptr) {
#pragma unroll
                    for (int k = 0; k < NC; ++k) {
                        const double corr = hang_sn_corr(m, a.grad_lsq, k, o, n, dl[s], h);
                        const double cs = (gf * msf[s]) * corr;
                        src[k] += a.lap_sign * (side == 0 ? -cs : cs);
                        ffc_k[k] = cs;
                    }
                }
            }
            if (a.ffc != nullptr && side == 0) {
#pragma unroll
                for (int k = 0; k < NC; ++k) a.ffc[k * (int64_t)F + f] = ffc_k[k];
            }
        } else if (!empty) {
            const int b = f >= F ? f - F : (int)m.n_domain + (side ? (int)m.n_imm : 0) + imm[s];
            if (a.bc_kind[b] != GF_BC_NONE) {
                const double fr = a.frac[b];
                const double mag_d = __ldg(m.bnd_mag_d + b);
                if (CONV) {
                    const double flux = a.phi[F + b];
                    diag += a.div_sign * (flux * (1.0 - fr));
#pragma unroll
                    for (int k = 0; k < NC; ++k) {
                        const double bsrc = fr * a.refv[k * nb + b] + (1.0 - fr) * mag_d * a.refg[k * nb + b];
                        src[k] += -a.div_sign * (flux * bsrc);
                    }
                }
                if (LAP) {
                    const double g = a.gamma ? a.gamma[c] : a.gamma_scalar;
                    const double cond = g * __ldg(m.bnd_mag_sf + b);
                    const double cv = cond * value_grad_coeff(m, b, fr);
                    const double cg = cond * (1.0 - fr);
                    diag += a.lap_sign * (-cv);
#pragma unroll
                    for (int k = 0; k < NC; ++k) {
                        const double ls = cv * a.refv[k * nb + b] + cg * a.refg[k * nb + b];
                        src[k] += a.lap_sign * (-ls);
                    }
                }
            }
        }
        a.val[(s0 + s) * C + c] = val;
    }
}

// k_assemble for octree rows (6 < W <= 12) and schemes without a TVD
// correction: a row's slots in staged groups of three (three slots' face
// data in registers at once; six spill), the groups from slot 6 on only
// where their first slot is used (cells with hanging faces; a row's used
// slots come first, and every row of the axis-projected grid has at least
// six), zeros written to the unused slots without reading them.  Same
// contributions in the same order as k_assemble (same bits).
template <int NC, bool CONV, bool LAP>
__global__ void __launch_bounds__(256, 2) k_assemble12(gf_mesh_t m, gf_assembly_t a) {
    const int64_t C = m.n_cells;
    const int W = m.ell_width;
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < C;
         c += (int64_t)gridDim.x * blockDim.x) {
        double diag = 0.0;
        double src[NC];
#pragma unroll
        for (int k = 0; k < NC; ++k) src[k] = 0.0;
        if (a.use_ddt) {
            const double vdt = __ldg(m.volume + c) / a.dt;
            diag += a.ddt_a * vdt;
#pragma unroll
            for (int k = 0; k < NC; ++k) {
                double hist = a.ddt_b * a.psi_old[k * C + c];
                if (a.ddt_c != 0.0) hist = hist - a.ddt_c * a.psi_older[k * C + c];
                src[k] += vdt * hist;
            }
        }
        constexpr int G = 3;
        for (int s0 = 0; s0 < W; s0 += G) {
            if (s0 >= 6 && __ldg(m.ell_code + s0 * C + c) < 0) {
                for (int s = s0; s < W; ++s) a.val[s * C + c] = 0.0;
                break;
            }
            assemble_slots<NC, CONV, LAP, G>(m, a, c, s0, W, diag, src);
        }
        a.diag[c] = diag;
#pragma unroll
        for (int k = 0; k < NC; ++k) a.source[k * C + c] = src[k];
    }
}

__global__ void k_momentum_finalize(int64_t C, int nc, double relax, const double* __restrict__ vol,
                                    const double* __restrict__ psi, const double* __restrict__ grad,
                                    double* __restrict__ diag, double* __restrict__ source,
                                    double* __restrict__ pred) {
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < C;
         c += (int64_t)gridDim.x * blockDim.x) {
        if (relax > 0.0) {
            const double a_old = diag[c];
            diag[c] = a_old / relax;
            const double rc = ((1.0 - relax) / relax) * a_old;
            for (int k = 0; k < nc; ++k) source[k * C + c] = source[k * C + c] + rc * psi[k * C + c];
        }
        if (pred != nullptr) {
            const double v = vol[c];
            for (int k = 0; k < nc; ++k)
                pred[k * C + c] = source[k * C + c] - (grad ? v * grad[k * C + c] : 0.0);
        }
    }
}

// Face sum of a face field for cell c (fv/fvc/div.py:33-64, before / V).
__device__ __forceinline__ double face_sum(const gf_mesh_t& m, int64_t c, const double* __restrict__ phi) {
    const int64_t C = m.n_cells;
    const int64_t F = m.n_faces;
    double sum = 0.0;
    for (int s = 0; s < m.ell_width; ++s) {
        const int32_t code = __ldg(m.ell_code + s * C + c);
        const Slot sl = decode_slot(m, code);
        if (sl.kind == kInternal) {
            const double v = phi[sl.face];
            sum += sl.side ? -v : v;
        } else if (sl.kind == kBoundary) {
            sum += phi[F + sl.bnd];
        }
    }
    return sum;
}

__global__ void k_pressure_finalize(gf_mesh_t m, const double* __restrict__ phi, double* __restrict__ diag,
                                    double* __restrict__ source, double* __restrict__ div_out,
                                    int64_t ref_cell, double ref_value) {
    const int64_t C = m.n_cells;
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < C;
         c += (int64_t)gridDim.x * blockDim.x) {
        const double v = __ldg(m.volume + c);
        const double div = face_sum(m, c, phi) / v;
        if (div_out) div_out[c] = div;
        double src = source[c] - div * v;
        if (c == ref_cell) {
            const double d = diag[c];
            diag[c] = d + d;
            src += d * ref_value;
        }
        source[c] = src;
    }
}

__global__ void k_fvc_div(gf_mesh_t m, int nc, const double* __restrict__ phi, double* __restrict__ out) {
    const int64_t C = m.n_cells;
    const int64_t rows = m.n_faces + m.n_bnd;
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < C;
         c += (int64_t)gridDim.x * blockDim.x) {
        const double v = __ldg(m.volume + c);
        for (int k = 0; k < nc; ++k) out[k * C + c] = face_sum(m, c, phi + k * rows) / v;
    }
}

// Green-Gauss gradient from face values (fv/kernels/gauss_gradient.py:15-73):
// grad(c) = sum over the faces of c of psi_f Sf (Sf outward from c) / V.
// psi_f is a face field in the extended layout [F | Nb] (fvc.interpolate);
// internal faces enter with +Sf on the owner side and -Sf on the neighbour
// side, boundary and immersed faces with their outward Sf.
template <int NC>
__global__ void k_gauss_grad(gf_mesh_t m, const double* __restrict__ psif, double* __restrict__ grad) {
    const int64_t C = m.n_cells;
    const int64_t F = m.n_faces;
    const int64_t Nb = m.n_bnd;
    const int64_t rows = F + Nb;
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < C;
         c += (int64_t)gridDim.x * blockDim.x) {
        double g[NC][3];
#pragma unroll
        for (int k = 0; k < NC; ++k) g[k][0] = g[k][1] = g[k][2] = 0.0;
        for (int s = 0; s < m.ell_width; ++s) {
            const Slot sl = decode_slot(m, __ldg(m.ell_code + s * C + c));
            double S[3];
            int64_t row;
            if (sl.kind == kInternal) {
                const double sign = sl.side ? -1.0 : 1.0;
#pragma unroll
                for (int j = 0; j < 3; ++j) S[j] = sign * __ldg(m.sf + j * F + sl.face);
                row = sl.face;
            } else if (sl.kind == kBoundary) {
#pragma unroll
                for (int j = 0; j < 3; ++j) S[j] = __ldg(m.bnd_sf + j * Nb + sl.bnd);
                row = F + sl.bnd;
            } else {
                continue;
            }
#pragma unroll
            for (int k = 0; k < NC; ++k) {
                const double v = psif[k * rows + row];
#pragma unroll
                for (int j = 0; j < 3; ++j) g[k][j] += v * S[j];
            }
        }
        const double vol = __ldg(m.volume + c);
#pragma unroll
        for (int k = 0; k < NC; ++k)
#pragma unroll
            for (int j = 0; j < 3; ++j) grad[(k * 3 + j) * C + c] = g[k][j] / vol;
    }
}

// ---------------------------------------------------------------------------
// Deterministic reductions (single pass of block partials + one final block)
// ---------------------------------------------------------------------------
constexpr int kReduceBlocks = 256;

__device__ __forceinline__ double block_sum(double v, double* sh) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    const int nw = blockDim.x >> 5;
    v = (threadIdx.x < nw) ? sh[threadIdx.x] : 0.0;
    if (warp == 0)
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;  // valid in thread 0
}

__global__ void k_diag_sum_partial(int64_t n, const double* __restrict__ x, double* __restrict__ part) {
    __shared__ double sh[32];
    double acc = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        acc += x[i];
    acc = block_sum(acc, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = acc;
}

__global__ void k_finish_sum(int nparts, const double* __restrict__ part, double* __restrict__ out) {
    __shared__ double sh[32];
    double acc = 0.0;
    for (int i = threadIdx.x; i < nparts; i += blockDim.x) acc += part[i];
    acc = block_sum(acc, sh);
    if (threadIdx.x == 0) out[0] = acc;
}

// ---------------------------------------------------------------------------
// with_fixed_values (core/fvmatrix.py:325-394)
// ---------------------------------------------------------------------------
template <int NC>
__global__ void k_fixed_values(gf_mesh_t m, const double* __restrict__ diag, const double* __restrict__ val,
                               const double* __restrict__ source, const uint8_t* __restrict__ fixed,
                               const double* __restrict__ prescribed, const double* __restrict__ diag_sum,
                               double* __restrict__ odiag, double* __restrict__ oval, double* __restrict__ osrc) {
    const int64_t C = m.n_cells;
    const int W = m.ell_width;
    const double unit = diag_sum[0] < 0.0 ? -1.0 : 1.0;
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < C;
         c += (int64_t)gridDim.x * blockDim.x) {
        const double d = diag[c];
        if (fixed[c]) {
            const double cd = d != 0.0 ? d : unit;
            odiag[c] = cd;
            for (int s = 0; s < W; ++s) oval[s * C + c] = 0.0;
#pragma unroll
            for (int k = 0; k < NC; ++k) osrc[k * C + c] = cd * prescribed[k * C + c];
            continue;
        }
        odiag[c] = d;
        double src[NC];
#pragma unroll
        for (int k = 0; k < NC; ++k) src[k] = source[k * C + c];
        for (int s = 0; s < W; ++s) {
            const int n = __ldg(m.ell_nbr + s * C + c);
            const double v = val[s * C + c];
            if (n != c && fixed[n]) {
#pragma unroll
                for (int k = 0; k < NC; ++k) src[k] += -v * prescribed[k * C + n];
                oval[s * C + c] = 0.0;
            } else {
                oval[s * C + c] = v;
            }
        }
#pragma unroll
        for (int k = 0; k < NC; ++k) osrc[k * C + c] = src[k];
    }
}

// ---------------------------------------------------------------------------
// SpMV, H / A / H1 (core/fvmatrix.py:242-323)
// ---------------------------------------------------------------------------
template <int NC>
__global__ void k_spmv(gf_mesh_t m, const double* __restrict__ diag, const double* __restrict__ val,
                       const double* __restrict__ x, double* __restrict__ y) {
    const int64_t C = m.n_cells;
    const int W = m.ell_width;
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < C;
         c += (int64_t)gridDim.x * blockDim.x) {
        const double d = diag[c];
        double acc[NC];
#pragma unroll
        for (int k = 0; k < NC; ++k) acc[k] = d * x[k * C + c];
        const int Wc = m.ell_len ? (int)__ldg(m.ell_len + c) : W;
        for (int s = 0; s < Wc; ++s) {
            const double v = val[s * C + c];
            const int n = __ldg(m.ell_nbr + s * C + c);
#pragma unroll
            for (int k = 0; k < NC; ++k) acc[k] += v * x[k * C + n];
        }
#pragma unroll
        for (int k = 0; k < NC; ++k) y[k * C + c] = acc[k];
    }
}

template <int NC>
__global__ void k_rau_hbya(gf_mesh_t m, const double* __restrict__ diag, const double* __restrict__ val,
                           const double* __restrict__ source, const double* __restrict__ psi,
                           double* __restrict__ rau, double* __restrict__ hbya, double* __restrict__ h1) {
    const int64_t C = m.n_cells;
    const int W = m.ell_width;
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < C;
         c += (int64_t)gridDim.x * blockDim.x) {
        const double d = diag[c];
        const double v = __ldg(m.volume + c);
        double off[NC];
        double hsum = 0.0;
#pragma unroll
        for (int k = 0; k < NC; ++k) off[k] = 0.0;
        const int Wc = m.ell_len ? (int)__ldg(m.ell_len + c) : W;
        for (int s = 0; s < Wc; ++s) {
            const double a = val[s * C + c];
            const int n = __ldg(m.ell_nbr + s * C + c);
            hsum += -a;
#pragma unroll
            for (int k = 0; k < NC; ++k) off[k] += a * psi[k * C + n];
        }
        const double r = 1.0 / (d / v);
        if (rau) rau[c] = r;
        if (h1) h1[c] = hsum / v;
        if (hbya) {
#pragma unroll
            for (int k = 0; k < NC; ++k) {
                const double x = psi[k * C + c];
                const double ax = d * x + off[k];
                hbya[k * C + c] = r * ((source[k * C + c] - ax + d * x) / v);
            }
        }
    }
}

__global__ void k_simplec_ratu(int64_t C, const double* __restrict__ rau, const double* __restrict__ h1,
                               double* __restrict__ ratu) {
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < C;
         c += (int64_t)gridDim.x * blockDim.x) {
        const double r = rau[c];
        double inv = 1.0 / r - h1[c];
        inv = fmax(inv, 0.1 / r);
        ratu[c] = 1.0 / inv;
    }
}

// ---------------------------------------------------------------------------
// Face fluxes (fv/flux.py:32-162, fv/fvc/ddt_corr.py:13-78)
// ---------------------------------------------------------------------------
// Rows first .. F + Nb of the extended face layout (first = F: boundary
// faces only, the internal ones done by k_face_flux_axis).
__global__ void k_face_flux(gf_mesh_t m, int mode, const double* __restrict__ vel,
                            const int8_t* __restrict__ u_kind, const double* __restrict__ u_psib,
                            gf_ddtcorr_t ddt, int has_ddt, const double* __restrict__ grad,
                            double* __restrict__ phi, int64_t first) {
    const int64_t C = m.n_cells;
    const int64_t F = m.n_faces;
    const int64_t nb = m.n_bnd;
    const int64_t total = F + nb;
    for (int64_t i = first + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
         i += (int64_t)gridDim.x * blockDim.x) {
        if (i < F) {
            const int f = (int)i;
            if (m.imm_index && __ldg(m.imm_index + f) >= 0) {
                phi[f] = 0.0;
                continue;
            }
            const int o = __ldg(m.owner + f), n = __ldg(m.neighbour + f);
            const double w = __ldg(m.weight + f);
            const int h = grad ? hang_of(m, f) : -1;
            // Sf has one non-zero component (the face axis) on this grid:
            // with face_axis only that component is read, and the products
            // of the two zero components (exact zeros) are not formed.
            const int ax = m.face_axis ? __ldg(m.face_axis + f) : -1;
            double flux = 0.0;
            double sf[3];
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const bool on = ax < 0 || k == ax;
                sf[k] = on ? __ldg(m.sf + k * F + f) : 0.0;
                if (on) {
                    double vf = w * vel[k * C + o] + (1.0 - w) * vel[k * C + n];
                    if (h >= 0) vf = vf + hang_value_corr(m, grad, k, o, n, w, h);
                    flux += vf * sf[k];
                }
            }
            if (has_ddt) {
                double u0f_sf = 0.0;
#pragma unroll
                for (int k = 0; k < 3; ++k)
                    if (ax < 0 || k == ax)
                        u0f_sf += (w * ddt.u_old[k * C + o] + (1.0 - w) * ddt.u_old[k * C + n]) * sf[k];
                const double phi0 = ddt.phi_old[f];
                const double corr = phi0 - u0f_sf;
                double hist = ddt.b * corr;
                if (ddt.c != 0.0) {
                    double u00f_sf = 0.0;
#pragma unroll
                    for (int k = 0; k < 3; ++k)
                        if (ax < 0 || k == ax)
                            u00f_sf += (w * ddt.u_older[k * C + o] + (1.0 - w) * ddt.u_older[k * C + n]) * sf[k];
                    hist = hist - ddt.c * (ddt.phi_older[f] - u00f_sf);
                }
                const double tiny = 2.2250738585072014e-308;
                const double coupling = 1.0 - fmin(fabs(corr) / (fabs(phi0) + tiny), 1.0);
                const double rau_f = w * ddt.rau[o] + (1.0 - w) * ddt.rau[n];
                flux = flux + rau_f * (coupling * hist / ddt.dt);
            }
            phi[f] = flux;
        } else {
            const int b = (int)(i - F);
            const int c = __ldg(m.bnd_cell + b);
            const int kind = u_kind[b];
            const bool domain = b < m.n_domain;
            double flux = 0.0;
            const bool use_bc = (mode == 0) ? (kind != GF_BC_NONE) : nonassignable(kind);
            if (kind == GF_BC_NONE && domain) {
                flux = 0.0;
            } else if (use_bc) {
                for (int k = 0; k < 3; ++k) flux += u_psib[k * nb + b] * __ldg(m.bnd_sf + k * nb + b);
            } else {
                for (int k = 0; k < 3; ++k) flux += vel[k * C + c] * __ldg(m.bnd_sf + k * nb + b);
            }
            phi[i] = flux;
        }
    }
}

// Internal faces of an axis-aligned grid without hanging faces
// (face_axis given, no gradient correction): the arithmetic of k_face_flux
// for the one non-zero Sf component, two faces per thread per pass with
// every load of both faces issued before the loads that depend on them
// (indices, then gathers), and no branch between the two levels.
template <bool DDT>
__global__ void __launch_bounds__(256, 3) k_face_flux_axis(gf_mesh_t m, const double* __restrict__ vel,
                                                        gf_ddtcorr_t ddt, double* __restrict__ phi) {
    constexpr int U = 2;
    const int64_t C = m.n_cells;
    const int F = (int)m.n_faces;
    const int stride = gridDim.x * blockDim.x;
    const bool older = DDT && ddt.c != 0.0;
    for (int f0 = blockIdx.x * blockDim.x + threadIdx.x; f0 < F; f0 += U * stride) {
        int f[U], o[U], n[U], ax[U], imm[U];
        double w[U], p0[U], p00[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            f[u] = f0 + u * stride;
            const int g = f[u] < F ? f[u] : f0;  // the tail re-reads face f0
            o[u] = __ldg(m.owner + g);
            n[u] = __ldg(m.neighbour + g);
            w[u] = __ldg(m.weight + g);
            ax[u] = __ldg(m.face_axis + g);
            imm[u] = m.imm_index ? __ldg(m.imm_index + g) : -1;
            if (DDT) {
                p0[u] = __ldg(ddt.phi_old + g);
                p00[u] = older ? __ldg(ddt.phi_older + g) : 0.0;
            }
        }
        double sfa[U], vo[U], vn[U], uo[U], un[U], uoo[U], unn[U], ro[U], rn[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int g = f[u] < F ? f[u] : f0;
            const int64_t kC = (int64_t)ax[u] * C;
            sfa[u] = __ldg(m.sf + (int64_t)ax[u] * F + g);
            vo[u] = __ldg(vel + kC + o[u]);
            vn[u] = __ldg(vel + kC + n[u]);
            if (DDT) {
                uo[u] = __ldg(ddt.u_old + kC + o[u]);
                un[u] = __ldg(ddt.u_old + kC + n[u]);
                ro[u] = __ldg(ddt.rau + o[u]);
                rn[u] = __ldg(ddt.rau + n[u]);
                if (older) {
                    uoo[u] = __ldg(ddt.u_older + kC + o[u]);
                    unn[u] = __ldg(ddt.u_older + kC + n[u]);
                }
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            if (f[u] >= F) continue;
            double flux = 0.0;
            const double vf = w[u] * vo[u] + (1.0 - w[u]) * vn[u];
            flux += vf * sfa[u];
            if (DDT) {
                double u0f_sf = 0.0;
                u0f_sf += (w[u] * uo[u] + (1.0 - w[u]) * un[u]) * sfa[u];
                const double corr = p0[u] - u0f_sf;
                double hist = ddt.b * corr;
                if (older) {
                    double u00f_sf = 0.0;
                    u00f_sf += (w[u] * uoo[u] + (1.0 - w[u]) * unn[u]) * sfa[u];
                    hist = hist - ddt.c * (p00[u] - u00f_sf);
                }
                const double tiny = 2.2250738585072014e-308;
                const double coupling = 1.0 - fmin(fabs(corr) / (fabs(p0[u]) + tiny), 1.0);
                const double rau_f = w[u] * ro[u] + (1.0 - w[u]) * rn[u];
                flux = flux + rau_f * (coupling * hist / ddt.dt);
            }
            phi[f[u]] = imm[u] >= 0 ? 0.0 : flux;
        }
    }
}

__global__ void k_interpolate(gf_mesh_t m, int nc, const double* __restrict__ psi,
                              const int8_t* __restrict__ kind, const double* __restrict__ psib,
                              const double* __restrict__ grad, double* __restrict__ out) {
    const int64_t C = m.n_cells;
    const int64_t F = m.n_faces;
    const int64_t nb = m.n_bnd;
    const int64_t total = F + nb;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
         i += (int64_t)gridDim.x * blockDim.x) {
        if (i < F) {
            const int f = (int)i;
            const bool imm = m.imm_index && __ldg(m.imm_index + f) >= 0;
            const int o = __ldg(m.owner + f), n = __ldg(m.neighbour + f);
            const double w = __ldg(m.weight + f);
            const int h = (grad && !imm) ? hang_of(m, f) : -1;
            for (int k = 0; k < nc; ++k) {
                double v = imm ? 0.0 : w * psi[k * C + o] + (1.0 - w) * psi[k * C + n];
                if (h >= 0) v = v + hang_value_corr(m, grad, k, o, n, w, h);
                out[k * total + f] = v;
            }
        } else {
            const int b = (int)(i - F);
            const int c = __ldg(m.bnd_cell + b);
            const bool cov = kind && kind[b] != GF_BC_NONE;
            for (int k = 0; k < nc; ++k) out[k * total + i] = cov ? psib[k * nb + b] : psi[k * C + c];
        }
    }
}

__global__ void k_sn_grad(gf_mesh_t m, int nc, const double* __restrict__ psi, const int8_t* __restrict__ kind,
                          const double* __restrict__ frac, const double* __restrict__ refv,
                          const double* __restrict__ refg, const double* __restrict__ grad,
                          double* __restrict__ out) {
    const int64_t C = m.n_cells;
    const int64_t F = m.n_faces;
    const int64_t nb = m.n_bnd;
    const int64_t total = F + nb;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
         i += (int64_t)gridDim.x * blockDim.x) {
        if (i < F) {
            const int f = (int)i;
            const bool imm = m.imm_index && __ldg(m.imm_index + f) >= 0;
            const int o = __ldg(m.owner + f), n = __ldg(m.neighbour + f);
            const double dc = __ldg(m.delta + f);
            const int h = (grad && !imm) ? hang_of(m, f) : -1;
            for (int k = 0; k < nc; ++k) {
                double v = imm ? 0.0 : dc * (psi[k * C + n] - psi[k * C + o]);
                if (h >= 0) v = v + hang_sn_corr(m, grad, k, o, n, dc, h);
                out[k * total + f] = v;
            }
        } else {
            const int b = (int)(i - F);
            const int c = __ldg(m.bnd_cell + b);
            if (kind[b] == GF_BC_NONE) {
                for (int k = 0; k < nc; ++k) out[k * total + i] = 0.0;
                continue;
            }
            const double fr = frac[b];
            const double vg = value_grad_coeff(m, b, fr);
            for (int k = 0; k < nc; ++k)
                out[k * total + i] = vg * (refv[k * nb + b] - psi[k * C + c]) + (1.0 - fr) * refg[k * nb + b];
        }
    }
}

// ---------------------------------------------------------------------------
// Pressure-velocity corrections (algorithms/utils/pressure_correction.py)
// ---------------------------------------------------------------------------
__global__ void k_correct_phi(gf_mesh_t m, const double* __restrict__ pred, const double* __restrict__ coeff,
                              const double* __restrict__ p, const int8_t* __restrict__ kind,
                              const double* __restrict__ frac, const double* __restrict__ refv,
                              const double* __restrict__ refg, double sign, int simplec,
                              const double* __restrict__ grad_p, const double* __restrict__ ffc,
                              double* __restrict__ phi) {
    const int64_t F = m.n_faces;
    const int64_t nb = m.n_bnd;
    const int64_t total = F + nb;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
         i += (int64_t)gridDim.x * blockDim.x) {
        const double base = pred[i];
        if (i < F) {
            const int f = (int)i;
            if (m.imm_index && __ldg(m.imm_index + f) >= 0) {
                phi[f] = base;
                continue;
            }
            const int o = __ldg(m.owner + f), n = __ldg(m.neighbour + f);
            const double w = __ldg(m.weight + f);
            const double cf = w * coeff[o] + (1.0 - w) * coeff[n];
            if (simplec) {
                double sn = __ldg(m.delta + f) * (p[n] - p[o]);
                const int h = grad_p ? hang_of(m, f) : -1;
                if (h >= 0) sn = sn + hang_sn_corr(m, grad_p, 0, o, n, __ldg(m.delta + f), h);
                phi[f] = base + cf * __ldg(m.mag_sf + f) * sn;
            } else {
                const double g = cf * __ldg(m.mag_sf + f) * __ldg(m.delta + f);
                double flux = g * p[n] - g * p[o];
                if (ffc) flux = flux + ffc[f];
                phi[f] = base - flux;
            }
        } else {
            const int b = (int)(i - F);
            double out = base;
            if (kind[b] != GF_BC_NONE) {
                const int c = __ldg(m.bnd_cell + b);
                const double fr = frac[b];
                const double sn = value_grad_coeff(m, b, fr) * (refv[b] - p[c]) + (1.0 - fr) * refg[b];
                out = base + sign * coeff[c] * __ldg(m.bnd_mag_sf + b) * sn;
            }
            phi[i] = out;
        }
    }
}

__global__ void k_fixed_imbalance(gf_mesh_t m, int64_t n, const int32_t* __restrict__ faces,
                                  const double* __restrict__ phi, double* __restrict__ imb) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int b = faces[i];
        const int c = __ldg(m.bnd_cell + b);
        const double v = __ldg(m.volume + c);
        imb[i] = (face_sum(m, c, phi) / v) * v;
    }
}

__global__ void k_fixed_apply(gf_mesh_t m, int64_t n, const int32_t* __restrict__ faces,
                              const double* __restrict__ area_frac, const double* __restrict__ imb,
                              double* __restrict__ phi) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t row = m.n_faces + faces[i];
        phi[row] = phi[row] - area_frac[i] * imb[i];
    }
}

__global__ void k_correct_velocity(int64_t C, const double* __restrict__ base, const double* __restrict__ coeff,
                                   const double* __restrict__ grad, double* __restrict__ out) {
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < C;
         c += (int64_t)gridDim.x * blockDim.x) {
        const double r = coeff[c];
        for (int k = 0; k < 3; ++k) out[k * C + c] = base[k * C + c] - r * grad[k * C + c];
    }
}

__global__ void k_set_cell_values(int64_t C, int nc, int64_t n, const int32_t* __restrict__ cells,
                                  const double* __restrict__ values, int64_t stride, double* __restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int c = cells[i];
        for (int k = 0; k < nc; ++k) out[k * C + c] = values[k * stride + i];
    }
}

__global__ void k_gather_bnd(int64_t nb, int nc, int64_t n, const int32_t* __restrict__ faces,
                             const double* __restrict__ refv, double* __restrict__ values) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int b = faces[i];
        for (int k = 0; k < nc; ++k) values[k * n + i] = refv[k * nb + b];
    }
}

// fv/adjust_phi.py:44-127 on one block: sums over domain faces, then scaling.
__global__ void k_adjust_phi(gf_mesh_t m, const int8_t* __restrict__ cls, double* __restrict__ phi) {
    __shared__ double sh[32];
    __shared__ double s_corr;
    __shared__ int s_do;
    const int64_t nb = m.n_domain;
    double* bphi = phi + m.n_faces;
    double in = 0.0, fixed_out = 0.0, adj_out = 0.0;
    for (int64_t b = threadIdx.x; b < nb; b += blockDim.x) {
        const int k = cls[b];
        if (k == 0) continue;
        const double v = bphi[b];
        if (v < 0.0) in -= v;
        if (v > 0.0) {
            if (k == 1) fixed_out += v;
            else adj_out += v;
        }
    }
    in = block_sum(in, sh);
    __syncthreads();
    fixed_out = block_sum(fixed_out, sh);
    __syncthreads();
    adj_out = block_sum(adj_out, sh);
    if (threadIdx.x == 0) {
        s_do = adj_out > 0.0;
        s_corr = s_do ? (in - fixed_out) / adj_out : 1.0;
    }
    __syncthreads();
    if (!s_do) return;
    const double corr = s_corr;
    for (int64_t b = threadIdx.x; b < nb; b += blockDim.x) {
        if (cls[b] != 2) continue;
        const double v = bphi[b];
        if (v > 0.0) bphi[b] = v * corr;
    }
}

__global__ void k_relax_field(int64_t n, double alpha, const double* __restrict__ old, double* __restrict__ cur) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        cur[i] = old[i] + alpha * (cur[i] - old[i]);
}

__global__ void k_axpby(int64_t n, double a, const double* __restrict__ x, double b, const double* __restrict__ y,
                        double* __restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = a * x[i] + b * y[i];
}

__global__ void k_ell_to_ldu(gf_mesh_t m, const double* __restrict__ val, double* __restrict__ upper,
                             double* __restrict__ lower) {
    for (int64_t f = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; f < m.n_faces;
         f += (int64_t)gridDim.x * blockDim.x) {
        upper[f] = val[__ldg(m.face_pos_owner + f)];
        lower[f] = val[__ldg(m.face_pos_neigh + f)];
    }
}

__global__ void k_ldu_to_ell(gf_mesh_t m, const double* __restrict__ upper, const double* __restrict__ lower,
                             double* __restrict__ val) {
    for (int64_t f = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; f < m.n_faces;
         f += (int64_t)gridDim.x * blockDim.x) {
        const bool imm = m.imm_index && __ldg(m.imm_index + f) >= 0;
        val[__ldg(m.face_pos_owner + f)] = imm ? 0.0 : upper[f];
        val[__ldg(m.face_pos_neigh + f)] = imm ? 0.0 : lower[f];
    }
}

template <int NC>
__global__ void k_residual_partial(gf_mesh_t m, const double* __restrict__ diag, const double* __restrict__ val,
                                   const double* __restrict__ source, const double* __restrict__ psi,
                                   double* __restrict__ part) {
    __shared__ double sh[32];
    const int64_t C = m.n_cells;
    const int W = m.ell_width;
    double rr = 0.0, bb = 0.0;
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < C;
         c += (int64_t)gridDim.x * blockDim.x) {
        const double d = diag[c];
        double acc[NC];
#pragma unroll
        for (int k = 0; k < NC; ++k) acc[k] = d * psi[k * C + c];
        const int Wc = m.ell_len ? (int)__ldg(m.ell_len + c) : W;
        for (int s = 0; s < Wc; ++s) {
            const double v = val[s * C + c];
            const int n = __ldg(m.ell_nbr + s * C + c);
#pragma unroll
            for (int k = 0; k < NC; ++k) acc[k] += v * psi[k * C + n];
        }
#pragma unroll
        for (int k = 0; k < NC; ++k) {
            const double b = source[k * C + c];
            const double r = acc[k] - b;
            rr += r * r;
            bb += b * b;
        }
    }
    rr = block_sum(rr, sh);
    __syncthreads();
    bb = block_sum(bb, sh);
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = rr;
        part[2 * blockIdx.x + 1] = bb;
    }
}

__global__ void k_residual_finish(int nparts, const double* __restrict__ part, double* __restrict__ out) {
    __shared__ double sh[32];
    double rr = 0.0, bb = 0.0;
    for (int i = threadIdx.x; i < nparts; i += blockDim.x) {
        rr += part[2 * i];
        bb += part[2 * i + 1];
    }
    rr = block_sum(rr, sh);
    __syncthreads();
    bb = block_sum(bb, sh);
    if (threadIdx.x == 0) out[0] = sqrt(rr) / (sqrt(bb) + 2.220446049250313e-16);
}

template <int NC>
__global__ void k_matrix_flux(gf_mesh_t m, const double* __restrict__ val, const double* __restrict__ psi,
                              const double* __restrict__ ffc, double* __restrict__ out) {
    const int64_t C = m.n_cells;
    const int64_t F = m.n_faces;
    for (int64_t f = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; f < F;
         f += (int64_t)gridDim.x * blockDim.x) {
        const bool imm = m.imm_index && __ldg(m.imm_index + f) >= 0;
        const double up = val[__ldg(m.face_pos_owner + f)];
        const double lo = val[__ldg(m.face_pos_neigh + f)];
        const int o = __ldg(m.owner + f), n = __ldg(m.neighbour + f);
#pragma unroll
        for (int k = 0; k < NC; ++k) {
            double v = imm ? 0.0 : up * psi[k * C + n] - lo * psi[k * C + o];
            if (ffc && !imm) v = v + ffc[k * F + f];
            out[k * F + f] = v;
        }
    }
}

// fv/fvc/reconstruct.py:28-117: U_c = (sum_f |Sf| n n^T)^-1 sum_f n phi_f over
// every face of the cell (both sides of internal faces with the same sign;
// boundary faces with their outward Sf).  Diagonal on axis-aligned grids.
__global__ void k_reconstruct(gf_mesh_t m, const double* __restrict__ phi, double* __restrict__ U) {
    const int64_t C = m.n_cells, F = m.n_faces, nb = m.n_bnd;
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < C; c += (int64_t)gridDim.x * blockDim.x) {
        double num[3] = {0.0, 0.0, 0.0}, den[3] = {0.0, 0.0, 0.0};
        for (int s = 0; s < m.ell_width; ++s) {
            const Slot sl = decode_slot(m, __ldg(m.ell_code + s * C + c));
            double sf[3], flux;
            if (sl.kind == kInternal) {
                for (int k = 0; k < 3; ++k) sf[k] = __ldg(m.sf + k * F + sl.face);
                flux = phi[sl.face];
            } else if (sl.kind == kBoundary) {
                for (int k = 0; k < 3; ++k) sf[k] = __ldg(m.bnd_sf + k * nb + sl.bnd);
                flux = phi[F + sl.bnd];
            } else {
                continue;
            }
            const double mag = sqrt(sf[0] * sf[0] + sf[1] * sf[1] + sf[2] * sf[2]);
            for (int k = 0; k < 3; ++k) {
                const double n = sf[k] / mag;
                num[k] += flux * n;
                den[k] += mag * n * n;
            }
        }
        for (int k = 0; k < 3; ++k) U[k * C + c] = num[k] / den[k];
    }
}

static bool valid_mesh(const gf_mesh_t* m) {
    if (m == nullptr || m->n_cells <= 0 || m->ell_width <= 0 || m->ell_code == nullptr ||
        m->ell_nbr == nullptr || m->volume == nullptr) {
        set_error("invalid mesh descriptor");
        return false;
    }
    if (m->n_cells * (int64_t)m->ell_width > 2147483647LL) {
        set_error("mesh too large for 32-bit ELL positions");
        return false;
    }
    if (m->n_hang < 0 || (m->n_hang > 0 && (m->face_hang == nullptr || m->hang_offset == nullptr ||
                                            m->hang_move_o == nullptr || m->hang_move_n == nullptr))) {
        set_error("invalid mesh descriptor: hanging-face arrays missing");
        return false;
    }
    return true;
}

static bool valid_nc(int nc) {
    if (nc != 1 && nc != 3) {
        set_error("ncomp must be 1 or 3, got %d", nc);
        return false;
    }
    return true;
}

}  // namespace gf

using namespace gf;


extern "C" {

const char* gf_last_error(void) { return g_last_error.c_str(); }

int gf_version(void) { return 1; }

int gf_bc_state(const gf_mesh_t* m, const gf_bc_t* bc, const double* psi, const gf_bc_aux_t* aux,
                gf_bc_state_t* out, void* stream) {
    if (!valid_mesh(m) || bc == nullptr || out == nullptr || psi == nullptr) {
        if (bc == nullptr || out == nullptr) set_error("gf_bc_state: null argument");
        return GF_ERR_INVALID;
    }
    if (!valid_nc(bc->ncomp)) return GF_ERR_INVALID;
    if (m->n_bnd == 0) return GF_OK;
    gf_bc_aux_t a = aux ? *aux : gf_bc_aux_t{nullptr, nullptr, nullptr, nullptr, nullptr};
    k_bc_state<<<grid_for(m->n_bnd), kThreads, 0, GF_STREAM(stream)>>>(*m, *bc, psi, a, *out);
    return check_launch("gf_bc_state");
}

int gf_lsq_grad(const gf_mesh_t* m, int32_t ncomp, const double* psi, const int8_t* bc_kind, const double* psib,
                double* grad, void* stream) {
    if (!valid_mesh(m) || !valid_nc(ncomp) || m->lsq_ata_inv == nullptr) return GF_ERR_INVALID;
    const unsigned g = grid_for(m->n_cells);
    cudaStream_t st = GF_STREAM(stream);
    const bool six = m->ell_width == 6 && m->n_faces < (int64_t)INT32_MAX;
    // Octree rows (6 < W <= 12, every row at least six slots): staged slots,
    // each row read to its last used slot.
    const bool twelve = m->ell_width > 6 && m->ell_width <= 12 && m->n_faces > 0 && m->n_faces < (int64_t)INT32_MAX;
    if (twelve) {
        if (ncomp == 1) k_lsq_grad12<1><<<g, kThreads, 0, st>>>(*m, psi, bc_kind, psib, grad);
        else k_lsq_grad12<3><<<g, kThreads, 0, st>>>(*m, psi, bc_kind, psib, grad);
        return check_launch("gf_lsq_grad");
    }
    // One component: the per-slot kernel is as fast (fewer registers).
    if (ncomp == 1) {
        k_lsq_grad<1><<<g, kThreads, 0, st>>>(*m, psi, bc_kind, psib, grad);
    } else {
        if (six)
            k_lsq_grad6<3><<<g, kThreads, 0, st>>>(*m, psi, bc_kind, psib, grad);
        else
            k_lsq_grad<3><<<g, kThreads, 0, st>>>(*m, psi, bc_kind, psib, grad);
    }
    return check_launch("gf_lsq_grad");
}

int gf_assemble(const gf_mesh_t* m, const gf_assembly_t* a, void* stream) {
    if (!valid_mesh(m) || a == nullptr || !valid_nc(a->ncomp)) return GF_ERR_INVALID;
    if (a->diag == nullptr || a->val == nullptr || a->source == nullptr) {
        set_error("gf_assemble: null output");
        return GF_ERR_INVALID;
    }
    if (a->div_scheme < GF_DIV_NONE || a->div_scheme > GF_DIV_KOREN) {
        set_error("gf_assemble: unknown div scheme %d", a->div_scheme);
        return GF_ERR_INVALID;
    }
    if (a->div_scheme >= GF_DIV_VANLEER && (a->grad_psi == nullptr || a->psi == nullptr)) {
        set_error("gf_assemble: TVD scheme needs psi and grad_psi");
        return GF_ERR_INVALID;
    }
    if (a->use_ddt && (a->psi_old == nullptr || a->dt <= 0.0 || (a->ddt_c != 0.0 && a->psi_older == nullptr))) {
        set_error("gf_assemble: ddt term needs history and dt > 0");
        return GF_ERR_INVALID;
    }
    const bool fast = m->ell_width == 6 && m->n_hang == 0 && a->ffc == nullptr &&
                      a->div_scheme <= GF_DIV_LINEAR && m->n_faces < (int64_t)INT32_MAX;
    // Octree rows without a TVD correction: staged slots, each row read to
    // its last used slot.
    const bool twelve = m->ell_width > 6 && m->ell_width <= 12 && a->div_scheme <= GF_DIV_LINEAR &&
                        m->n_faces > 0 && m->n_faces < (int64_t)INT32_MAX;
    const bool conv = a->div_scheme != GF_DIV_NONE, lap = a->lap_sign != 0.0;
    cudaStream_t st = GF_STREAM(stream);
    const unsigned g = grid_for(m->n_cells);
    if (fast) {
        if (a->ncomp == 1) {
            if (conv && lap) k_assemble6<1, true, true><<<g, kThreads, 0, st>>>(*m, *a);
            else if (conv) k_assemble6<1, true, false><<<g, kThreads, 0, st>>>(*m, *a);
            else k_assemble6<1, false, true><<<g, kThreads, 0, st>>>(*m, *a);
        } else {
            if (conv && lap) k_assemble6<3, true, true><<<g, kThreads, 0, st>>>(*m, *a);
            else if (conv) k_assemble6<3, true, false><<<g, kThreads, 0, st>>>(*m, *a);
            else k_assemble6<3, false, true><<<g, kThreads, 0, st>>>(*m, *a);
        }
    } else if (twelve) {
        if (a->ncomp == 1) {
            if (conv && lap) k_assemble12<1, true, true><<<g, kThreads, 0, st>>>(*m, *a);
            else if (conv) k_assemble12<1, true, false><<<g, kThreads, 0, st>>>(*m, *a);
            else k_assemble12<1, false, true><<<g, kThreads, 0, st>>>(*m, *a);
        } else {
            if (conv && lap) k_assemble12<3, true, true><<<g, kThreads, 0, st>>>(*m, *a);
            else if (conv) k_assemble12<3, true, false><<<g, kThreads, 0, st>>>(*m, *a);
            else k_assemble12<3, false, true><<<g, kThreads, 0, st>>>(*m, *a);
        }
    } else if (a->ncomp == 1) {
        k_assemble<1><<<g, kThreads, 0, st>>>(*m, *a);
    } else {
        k_assemble<3><<<g, kThreads, 0, st>>>(*m, *a);
    }
    return check_launch("gf_assemble");
}

int gf_momentum_finalize(const gf_mesh_t* m, int32_t ncomp, double relax, const double* psi, const double* grad,
                         double* diag, double* source, double* pred_source, void* stream) {
    if (!valid_mesh(m) || !valid_nc(ncomp)) return GF_ERR_INVALID;
    if (relax > 0.0 && psi == nullptr) {
        set_error("gf_momentum_finalize: relaxation needs psi");
        return GF_ERR_INVALID;
    }
    k_momentum_finalize<<<grid_for(m->n_cells), kThreads, 0, GF_STREAM(stream)>>>(
        m->n_cells, ncomp, relax, m->volume, psi, grad, diag, source, pred_source);
    return check_launch("gf_momentum_finalize");
}

int gf_pressure_finalize(const gf_mesh_t* m, const double* phi, double* diag, double* source, double* div_out,
                         int64_t ref_cell, double ref_value, void* stream) {
    if (!valid_mesh(m)) return GF_ERR_INVALID;
    if (ref_cell >= m->n_cells) {
        set_error("gf_pressure_finalize: reference cell %lld out of range", (long long)ref_cell);
        return GF_ERR_INVALID;
    }
    k_pressure_finalize<<<grid_for(m->n_cells), kThreads, 0, GF_STREAM(stream)>>>(*m, phi, diag, source, div_out,
                                                                                  ref_cell, ref_value);
    return check_launch("gf_pressure_finalize");
}

int gf_fixed_values(const gf_mesh_t* m, int32_t ncomp, const double* diag, const double* val, const double* source,
                    int64_t n_fixed, const int32_t* cells, const double* values, const uint8_t* fixed_mask,
                    double* out_diag, double* out_val, double* out_source, double* scratch, void* stream) {
    // `cells`/`values` are accepted for documentation symmetry; the kernel
    // reads the dense prescribed field passed in `values` ([ncomp][C]).
    (void)cells;
    if (!valid_mesh(m) || !valid_nc(ncomp) || fixed_mask == nullptr || values == nullptr || scratch == nullptr)
        return GF_ERR_INVALID;
    if (n_fixed == 0) return GF_OK;
    cudaStream_t s = GF_STREAM(stream);
    k_diag_sum_partial<<<kReduceBlocks, kThreads, 0, s>>>(m->n_cells, diag, scratch + 1);
    k_finish_sum<<<1, kThreads, 0, s>>>(kReduceBlocks, scratch + 1, scratch);
    if (ncomp == 1)
        k_fixed_values<1><<<grid_for(m->n_cells), kThreads, 0, s>>>(*m, diag, val, source, fixed_mask, values,
                                                                   scratch, out_diag, out_val, out_source);
    else
        k_fixed_values<3><<<grid_for(m->n_cells), kThreads, 0, s>>>(*m, diag, val, source, fixed_mask, values,
                                                                   scratch, out_diag, out_val, out_source);
    return check_launch("gf_fixed_values");
}

int gf_spmv(const gf_mesh_t* m, int32_t ncomp, const double* diag, const double* val, const double* x, double* y,
            void* stream) {
    if (!valid_mesh(m) || !valid_nc(ncomp)) return GF_ERR_INVALID;
    if (ncomp == 1)
        k_spmv<1><<<grid_for(m->n_cells), kThreads, 0, GF_STREAM(stream)>>>(*m, diag, val, x, y);
    else
        k_spmv<3><<<grid_for(m->n_cells), kThreads, 0, GF_STREAM(stream)>>>(*m, diag, val, x, y);
    return check_launch("gf_spmv");
}

int gf_rau_hbya(const gf_mesh_t* m, int32_t ncomp, const double* diag, const double* val, const double* source,
                const double* psi, double* rau, double* hbya, double* h1, void* stream) {
    if (!valid_mesh(m) || !valid_nc(ncomp)) return GF_ERR_INVALID;
    if (ncomp == 1)
        k_rau_hbya<1><<<grid_for(m->n_cells), kThreads, 0, GF_STREAM(stream)>>>(*m, diag, val, source, psi, rau,
                                                                               hbya, h1);
    else
        k_rau_hbya<3><<<grid_for(m->n_cells), kThreads, 0, GF_STREAM(stream)>>>(*m, diag, val, source, psi, rau,
                                                                               hbya, h1);
    return check_launch("gf_rau_hbya");
}

int gf_simplec_rAtU(const gf_mesh_t* m, const double* rau, const double* h1, double* ratu, void* stream) {
    if (!valid_mesh(m)) return GF_ERR_INVALID;
    k_simplec_ratu<<<grid_for(m->n_cells), kThreads, 0, GF_STREAM(stream)>>>(m->n_cells, rau, h1, ratu);
    return check_launch("gf_simplec_rAtU");
}

int gf_face_flux(const gf_mesh_t* m, int32_t mode, const double* vel, const int8_t* u_kind, const double* u_psib,
                 const gf_ddtcorr_t* ddt, const double* grad_vel, double* phi, void* stream) {
    if (!valid_mesh(m) || (mode != 0 && mode != 1) || vel == nullptr || u_kind == nullptr) {
        set_error("gf_face_flux: invalid arguments");
        return GF_ERR_INVALID;
    }
    gf_ddtcorr_t d{};
    int has = 0;
    if (ddt != nullptr) {
        d = *ddt;
        has = 1;
        if (d.rau == nullptr || d.u_old == nullptr || d.phi_old == nullptr || d.dt <= 0.0 ||
            (d.c != 0.0 && (d.u_older == nullptr || d.phi_older == nullptr))) {
            set_error("gf_face_flux: incomplete ddtCorr history");
            return GF_ERR_INVALID;
        }
    }
    cudaStream_t st = GF_STREAM(stream);
    if (m->face_axis != nullptr && grad_vel == nullptr && m->n_faces > 0 && m->n_faces < (int64_t)INT32_MAX) {
        const unsigned g = grid_for((m->n_faces + 1) / 2);
        if (has)
            k_face_flux_axis<true><<<g, kThreads, 0, st>>>(*m, vel, d, phi);
        else
            k_face_flux_axis<false><<<g, kThreads, 0, st>>>(*m, vel, d, phi);
        if (m->n_bnd > 0)
            k_face_flux<<<grid_for(m->n_bnd), kThreads, 0, st>>>(*m, mode, vel, u_kind, u_psib, d, has, grad_vel,
                                                                  phi, m->n_faces);
    } else {
        k_face_flux<<<grid_for(m->n_faces + m->n_bnd), kThreads, 0, st>>>(*m, mode, vel, u_kind, u_psib, d, has,
                                                                          grad_vel, phi, 0);
    }
    return check_launch("gf_face_flux");
}

int gf_reconstruct(const gf_mesh_t* m, const double* phi, double* U, void* stream) {
    if (!valid_mesh(m) || phi == nullptr || U == nullptr || m->sf == nullptr || m->bnd_sf == nullptr) {
        set_error("gf_reconstruct: invalid arguments");
        return GF_ERR_INVALID;
    }
    k_reconstruct<<<grid_for(m->n_cells), kThreads, 0, GF_STREAM(stream)>>>(*m, phi, U);
    return check_launch("gf_reconstruct");
}

int gf_fvc_div(const gf_mesh_t* m, int32_t ncomp, const double* phi, double* out, void* stream) {
    if (!valid_mesh(m) || !valid_nc(ncomp)) return GF_ERR_INVALID;
    k_fvc_div<<<grid_for(m->n_cells), kThreads, 0, GF_STREAM(stream)>>>(*m, ncomp, phi, out);
    return check_launch("gf_fvc_div");
}

int gf_gauss_grad(const gf_mesh_t* m, int32_t ncomp, const double* psi_f, double* grad, void* stream) {
    if (!valid_mesh(m) || !valid_nc(ncomp) || psi_f == nullptr || grad == nullptr || m->sf == nullptr ||
        m->bnd_sf == nullptr) {
        set_error("gf_gauss_grad: invalid arguments");
        return GF_ERR_INVALID;
    }
    const unsigned g = grid_for(m->n_cells);
    cudaStream_t st = GF_STREAM(stream);
    if (ncomp == 1) k_gauss_grad<1><<<g, kThreads, 0, st>>>(*m, psi_f, grad);
    else if (ncomp == 2) k_gauss_grad<2><<<g, kThreads, 0, st>>>(*m, psi_f, grad);
    else k_gauss_grad<3><<<g, kThreads, 0, st>>>(*m, psi_f, grad);
    return check_launch("gf_gauss_grad");
}

int gf_interpolate(const gf_mesh_t* m, int32_t ncomp, const double* psi, const int8_t* bc_kind, const double* psib,
                   const double* grad, double* out, void* stream) {
    if (!valid_mesh(m) || !valid_nc(ncomp)) return GF_ERR_INVALID;
    k_interpolate<<<grid_for(m->n_faces + m->n_bnd), kThreads, 0, GF_STREAM(stream)>>>(*m, ncomp, psi, bc_kind,
                                                                                       psib, grad, out);
    return check_launch("gf_interpolate");
}

int gf_sn_grad(const gf_mesh_t* m, int32_t ncomp, const double* psi, const int8_t* bc_kind, const double* frac,
               const double* refv, const double* refg, const double* grad, double* out, void* stream) {
    if (!valid_mesh(m) || !valid_nc(ncomp)) return GF_ERR_INVALID;
    k_sn_grad<<<grid_for(m->n_faces + m->n_bnd), kThreads, 0, GF_STREAM(stream)>>>(*m, ncomp, psi, bc_kind, frac,
                                                                                   refv, refg, grad, out);
    return check_launch("gf_sn_grad");
}

int gf_correct_phi(const gf_mesh_t* m, const double* phi_pred, const double* coeff, const double* p,
                   const int8_t* p_kind, const double* frac, const double* refv, const double* refg, double sign,
                   int32_t simplec, const double* grad_p, const double* ffc, double* phi, void* stream) {
    if (!valid_mesh(m)) return GF_ERR_INVALID;
    k_correct_phi<<<grid_for(m->n_faces + m->n_bnd), kThreads, 0, GF_STREAM(stream)>>>(
        *m, phi_pred, coeff, p, p_kind, frac, refv, refg, sign, simplec, grad_p, ffc, phi);
    return check_launch("gf_correct_phi");
}

int gf_close_fixed_flux(const gf_mesh_t* m, int64_t n_faces, const int32_t* face_list, const double* area_frac,
                        double* phi, double* scratch, void* stream) {
    if (!valid_mesh(m)) return GF_ERR_INVALID;
    if (n_faces == 0) return GF_OK;
    cudaStream_t s = GF_STREAM(stream);
    k_fixed_imbalance<<<grid_for(n_faces), kThreads, 0, s>>>(*m, n_faces, face_list, phi, scratch);
    k_fixed_apply<<<grid_for(n_faces), kThreads, 0, s>>>(*m, n_faces, face_list, area_frac, scratch, phi);
    return check_launch("gf_close_fixed_flux");
}

int gf_correct_velocity(const gf_mesh_t* m, const double* base, const double* coeff, const double* grad,
                        double* out, void* stream) {
    if (!valid_mesh(m)) return GF_ERR_INVALID;
    k_correct_velocity<<<grid_for(m->n_cells), kThreads, 0, GF_STREAM(stream)>>>(m->n_cells, base, coeff, grad,
                                                                                 out);
    return check_launch("gf_correct_velocity");
}

int gf_set_cell_values(int64_t n_cells, int32_t ncomp, int64_t n_set, const int32_t* cells, const double* values,
                       int64_t values_stride, double* out, void* stream) {
    if (n_set == 0) return GF_OK;
    if (!valid_nc(ncomp) || cells == nullptr || values == nullptr || out == nullptr) return GF_ERR_INVALID;
    k_set_cell_values<<<grid_for(n_set), kThreads, 0, GF_STREAM(stream)>>>(n_cells, ncomp, n_set, cells, values,
                                                                          values_stride, out);
    return check_launch("gf_set_cell_values");
}

int gf_gather_bnd(int64_t n_bnd, int32_t ncomp, int64_t n, const int32_t* faces, const double* refv, double* values,
                  void* stream) {
    if (n == 0) return GF_OK;
    if (!valid_nc(ncomp)) return GF_ERR_INVALID;
    k_gather_bnd<<<grid_for(n), kThreads, 0, GF_STREAM(stream)>>>(n_bnd, ncomp, n, faces, refv, values);
    return check_launch("gf_gather_bnd");
}

int gf_adjust_phi(const gf_mesh_t* m, const int8_t* face_class, double* phi, void* stream) {
    if (!valid_mesh(m) || face_class == nullptr) return GF_ERR_INVALID;
    if (m->n_domain == 0) return GF_OK;
    k_adjust_phi<<<1, 1024, 0, GF_STREAM(stream)>>>(*m, face_class, phi);
    return check_launch("gf_adjust_phi");
}

int gf_relax_field(int64_t n, double alpha, const double* old, double* cur, void* stream) {
    k_relax_field<<<grid_for(n), kThreads, 0, GF_STREAM(stream)>>>(n, alpha, old, cur);
    return check_launch("gf_relax_field");
}

int gf_axpby(int64_t n, double a, const double* x, double b, const double* y, double* out, void* stream) {
    if (n == 0) return GF_OK;
    k_axpby<<<grid_for(n), kThreads, 0, GF_STREAM(stream)>>>(n, a, x, b, y, out);
    return check_launch("gf_axpby");
}

int gf_ell_to_ldu(const gf_mesh_t* m, const double* val, double* upper, double* lower, void* stream) {
    if (!valid_mesh(m) || m->face_pos_owner == nullptr) return GF_ERR_INVALID;
    if (m->n_faces == 0) return GF_OK;
    k_ell_to_ldu<<<grid_for(m->n_faces), kThreads, 0, GF_STREAM(stream)>>>(*m, val, upper, lower);
    return check_launch("gf_ell_to_ldu");
}

int gf_ldu_to_ell(const gf_mesh_t* m, const double* upper, const double* lower, double* val, void* stream) {
    if (!valid_mesh(m) || m->face_pos_owner == nullptr) return GF_ERR_INVALID;
    cudaStream_t s = GF_STREAM(stream);
    cudaMemsetAsync(val, 0, sizeof(double) * m->n_cells * m->ell_width, s);
    if (m->n_faces == 0) return check_launch("gf_ldu_to_ell");
    k_ldu_to_ell<<<grid_for(m->n_faces), kThreads, 0, s>>>(*m, upper, lower, val);
    return check_launch("gf_ldu_to_ell");
}

int gf_field_residual(const gf_mesh_t* m, int32_t ncomp, const double* diag, const double* val, const double* source,
                      const double* psi, double* scratch, double* out, void* stream) {
    if (!valid_mesh(m) || !valid_nc(ncomp) || scratch == nullptr) return GF_ERR_INVALID;
    cudaStream_t s = GF_STREAM(stream);
    if (ncomp == 1)
        k_residual_partial<1><<<kReduceBlocks, kThreads, 0, s>>>(*m, diag, val, source, psi, scratch);
    else
        k_residual_partial<3><<<kReduceBlocks, kThreads, 0, s>>>(*m, diag, val, source, psi, scratch);
    k_residual_finish<<<1, kThreads, 0, s>>>(kReduceBlocks, scratch, out);
    return check_launch("gf_field_residual");
}

int gf_matrix_flux(const gf_mesh_t* m, int32_t ncomp, const double* val, const double* psi, const double* ffc,
                   double* out, void* stream) {
    if (!valid_mesh(m) || !valid_nc(ncomp)) return GF_ERR_INVALID;
    if (m->n_faces == 0) return GF_OK;
    if (ncomp == 1)
        k_matrix_flux<1><<<grid_for(m->n_faces), kThreads, 0, GF_STREAM(stream)>>>(*m, val, psi, ffc, out);
    else
        k_matrix_flux<3><<<grid_for(m->n_faces), kThreads, 0, GF_STREAM(stream)>>>(*m, val, psi, ffc, out);
    return check_launch("gf_matrix_flux");
}

}  // extern "C"
