// Post-processing kernels (sm_100a): the immersed-surface force integral
// (post/forces/sampling.py:69-168, post/forces/integration.py:76-187).
//
// One thread per axis-projected boundary sample of the patch: the sample is
// kept when its outward direction points into the body (n_hat . S_body > 0,
// S_body the body-inward surface normal of its anchor); its pressure force
// is rho p_b Sf and its viscous force -rho nu (gradU + gradU^T) Sf with
// gradU = (U_b - U_P) / wall_dist (x) n_surface.  Per-sample forces and
// moments go to a buffer; one block then sums them in a fixed order.
#include "gf_common.cuh"

namespace gf {

constexpr int kSampleRows = 12;  // pressure[3], viscous[3], force[3], moment[3]

__device__ __forceinline__ double side_value(const int8_t* kind, const gf_bc_state_t& st, const double* psi,
                                             int64_t C, int64_t nb, int k, int b, int c, double mag_d) {
    const double pc = psi[k * C + c];
    if (kind[b] == GF_BC_NONE) return pc;  // sampling.py:58-59: no condition on the patch
    const double f = st.frac[b];
    return f * st.refv[k * nb + b] + (1.0 - f) * (pc + mag_d * st.refg[k * nb + b]);
}

__global__ void k_force_samples(gf_mesh_t m, int64_t n, const int32_t* __restrict__ faces,
                                const double* __restrict__ anchor_normal, const int8_t* __restrict__ p_kind,
                                gf_bc_state_t ps, const double* __restrict__ p, const int8_t* __restrict__ u_kind,
                                gf_bc_state_t us, const double* __restrict__ U, const double* __restrict__ nu,
                                double nu_scalar, double rho, double cx, double cy, double cz,
                                double* __restrict__ out) {
    const int64_t C = m.n_cells, nb = m.n_bnd, Fi = m.n_imm;
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x) {
        const int b = faces[j];
        int64_t a = b - m.n_domain;
        if (a >= Fi) a -= Fi;
        const int c = __ldg(m.bnd_cell + b);
        const double mag_sf = __ldg(m.bnd_mag_sf + b), mag_d = __ldg(m.bnd_mag_d + b);
        double sf[3], nh[3], sb[3];
        double align = 0.0, area2 = 0.0;
        for (int k = 0; k < 3; ++k) {
            sf[k] = __ldg(m.bnd_sf + k * nb + b);
            nh[k] = sf[k] / mag_sf;
            sb[k] = -anchor_normal[k * Fi + a];
            align += nh[k] * sb[k];
            area2 += sb[k] * sb[k];
        }
        double row[kSampleRows];
        for (int r = 0; r < kSampleRows; ++r) row[r] = 0.0;
        if (align > 0.0) {
            const double area = sqrt(area2);
            double ns[3], nal = 0.0;
            for (int k = 0; k < 3; ++k) {
                ns[k] = sb[k] / area;
                nal += nh[k] * ns[k];
            }
            const double wall = mag_d * fmax(nal, 1.0e-12);
            double dudn[3];
            for (int k = 0; k < 3; ++k)
                dudn[k] = (side_value(u_kind, us, U, C, nb, k, b, c, mag_d) - U[k * C + c]) / wall;
            const double pb = side_value(p_kind, ps, p, C, nb, 0, b, c, mag_d);
            const double nuc = nu ? nu[c] : nu_scalar;
            const double fc[3] = {__ldg(m.center + c) + mag_d * nh[0] - cx,
                                  __ldg(m.center + C + c) + mag_d * nh[1] - cy,
                                  __ldg(m.center + 2 * C + c) + mag_d * nh[2] - cz};
            double ff[3];
            for (int i = 0; i < 3; ++i) {
                const double pf = (rho * pb) * sf[i];
                double vf = 0.0;
                for (int k = 0; k < 3; ++k) {
                    const double s = rho * nuc * (dudn[i] * ns[k] + dudn[k] * ns[i]);
                    vf += s * sf[k];
                }
                vf = -vf;
                row[i] = pf;
                row[3 + i] = vf;
                ff[i] = pf + vf;
                row[6 + i] = ff[i];
            }
            row[9] = fc[1] * ff[2] - fc[2] * ff[1];
            row[10] = fc[2] * ff[0] - fc[0] * ff[2];
            row[11] = fc[0] * ff[1] - fc[1] * ff[0];
        }
        for (int r = 0; r < kSampleRows; ++r) out[r * n + j] = row[r];
    }
}

// total[0:3] = sum force, total[3:6] = sum moment, in a fixed order.
__global__ void k_force_sum(int64_t n, const double* __restrict__ samples, double* __restrict__ total) {
    __shared__ double sh[kThreads];
    for (int r = 0; r < 6; ++r) {
        const double* row = samples + (6 + r) * n;
        double acc = 0.0;
        for (int64_t j = threadIdx.x; j < n; j += blockDim.x) acc += row[j];
        sh[threadIdx.x] = acc;
        __syncthreads();
        for (int s = blockDim.x / 2; s > 0; s >>= 1) {
            if ((int)threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
            __syncthreads();
        }
        if (threadIdx.x == 0) total[r] = sh[0];
        __syncthreads();
    }
}

// Continuity-error sums over cells: blocks of kContBlocks fixed ranges, then
// one block over the block partials, both in a fixed order, so the sums are
// the same bits on every launch and every device.
constexpr int kContBlocks = 256;

__global__ void k_cont_partials(int64_t n, const double* __restrict__ div, const double* __restrict__ vol,
                                double* __restrict__ part) {
    __shared__ double sh[3][kThreads];
    const int64_t per = (n + kContBlocks - 1) / kContBlocks;
    const int64_t b0 = blockIdx.x * per;
    const int64_t b1 = b0 + per < n ? b0 + per : n;
    double a = 0.0, g = 0.0, v = 0.0;
    for (int64_t c = b0 + threadIdx.x; c < b1; c += blockDim.x) {
        const double d = div[c], w = vol[c];
        a += fabs(d) * w;
        g += d * w;
        v += w;
    }
    sh[0][threadIdx.x] = a;
    sh[1][threadIdx.x] = g;
    sh[2][threadIdx.x] = v;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s)
            for (int r = 0; r < 3; ++r) sh[r][threadIdx.x] += sh[r][threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x < 3) part[threadIdx.x * kContBlocks + blockIdx.x] = sh[threadIdx.x][0];
}

__global__ void k_cont_final(const double* __restrict__ part, double* __restrict__ out) {
    __shared__ double sh[kContBlocks];
    for (int r = 0; r < 3; ++r) {
        sh[threadIdx.x] = part[r * kContBlocks + threadIdx.x];
        __syncthreads();
        for (int s = kContBlocks / 2; s > 0; s >>= 1) {
            if ((int)threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
            __syncthreads();
        }
        if (threadIdx.x == 0) out[r] = sh[0];
        __syncthreads();
    }
}

}  // namespace gf

using namespace gf;

extern "C" {

int gf_force_integral(const gf_mesh_t* m, int64_t n, const int32_t* faces, const double* anchor_normal,
                      const int8_t* p_kind, const gf_bc_state_t* p_state, const double* p, const int8_t* u_kind,
                      const gf_bc_state_t* u_state, const double* U, const double* nu_eff, double nu_scalar,
                      double rho, double cx, double cy, double cz, double* samples, double* total, void* stream) {
    if (m == nullptr || n < 0 || (n > 0 && (faces == nullptr || anchor_normal == nullptr)) || p_kind == nullptr ||
        p_state == nullptr || p == nullptr || u_kind == nullptr || u_state == nullptr || U == nullptr ||
        samples == nullptr || total == nullptr || m->n_imm <= 0) {
        set_error("gf_force_integral: invalid arguments");
        return GF_ERR_INVALID;
    }
    if (n > 0)
        k_force_samples<<<grid_for(n), kThreads, 0, GF_STREAM(stream)>>>(*m, n, faces, anchor_normal, p_kind,
                                                                         *p_state, p, u_kind, *u_state, U, nu_eff,
                                                                         nu_scalar, rho, cx, cy, cz, samples);
    k_force_sum<<<1, kThreads, 0, GF_STREAM(stream)>>>(n, samples, total);
    return check_launch("gf_force_integral");
}

int64_t gf_continuity_scratch_doubles(void) { return 3 * (int64_t)kContBlocks; }

int gf_continuity_sums(int64_t n, const double* div, const double* vol, double* scratch, double* out,
                       void* stream) {
    if (n < 0 || (n > 0 && (div == nullptr || vol == nullptr)) || scratch == nullptr || out == nullptr) {
        set_error("gf_continuity_sums: invalid arguments");
        return GF_ERR_INVALID;
    }
    static_assert(kContBlocks == kThreads, "one final block reduces one partial per thread");
    k_cont_partials<<<kContBlocks, kThreads, 0, GF_STREAM(stream)>>>(n, div, vol, scratch);
    k_cont_final<<<1, kContBlocks, 0, GF_STREAM(stream)>>>(scratch, out);
    return check_launch("gf_continuity_sums");
}

}  // extern "C"
