// Shared device helpers for the gridfoam_b200 kernels (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdarg>
#include <cstdio>
#include <string>

#include "../../include/gridfoam_b200.h"

namespace gf {

constexpr int kThreads = 256;

// Thread-local last error message, returned by gf_last_error().
void set_error(const char* fmt, ...);

inline int check_launch(const char* what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error("%s: %s", what, cudaGetErrorString(e));
        return GF_ERR_CUDA;
    }
    return GF_OK;
}

#define GF_STREAM(s) (reinterpret_cast<cudaStream_t>(s))

inline unsigned grid_for(int64_t n, int threads = kThreads) {
    int64_t g = (n + threads - 1) / threads;
    if (g < 1) g = 1;
    if (g > 2147483647LL) g = 2147483647LL;
    return (unsigned)g;
}

// Slot decoding of the ELL adjacency.
enum SlotKind { kEmpty = 0, kInternal = 1, kBoundary = 2 };

struct Slot {
    int kind;
    int face;  // internal face index (kInternal) or -1
    int side;  // 0: cell is owner, 1: cell is neighbour
    int bnd;   // boundary face index (kBoundary)
};

__device__ __forceinline__ Slot decode_slot(const gf_mesh_t& m, int32_t code) {
    Slot s;
    s.face = -1;
    s.bnd = -1;
    s.side = 0;
    if (code < 0) {
        s.kind = kEmpty;
        return s;
    }
    const int f = code >> 1;
    s.side = code & 1;
    if (f >= m.n_faces) {
        s.kind = kBoundary;
        s.bnd = f - (int)m.n_faces;
        return s;
    }
    const int imm = m.imm_index ? __ldg(m.imm_index + f) : -1;
    if (imm >= 0) {
        s.kind = kBoundary;
        s.bnd = (int)m.n_domain + (s.side ? (int)m.n_imm : 0) + imm;
        return s;
    }
    s.kind = kInternal;
    s.face = f;
    return s;
}

__device__ __forceinline__ double sgn(double x) {
    return (x > 0.0) ? 1.0 : ((x < 0.0) ? -1.0 : 0.0);
}

// Boundary-normal-gradient value coefficient (fv/boundary_ops.py:405-422).
__device__ __forceinline__ double value_grad_coeff(const gf_mesh_t& m, int b, double frac) {
    const bool near = m.bnd_near ? (__ldg(m.bnd_near + b) != 0) : false;
    const bool fixed = near && (frac == 1.0) && (b >= m.n_domain);
    const bool active = (frac != 0.0) && !fixed;
    if (!active) return 0.0;
    return frac / __ldg(m.bnd_mag_d + b);
}

__device__ __forceinline__ bool nonassignable(int kind) {
    return kind == GF_BC_DIRICHLET || kind == GF_BC_SLIP;
}

// Hanging ordinal of internal face f, or -1 (also when the mesh has none).
__device__ __forceinline__ int hang_of(const gf_mesh_t& m, int f) {
    return m.n_hang > 0 ? __ldg(m.face_hang + f) : -1;
}

// Offset correction of the linear face value of component k on hanging face
// h: (w grad_O + (1 - w) grad_N) . offset (face_interpolation.py:81-96).
// grad is [ncomp*3][C].
__device__ __forceinline__ double hang_value_corr(const gf_mesh_t& m, const double* __restrict__ grad, int k,
                                                  int o, int n, double w, int h) {
    const int64_t C = m.n_cells, H = m.n_hang;
    double acc = 0.0;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        const double gf = w * grad[(k * 3 + j) * C + o] + (1.0 - w) * grad[(k * 3 + j) * C + n];
        acc += gf * __ldg(m.hang_offset + j * H + h);
    }
    return acc;
}

// Skewness correction of the normal gradient of component k on hanging face
// h: delta (grad_N . move_N - grad_O . move_O) (face_interpolation.py:99-145).
__device__ __forceinline__ double hang_sn_corr(const gf_mesh_t& m, const double* __restrict__ grad, int k, int o,
                                               int n, double delta, int h) {
    const int64_t C = m.n_cells, H = m.n_hang;
    double cn = 0.0, co = 0.0;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        cn += grad[(k * 3 + j) * C + n] * __ldg(m.hang_move_n + j * H + h);
        co += grad[(k * 3 + j) * C + o] * __ldg(m.hang_move_o + j * H + h);
    }
    return delta * (cn - co);
}

}  // namespace gf
