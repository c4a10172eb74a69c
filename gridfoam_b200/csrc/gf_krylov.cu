// Persistent cooperative Krylov solvers (sm_100a).
//
// One launch runs a whole solve (all iterations, up to three right-hand
// sides sharing the matrix).  Blocks synchronise through a grid barrier that
// also finishes every dot product: each block writes its partial sums, the
// last block to arrive reduces them in a fixed order and releases the
// others, so each reduction costs one barrier and is bitwise reproducible.
// Every wait is bounded; on expiry the kernel raises an error flag and
// returns instead of hanging.  The launch is cooperative, so all blocks are
// co-resident and the barrier is always reachable.
#include "gf_common.cuh"

#include <mutex>

namespace gf {

constexpr int kKThreads = 512;
constexpr int kCgThreads = 256;
constexpr int kMaxBlocks = 1024;
constexpr int kMaxNV = 16;
constexpr int kCtlDoubles = 32;
constexpr long long kSpinLimit = 30000000LL;  // x ~40 ns polls: about a second

struct KCtl {
    unsigned int count;
    unsigned int gen;
    int error;
    int pad;
    double results[kMaxNV];
};

__device__ __forceinline__ unsigned vload(const unsigned* p) { return *(const volatile unsigned*)p; }
__device__ __forceinline__ int vload(const int* p) { return *(const volatile int*)p; }

__device__ __forceinline__ double nmax(double a, double b) {
    if (a != a || b != b) return __longlong_as_double(0x7ff8000000000000LL);
    return fmax(a, b);
}

__device__ __forceinline__ double inv_diag(const double* __restrict__ diag, int64_t c, bool jac) {
    if (!jac) return 1.0;
    const double d = __ldg(diag + c);
    return fabs(d) < 2.220446049250313e-16 ? 1.0 : 1.0 / d;
}

// Grid-wide reduction of NV values per thread (sum, or max where maxmask
// has the bit set), fused with the grid barrier.  Returns false when the
// barrier wait expired.
template <int NV, int THREADS = kKThreads>
__device__ bool grid_reduce(KCtl* ctl, double* partials, double (&v)[NV], unsigned maxmask) {
    __shared__ double sm[kMaxNV * 32];
    __shared__ double s_res[kMaxNV];
    __shared__ int s_last, s_err;
    __shared__ unsigned s_gen;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int j = 0; j < NV; ++j) {
        const bool mx = (maxmask >> j) & 1u;
        double x = v[j];
        for (int o = 16; o > 0; o >>= 1) {
            const double y = __shfl_xor_sync(0xffffffffu, x, o);
            x = mx ? nmax(x, y) : x + y;
        }
        if (lane == 0) sm[j * 32 + warp] = x;
    }
    __syncthreads();
    if (threadIdx.x < NV) {
        const int j = threadIdx.x;
        const bool mx = (maxmask >> j) & 1u;
        double x = sm[j * 32];
        for (int w = 1; w < nw; ++w) x = mx ? nmax(x, sm[j * 32 + w]) : x + sm[j * 32 + w];
        __stcg(partials + (int64_t)blockIdx.x * NV + j, x);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        // Release: the CTA barrier orders every thread's writes of this phase
        // before this fence, which orders them before the arrival.
        __threadfence();
        const unsigned gen = vload(&ctl->gen);
        const unsigned prev = atomicAdd(&ctl->count, 1u);
        s_gen = gen;
        s_last = (prev == gridDim.x - 1);
        s_err = 0;
    }
    __syncthreads();
    if (s_last) {
        // Every thread loads its (at most kMaxBlocks / blockDim) partials of
        // each value at once, then a fixed-order block reduction: one L2
        // round trip instead of a chain of dependent loads.
        double acc[NV];
#pragma unroll
        for (int j = 0; j < NV; ++j) acc[j] = 0.0;
        constexpr int kPer = (kMaxBlocks + THREADS - 1) / THREADS;
        double y[kPer][NV];
#pragma unroll
        for (int i = 0; i < kPer; ++i) {
            const int b = threadIdx.x + i * blockDim.x;
#pragma unroll
            for (int j = 0; j < NV; ++j) y[i][j] = b < (int)gridDim.x ? __ldcg(partials + (int64_t)b * NV + j) : 0.0;
        }
#pragma unroll
        for (int i = 0; i < kPer; ++i) {
#pragma unroll
            for (int j = 0; j < NV; ++j) {
                const bool mx = (maxmask >> j) & 1u;
                acc[j] = mx ? nmax(acc[j], y[i][j]) : acc[j] + y[i][j];
            }
        }
#pragma unroll
        for (int j = 0; j < NV; ++j) {
            const bool mx = (maxmask >> j) & 1u;
            double x = acc[j];
            for (int o = 16; o > 0; o >>= 1) {
                const double t = __shfl_xor_sync(0xffffffffu, x, o);
                x = mx ? nmax(x, t) : x + t;
            }
            if (lane == 0) sm[j * 32 + warp] = x;
        }
        __syncthreads();
        if (threadIdx.x < NV) {
            const int j = threadIdx.x;
            const bool mx = (maxmask >> j) & 1u;
            double x = sm[j * 32];
            for (int w = 1; w < nw; ++w) x = mx ? nmax(x, sm[j * 32 + w]) : x + sm[j * 32 + w];
            __stcg(&ctl->results[j], x);
            s_res[j] = x;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            atomicExch(&ctl->count, 0u);
            __threadfence();
            atomicAdd(&ctl->gen, 1u);
            s_err = vload(&ctl->error);
        }
    } else if (threadIdx.x == 0) {
        long long it = 0;
        while (vload(&ctl->gen) == s_gen) {
            __nanosleep(20);
            if (++it > kSpinLimit) {
                atomicExch(&ctl->error, 1);
                break;
            }
        }
        __threadfence();  // acquire side of the release above
#pragma unroll
        for (int j = 0; j < NV; ++j) s_res[j] = __ldcg(&ctl->results[j]);
        s_err = vload(&ctl->error);
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < NV; ++j) v[j] = s_res[j];
    return s_err == 0;
}

// y_k(c) = diag(c) * g(k, c) + sum_s val(s, c) * g(k, nbr(s, c))
template <int NC, class G>
__device__ __forceinline__ void row_apply(const gf_krylov_t& K, int64_t c, const G& g, double (&out)[NC]) {
    const int64_t n = K.n;
    const double d = __ldg(K.diag + c);
#pragma unroll
    for (int k = 0; k < NC; ++k) out[k] = d * g(k, c);
    for (int s = 0; s < K.width; ++s) {
        const double a = __ldg(K.val + s * n + c);
        const int nb = __ldg(K.nbr + s * n + c);
#pragma unroll
        for (int k = 0; k < NC; ++k) out[k] += a * g(k, nb);
    }
}

__device__ __forceinline__ double norm_acc(double acc, double r, bool linf) {
    return linf ? nmax(acc, fabs(r)) : acc + r * r;
}

__device__ __forceinline__ double norm_fin(double acc, bool linf) { return linf ? acc : sqrt(acc); }

struct CgState {
    double thresh, r0, final, rz_old, alpha, beta;
    int done, its, converged, status;
};

template <int NC>
__global__ void __launch_bounds__(kKThreads) k_pcg(gf_krylov_t K) {
    __shared__ CgState st[NC];
    __shared__ int s_all_done;
    KCtl* ctl = reinterpret_cast<KCtl*>(K.work);
    double* partials = K.work + kCtlDoubles;
    double* vec = partials + kMaxBlocks * kMaxNV;
    const int64_t n = K.n;
    double* r = vec;
    double* p = vec + NC * n;
    double* q = vec + 2 * NC * n;
    double* x = K.x;
    const bool jac = K.jacobi != 0, linf = K.norm_inf != 0;
    const unsigned nmask = linf ? ((1u << NC) - 1u) : 0u;
    const int64_t t0 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    bool ok = true;

    {  // r = b - A x, z = M r, p = z; reduce |r| and r.z
        double loc[2 * NC];
#pragma unroll
        for (int j = 0; j < 2 * NC; ++j) loc[j] = 0.0;
        auto gx = [&](int k, int64_t i) { return __ldcg(x + k * n + i); };
        for (int64_t c = t0; c < n; c += stride) {
            double ax[NC];
            row_apply<NC>(K, c, gx, ax);
            const double ic = inv_diag(K.diag, c, jac);
#pragma unroll
            for (int k = 0; k < NC; ++k) {
                const double rk = __ldg(K.rhs + k * n + c) - ax[k];
                const double zk = ic * rk;
                __stcg(r + k * n + c, rk);
                __stcg(p + k * n + c, zk);
                loc[k] = norm_acc(loc[k], rk, linf);
                loc[NC + k] += rk * zk;
            }
        }
        ok = grid_reduce<2 * NC>(ctl, partials, loc, nmask);
        if (threadIdx.x == 0) {
            for (int k = 0; k < NC; ++k) {
                const double r0 = norm_fin(loc[k], linf);
                st[k].r0 = r0;
                st[k].final = r0;
                st[k].thresh = fmax(K.atol, K.rtol * r0);
                st[k].rz_old = loc[NC + k];
                st[k].its = 0;
                st[k].converged = 0;
                st[k].status = GF_MAX_ITER;
                st[k].done = 0;
                if (r0 < st[k].thresh) {
                    st[k].done = 1;
                    st[k].converged = 1;
                    st[k].status = GF_OK;
                } else if (!isfinite(r0)) {
                    st[k].done = 1;
                    st[k].status = GF_NONFINITE;
                }
            }
        }
        __syncthreads();
    }

    for (int it = 1; ok && it <= K.max_iter; ++it) {
        if (threadIdx.x == 0) {
            int all = 1;
            for (int k = 0; k < NC; ++k) all &= st[k].done;
            s_all_done = all;
        }
        __syncthreads();
        if (s_all_done) break;

        {  // q = A p, p.q
            double loc[NC];
#pragma unroll
            for (int k = 0; k < NC; ++k) loc[k] = 0.0;
            auto gp = [&](int k, int64_t i) { return __ldcg(p + k * n + i); };
            for (int64_t c = t0; c < n; c += stride) {
                double ap[NC];
                row_apply<NC>(K, c, gp, ap);
#pragma unroll
                for (int k = 0; k < NC; ++k) {
                    if (st[k].done) continue;
                    __stcg(q + k * n + c, ap[k]);
                    loc[k] += __ldcg(p + k * n + c) * ap[k];
                }
            }
            ok = grid_reduce<NC>(ctl, partials, loc, 0u);
            if (!ok) break;
            if (threadIdx.x == 0)
                for (int k = 0; k < NC; ++k)
                    if (!st[k].done) st[k].alpha = st[k].rz_old / loc[k];
            __syncthreads();
        }
        {  // x += alpha p, r -= alpha q, |r|, r.z
            double loc[2 * NC];
#pragma unroll
            for (int j = 0; j < 2 * NC; ++j) loc[j] = 0.0;
            for (int64_t c = t0; c < n; c += stride) {
                const double ic = inv_diag(K.diag, c, jac);
#pragma unroll
                for (int k = 0; k < NC; ++k) {
                    if (st[k].done) continue;
                    const double a = st[k].alpha;
                    const double pk = __ldcg(p + k * n + c);
                    __stcg(x + k * n + c, __ldcg(x + k * n + c) + a * pk);
                    const double rk = __ldcg(r + k * n + c) - a * __ldcg(q + k * n + c);
                    __stcg(r + k * n + c, rk);
                    loc[k] = norm_acc(loc[k], rk, linf);
                    loc[NC + k] += rk * (ic * rk);
                }
            }
            ok = grid_reduce<2 * NC>(ctl, partials, loc, nmask);
            if (!ok) break;
            if (threadIdx.x == 0) {
                int all = 1;
                for (int k = 0; k < NC; ++k) {
                    if (st[k].done) continue;
                    const double fin = norm_fin(loc[k], linf);
                    st[k].final = fin;
                    if (fin < st[k].thresh) {
                        st[k].done = 1;
                        st[k].converged = 1;
                        st[k].its = it;
                        st[k].status = GF_OK;
                    } else if (!isfinite(fin)) {
                        st[k].done = 1;
                        st[k].its = it;
                        st[k].status = GF_NONFINITE;
                    } else {
                        st[k].beta = loc[NC + k] / st[k].rz_old;
                        st[k].rz_old = loc[NC + k];
                    }
                    all &= st[k].done;
                }
                for (int k = 0; k < NC; ++k) all &= st[k].done;
                s_all_done = all;
            }
            __syncthreads();
            if (s_all_done) break;
        }
        {  // p = z + p beta
            double dummy[1] = {0.0};
            for (int64_t c = t0; c < n; c += stride) {
                const double ic = inv_diag(K.diag, c, jac);
#pragma unroll
                for (int k = 0; k < NC; ++k) {
                    if (st[k].done) continue;
                    const double rk = __ldcg(r + k * n + c);
                    __stcg(p + k * n + c, ic * rk + __ldcg(p + k * n + c) * st[k].beta);
                }
            }
            ok = grid_reduce<1>(ctl, partials, dummy, 0u);
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        for (int k = 0; k < NC; ++k) {
            double* s = K.stats + 5 * k;
            s[0] = st[k].r0;
            s[1] = st[k].final;
            s[2] = st[k].done ? st[k].its : K.max_iter;
            s[3] = st[k].converged;
            s[4] = ok ? st[k].status : GF_ERR_TIMEOUT;
        }
    }
}

// Row products A_c . g for the single-system CG kernels.  EllRows gathers
// through the neighbour table; BoxRows uses implicit neighbours of a
// uniform lexicographic box (slot order -x,+x,-y,+y,-z,+z; the coefficient
// of a boundary slot is zero, so clamped neighbour indices are harmless).
// With SYM the "-" coefficient of cell c is the "+" coefficient of
// c - stride, so only three coefficient arrays are read.  T is the storage
// type of the coefficients; COMPACT means the array holds only the needed
// slots (3 for SYM) instead of the 6-slot ELL layout.
// Coefficient loads: FP64 coefficients are kernel inputs (read-only path);
// the FP32 copies are written inside the kernel, so they bypass L1.
__device__ __forceinline__ double ld_coef(const double* p) { return __ldg(p); }
__device__ __forceinline__ float ld_coef(const float* p) { return __ldcg(p); }

template <typename T, int WIDTH>
struct EllRows {
    const T* val;
    const int32_t* nbr;
    int64_t n;
    int w;
    template <typename A, class G>
    __device__ __forceinline__ A apply(int64_t c, A dc, const G& g) const {
        A acc = dc * g(c);
        if (WIDTH > 0) {
            int nb[WIDTH > 0 ? WIDTH : 1];
            A a[WIDTH > 0 ? WIDTH : 1];
#pragma unroll
            for (int s = 0; s < (WIDTH > 0 ? WIDTH : 1); ++s) {
                nb[s] = __ldg(nbr + s * n + c);
                a[s] = (A)ld_coef(val + s * n + c);
            }
#pragma unroll
            for (int s = 0; s < (WIDTH > 0 ? WIDTH : 1); ++s) acc += a[s] * g(nb[s]);
        } else {
            for (int s = 0; s < w; ++s) acc += (A)ld_coef(val + s * n + c) * g(__ldg(nbr + s * n + c));
        }
        return acc;
    }
};

template <typename T, bool SYM, bool COMPACT>
struct BoxRows {
    const T* val;
    int64_t n, sy, sz;
    // COMPACT arrays hold only the three '+' slots, which only SYM uses.
    __device__ __forceinline__ int64_t plus_slot(int a) const { return (COMPACT && SYM) ? a : 2 * a + 1; }
    template <typename A, class G>
    __device__ __forceinline__ A apply(int64_t c, A dc, const G& g) const {
        const int64_t st[3] = {1, sy, sz};
        A ap[3], am[3];
        int64_t ip[3], im[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const int64_t s = st[a];
            const T* pv = val + plus_slot(a) * n;
            ap[a] = (A)ld_coef(pv + c);
            if (SYM) {
                am[a] = c >= s ? (A)ld_coef(pv + c - s) : (A)0;
            } else {
                am[a] = (A)ld_coef(val + (2 * a) * n + c);
            }
            im[a] = c >= s ? c - s : c;
            ip[a] = c + s < n ? c + s : c;
        }
        // Same accumulation order as the ELL slots (-x, +x, -y, +y, -z, +z),
        // so both layouts give bitwise identical products.
        A acc = dc * g(c);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            acc += am[a] * g(im[a]);
            acc += ap[a] * g(ip[a]);
        }
        return acc;
    }
};

// Single-system Jacobi-PCG with the direction update fused into the SpMV
// pass: p_new = z + p_old beta is stored for the own cell and recomputed
// (bitwise identically) at the neighbours, so an iteration needs two grid
// reductions (p.Ap, then |r| and r.z) instead of three.

template <int U, class Rows>
__device__ void pcg1_body(const gf_krylov_t& K, const Rows& rows) {
    __shared__ CgState st;
    KCtl* ctl = reinterpret_cast<KCtl*>(K.work);
    double* partials = K.work + kCtlDoubles;
    double* vec = partials + kMaxBlocks * kMaxNV;
    const int64_t n = K.n;
    double* r = vec;
    double* z = vec + n;
    double* pa = vec + 2 * n;
    double* pb = vec + 3 * n;
    double* q = vec + 4 * n;
    double* x = K.x;
    const bool jac = K.jacobi != 0, linf = K.norm_inf != 0;
    const int64_t t0 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    bool ok = true;
    {
        double loc[2] = {0.0, 0.0};
        auto gx = [&](int64_t i) { return __ldcg(x + i); };
        for (int64_t c = t0; c < n; c += stride) {
            const double ax = rows.apply(c, __ldg(K.diag + c), gx);
            const double rk = __ldg(K.rhs + c) - ax;
            const double zk = inv_diag(K.diag, c, jac) * rk;
            __stcg(r + c, rk);
            __stcg(z + c, zk);
            __stcg(pa + c, 0.0);
            loc[0] = norm_acc(loc[0], rk, linf);
            loc[1] += rk * zk;
        }
        ok = grid_reduce<2, kCgThreads>(ctl, partials, loc, linf ? 1u : 0u);
        if (threadIdx.x == 0) {
            const double r0 = norm_fin(loc[0], linf);
            st.r0 = r0;
            st.final = r0;
            st.thresh = fmax(K.atol, K.rtol * r0);
            st.rz_old = loc[1];
            st.beta = 0.0;
            st.its = 0;
            st.converged = 0;
            st.status = GF_MAX_ITER;
            st.done = 0;
            if (r0 < st.thresh) {
                st.done = 1;
                st.converged = 1;
                st.status = GF_OK;
            } else if (!isfinite(r0)) {
                st.done = 1;
                st.status = GF_NONFINITE;
            }
        }
        __syncthreads();
    }
    double* p_old = pa;
    double* p_new = pb;
    for (int it = 1; ok && !st.done && it <= K.max_iter; ++it) {
        const double beta = st.beta;
        {  // p_new = z + p_old beta; q = A p_new; p_new . q
            double loc[1] = {0.0};
            auto gp = [&](int64_t i) { return __ldcg(z + i) + __ldcg(p_old + i) * beta; };
            // U cells per thread per pass: all loads of the U rows are issued
            // before any store, and loc accumulates in the U = 1 order.
            for (int64_t c0 = t0; c0 < n; c0 += U * stride) {
                double pc[U], ap[U];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int64_t c = c0 + u * stride;
                    if (c < n) pc[u] = gp(c);
                }
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int64_t c = c0 + u * stride;
                    if (c < n) ap[u] = rows.apply(c, __ldg(K.diag + c), gp);
                }
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int64_t c = c0 + u * stride;
                    if (c < n) {
                        __stcg(p_new + c, pc[u]);
                        __stcg(q + c, ap[u]);
                        loc[0] += pc[u] * ap[u];
                    }
                }
            }
            ok = grid_reduce<1, kCgThreads>(ctl, partials, loc, 0u);
            if (!ok) break;
            if (threadIdx.x == 0) st.alpha = st.rz_old / loc[0];
            __syncthreads();
        }
        {  // x += alpha p; r -= alpha q; z = M r; |r|, r.z
            const double alpha = st.alpha;
            double loc[2] = {0.0, 0.0};
            for (int64_t c0 = t0; c0 < n; c0 += U * stride) {
                double pc[U], xo[U], ro[U], qo[U], dg[U];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int64_t c = c0 + u * stride;
                    if (c < n) {
                        pc[u] = __ldcg(p_new + c);
                        xo[u] = __ldcg(x + c);
                        ro[u] = __ldcg(r + c);
                        qo[u] = __ldcg(q + c);
                        dg[u] = inv_diag(K.diag, c, jac);
                    }
                }
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int64_t c = c0 + u * stride;
                    if (c < n) {
                        __stcg(x + c, xo[u] + alpha * pc[u]);
                        const double rk = ro[u] - alpha * qo[u];
                        const double zk = dg[u] * rk;
                        __stcg(r + c, rk);
                        __stcg(z + c, zk);
                        loc[0] = norm_acc(loc[0], rk, linf);
                        loc[1] += rk * zk;
                    }
                }
            }
            ok = grid_reduce<2, kCgThreads>(ctl, partials, loc, linf ? 1u : 0u);
            if (!ok) break;
            if (threadIdx.x == 0) {
                const double fin = norm_fin(loc[0], linf);
                st.final = fin;
                if (fin < st.thresh) {
                    st.done = 1;
                    st.converged = 1;
                    st.its = it;
                    st.status = GF_OK;
                } else if (!isfinite(fin)) {
                    st.done = 1;
                    st.its = it;
                    st.status = GF_NONFINITE;
                } else {
                    st.beta = loc[1] / st.rz_old;
                    st.rz_old = loc[1];
                }
            }
            __syncthreads();
        }
        double* tmp = p_old;
        p_old = p_new;
        p_new = tmp;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        double* o = K.stats;
        o[0] = st.r0;
        o[1] = st.final;
        o[2] = st.done ? st.its : K.max_iter;
        o[3] = st.converged;
        o[4] = ok ? st.status : GF_ERR_TIMEOUT;
    }
}

template <int WIDTH>
__global__ void __launch_bounds__(kCgThreads, 4) k_pcg1(gf_krylov_t K) {
    EllRows<double, WIDTH> rows{K.val, K.nbr, K.n, K.width};
    pcg1_body<1>(K, rows);
}

// Box kernels come in tuning variants: MINB resident blocks per SM (the
// register budget follows from it) and U cells per thread per pass.
template <bool SYM, int MINB, int U>
__global__ void __launch_bounds__(kCgThreads, MINB) k_pcg1_box(gf_krylov_t K) {
    BoxRows<double, SYM, false> rows{K.val, K.n, K.stride_y, K.stride_z};
    pcg1_body<U>(K, rows);
}

// Mixed precision: FP32 inner Jacobi-PCG cycles inside FP64 iterative
// refinement.  Each cycle starts from the true FP64 residual r = b - A x
// (also the stopping test, |r| < max(atol, rtol |r0|) as in FP64), runs
// FP32 CG on A d = r with FP64-accumulated dot products until the recurrence
// residual falls below max(eta |r|, thresh / 2), then folds x += d in FP64.
// The FP32 copy of the matrix coefficients (all ELL slots, or the three "+"
// slots of a symmetric box) is made once per solve.
constexpr int kMaxEll = 32;

template <int U, class Rows64, class Rows32>
__device__ void pcg1_mixed_body(const gf_krylov_t& K, const Rows64& rows64, Rows32 rows32, int ncoef) {
    __shared__ CgState st;
    __shared__ double s_target;
    __shared__ int s_cycle_done;
    KCtl* ctl = reinterpret_cast<KCtl*>(K.work);
    double* partials = K.work + kCtlDoubles;
    double* base = partials + kMaxBlocks * kMaxNV;
    const int64_t n = K.n;
    float* f = reinterpret_cast<float*>(base + n);
    float* val32 = f;
    float* diag32 = f + (int64_t)ncoef * n;
    float* inv32 = diag32 + n;
    float* r = inv32 + n;
    float* z = r + n;
    float* pa = z + n;
    float* pb = pa + n;
    float* q = pb + n;
    float* d = q + n;
    double* x = K.x;
    const bool jac = K.jacobi != 0, linf = K.norm_inf != 0;
    const int64_t t0 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const bool sym_box = K.stride_y > 0 && K.symmetric;
    bool ok = true;
    int its = 0;
    rows32.val = val32;

    for (int64_t c = t0; c < n; c += stride) {
        for (int s = 0; s < ncoef; ++s) {
            const int64_t src = sym_box ? (2 * s + 1) : s;
            __stcg(val32 + s * n + c, (float)__ldg(K.val + src * n + c));
        }
        __stcg(diag32 + c, (float)__ldg(K.diag + c));
        __stcg(inv32 + c, (float)inv_diag(K.diag, c, jac));
    }
    if (threadIdx.x == 0) {
        st.its = 0;
        st.converged = 0;
        st.status = GF_MAX_ITER;
        st.done = 0;
    }
    bool pending = false;
    // max_outer inner cycles, each preceded by a true-residual evaluation,
    // plus a final evaluation that verifies the last correction.
    for (int cycle = 0; ok && cycle <= K.max_outer; ++cycle) {
        {  // fold the pending correction, then the true residual in FP64
            double loc[2] = {0.0, 0.0};
            if (pending) {
                for (int64_t c = t0; c < n; c += stride) __stcg(x + c, __ldcg(x + c) + (double)__ldcg(d + c));
                pending = false;
            }
            // The barrier also publishes the FP32 coefficients (cycle 0).
            double dummy[1] = {0.0};
            ok = grid_reduce<1, kCgThreads>(ctl, partials, dummy, 0u);
            if (!ok) break;
            auto gx = [&](int64_t i) { return __ldcg(x + i); };
            for (int64_t c = t0; c < n; c += stride) {
                const double ax = rows64.apply(c, __ldg(K.diag + c), gx);
                const double rk = __ldg(K.rhs + c) - ax;
                const float r32 = (float)rk;
                const float z32 = __ldcg(inv32 + c) * r32;
                __stcg(r + c, r32);
                __stcg(z + c, z32);
                __stcg(pa + c, 0.0f);
                __stcg(d + c, 0.0f);
                loc[0] = norm_acc(loc[0], rk, linf);
                loc[1] += (double)r32 * (double)z32;
            }
            ok = grid_reduce<2, kCgThreads>(ctl, partials, loc, linf ? 1u : 0u);
            if (!ok) break;
            if (threadIdx.x == 0) {
                const double nr = norm_fin(loc[0], linf);
                if (cycle == 0) {
                    st.r0 = nr;
                    st.thresh = fmax(K.atol, K.rtol * nr);
                }
                st.final = nr;
                if (nr < st.thresh) {
                    st.done = 1;
                    st.converged = 1;
                    st.status = GF_OK;
                } else if (!isfinite(nr)) {
                    st.done = 1;
                    st.status = GF_NONFINITE;
                }
                st.rz_old = loc[1];
                st.beta = 0.0;
                s_target = fmax(K.inner_eta * nr, 0.5 * st.thresh);
                s_cycle_done = 0;
            }
            __syncthreads();
            if (st.done || cycle == K.max_outer || its >= K.max_iter) break;
        }
        pending = true;
        float* p_old = pa;
        float* p_new = pb;
        while (ok && !s_cycle_done && its < K.max_iter) {
            ++its;
            const float beta = (float)st.beta;
            {
                double loc[1] = {0.0};
                auto gp = [&](int64_t i) { return __ldcg(z + i) + __ldcg(p_old + i) * beta; };
                for (int64_t c0 = t0; c0 < n; c0 += U * stride) {
                    float pc[U], ap[U];
#pragma unroll
                    for (int u = 0; u < U; ++u) {
                        const int64_t c = c0 + u * stride;
                        if (c < n) pc[u] = gp(c);
                    }
#pragma unroll
                    for (int u = 0; u < U; ++u) {
                        const int64_t c = c0 + u * stride;
                        if (c < n) ap[u] = rows32.apply(c, __ldcg(diag32 + c), gp);
                    }
#pragma unroll
                    for (int u = 0; u < U; ++u) {
                        const int64_t c = c0 + u * stride;
                        if (c < n) {
                            __stcg(p_new + c, pc[u]);
                            __stcg(q + c, ap[u]);
                            loc[0] += (double)pc[u] * (double)ap[u];
                        }
                    }
                }
                ok = grid_reduce<1, kCgThreads>(ctl, partials, loc, 0u);
                if (!ok) break;
                if (threadIdx.x == 0) st.alpha = st.rz_old / loc[0];
                __syncthreads();
            }
            {
                const float alpha = (float)st.alpha;
                double loc[2] = {0.0, 0.0};
                for (int64_t c0 = t0; c0 < n; c0 += U * stride) {
                    float pc[U], dd[U], ro[U], qo[U], iv[U];
#pragma unroll
                    for (int u = 0; u < U; ++u) {
                        const int64_t c = c0 + u * stride;
                        if (c < n) {
                            pc[u] = __ldcg(p_new + c);
                            dd[u] = __ldcg(d + c);
                            ro[u] = __ldcg(r + c);
                            qo[u] = __ldcg(q + c);
                            iv[u] = __ldcg(inv32 + c);
                        }
                    }
#pragma unroll
                    for (int u = 0; u < U; ++u) {
                        const int64_t c = c0 + u * stride;
                        if (c < n) {
                            __stcg(d + c, dd[u] + alpha * pc[u]);
                            const float rk = ro[u] - alpha * qo[u];
                            const float zk = iv[u] * rk;
                            __stcg(r + c, rk);
                            __stcg(z + c, zk);
                            loc[0] = norm_acc(loc[0], (double)rk, linf);
                            loc[1] += (double)rk * (double)zk;
                        }
                    }
                }
                ok = grid_reduce<2, kCgThreads>(ctl, partials, loc, linf ? 1u : 0u);
                if (!ok) break;
                if (threadIdx.x == 0) {
                    const double nr = norm_fin(loc[0], linf);
                    if (!(nr >= s_target) || !isfinite(nr)) {
                        s_cycle_done = 1;
                    } else {
                        st.beta = loc[1] / st.rz_old;
                        st.rz_old = loc[1];
                    }
                }
                __syncthreads();
            }
            float* tmp = p_old;
            p_old = p_new;
            p_new = tmp;
        }
    }
    if (ok && pending) {
        // iteration budget spent inside a cycle: keep its correction
        for (int64_t c = t0; c < n; c += stride) __stcg(x + c, __ldcg(x + c) + (double)__ldcg(d + c));
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        double* o = K.stats;
        o[0] = st.r0;
        o[1] = st.final;
        o[2] = its;
        o[3] = st.converged;
        o[4] = ok ? st.status : GF_ERR_TIMEOUT;
    }
}

template <int WIDTH>
__global__ void __launch_bounds__(kCgThreads, 4) k_pcg1_mixed(gf_krylov_t K) {
    EllRows<double, WIDTH> rows64{K.val, K.nbr, K.n, K.width};
    EllRows<float, WIDTH> rows32{nullptr, K.nbr, K.n, K.width};
    pcg1_mixed_body<1>(K, rows64, rows32, K.width);
}

template <bool SYM, int MINB, int U>
__global__ void __launch_bounds__(kCgThreads, MINB) k_pcg1_mixed_box(gf_krylov_t K) {
    BoxRows<double, SYM, false> rows64{K.val, K.n, K.stride_y, K.stride_z};
    BoxRows<float, SYM, SYM> rows32{nullptr, K.n, K.stride_y, K.stride_z};
    pcg1_mixed_body<U>(K, rows64, rows32, SYM ? 3 : 6);
}

// Tuning variants of the box kernels: {MINB, U}.
constexpr int kBoxVariants = 5;

template <bool MIXED, bool SYM>
static void* box_kernel(int variant) {
    switch (variant) {
        case 1:
            return MIXED ? (void*)k_pcg1_mixed_box<SYM, 4, 2> : (void*)k_pcg1_box<SYM, 4, 2>;
        case 2:
            return MIXED ? (void*)k_pcg1_mixed_box<SYM, 6, 1> : (void*)k_pcg1_box<SYM, 6, 1>;
        case 3:
            return MIXED ? (void*)k_pcg1_mixed_box<SYM, 8, 1> : (void*)k_pcg1_box<SYM, 8, 1>;
        case 4:
            return MIXED ? (void*)k_pcg1_mixed_box<SYM, 6, 2> : (void*)k_pcg1_box<SYM, 6, 2>;
        default:
            return MIXED ? (void*)k_pcg1_mixed_box<SYM, 4, 1> : (void*)k_pcg1_box<SYM, 4, 1>;
    }
}

// BiCGStab per-component modes.
enum { kDone = 0, kRun = 1, kRestart = 2, kIdle = 3, kConvS = 4 };

struct BiState {
    double thresh, r0, final, rho_old, alpha, omega, beta;
    int mode, restarts, its, converged, status;
};

__device__ __forceinline__ void breakdown(BiState& s, int it, int max_restart) {
    if (s.restarts >= max_restart) {
        s.mode = kDone;
        s.its = it;
        s.status = GF_BREAKDOWN;
    } else {
        s.restarts += 1;
        s.mode = kRestart;
    }
}

template <int NC>
__global__ void __launch_bounds__(kKThreads) k_bicgstab(gf_krylov_t K) {
    __shared__ BiState st[NC];
    __shared__ int s_any;
    KCtl* ctl = reinterpret_cast<KCtl*>(K.work);
    double* partials = K.work + kCtlDoubles;
    double* vec = partials + kMaxBlocks * kMaxNV;
    const int64_t n = K.n;
    double* r = vec;
    double* rh = vec + NC * n;
    double* p = vec + 2 * NC * n;
    double* v = vec + 3 * NC * n;
    double* s = vec + 4 * NC * n;
    double* t = vec + 5 * NC * n;
    double* x = K.x;
    const bool jac = K.jacobi != 0, linf = K.norm_inf != 0;
    const int64_t t0 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    bool ok = true;

    {  // r = b - A x; r_hat = p = r; |r|, r.r
        double loc[2 * NC];
#pragma unroll
        for (int j = 0; j < 2 * NC; ++j) loc[j] = 0.0;
        auto gx = [&](int k, int64_t i) { return __ldcg(x + k * n + i); };
        for (int64_t c = t0; c < n; c += stride) {
            double ax[NC];
            row_apply<NC>(K, c, gx, ax);
#pragma unroll
            for (int k = 0; k < NC; ++k) {
                const double rk = __ldg(K.rhs + k * n + c) - ax[k];
                __stcg(r + k * n + c, rk);
                __stcg(rh + k * n + c, rk);
                __stcg(p + k * n + c, rk);
                loc[k] = norm_acc(loc[k], rk, linf);
                loc[NC + k] += rk * rk;
            }
        }
        ok = grid_reduce<2 * NC>(ctl, partials, loc, linf ? ((1u << NC) - 1u) : 0u);
        if (threadIdx.x == 0) {
            for (int k = 0; k < NC; ++k) {
                BiState& b = st[k];
                const double r0 = norm_fin(loc[k], linf);
                b.r0 = r0;
                b.final = r0;
                b.thresh = fmax(K.atol, K.rtol * r0);
                b.rho_old = loc[NC + k];
                b.restarts = 0;
                b.its = 0;
                b.converged = 0;
                b.status = GF_MAX_ITER;
                b.mode = kRun;
                if (r0 < b.thresh) {
                    b.mode = kDone;
                    b.converged = 1;
                    b.status = GF_OK;
                } else if (!isfinite(r0)) {
                    b.mode = kDone;
                    b.status = GF_NONFINITE;
                }
            }
        }
        __syncthreads();
    }

    for (int it = 1; ok && it <= K.max_iter; ++it) {
        if (threadIdx.x == 0) {
            int any = 0;
            for (int k = 0; k < NC; ++k) {
                if (st[k].mode == kIdle) st[k].mode = kRun;
                any |= (st[k].mode == kRun);
            }
            s_any = any;
        }
        __syncthreads();
        if (!s_any) break;

        // P1: y = M p, v = A y; r_hat.v, |r_hat|^2, |v|^2
        {
            double loc[3 * NC];
#pragma unroll
            for (int j = 0; j < 3 * NC; ++j) loc[j] = 0.0;
            auto gy = [&](int k, int64_t i) { return inv_diag(K.diag, i, jac) * __ldcg(p + k * n + i); };
            for (int64_t c = t0; c < n; c += stride) {
                double av[NC];
                row_apply<NC>(K, c, gy, av);
#pragma unroll
                for (int k = 0; k < NC; ++k) {
                    if (st[k].mode != kRun) continue;
                    __stcg(v + k * n + c, av[k]);
                    const double h = __ldcg(rh + k * n + c);
                    loc[k] += h * av[k];
                    loc[NC + k] += h * h;
                    loc[2 * NC + k] += av[k] * av[k];
                }
            }
            ok = grid_reduce<3 * NC>(ctl, partials, loc, 0u);
            if (!ok) break;
            if (threadIdx.x == 0) {
                for (int k = 0; k < NC; ++k) {
                    BiState& b = st[k];
                    if (b.mode != kRun) continue;
                    const double da = loc[k];
                    if (fabs(da) <= 1e-6 * sqrt(loc[NC + k]) * sqrt(loc[2 * NC + k]))
                        breakdown(b, it, K.max_restart);
                    else
                        b.alpha = b.rho_old / da;
                }
            }
            __syncthreads();
        }
        // P2: s = r - alpha v, |s|; restarting systems copy r and reduce r.r
        {
            double loc[2 * NC];
#pragma unroll
            for (int j = 0; j < 2 * NC; ++j) loc[j] = 0.0;
            for (int64_t c = t0; c < n; c += stride) {
#pragma unroll
                for (int k = 0; k < NC; ++k) {
                    const int md = st[k].mode;
                    if (md == kRun) {
                        const double sk = __ldcg(r + k * n + c) - st[k].alpha * __ldcg(v + k * n + c);
                        __stcg(s + k * n + c, sk);
                        loc[k] = norm_acc(loc[k], sk, linf);
                    } else if (md == kRestart) {
                        const double rk = __ldcg(r + k * n + c);
                        __stcg(rh + k * n + c, rk);
                        __stcg(p + k * n + c, rk);
                        loc[NC + k] += rk * rk;
                    }
                }
            }
            ok = grid_reduce<2 * NC>(ctl, partials, loc, linf ? ((1u << NC) - 1u) : 0u);
            if (!ok) break;
            if (threadIdx.x == 0) {
                for (int k = 0; k < NC; ++k) {
                    BiState& b = st[k];
                    if (b.mode == kRestart) {
                        b.rho_old = loc[NC + k];
                        b.mode = kIdle;
                    } else if (b.mode == kRun) {
                        const double fin = norm_fin(loc[k], linf);
                        b.final = fin;
                        if (fin < b.thresh) {
                            b.mode = kConvS;
                            b.converged = 1;
                            b.its = it;
                            b.status = GF_OK;
                        } else if (!isfinite(fin)) {
                            b.mode = kDone;
                            b.its = it;
                            b.status = GF_NONFINITE;
                        }
                    }
                }
            }
            __syncthreads();
        }
        // P3: converged-on-s systems take x += alpha y; others z = M s, t = A z
        {
            double loc[2 * NC];
#pragma unroll
            for (int j = 0; j < 2 * NC; ++j) loc[j] = 0.0;
            auto gz = [&](int k, int64_t i) { return inv_diag(K.diag, i, jac) * __ldcg(s + k * n + i); };
            for (int64_t c = t0; c < n; c += stride) {
                double at[NC];
                row_apply<NC>(K, c, gz, at);
                const double ic = inv_diag(K.diag, c, jac);
#pragma unroll
                for (int k = 0; k < NC; ++k) {
                    const int md = st[k].mode;
                    if (md == kConvS) {
                        const double y = ic * __ldcg(p + k * n + c);
                        __stcg(x + k * n + c, __ldcg(x + k * n + c) + st[k].alpha * y);
                    } else if (md == kRun) {
                        __stcg(t + k * n + c, at[k]);
                        loc[k] += at[k] * at[k];
                        loc[NC + k] += at[k] * __ldcg(s + k * n + c);
                    }
                }
            }
            ok = grid_reduce<2 * NC>(ctl, partials, loc, 0u);
            if (!ok) break;
            if (threadIdx.x == 0) {
                for (int k = 0; k < NC; ++k) {
                    BiState& b = st[k];
                    if (b.mode == kConvS) {
                        b.mode = kDone;
                        continue;
                    }
                    if (b.mode != kRun) continue;
                    const double dd = loc[k];
                    const double tn = sqrt(loc[k]);
                    if (fabs(dd) <= 1e-6 * tn * tn) {
                        breakdown(b, it, K.max_restart);
                        continue;
                    }
                    b.omega = loc[NC + k] / dd;
                    if (fabs(b.omega) <= 1e-6) breakdown(b, it, K.max_restart);
                }
            }
            __syncthreads();
        }
        // P4: x += alpha y + omega z, r = s - omega t; |r|, r_hat.r, |r_hat|^2, |r|^2
        {
            double loc[4 * NC];
#pragma unroll
            for (int j = 0; j < 4 * NC; ++j) loc[j] = 0.0;
            for (int64_t c = t0; c < n; c += stride) {
                const double ic = inv_diag(K.diag, c, jac);
#pragma unroll
                for (int k = 0; k < NC; ++k) {
                    const int md = st[k].mode;
                    if (md == kRun) {
                        const double sk = __ldcg(s + k * n + c);
                        const double y = ic * __ldcg(p + k * n + c);
                        const double z = ic * sk;
                        __stcg(x + k * n + c, __ldcg(x + k * n + c) + st[k].alpha * y + st[k].omega * z);
                        const double rk = sk - st[k].omega * __ldcg(t + k * n + c);
                        __stcg(r + k * n + c, rk);
                        const double h = __ldcg(rh + k * n + c);
                        loc[k] = norm_acc(loc[k], rk, linf);
                        loc[NC + k] += h * rk;
                        loc[2 * NC + k] += h * h;
                        loc[3 * NC + k] += rk * rk;
                    } else if (md == kRestart) {
                        const double rk = __ldcg(r + k * n + c);
                        __stcg(rh + k * n + c, rk);
                        __stcg(p + k * n + c, rk);
                        loc[3 * NC + k] += rk * rk;
                    }
                }
            }
            ok = grid_reduce<4 * NC>(ctl, partials, loc, linf ? ((1u << NC) - 1u) : 0u);
            if (!ok) break;
            if (threadIdx.x == 0) {
                for (int k = 0; k < NC; ++k) {
                    BiState& b = st[k];
                    if (b.mode == kRestart) {
                        b.rho_old = loc[3 * NC + k];
                        b.mode = kIdle;
                        continue;
                    }
                    if (b.mode != kRun) continue;
                    const double fin = norm_fin(loc[k], linf);
                    b.final = fin;
                    if (fin < b.thresh) {
                        b.mode = kDone;
                        b.converged = 1;
                        b.its = it;
                        b.status = GF_OK;
                        continue;
                    }
                    if (!isfinite(fin)) {
                        b.mode = kDone;
                        b.its = it;
                        b.status = GF_NONFINITE;
                        continue;
                    }
                    const double rho_new = loc[NC + k];
                    if (fabs(rho_new) <= 1e-6 * sqrt(loc[2 * NC + k]) * sqrt(loc[3 * NC + k])) {
                        breakdown(b, it, K.max_restart);
                        continue;
                    }
                    b.beta = (rho_new / b.rho_old) * (b.alpha / b.omega);
                    b.rho_old = rho_new;
                }
            }
            __syncthreads();
        }
        // P5: p = r + beta (p - omega v); restarting systems copy r
        {
            double loc[NC];
#pragma unroll
            for (int k = 0; k < NC; ++k) loc[k] = 0.0;
            for (int64_t c = t0; c < n; c += stride) {
#pragma unroll
                for (int k = 0; k < NC; ++k) {
                    const int md = st[k].mode;
                    if (md == kRun) {
                        const double pk = __ldcg(p + k * n + c);
                        __stcg(p + k * n + c,
                               __ldcg(r + k * n + c) + st[k].beta * (pk - st[k].omega * __ldcg(v + k * n + c)));
                    } else if (md == kRestart) {
                        const double rk = __ldcg(r + k * n + c);
                        __stcg(rh + k * n + c, rk);
                        __stcg(p + k * n + c, rk);
                        loc[k] += rk * rk;
                    }
                }
            }
            ok = grid_reduce<NC>(ctl, partials, loc, 0u);
            if (!ok) break;
            if (threadIdx.x == 0) {
                for (int k = 0; k < NC; ++k) {
                    if (st[k].mode == kRestart) {
                        st[k].rho_old = loc[k];
                        st[k].mode = kIdle;
                    }
                }
            }
            __syncthreads();
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        for (int k = 0; k < NC; ++k) {
            double* o = K.stats + 5 * k;
            const bool fin = st[k].mode == kDone;
            o[0] = st[k].r0;
            o[1] = st[k].final;
            o[2] = fin ? st[k].its : K.max_iter;
            o[3] = st[k].converged;
            o[4] = ok ? (fin ? st[k].status : GF_MAX_ITER) : GF_ERR_TIMEOUT;
        }
    }
}

template <class Kern>
static int launch_persistent(Kern kern, const gf_krylov_t* k, void* stream, const char* what,
                             int threads = kKThreads, int unroll = 1) {
    int dev = 0;
    cudaGetDevice(&dev);
    int sms = 0, coop = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
    if (!coop) {
        set_error("%s: device does not support cooperative launch", what);
        return GF_ERR_CUDA;
    }
    int per_sm = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)kern, threads, 0);
    if (e != cudaSuccess || per_sm < 1) {
        set_error("%s: occupancy query failed: %s", what, cudaGetErrorString(e));
        return GF_ERR_CUDA;
    }
    int64_t want = (k->n + threads - 1) / threads;
    if (unroll > 1) want = (want + unroll - 1) / unroll;
    int64_t cap = (int64_t)per_sm * sms;
    if (cap > kMaxBlocks) cap = kMaxBlocks;
    if (k->block_cap > 0 && k->block_cap < cap) cap = k->block_cap;
    int grid = (int)(want < cap ? want : cap);
    if (grid < 1) grid = 1;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    e = cudaMemsetAsync(k->work, 0, sizeof(KCtl), s);
    if (e != cudaSuccess) {
        set_error("%s: %s", what, cudaGetErrorString(e));
        return GF_ERR_CUDA;
    }
    gf_krylov_t arg = *k;
    void* args[] = {&arg};
    e = cudaLaunchCooperativeKernel((const void*)kern, dim3(grid), dim3(threads), args, 0, s);
    if (e != cudaSuccess) {
        set_error("%s: cooperative launch failed: %s", what, cudaGetErrorString(e));
        return GF_ERR_CUDA;
    }
    return GF_OK;
}

static bool valid_krylov(const gf_krylov_t* k, int nvec, const char* what) {
    if (k == nullptr || k->n <= 0 || k->width <= 0 || k->ncomp < 1 || k->ncomp > 3 || k->nbr == nullptr ||
        k->diag == nullptr || k->val == nullptr || k->rhs == nullptr || k->x == nullptr || k->work == nullptr ||
        k->stats == nullptr || k->max_iter < 0) {
        set_error("%s: invalid arguments", what);
        return false;
    }
    const int64_t need = kCtlDoubles + (int64_t)kMaxBlocks * kMaxNV + (int64_t)nvec * k->ncomp * k->n;
    if (k->work_len < need) {
        set_error("%s: workspace holds %lld doubles, %lld needed", what, (long long)k->work_len, (long long)need);
        return false;
    }
    if (k->n * (int64_t)k->width > 2147483647LL) {
        set_error("%s: system too large", what);
        return false;
    }
    return true;
}

}  // namespace gf

using namespace gf;

extern "C" {

int64_t gf_krylov_workspace_size(int64_t n, int32_t ncomp, int32_t kind) {
    // kind 2 + 100 * width: mixed-precision CG for an ELL of that width.
    if (kind >= 2) {
        const int64_t width = (kind - 2) / 100 > 0 ? (kind - 2) / 100 : kMaxEll;
        const int64_t floats = (width + 8) * n;
        return kCtlDoubles + (int64_t)kMaxBlocks * kMaxNV + n + (floats + 1) / 2 + 1;
    }
    const int bicgstab = kind == 1;
    const int nvec = bicgstab ? 6 : (ncomp == 1 ? 5 : 3);
    return kCtlDoubles + (int64_t)kMaxBlocks * kMaxNV + (int64_t)nvec * ncomp * n;
}

int gf_pcg_solve(const gf_krylov_t* k, void* stream) {
    if (k == nullptr) {
        set_error("gf_pcg_solve: invalid arguments (null descriptor)");
        return GF_ERR_INVALID;
    }
    const bool box = k->stride_y > 0;
    if (box && (k->width != 6 || k->stride_z < k->stride_y || k->stride_y < 1)) {
        set_error("gf_pcg_solve: a box layout needs width 6 and strides 1 <= stride_y <= stride_z");
        return GF_ERR_INVALID;
    }
    if (k->mixed) {
        if (k->ncomp != 1 || k->max_outer < 1 || k->width > kMaxEll) {
            set_error("gf_pcg_solve: mixed precision needs one system, max_outer >= 1, width <= %d", kMaxEll);
            return GF_ERR_INVALID;
        }
        if (!valid_krylov(k, 0, "gf_pcg_solve")) return GF_ERR_INVALID;
        const int64_t need = gf_krylov_workspace_size(k->n, 1, 2 + 100 * k->width);
        if (k->work_len < need) {
            set_error("gf_pcg_solve: mixed workspace holds %lld doubles, %lld needed", (long long)k->work_len,
                      (long long)need);
            return GF_ERR_INVALID;
        }
        if (box) {
            const int v = (k->variant >= 0 && k->variant < kBoxVariants) ? k->variant : 0;
            void* kern = k->symmetric ? box_kernel<true, true>(v) : box_kernel<true, false>(v);
            return launch_persistent(kern, k, stream, "gf_pcg_solve", kCgThreads, (v == 1 || v == 4) ? 2 : 1);
        }
        if (k->width == 6) return launch_persistent(k_pcg1_mixed<6>, k, stream, "gf_pcg_solve", kCgThreads);
        return launch_persistent(k_pcg1_mixed<0>, k, stream, "gf_pcg_solve", kCgThreads);
    }
    if (!valid_krylov(k, k->ncomp == 1 ? 5 : 3, "gf_pcg_solve")) return GF_ERR_INVALID;
    switch (k->ncomp) {
        case 1:
            if (box) {
                const int v = (k->variant >= 0 && k->variant < kBoxVariants) ? k->variant : 0;
                void* kern = k->symmetric ? box_kernel<false, true>(v) : box_kernel<false, false>(v);
                return launch_persistent(kern, k, stream, "gf_pcg_solve", kCgThreads, (v == 1 || v == 4) ? 2 : 1);
            }
            if (k->width == 6) return launch_persistent(k_pcg1<6>, k, stream, "gf_pcg_solve", kCgThreads);
            return launch_persistent(k_pcg1<0>, k, stream, "gf_pcg_solve", kCgThreads);
        case 2:
            return launch_persistent(k_pcg<2>, k, stream, "gf_pcg_solve");
        default:
            return launch_persistent(k_pcg<3>, k, stream, "gf_pcg_solve");
    }
}

int gf_bicgstab_solve(const gf_krylov_t* k, void* stream) {
    if (!valid_krylov(k, 6, "gf_bicgstab_solve")) return GF_ERR_INVALID;
    switch (k->ncomp) {
        case 1:
            return launch_persistent(k_bicgstab<1>, k, stream, "gf_bicgstab_solve");
        case 2:
            return launch_persistent(k_bicgstab<2>, k, stream, "gf_bicgstab_solve");
        default:
            return launch_persistent(k_bicgstab<3>, k, stream, "gf_bicgstab_solve");
    }
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free CG entry point.
//
// Some callers cannot allocate device memory at solve time: a host
// framework that has already reserved the device pool for its own caching
// allocator (so a raw cudaMalloc would fail or fragment it), or a serving
// loop that must not allocate after start-up to keep its latency and memory
// footprint fixed.  gf_pcg_solve_static runs the same persistent CG as
// gf_pcg_solve, but its scratch (barrier control block, block partials and
// Krylov vectors) lives in the file-scope device array below instead of a
// caller workspace.  Every GPU that loads this library holds that array
// until the process exits.
// ---------------------------------------------------------------------------
namespace gf {

// One FP64 system of up to 262,144 cells (10.1 MiB).
constexpr int64_t kStaticScratchCells = 262144;
constexpr int64_t kStaticScratchDoubles =
    kCtlDoubles + (int64_t)kMaxBlocks * kMaxNV + 5 * kStaticScratchCells;

static __device__ __align__(256) double g_static_scratch[kStaticScratchDoubles];

constexpr int kMaxDevices = 128;
static std::mutex g_static_mutex;
static double* g_static_addr[kMaxDevices] = {};

// Device address of g_static_scratch on the current device.  In host code
// the array's name is only a host-side stand-in, so the address is looked
// up once per device (with that device current) and cached.
static int static_scratch(double** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        set_error("gf_pcg_solve_static: cudaGetDevice failed: %s", cudaGetErrorString(e));
        return GF_ERR_CUDA;
    }
    if (dev < 0 || dev >= kMaxDevices) {
        set_error("gf_pcg_solve_static: device ordinal %d out of range", dev);
        return GF_ERR_INVALID;
    }
    std::lock_guard<std::mutex> lock(g_static_mutex);
    if (g_static_addr[dev] == nullptr) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_static_scratch);
        if (e != cudaSuccess || p == nullptr) {
            set_error("gf_pcg_solve_static: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
            return GF_ERR_CUDA;
        }
        g_static_addr[dev] = static_cast<double*>(p);
    }
    *out = g_static_addr[dev];
    return GF_OK;
}

}  // namespace gf

extern "C" {

int64_t gf_pcg_static_scratch_doubles(void) { return kStaticScratchDoubles; }

int gf_pcg_solve_static(const gf_krylov_t* k, void* stream) {
    if (k == nullptr) {
        set_error("gf_pcg_solve_static: invalid arguments (null descriptor)");
        return GF_ERR_INVALID;
    }
    const int32_t kind = k->mixed ? 2 + 100 * k->width : 0;
    const int64_t need = gf_krylov_workspace_size(k->n, k->ncomp, kind);
    if (k->n <= 0 || need > kStaticScratchDoubles) {
        set_error("gf_pcg_solve_static: the system needs %lld scratch doubles but the static scratch holds "
                  "%lld (at most %lld cells for one FP64 system); use gf_pcg_solve with a caller workspace",
                  (long long)need, (long long)kStaticScratchDoubles, (long long)kStaticScratchCells);
        return GF_ERR_INVALID;
    }
    double* scratch = nullptr;
    const int st = static_scratch(&scratch);
    if (st != GF_OK) return st;
    gf_krylov_t local = *k;
    local.work = scratch;
    local.work_len = kStaticScratchDoubles;
    // gf_pcg_solve clears the barrier control block before its launch; the
    // partials and vectors are written before they are read.
    return gf_pcg_solve(&local, stream);
}

}  // extern "C"
