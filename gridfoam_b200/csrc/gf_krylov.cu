// Persistent cooperative Krylov solvers (sm_100a).
//
// One launch runs a whole solve (all iterations, up to three right-hand
// sides sharing the matrix).  Blocks synchronise through a grid barrier that
// also finishes every dot product: each block writes its partial sums,
// arrives on a monotonic counter, and once every block has arrived each
// block reduces all partials itself in one fixed order, so every block gets
// the same bitwise-reproducible value without a second publish step.  Every
// wait is bounded; on expiry the kernel raises an error flag and returns
// instead of hanging.  The launch is cooperative, so all blocks are
// co-resident and the barrier is always reachable.
#include "gf_common.cuh"

#include <cstdlib>
#include <cstring>
#include <mutex>

namespace gf {

constexpr int kKThreads = 512;
constexpr int kCgThreads = 256;
constexpr int kMaxBlocks = 1024;
constexpr int kMaxNV = 16;
constexpr int kCtlDoubles = 32;
constexpr long long kSpinLimit = 30000000LL;  // x ~40 ns polls: about a second
// Slots of a runtime-width matrix row whose loads are issued together.
constexpr int kSlotGroup = 8;

// Partial sums are double-buffered by barrier parity: a block may write the
// next barrier's partials while a slower block still reads this one's, but
// not the one after (that needs the slow block's arrival).
constexpr int64_t kPartials = 2LL * kMaxBlocks * kMaxNV;
constexpr int64_t kHeader = kCtlDoubles + kPartials;

struct KCtl {
    unsigned long long count;  // barrier arrivals since launch (zeroed per launch)
    int error;
    int pad;
};

// Barriers this block has passed since the kernel started, and the poll
// limit of every bounded wait of this launch; barrier_init() must run at the
// top of every kernel that waits on other blocks.
// g_nblk / g_bid: the blocks taking part in this solve's reductions and
// this block's index among them (the whole grid, or one system's share of a
// batched launch).
__shared__ unsigned g_epoch;
__shared__ long long g_spin;
__shared__ int g_nblk, g_bid;

__device__ __forceinline__ void barrier_init_v(const gf_krylov_t& K, int nblk, int bid) {
    if (threadIdx.x == 0) {
        g_epoch = 0;
        g_spin = K.spin_limit > 0 ? K.spin_limit : kSpinLimit;
        g_nblk = nblk;
        g_bid = bid;
    }
}

__device__ __forceinline__ void barrier_init(const gf_krylov_t& K) {
    barrier_init_v(K, (int)gridDim.x, (int)blockIdx.x);
}

__device__ __forceinline__ int vload(const int* p) { return *(const volatile int*)p; }

// Release-add / acquire-load pair of the grid barrier (the CTA barrier
// before the add makes it cumulative over the whole block's writes).
__device__ __forceinline__ void arrive_release(unsigned long long* p) {
    asm volatile("fence.acq_rel.gpu;\n\tred.relaxed.gpu.global.add.u64 [%0], 1;" ::"l"(p) : "memory");
}

__device__ __forceinline__ unsigned long long load_acquire(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

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
// barrier wait expired or another block reported an error.  Every block
// sums the per-block partials in the same fixed order, so all blocks hold
// the same bits.  The cost is in the CTA barriers, the shuffle trees and
// the L2 round trips; an empty reduction of 148 x 1024 threads measured
// 2.26 / 2.83 / 3.42 us (NV = 1 / 2 / 3) with grid_reduce_all and 2.07 /
// 2.75 us (NV = 1 / 3) with grid_reduce_w0, against 1.33 us for the bare
// counter barrier.
constexpr int kW0Loads = 5;
constexpr int kW0Blocks = 32 * kW0Loads;

__device__ __forceinline__ double comb(double x, double y, bool mx) { return mx ? nmax(x, y) : x + y; }

// Staging of the partials in grid_reduce_w0 (warp 0 only, between its wait
// and the CTA barrier that ends the reduction).
__shared__ __align__(16) double g_stage[3 * kW0Blocks + 2];

// Reduction scratch, one per NV, shared by the two forms.
template <int NV>
struct RedBuf {
    double sm1[NV * 32];
    double sm2[NV * 32];
    int err;
};
template <int NV>
__device__ __forceinline__ RedBuf<NV>& red_buf() {
    __shared__ RedBuf<NV> b;
    return b;
}

// All threads load the partials: the general form (any block size, any
// grid, any NV).
template <int NV, int THREADS>
__device__ bool grid_reduce_all(KCtl* ctl, double* partials, double (&v)[NV], unsigned maxmask) {
    RedBuf<NV>& rb = red_buf<NV>();
    double* sm1 = rb.sm1;
    double* sm2 = rb.sm2;
    int& s_err = rb.err;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int j = 0; j < NV; ++j) {
        const bool mx = (maxmask >> j) & 1u;
        double x = v[j];
        for (int o = 16; o > 0; o >>= 1) {
            const double y = __shfl_xor_sync(0xffffffffu, x, o);
            x = mx ? nmax(x, y) : x + y;
        }
        if (lane == 0) sm1[j * 32 + warp] = x;
    }
    __syncthreads();
    const unsigned ep = g_epoch;
    double* part = partials + (ep & 1u) * (kPartials / 2);
    if (THREADS == 1024) {
        // 32 warp sums: a shuffle tree in warp 0 is shorter than a serial sum.
        if (warp == 0) {
#pragma unroll
            for (int j = 0; j < NV; ++j) {
                const bool mx = (maxmask >> j) & 1u;
                double x = sm1[j * 32 + lane];
                for (int o = 16; o > 0; o >>= 1) {
                    const double y = __shfl_xor_sync(0xffffffffu, x, o);
                    x = mx ? nmax(x, y) : x + y;
                }
                if (lane == 0) __stcg(part + (int64_t)g_bid * NV + j, x);
            }
        }
    } else if (threadIdx.x < NV) {
        const int j = threadIdx.x;
        const bool mx = (maxmask >> j) & 1u;
        double x = sm1[j * 32];
        for (int w = 1; w < nw; ++w) x = mx ? nmax(x, sm1[j * 32 + w]) : x + sm1[j * 32 + w];
        __stcg(part + (int64_t)g_bid * NV + j, x);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        arrive_release(&ctl->count);
        const unsigned long long target = (unsigned long long)(ep + 1u) * (unsigned)g_nblk;
        int err = 0;
        long long it = 0;
        while (load_acquire(&ctl->count) < target) {
            __nanosleep(20);
            ++it;
            if ((it & 255) == 0 && vload(&ctl->error) != 0) {
                err = 1;
                break;
            }
            if (it > g_spin) {
                atomicExch(&ctl->error, 1);
                err = 1;
                break;
            }
        }
        // A block that gave up raised the flag; the others see it at their
        // next wait (checked every 256 polls) and leave as well.
        s_err = err;
        g_epoch = ep + 1u;
    }
    __syncthreads();
    if (s_err) return false;
    // Every thread loads its (at most kMaxBlocks / THREADS) partials of each
    // value at once, then a fixed-order block reduction: one L2 round trip,
    // and every block computes the same bits.
    double acc[NV];
#pragma unroll
    for (int j = 0; j < NV; ++j) acc[j] = 0.0;
    constexpr int kPer = (kMaxBlocks + THREADS - 1) / THREADS;
#pragma unroll
    for (int i = 0; i < kPer; ++i) {
        const int b = threadIdx.x + i * blockDim.x;
#pragma unroll
        for (int j = 0; j < NV; ++j) {
            const bool mx = (maxmask >> j) & 1u;
            const double y = b < g_nblk ? __ldcg(part + (int64_t)b * NV + j) : 0.0;
            acc[j] = mx ? nmax(acc[j], y) : acc[j] + y;
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
        if (lane == 0) sm2[j * 32 + warp] = x;
    }
    __syncthreads();
    // sm2 is next written after the first CTA barrier of the next call, and
    // sm1 is next read after the second: no trailing barrier is needed.
#pragma unroll
    for (int j = 0; j < NV; ++j) {
        const bool mx = (maxmask >> j) & 1u;
        double x;
        if (THREADS == 1024) {
            // Every warp runs the same butterfly; its additions commute
            // exactly, so all lanes of all warps hold the same bits.
            x = sm2[j * 32 + lane];
            for (int o = 16; o > 0; o >>= 1) {
                const double t = __shfl_xor_sync(0xffffffffu, x, o);
                x = mx ? nmax(x, t) : x + t;
            }
        } else {
            x = sm2[j * 32];
            for (int w = 1; w < nw; ++w) x = mx ? nmax(x, sm2[j * 32 + w]) : x + sm2[j * 32 + w];
        }
        v[j] = x;
    }
    return true;
}

// 1024-thread blocks on grids of at most kW0Blocks (one block an SM) and a
// 16-byte aligned workspace: one warp on the critical path after the warp
// sums.  Warp 0 forms the block partial, thread 0 publishes it, warp 0
// waits, copies every partial to shared memory with all copies in flight
// and sums them in a fixed order; a second CTA barrier hands the result out
// (grid_reduce_all: four CTA barriers, and every warp runs two more shuffle
// trees).  The shuffle trees of the NV values are interleaved level by
// level.
//
// SIDE(t, nt) runs on the other 31 warps (t = threadIdx.x - 32 of nt =
// blockDim.x - 32) while warp 0 waits for the grid: block-local work that
// needs neither the reduction's result nor other blocks' data.
struct NoSide {
    __device__ __forceinline__ void operator()(int, int) const {}
};

template <int NV, class SIDE = NoSide>
__device__ bool grid_reduce_w0(KCtl* ctl, double* partials, double (&v)[NV], unsigned maxmask,
                               const SIDE& side = SIDE()) {
    RedBuf<NV>& rb = red_buf<NV>();
    double* sm1 = rb.sm1;
    double* sm2 = rb.sm2;
    int& s_err = rb.err;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    double x[NV];
#pragma unroll
    for (int j = 0; j < NV; ++j) x[j] = v[j];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
        for (int j = 0; j < NV; ++j) x[j] = comb(x[j], __shfl_xor_sync(0xffffffffu, x[j], o), (maxmask >> j) & 1u);
    if (lane == 0)
#pragma unroll
        for (int j = 0; j < NV; ++j) sm1[j * 32 + warp] = x[j];
    __syncthreads();
    if (warp == 0) {
        // Only warp 0 uses the epoch; lane 0 reads it (after the CTA barrier
        // that follows barrier_init) and advances it after its wait.
        const unsigned ep = __shfl_sync(0xffffffffu, lane == 0 ? g_epoch : 0u, 0);
        double* part = partials + (ep & 1u) * (kPartials / 2);
        // Block partial (0 is the identity of both: the max values are norms).
#pragma unroll
        for (int j = 0; j < NV; ++j) x[j] = lane < nw ? sm1[j * 32 + lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
#pragma unroll
            for (int j = 0; j < NV; ++j)
                x[j] = comb(x[j], __shfl_xor_sync(0xffffffffu, x[j], o), (maxmask >> j) & 1u);
        if (lane == 0) {
#pragma unroll
            for (int j = 0; j < NV; ++j) __stcg(part + (int64_t)g_bid * NV + j, x[j]);
            // The CTA barrier above orders the other warps' writes before
            // this release (cumulativity).
            arrive_release(&ctl->count);
        }
        __syncwarp();
        {
            // The whole warp polls (one request a poll).  Lane 0 polling
            // alone with __nanosleep while the other lanes waited at a warp
            // barrier left the blocks microseconds apart on leaving (CG
            // iterations 40-60 % slower).
            const unsigned long long target = (unsigned long long)(ep + 1u) * (unsigned)g_nblk;
            int err = 0;
            long long it = 0;
            while (true) {
                const unsigned long long c = load_acquire(&ctl->count);
                if (__all_sync(0xffffffffu, c >= target)) break;
                __nanosleep(20);
                ++it;
                if ((it & 255) == 0 && __any_sync(0xffffffffu, vload(&ctl->error) != 0)) {
                    err = 1;
                    break;
                }
                if (it > g_spin) {
                    if (lane == 0) atomicExch(&ctl->error, 1);
                    err = 1;
                    break;
                }
            }
            // A block that gave up raised the flag; the others see it at
            // their next wait (checked every 256 polls) and leave as well.
            if (lane == 0) {
                s_err = err;
                g_epoch = ep + 1u;
            }
        }
        __syncwarp();
        if (!s_err) {
            // All partials in flight at once through 16-byte L2 copies into
            // shared memory (register loads would be serialised in the
            // register-capped CG kernels).  The last copy may read one
            // double past the partials, inside the same half.
            const int nd = g_nblk * NV;
            for (int q = lane; 2 * q < nd; q += 32) {
                const unsigned dst = (unsigned)__cvta_generic_to_shared(g_stage + 2 * q);
                asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(part + 2 * q) : "memory");
            }
            asm volatile("cp.async.commit_group;\n\tcp.async.wait_all;" ::: "memory");
            __syncwarp();
#pragma unroll
            for (int j = 0; j < NV; ++j) x[j] = lane < g_nblk ? g_stage[lane * NV + j] : 0.0;
#pragma unroll
            for (int k = 1; k < kW0Loads; ++k) {
                const int b = lane + 32 * k;
                if (b < g_nblk)
#pragma unroll
                    for (int j = 0; j < NV; ++j) x[j] = comb(x[j], g_stage[b * NV + j], (maxmask >> j) & 1u);
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1)
#pragma unroll
                for (int j = 0; j < NV; ++j)
                    x[j] = comb(x[j], __shfl_xor_sync(0xffffffffu, x[j], o), (maxmask >> j) & 1u);
            if (lane == 0)
#pragma unroll
                for (int j = 0; j < NV; ++j) sm2[j] = x[j];
        }
    } else {
        side((int)threadIdx.x - 32, (int)blockDim.x - 32);
    }
    __syncthreads();
    // No trailing barrier: sm1 is read only before the barrier above (the
    // next call writes it before its first one), and sm2 is next written
    // after the next call's first barrier, which every thread reaches only
    // after reading it here.
    if (s_err) return false;
#pragma unroll
    for (int j = 0; j < NV; ++j) v[j] = sm2[j];
    return true;
}

// With side work (see grid_reduce_w0); the general form runs it first on
// every thread.
template <int NV, int THREADS, class SIDE>
__device__ __forceinline__ bool grid_reduce_side(KCtl* ctl, double* partials, double (&v)[NV], unsigned maxmask,
                                                 const SIDE& side) {
    if constexpr (THREADS == 1024 && NV <= 3) {
        if (gridDim.x <= (unsigned)kW0Blocks && (reinterpret_cast<uintptr_t>(partials) & 15u) == 0)
            return grid_reduce_w0<NV>(ctl, partials, v, maxmask, side);
    }
    side((int)threadIdx.x, (int)blockDim.x);
    return grid_reduce_all<NV, THREADS>(ctl, partials, v, maxmask);
}

template <int NV, int THREADS = kKThreads>
__device__ __forceinline__ bool grid_reduce(KCtl* ctl, double* partials, double (&v)[NV], unsigned maxmask) {
    if constexpr (THREADS == 1024 && NV <= 3) {
        // (the 16-byte copies of the partials need a 16-byte aligned workspace)
        if (gridDim.x <= (unsigned)kW0Blocks && (reinterpret_cast<uintptr_t>(partials) & 15u) == 0)
            return grid_reduce_w0<NV>(ctl, partials, v, maxmask);
    }
    return grid_reduce_all<NV, THREADS>(ctl, partials, v, maxmask);
}

// y_k(c) = diag(c) * g(k, c) + sum_s val(s, c) * g(k, nbr(s, c)); WIDTH > 0
// fixes the row width at compile time (the slots are unrolled).
template <int NC, int WIDTH = 0, class G>
__device__ __forceinline__ void row_apply(const gf_krylov_t& K, int64_t c, const G& g, double (&out)[NC]) {
    const int64_t n = K.n;
    const double d = __ldg(K.diag + c);
#pragma unroll
    for (int k = 0; k < NC; ++k) out[k] = d * g(k, c);
    if (WIDTH > 0) {
#pragma unroll
        for (int s = 0; s < (WIDTH > 0 ? WIDTH : 1); ++s) {
            const double a = __ldg(K.val + s * n + c);
            const int nb = __ldg(K.nbr + s * n + c);
#pragma unroll
            for (int k = 0; k < NC; ++k) out[k] += a * g(k, nb);
        }
        return;
    }
    // Runtime row length: loads of a slot group first (see EllRows).
    const int W = K.row_len ? (int)__ldg(K.row_len + c) : K.width;
    for (int s0 = 0; s0 < W; s0 += kSlotGroup) {
        int nb[kSlotGroup];
        double a[kSlotGroup];
#pragma unroll
        for (int j = 0; j < kSlotGroup; ++j) {
            const int s = s0 + j;
            nb[j] = s < W ? __ldg(K.nbr + s * n + c) : (int)c;
            a[j] = s < W ? __ldg(K.val + s * n + c) : 0.0;
        }
#pragma unroll
        for (int j = 0; j < kSlotGroup; ++j)
            if (s0 + j < W)
#pragma unroll
                for (int k = 0; k < NC; ++k) out[k] += a[j] * g(k, nb[j]);
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
    barrier_init(K);
    double* partials = K.work + kCtlDoubles;
    double* vec = partials + kPartials;
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

// I: the cell index type (int32_t where n times the row width fits); GRP:
// slots of a runtime-width row whose loads are issued together.
template <typename T, int WIDTH, typename I = int64_t, int GRP = kSlotGroup>
struct EllRows {
    const T* val;
    const int32_t* nbr;
    I n;
    int w;
    // Row lengths (gf_krylov_t row_len) or nullptr: row c stops at len[c].
    const uint8_t* len = nullptr;
    template <typename A, class G>
    __device__ __forceinline__ A apply(I c, A dc, const G& g) const {
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
            // Slots in groups of kSlotGroup: every coefficient and index load
            // of a group is issued before its gathers, so a thread keeps
            // many loads in flight (a plain loop over a runtime row length
            // waits for each slot's index before its gather).  The products
            // are added in slot order, as in the plain loop.
            const int ws = len ? (int)__ldg(len + c) : w;
            for (int s0 = 0; s0 < ws; s0 += GRP) {
                int nb[GRP];
                A a[GRP];
#pragma unroll
                for (int j = 0; j < GRP; ++j) {
                    const int s = s0 + j;
                    nb[j] = s < ws ? __ldg(nbr + s * n + c) : (int)c;
                    a[j] = s < ws ? (A)ld_coef(val + s * n + c) : (A)0;
                }
                A gv[GRP];
#pragma unroll
                for (int j = 0; j < GRP; ++j) gv[j] = s0 + j < ws ? g(nb[j]) : (A)0;
#pragma unroll
                for (int j = 0; j < GRP; ++j)
                    if (s0 + j < ws) acc += a[j] * gv[j];
            }
        }
        return acc;
    }
    // Smallest and largest cell index that apply(c) reads, folded into lo/hi.
    __device__ __forceinline__ void span(I c, I& lo, I& hi) const {
        lo = c < lo ? c : lo;
        hi = c > hi ? c : hi;
        for (int s = 0; s < w; ++s) {
            const I j = __ldg(nbr + s * n + c);
            lo = j < lo ? j : lo;
            hi = j > hi ? j : hi;
        }
    }
};

template <typename T, bool SYM, bool COMPACT, typename I = int64_t>
struct BoxRows {
    const T* val;
    I n, sy, sz;
    // COMPACT arrays hold only the three '+' slots, which only SYM uses.
    __device__ __forceinline__ I plus_slot(int a) const { return (COMPACT && SYM) ? a : 2 * a + 1; }
    template <typename A, class G>
    __device__ __forceinline__ A apply(I c, A dc, const G& g) const {
        const I st[3] = {1, sy, sz};
        A ap[3], am[3];
        I ip[3], im[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const I s = st[a];
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
    __device__ __forceinline__ void span(I c, I& lo, I& hi) const {
        const I st[3] = {1, sy, sz};
        lo = c < lo ? c : lo;
        hi = c > hi ? c : hi;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            if (c >= st[a] && c - st[a] < lo) lo = c - st[a];
            if (c + st[a] < n && c + st[a] > hi) hi = c + st[a];
        }
    }
};

// Single-system Jacobi-PCG with the direction update fused into the SpMV
// pass: p_new = z + p_old beta is stored for the own cell and recomputed
// (bitwise identically) at the neighbours, so an iteration needs two grid
// reductions (p.Ap, then |r| and r.z) instead of three.

// vb / vn (>= 0): this block's index among the vn blocks of its system in a
// batched launch (gf_pcg_solve_batched); by default the whole grid.
template <int THREADS, int U, class Rows>
__device__ void pcg1_body(const gf_krylov_t& K, const Rows& rows, int vb = -1, int vn = -1) {
    __shared__ CgState st;
    KCtl* ctl = reinterpret_cast<KCtl*>(K.work);
    const int bk = vb >= 0 ? vb : (int)blockIdx.x;
    const int nbk = vn >= 0 ? vn : (int)gridDim.x;
    barrier_init_v(K, nbk, bk);
    double* partials = K.work + kCtlDoubles;
    double* vec = partials + kPartials;
    const int64_t n = K.n;
    double* r = vec;
    double* z = vec + n;
    double* pa = vec + 2 * n;
    double* pb = vec + 3 * n;
    double* q = vec + 4 * n;
    double* x = K.x;
    const bool jac = K.jacobi != 0, linf = K.norm_inf != 0;
    const int64_t t0 = bk * (int64_t)blockDim.x + threadIdx.x;
    const int64_t stride = (int64_t)nbk * blockDim.x;
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
        ok = grid_reduce<2, THREADS>(ctl, partials, loc, linf ? 1u : 0u);
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
            ok = grid_reduce<1, THREADS>(ctl, partials, loc, 0u);
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
            ok = grid_reduce<2, THREADS>(ctl, partials, loc, linf ? 1u : 0u);
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
    if (bk == 0 && threadIdx.x == 0) {
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
    EllRows<double, WIDTH> rows{K.val, K.nbr, K.n, K.width, K.row_len};
    pcg1_body<kCgThreads, 1>(K, rows);
}

// Single-reduction Jacobi-PCG (A. T. Chronopoulos and C. W. Gear, "s-step
// iterative methods for symmetric linear systems", J. Comput. Appl. Math.
// 25 (1989)).  With u = M r and w = A u the recurrences
//   gamma = r.u, delta = w.u, beta = gamma / gamma_old,
//   alpha = gamma / (delta - beta gamma / alpha_old),
//   p = u + beta p, s = w + beta s, x += alpha p, r -= alpha s
// are those of PCG (s = A p, delta - beta gamma / alpha_old = p.Ap), and
// both inner products of an iteration come from one grid reduction.  One
// pass per iteration: the new u is recomputed at the neighbours from the
// previous pass's r, w and s (double-buffered, since other blocks overwrite
// them in the same pass), so w = A u needs no second barrier.  Stopping
// test, iteration count and statistics are those of pcg1_body.
template <int THREADS, class Rows>
__device__ void pcg1_sr_body(const gf_krylov_t& K, const Rows& rows) {
    __shared__ CgState st;
    KCtl* ctl = reinterpret_cast<KCtl*>(K.work);
    barrier_init(K);
    double* partials = K.work + kCtlDoubles;
    double* vec = partials + kPartials;
    const int64_t n = K.n;
    double* rb[2] = {vec, vec + n};
    double* wb[2] = {vec + 2 * n, vec + 3 * n};
    double* sb[2] = {vec + 4 * n, vec + 5 * n};
    double* p = vec + 6 * n;
    double* x = K.x;
    const bool jac = K.jacobi != 0, linf = K.norm_inf != 0;
    const int64_t t0 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    bool ok = true;
    {  // r = b - A x, p = s = 0; |r|, gamma = r.u
        double loc[2] = {0.0, 0.0};
        auto gx = [&](int64_t i) { return __ldcg(x + i); };
        for (int64_t c = t0; c < n; c += stride) {
            const double ax = rows.apply(c, __ldg(K.diag + c), gx);
            const double rk = __ldg(K.rhs + c) - ax;
            const double uk = inv_diag(K.diag, c, jac) * rk;
            __stcg(rb[0] + c, rk);
            __stcg(sb[0] + c, 0.0);
            __stcg(p + c, 0.0);
            loc[0] = norm_acc(loc[0], rk, linf);
            loc[1] += rk * uk;
        }
        ok = grid_reduce<2, THREADS>(ctl, partials, loc, linf ? 1u : 0u);
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
    if (ok && !st.done) {  // w = A u; alpha = gamma / (w.u)
        double loc[1] = {0.0};
        const double* r0v = rb[0];
        auto gu = [&](int64_t i) { return inv_diag(K.diag, i, jac) * __ldcg(r0v + i); };
        for (int64_t c = t0; c < n; c += stride) {
            const double wk = rows.apply(c, __ldg(K.diag + c), gu);
            __stcg(wb[0] + c, wk);
            loc[0] += wk * gu(c);
        }
        ok = grid_reduce<1, THREADS>(ctl, partials, loc, 0u);
        if (threadIdx.x == 0) st.alpha = st.rz_old / loc[0];
        __syncthreads();
    }
    int a = 0;
    for (int it = 1; ok && !st.done && it <= K.max_iter; ++it) {
        const double alpha = st.alpha, beta = st.beta;
        const double* ra = rb[a];
        const double* wa = wb[a];
        const double* sa = sb[a];
        double* rn = rb[a ^ 1];
        double* wn = wb[a ^ 1];
        double* sn = sb[a ^ 1];
        // s and the new u of any cell from the previous pass's vectors; the
        // own cell and its neighbours evaluate the same expressions.
        auto gs = [&](int64_t i) { return __ldcg(wa + i) + beta * __ldcg(sa + i); };
        auto gr = [&](int64_t i) { return __ldcg(ra + i) - alpha * gs(i); };
        auto gu = [&](int64_t i) { return inv_diag(K.diag, i, jac) * gr(i); };
        double loc[3] = {0.0, 0.0, 0.0};
        for (int64_t c = t0; c < n; c += stride) {
            const double dinv = inv_diag(K.diag, c, jac);
            const double si = gs(c);
            const double pi = dinv * __ldcg(ra + c) + beta * __ldcg(p + c);
            const double rk = gr(c);
            const double uk = dinv * rk;
            const double wk = rows.apply(c, __ldg(K.diag + c), gu);
            __stcg(x + c, __ldcg(x + c) + alpha * pi);
            __stcg(p + c, pi);
            __stcg(sn + c, si);
            __stcg(rn + c, rk);
            __stcg(wn + c, wk);
            loc[0] = norm_acc(loc[0], rk, linf);
            loc[1] += rk * uk;
            loc[2] += wk * uk;
        }
        ok = grid_reduce<3, THREADS>(ctl, partials, loc, linf ? 1u : 0u);
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
                const double b = loc[1] / st.rz_old;
                st.alpha = loc[1] / (loc[2] - b * loc[1] / st.alpha);
                st.beta = b;
                st.rz_old = loc[1];
            }
        }
        __syncthreads();
        a ^= 1;
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
__global__ void __launch_bounds__(kCgThreads, 4) k_pcg1_sr(gf_krylov_t K) {
    EllRows<double, WIDTH> rows{K.val, K.nbr, K.n, K.width, K.row_len};
    pcg1_sr_body<kCgThreads>(K, rows);
}

template <bool SYM, int THREADS>
__global__ void __launch_bounds__(THREADS, 1024 / THREADS) k_pcg1_sr_box(gf_krylov_t K) {
    BoxRows<double, SYM, false> rows{K.val, K.n, K.stride_y, K.stride_z};
    pcg1_sr_body<THREADS>(K, rows);
}

// Box kernels come in tuning variants: MINB resident blocks per SM (the
// register budget follows from it) and U cells per thread per pass.
template <bool SYM, int THREADS, int U>
__global__ void __launch_bounds__(THREADS, 1024 / THREADS) k_pcg1_box(gf_krylov_t K) {
    BoxRows<double, SYM, false> rows{K.val, K.n, K.stride_y, K.stride_z};
    pcg1_body<THREADS, U>(K, rows);
}

// Mixed precision: FP32 inner Jacobi-PCG cycles inside FP64 iterative
// refinement.  Each cycle starts from the true FP64 residual r = b - A x
// (also the stopping test, |r| < max(atol, rtol |r0|) as in FP64), runs
// FP32 CG on A d = r with FP64-accumulated dot products until the recurrence
// residual falls below max(eta |r|, thresh / 2), then folds x += d in FP64.
// The FP32 copy of the matrix coefficients (all ELL slots, or the three "+"
// slots of a symmetric box) is made once per solve.
constexpr int kMaxEll = 32;

template <int THREADS, int U, class Rows64, class Rows32>
__device__ void pcg1_mixed_body(const gf_krylov_t& K, const Rows64& rows64, Rows32 rows32, int ncoef,
                                int vb = -1, int vn = -1) {
    const int bk = vb >= 0 ? vb : (int)blockIdx.x;
    const int nbk = vn >= 0 ? vn : (int)gridDim.x;
    __shared__ CgState st;
    __shared__ double s_target;
    __shared__ int s_cycle_done;
    KCtl* ctl = reinterpret_cast<KCtl*>(K.work);
    barrier_init_v(K, nbk, bk);
    double* partials = K.work + kCtlDoubles;
    double* base = partials + kPartials;
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
    const int64_t t0 = bk * (int64_t)blockDim.x + threadIdx.x;
    const int64_t stride = (int64_t)nbk * blockDim.x;
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
            ok = grid_reduce<1, THREADS>(ctl, partials, dummy, 0u);
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
            ok = grid_reduce<2, THREADS>(ctl, partials, loc, linf ? 1u : 0u);
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
                s_target = fmax(K.inner_eta * nr, (K.inner_margin > 0.0 ? K.inner_margin : 0.5) * st.thresh);
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
                ok = grid_reduce<1, THREADS>(ctl, partials, loc, 0u);
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
                ok = grid_reduce<2, THREADS>(ctl, partials, loc, linf ? 1u : 0u);
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
    if (bk == 0 && threadIdx.x == 0) {
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
    EllRows<double, WIDTH> rows64{K.val, K.nbr, K.n, K.width, K.row_len};
    EllRows<float, WIDTH> rows32{nullptr, K.nbr, K.n, K.width, K.row_len};
    pcg1_mixed_body<kCgThreads, 1>(K, rows64, rows32, K.width);
}

template <bool SYM, int THREADS, int U>
__global__ void __launch_bounds__(THREADS, 1024 / THREADS) k_pcg1_mixed_box(gf_krylov_t K) {
    BoxRows<double, SYM, false> rows64{K.val, K.n, K.stride_y, K.stride_z};
    BoxRows<float, SYM, SYM> rows32{nullptr, K.n, K.stride_y, K.stride_z};
    pcg1_mixed_body<THREADS, U>(K, rows64, rows32, SYM ? 3 : 6);
}

// Tuning variants of the box kernels: threads per block and U cells per
// thread per pass.  Every variant keeps 1024 resident threads per SM (64
// registers a thread); fewer, larger blocks mean fewer barrier arrivals.
struct BoxVariant {
    void* kern;
    int threads, unroll;
};
constexpr int kBoxVariants = 5;
// FP64 symmetric box CG with shared-memory tiles (k_pcg1_box_staged); falls
// back to variant 0 when the system does not qualify.
constexpr int kStagedVariant = 5;
// FP64 CG with the own-cell vectors in shared memory (pcg1_smem_body), box
// or ELL, 512-thread (6) or 1024-thread (7) blocks; falls back when the
// system is too large for it.
constexpr int kSmemVariant = 6;
// q-recurrence CG with shared-memory-resident vectors (pcg1_qrec_body),
// 1024-thread blocks, one (8) or two (9) cells per thread per gather pass.
constexpr int kQrecVariant = 8;
// Single-reduction CG with a halo sync (pcg1_halo_body), 1024-thread
// blocks, one (10) or two (11) cells per thread per gather pass; falls back
// to variant 8 when its four vectors do not fit.
constexpr int kHaloVariant = 10;
// Streaming q-recurrence CG with the vectors in the workspace
// (pcg1_stream_body): 512-thread blocks, two an SM (12); 1024-thread
// blocks (13); 256-thread blocks, four an SM (14).  FP64, one system.
constexpr int kStreamVariant = 12;
constexpr int kStreamVariants = 3;

// ELL (octree) FP64 CG in the launch shapes of the box variants 0-4.
template <int WIDTH, int THREADS, int U>
__global__ void __launch_bounds__(THREADS, 1024 / THREADS) k_pcg1_ellv(gf_krylov_t K) {
    EllRows<double, WIDTH> rows{K.val, K.nbr, K.n, K.width, K.row_len};
    pcg1_body<THREADS, U>(K, rows);
}

// Lean register form of pcg1_body for ELL rows: 32-bit cell indices,
// L1-cacheable gathers of z and p (both are written only before the grid
// barrier that precedes their next read, see pcg1_smem_body), and the
// x += alpha p of iteration k moved into the gather pass of iteration k + 1,
// which reads p anyway (the same additions in the same order; once more
// after the last iteration).  About 169 bytes a cell an iteration against
// 177 for pcg1_body.
// PF: before a cell is processed, the lines of the cell one grid stride on
// (its row slots, own vector entries) are prefetched into L2, so that
// cell's loads return at L2 rather than DRAM latency.
__device__ __forceinline__ void prefetch_l2(const void* p) {
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

template <int THREADS, class Rows, bool PF = false>
__device__ void pcg1_ell32_body(const gf_krylov_t& K, const Rows& rows) {
    __shared__ CgState st;
    KCtl* ctl = reinterpret_cast<KCtl*>(K.work);
    barrier_init(K);
    double* partials = K.work + kCtlDoubles;
    double* vec = partials + kPartials;
    const int n = (int)K.n;
    double* r = vec;
    double* z = vec + n;
    double* pa = vec + 2 * (int64_t)n;
    double* pb = vec + 3 * (int64_t)n;
    double* q = vec + 4 * (int64_t)n;
    double* x = K.x;
    const bool jac = K.jacobi != 0, linf = K.norm_inf != 0;
    const int t0 = blockIdx.x * THREADS + threadIdx.x;
    const int stride = gridDim.x * THREADS;
    bool ok = true;
    {
        double loc[2] = {0.0, 0.0};
        auto gx = [&](int i) { return __ldcg(x + i); };
        for (int c = t0; c < n; c += stride) {
            const double ax = rows.apply(c, __ldg(K.diag + c), gx);
            const double rk = __ldg(K.rhs + c) - ax;
            const double zk = inv_diag(K.diag, c, jac) * rk;
            __stcg(r + c, rk);
            __stcg(z + c, zk);
            __stcg(pa + c, 0.0);
            loc[0] = norm_acc(loc[0], rk, linf);
            loc[1] += rk * zk;
        }
        ok = grid_reduce<2, THREADS>(ctl, partials, loc, linf ? 1u : 0u);
        if (threadIdx.x == 0) {
            const double r0 = norm_fin(loc[0], linf);
            st.r0 = r0;
            st.final = r0;
            st.thresh = fmax(K.atol, K.rtol * r0);
            st.rz_old = loc[1];
            st.beta = 0.0;
            st.alpha = 0.0;
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
    bool pending = false;
    for (int it = 1; ok && !st.done && it <= K.max_iter; ++it) {
        const double beta = st.beta;
        {  // x += alpha_(k-1) p_old; p_new = z + p_old beta; q = A p_new; p_new . q
            const double alpha_prev = st.alpha;
            double loc[1] = {0.0};
            auto gp = [&](int i) { return z[i] + p_old[i] * beta; };
            for (int c = t0; c < n; c += stride) {
                if (PF) {
                    const int cn = c + stride;
                    if (cn < n) {
#pragma unroll
                        for (int sl = 0; sl < 6; ++sl) {
                            prefetch_l2(K.val + (int64_t)sl * n + cn);
                            prefetch_l2(K.nbr + (int64_t)sl * n + cn);
                        }
                        prefetch_l2(K.diag + cn);
                        prefetch_l2(z + cn);
                        prefetch_l2(p_old + cn);
                        prefetch_l2(x + cn);
                    }
                }
                const double pold = p_old[c];
                const double pc = z[c] + pold * beta;
                const double ap = rows.apply(c, __ldg(K.diag + c), gp);
                if (pending) __stcg(x + c, __ldcg(x + c) + alpha_prev * pold);
                __stcg(p_new + c, pc);
                __stcg(q + c, ap);
                loc[0] += pc * ap;
            }
            ok = grid_reduce<1, THREADS>(ctl, partials, loc, 0u);
            if (!ok) break;
            if (threadIdx.x == 0) st.alpha = st.rz_old / loc[0];
            __syncthreads();
        }
        {  // r -= alpha q; z = M r; |r|, r.z
            const double alpha = st.alpha;
            double loc[2] = {0.0, 0.0};
            for (int c = t0; c < n; c += stride) {
                if (PF) {
                    const int cn = c + stride;
                    if (cn < n) {
                        prefetch_l2(r + cn);
                        prefetch_l2(q + cn);
                        prefetch_l2(K.diag + cn);
                    }
                }
                const double rk = __ldcg(r + c) - alpha * __ldcg(q + c);
                const double zk = inv_diag(K.diag, c, jac) * rk;
                __stcg(r + c, rk);
                __stcg(z + c, zk);
                loc[0] = norm_acc(loc[0], rk, linf);
                loc[1] += rk * zk;
            }
            pending = true;
            ok = grid_reduce<2, THREADS>(ctl, partials, loc, linf ? 1u : 0u);
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
    if (ok && pending) {  // the last iteration's x += alpha p (p_old after the swap)
        const double alpha = st.alpha;
        for (int c = t0; c < n; c += stride) __stcg(x + c, __ldcg(x + c) + alpha * __ldcg(p_old + c));
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

template <int WIDTH, int THREADS, int MINB, int GRP, bool PF = false>
__global__ void __launch_bounds__(THREADS, MINB) k_pcg1_ell32(gf_krylov_t K) {
    EllRows<double, WIDTH, int, GRP> rows{K.val, K.nbr, (int)K.n, K.width, K.row_len};
    pcg1_ell32_body<THREADS, EllRows<double, WIDTH, int, GRP>, PF>(K, rows);
}

// Lean ELL CG shapes (FP64, one system, 32-bit indices): 15: 256 threads, 4
// blocks an SM, slot groups of 8; 16: 5 blocks an SM; 17: 6 blocks an SM,
// groups of 4; 18: as 17 with the next cell's lines prefetched into L2.
constexpr int kOccVariant = 15;
constexpr int kOccVariants = 4;

template <int WIDTH>
static BoxVariant ell_occ_kernel(int which) {
    switch (which) {
        case 1:
            return {(void*)k_pcg1_ell32<WIDTH, 256, 5, 8>, 256, 1};
        case 2:
            return {(void*)k_pcg1_ell32<WIDTH, 256, 6, 4>, 256, 1};
        case 3:
            return {(void*)k_pcg1_ell32<WIDTH, 256, 6, 4, true>, 256, 1};
        default:
            return {(void*)k_pcg1_ell32<WIDTH, 256, 4, 8>, 256, 1};
    }
}

template <int WIDTH>
static BoxVariant ell_kernel(int variant) {
    switch (variant) {
        case 1:
            return {(void*)k_pcg1_ellv<WIDTH, 256, 2>, 256, 2};
        case 2:
            return {(void*)k_pcg1_ellv<WIDTH, 512, 1>, 512, 1};
        case 3:
            return {(void*)k_pcg1_ellv<WIDTH, 1024, 1>, 1024, 1};
        case 4:
            return {(void*)k_pcg1_ellv<WIDTH, 1024, 2>, 1024, 2};
        default:
            return {(void*)k_pcg1<WIDTH>, kCgThreads, 1};
    }
}

template <bool MIXED, bool SYM, int THREADS, int U>
static BoxVariant box_variant() {
    void* k = MIXED ? (void*)k_pcg1_mixed_box<SYM, THREADS, U> : (void*)k_pcg1_box<SYM, THREADS, U>;
    return {k, THREADS, U};
}

template <bool MIXED, bool SYM>
static BoxVariant box_kernel(int variant) {
    switch (variant) {
        case 1:
            return box_variant<MIXED, SYM, 256, 2>();
        case 2:
            return box_variant<MIXED, SYM, 512, 1>();
        case 3:
            return box_variant<MIXED, SYM, 1024, 1>();
        case 4:
            return box_variant<MIXED, SYM, 1024, 2>();
        default:
            return box_variant<MIXED, SYM, 256, 1>();
    }
}

// ---------------------------------------------------------------------------
// Box CG with shared-memory tiles filled by bulk asynchronous copies.
//
// The register-resident kernels keep only a few loads per thread in flight,
// which at a million cells leaves them bound by memory latency rather than
// bandwidth.  Here each block walks tiles of T consecutive cells; one thread
// issues 1-D bulk copies (cp.async.bulk, completion counted on an mbarrier)
// of every window a tile reads into one of two shared-memory stages, so the
// next tile (~90 KB) is in flight while the current one is computed.
//   SpMV pass, cells [c0, c1): z and p_old over [c0-sz, c1-sz),
//   [c0-sy, c1+sy) and [c0+sz, c1+sz); the '+' coefficient slots over
//   [c0-1, c1), [c0-sy, c1), [c0-sz, c1-sz) and [c0, c1); diag over [c0, c1).
//   Update pass: p, q, x, r and diag over [c0, c1).
// Per cell the arithmetic and its order are those of BoxRows, so matrix
// products are bitwise those of k_pcg1_box.  Requires a symmetric box, even
// n and 16-byte aligned arrays (the host checks; other systems use
// k_pcg1_box).  Every copy reads this GPU's own memory into the issuing
// block's own shared memory.
constexpr int kStThreads = 512;
constexpr int kStMaxSmem = 220 * 1024;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* b) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(b)) : "memory");
}

__device__ __forceinline__ void mbar_expect(uint64_t* b, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_test(uint64_t* b, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(b)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for the phase with this parity; false when it expired.
__device__ __forceinline__ bool mbar_wait(uint64_t* b, uint32_t parity) {
    long long it = 0;
    while (!mbar_test(b, parity)) {
        if (++it > 1024) __nanosleep(20);
        if (it > g_spin) return false;
    }
    return true;
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* b) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(b))
        : "memory");
}

// Shared-memory slots of one stage (in doubles, all even so every slot
// starts 16-byte aligned): eight short ones (T + 4) and three long ones
// (T + 2 sy + 4) for the windows that carry the y halo.
struct StLayout {
    int a, b;  // slot lengths
    __host__ __device__ StLayout(int T, int64_t sy) : a(T + 4), b(T + 2 * (int)sy + 4) {}
    __host__ __device__ int stage() const { return 8 * a + 3 * b; }
    // SpMV pass
    __host__ __device__ int zm() const { return 0; }
    __host__ __device__ int zo() const { return a; }
    __host__ __device__ int zp() const { return a + b; }
    __host__ __device__ int pm() const { return 2 * a + b; }
    __host__ __device__ int po() const { return 3 * a + b; }
    __host__ __device__ int pp() const { return 3 * a + 2 * b; }
    __host__ __device__ int cx() const { return 4 * a + 2 * b; }
    __host__ __device__ int cy() const { return 5 * a + 2 * b; }
    __host__ __device__ int czm() const { return 5 * a + 3 * b; }
    __host__ __device__ int czo() const { return 6 * a + 3 * b; }
    __host__ __device__ int dg() const { return 7 * a + 3 * b; }
};

// Window [lo, hi) of an array, clamped to [0, n) and widened to even ends
// (n is even, arrays 16-byte aligned): its first index, and its bytes.
struct Window {
    int64_t base;
    uint32_t bytes;
};

__device__ __forceinline__ Window window(int64_t lo, int64_t hi, int64_t n) {
    lo = lo < 0 ? 0 : lo;
    hi = hi > n ? n : hi;
    if (hi <= lo) return {lo & ~1LL, 0u};
    const int64_t a = lo & ~1LL, e = (hi + 1) & ~1LL;
    return {a, (uint32_t)((e - a) * 8)};
}

struct StGeom {  // window first indices of one SpMV tile
    int64_t c0, c1, bm, bo, bp, bx, by;
};

__device__ __forceinline__ StGeom st_geom(int64_t t, int T, int64_t n, int64_t sy, int64_t sz) {
    StGeom g;
    g.c0 = t * T;
    g.c1 = g.c0 + T < n ? g.c0 + T : n;
    g.bm = window(g.c0 - sz, g.c1 - sz, n).base;
    g.bo = window(g.c0 - sy, g.c1 + sy, n).base;
    g.bp = window(g.c0 + sz, g.c1 + sz, n).base;
    g.bx = window(g.c0 - 1, g.c1, n).base;
    g.by = window(g.c0 - sy, g.c1, n).base;
    return g;
}

// Thread 0: expect the tile's bytes on the stage barrier, then issue every
// window copy of the list (array, window, slot offset).
struct StCopy {
    const double* src;
    Window w;
    int off;
};

template <int N>
__device__ __forceinline__ void st_issue(const StCopy (&cp)[N], double* stage, uint64_t* bar) {
    uint32_t total = 0;
#pragma unroll
    for (int i = 0; i < N; ++i) total += cp[i].w.bytes;
    mbar_expect(bar, total);
#pragma unroll
    for (int i = 0; i < N; ++i)
        if (cp[i].w.bytes) bulk_g2s(stage + cp[i].off, cp[i].src + cp[i].w.base, cp[i].w.bytes, bar);
}

__device__ __forceinline__ void st_issue_spmv(int64_t t, int T, const gf_krylov_t& K, const double* z,
                                              const double* pold, const StLayout& L, double* stage,
                                              uint64_t* bar) {
    const int64_t n = K.n, sy = K.stride_y, sz = K.stride_z;
    const int64_t c0 = t * T, c1 = c0 + T < n ? c0 + T : n;
    const Window wm = window(c0 - sz, c1 - sz, n), wo = window(c0 - sy, c1 + sy, n),
                 wp = window(c0 + sz, c1 + sz, n);
    const double* vx = K.val + 1 * n;  // '+' slots of the box ELL: 1, 3, 5
    const double* vy = K.val + 3 * n;
    const double* vz = K.val + 5 * n;
    const StCopy cp[11] = {
        {z, wm, L.zm()},    {z, wo, L.zo()},    {z, wp, L.zp()},
        {pold, wm, L.pm()}, {pold, wo, L.po()}, {pold, wp, L.pp()},
        {vx, window(c0 - 1, c1, n), L.cx()},     {vy, window(c0 - sy, c1, n), L.cy()},
        {vz, wm, L.czm()},  {vz, window(c0, c1, n), L.czo()},
        {K.diag, window(c0, c1, n), L.dg()},
    };
    st_issue(cp, stage, bar);
}

__device__ __forceinline__ void st_issue_update(int64_t t, int T, const gf_krylov_t& K, const double* p,
                                                const double* q, const double* r, const StLayout& L,
                                                double* stage, uint64_t* bar) {
    const int64_t n = K.n;
    const int64_t c0 = t * T, c1 = c0 + T < n ? c0 + T : n;
    const Window w = window(c0, c1, n);
    const StCopy cp[5] = {{p, w, 0 * L.a}, {q, w, 1 * L.a}, {K.x, w, 2 * L.a}, {r, w, 3 * L.a}, {K.diag, w, 4 * L.a}};
    st_issue(cp, stage, bar);
}

// One pass over this block's tiles (t = blockIdx.x, + gridDim.x, ...) with a
// two-stage pipeline.  issue(t, stage, bar) runs on thread 0; compute(t,
// stage) on all threads.  Returns false when a stage wait expired (after a
// second bounded wait so no copy is left landing in shared memory).
template <class Issue, class Compute>
__device__ bool st_pass(int64_t ntiles, double* st0, double* st1, uint64_t* bars, uint32_t& phase,
                        const Issue& issue, const Compute& compute) {
    const int64_t g = gridDim.x;
    const int64_t t0 = blockIdx.x;
    if (threadIdx.x == 0) {
        // Generic-proxy writes (this pass's inputs) before async-proxy reads.
        asm volatile("fence.proxy.async.global;" ::: "memory");
        if (t0 < ntiles) issue(t0, st0, &bars[0]);
        if (t0 + g < ntiles) issue(t0 + g, st1, &bars[1]);
    }
    int s = 0;
    for (int64_t t = t0; t < ntiles; t += g, s ^= 1) {
        const uint32_t par = (phase >> s) & 1u;
        // The vote keeps the block's control flow uniform if a wait expired.
        if (__syncthreads_or(!mbar_wait(&bars[s], par))) {
            // Drain both stages (bounded) before leaving.
            mbar_wait(&bars[s], par);
            if (t + g < ntiles) mbar_wait(&bars[s ^ 1], (phase >> (s ^ 1)) & 1u);
            return false;
        }
        phase ^= 1u << s;
        compute(t, s ? st1 : st0);
        __syncthreads();  // the stage is free again
        if (threadIdx.x == 0 && t + 2 * g < ntiles) issue(t + 2 * g, s ? st1 : st0, &bars[s]);
    }
    return true;
}

template <int THREADS>
__global__ void __launch_bounds__(THREADS, 1) k_pcg1_box_staged(gf_krylov_t K, int T) {
    __shared__ CgState st;
    __shared__ __align__(8) uint64_t bars[2];
    __shared__ int s_stage_err;
    extern __shared__ __align__(16) double smem[];
    KCtl* ctl = reinterpret_cast<KCtl*>(K.work);
    barrier_init(K);
    double* partials = K.work + kCtlDoubles;
    double* vec = partials + kPartials;
    const int64_t n = K.n, sy = K.stride_y, sz = K.stride_z;
    double* r = vec;
    double* z = vec + n;
    double* pa = vec + 2 * n;
    double* pb = vec + 3 * n;
    double* q = vec + 4 * n;
    double* x = K.x;
    const bool jac = K.jacobi != 0, linf = K.norm_inf != 0;
    const StLayout L(T, sy);
    double* st0 = smem;
    double* st1 = smem + L.stage();
    const int64_t ntiles = (n + T - 1) / T;
    uint32_t phase = 0;
    if (threadIdx.x == 0) {
        mbar_init(&bars[0]);
        mbar_init(&bars[1]);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_stage_err = 0;
    }
    __syncthreads();
    const BoxRows<double, true, false> rows{K.val, n, sy, sz};
    const int64_t gt0 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t gstride = (int64_t)gridDim.x * blockDim.x;
    bool ok = true;
    {  // r = b - A x, z = M r, p = 0; |r| and r.z (register path, once)
        double loc[2] = {0.0, 0.0};
        auto gx = [&](int64_t i) { return __ldcg(x + i); };
        for (int64_t c = gt0; c < n; c += gstride) {
            const double ax = rows.apply(c, __ldg(K.diag + c), gx);
            const double rk = __ldg(K.rhs + c) - ax;
            const double zk = inv_diag(K.diag, c, jac) * rk;
            __stcg(r + c, rk);
            __stcg(z + c, zk);
            __stcg(pa + c, 0.0);
            loc[0] = norm_acc(loc[0], rk, linf);
            loc[1] += rk * zk;
        }
        ok = grid_reduce<2, THREADS>(ctl, partials, loc, linf ? 1u : 0u);
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
            auto issue = [&](int64_t t, double* stage, uint64_t* bar) {
                st_issue_spmv(t, T, K, z, p_old, L, stage, bar);
            };
            auto compute = [&](int64_t t, const double* S) {
                const StGeom g = st_geom(t, T, n, sy, sz);
                for (int64_t c = g.c0 + threadIdx.x; c < g.c1; c += THREADS) {
                    auto po = [&](int64_t i) { return S[L.zo() + (i - g.bo)] + S[L.po() + (i - g.bo)] * beta; };
                    const double dc = S[L.dg() + (c - g.c0 + (g.c0 & 1))];
                    const double pc = po(c);
                    double acc = dc * pc;
                    {
                        const double am = c >= 1 ? S[L.cx() + (c - 1 - g.bx)] : 0.0;
                        const double ap = S[L.cx() + (c - g.bx)];
                        acc += am * po(c >= 1 ? c - 1 : c);
                        acc += ap * po(c + 1 < n ? c + 1 : c);
                    }
                    {
                        const double am = c >= sy ? S[L.cy() + (c - sy - g.by)] : 0.0;
                        const double ap = S[L.cy() + (c - g.by)];
                        acc += am * po(c >= sy ? c - sy : c);
                        acc += ap * po(c + sy < n ? c + sy : c);
                    }
                    {
                        const double am = c >= sz ? S[L.czm() + (c - sz - g.bm)] : 0.0;
                        const double ap = S[L.czo() + (c - g.c0 + (g.c0 & 1))];
                        const double gm =
                            c >= sz ? S[L.zm() + (c - sz - g.bm)] + S[L.pm() + (c - sz - g.bm)] * beta : pc;
                        const double gp =
                            c + sz < n ? S[L.zp() + (c + sz - g.bp)] + S[L.pp() + (c + sz - g.bp)] * beta : pc;
                        acc += am * gm;
                        acc += ap * gp;
                    }
                    __stcg(p_new + c, pc);
                    __stcg(q + c, acc);
                    loc[0] += pc * acc;
                }
            };
            ok = st_pass(ntiles, st0, st1, bars, phase, issue, compute);
            if (!ok) {
                if (threadIdx.x == 0) atomicExch(&ctl->error, 1);
                break;
            }
            ok = grid_reduce<1, THREADS>(ctl, partials, loc, 0u);
            if (!ok) break;
            if (threadIdx.x == 0) st.alpha = st.rz_old / loc[0];
            __syncthreads();
        }
        {  // x += alpha p; r -= alpha q; z = M r; |r|, r.z
            const double alpha = st.alpha;
            double loc[2] = {0.0, 0.0};
            auto issue = [&](int64_t t, double* stage, uint64_t* bar) {
                st_issue_update(t, T, K, p_new, q, r, L, stage, bar);
            };
            auto compute = [&](int64_t t, const double* S) {
                const int64_t c0 = t * T, c1 = c0 + T < n ? c0 + T : n;
                const int64_t b = c0 & ~1LL;
                for (int64_t c = c0 + threadIdx.x; c < c1; c += THREADS) {
                    const int i = (int)(c - b);
                    const double pc = S[0 * L.a + i], qo = S[1 * L.a + i], xo = S[2 * L.a + i],
                                 ro = S[3 * L.a + i], d = S[4 * L.a + i];
                    const double dg = jac ? (fabs(d) < 2.220446049250313e-16 ? 1.0 : 1.0 / d) : 1.0;
                    __stcg(x + c, xo + alpha * pc);
                    const double rk = ro - alpha * qo;
                    const double zk = dg * rk;
                    __stcg(r + c, rk);
                    __stcg(z + c, zk);
                    loc[0] = norm_acc(loc[0], rk, linf);
                    loc[1] += rk * zk;
                }
            };
            ok = st_pass(ntiles, st0, st1, bars, phase, issue, compute);
            if (!ok) {
                if (threadIdx.x == 0) atomicExch(&ctl->error, 1);
                break;
            }
            ok = grid_reduce<2, THREADS>(ctl, partials, loc, linf ? 1u : 0u);
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

// ---------------------------------------------------------------------------
// CG with each block's own-cell vectors resident in shared memory.
//
// Every block owns one contiguous chunk of cells for the whole solve and
// keeps x, r and q = A p of those cells in shared memory (3 doubles a cell,
// 4 with p: the 148 SMs' shared memory together holds them for about a
// million cells).  Only what neighbours read goes through global memory:
// z = M r and p, stored as interleaved pairs {z, p} so the 7-point gather
// of p_new = z + p_old beta is one 16-byte load a point.  Pair buffer k mod 2
// holds {z_k, p_(k-1)}: iteration k reads it and writes p_k and z_(k+1)
// into the other buffer, which no block reads until the grid barrier that
// ends iteration k.  The inverse diagonal is computed once per solve.  Cell
// indices are 32-bit (the host launches this kernel only when n times the
// row width is below 2^31).
// Arithmetic per cell is that of pcg1_body, so the iterates are the same.
template <int THREADS, int U, int V, bool KEEP_P, class Rows>
__device__ void pcg1_smem_body(const gf_krylov_t& K, const Rows& rows, int chunk) {
    __shared__ CgState st;
    extern __shared__ __align__(16) double sm[];
    KCtl* ctl = reinterpret_cast<KCtl*>(K.work);
    barrier_init(K);
    double* partials = K.work + kCtlDoubles;
    double* vec = partials + kPartials;
    const int n = (int)K.n;
    double2* zp0 = reinterpret_cast<double2*>(vec);
    double2* zp1 = reinterpret_cast<double2*>(vec + 2 * (int64_t)n);
    double* inv = vec + 4 * (int64_t)n;
    const int c0 = blockIdx.x * chunk;
    const int c1 = c0 + chunk < n ? c0 + chunk : n;
    const int m = c1 > c0 ? c1 - c0 : 0;
    double* xs = sm;
    double* rs = sm + chunk;
    double* qs = sm + 2 * chunk;
    double* ps = sm + 3 * chunk;  // only with KEEP_P (else p is re-read from global)
    const bool jac = K.jacobi != 0, linf = K.norm_inf != 0;
    bool ok = true;
    {  // r = b - A x, z = M r, p = 0; |r| and r.z
        double loc[2] = {0.0, 0.0};
        auto gx = [&](int i) { return __ldcg(K.x + i); };
        for (int i = threadIdx.x; i < m; i += THREADS) {
            const int c = c0 + i;
            const double ax = rows.apply(c, __ldg(K.diag + c), gx);
            const double rk = __ldg(K.rhs + c) - ax;
            const double iv = inv_diag(K.diag, c, jac);
            const double zk = iv * rk;
            xs[i] = __ldcg(K.x + c);
            rs[i] = rk;
            inv[c] = iv;
            __stcg(zp0 + c, make_double2(zk, 0.0));
            loc[0] = norm_acc(loc[0], rk, linf);
            loc[1] += rk * zk;
        }
        ok = grid_reduce<2, THREADS>(ctl, partials, loc, linf ? 1u : 0u);
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
    for (int it = 1; ok && !st.done && it <= K.max_iter; ++it) {
        const double2* cur = (it & 1) ? zp0 : zp1;
        double2* nxt = (it & 1) ? zp1 : zp0;
        {  // p_new = z + p_old beta; q = A p_new; p_new . q
            const double beta = st.beta;
            double loc[1] = {0.0};
            // Plain (L1-cacheable) loads: the pair buffer is written only
            // before the grid barrier, whose acquire makes this SM's L1
            // coherent again; a stencil's neighbours then mostly hit L1.
            auto gp = [&](int j) {
                const double2 v = cur[j];
                return v.x + v.y * beta;
            };
            // U cells per thread per pass: all their loads are issued before
            // any store, so U latency chains overlap.
            for (int i0 = threadIdx.x; i0 < m; i0 += U * THREADS) {
                double pc[U], ap[U];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int i = i0 + u * THREADS;
                    if (i < m) {
                        const int c = c0 + i;
                        pc[u] = gp(c);
                        ap[u] = rows.apply(c, __ldg(K.diag + c), gp);
                    }
                }
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int i = i0 + u * THREADS;
                    if (i < m) {
                        __stcg(&nxt[c0 + i].y, pc[u]);
                        if (KEEP_P) ps[i] = pc[u];
                        qs[i] = ap[u];
                        loc[0] += pc[u] * ap[u];
                    }
                }
            }
            ok = grid_reduce<1, THREADS>(ctl, partials, loc, 0u);
            if (!ok) break;
            if (threadIdx.x == 0) st.alpha = st.rz_old / loc[0];
            __syncthreads();
        }
        {  // x += alpha p; r -= alpha q; z = M r; |r|, r.z (own cells)
            const double alpha = st.alpha;
            double loc[2] = {0.0, 0.0};
            // V cells per thread per pass, global loads first: V L2 latencies
            // overlap instead of following one another.
            for (int i0 = threadIdx.x; i0 < m; i0 += V * THREADS) {
                double pv[V], iv[V];
#pragma unroll
                for (int u = 0; u < V; ++u) {
                    const int i = i0 + u * THREADS;
                    if (i < m) {
                        pv[u] = KEEP_P ? ps[i] : __ldcg(&nxt[c0 + i].y);
                        iv[u] = inv[c0 + i];
                    }
                }
#pragma unroll
                for (int u = 0; u < V; ++u) {
                    const int i = i0 + u * THREADS;
                    if (i < m) {
                        xs[i] = xs[i] + alpha * pv[u];
                        const double rk = rs[i] - alpha * qs[i];
                        const double zk = iv[u] * rk;
                        rs[i] = rk;
                        __stcg(&nxt[c0 + i].x, zk);
                        loc[0] = norm_acc(loc[0], rk, linf);
                        loc[1] += rk * zk;
                    }
                }
            }
            ok = grid_reduce<2, THREADS>(ctl, partials, loc, linf ? 1u : 0u);
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
    }
    // Every block writes its cells of x once, whatever the outcome.
    __syncthreads();
    for (int i = threadIdx.x; i < m; i += THREADS) K.x[c0 + i] = xs[i];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        double* o = K.stats;
        o[0] = st.r0;
        o[1] = st.final;
        o[2] = st.done ? st.its : K.max_iter;
        o[3] = st.converged;
        o[4] = ok ? st.status : GF_ERR_TIMEOUT;
    }
}

// Cells per thread per pass: 512-thread blocks (128 registers a thread)
// gather two cells at once and update four; 1024-thread blocks (64
// registers) gather one and update two.
// KEEP_P: p of the own cells in shared memory too (4 doubles a cell);
// otherwise 3 doubles a cell, which fits ~1.05M cells on 148 SMs.
__host__ __device__ constexpr int smem_gather_cells(int threads) { return threads <= 512 ? 2 : 1; }
__host__ __device__ constexpr int smem_update_cells(int threads) { return threads <= 512 ? 4 : 2; }

template <bool SYM, int THREADS, bool KEEP_P>
__global__ void __launch_bounds__(THREADS, 1) k_pcg1_smem_box(gf_krylov_t K, int chunk) {
    BoxRows<double, SYM, false, int> rows{K.val, (int)K.n, (int)K.stride_y, (int)K.stride_z};
    pcg1_smem_body<THREADS, smem_gather_cells(THREADS), smem_update_cells(THREADS), KEEP_P>(K, rows, chunk);
}

template <int WIDTH, int THREADS, bool KEEP_P>
__global__ void __launch_bounds__(THREADS, 1) k_pcg1_smem_ell(gf_krylov_t K, int chunk) {
    EllRows<double, WIDTH, int> rows{K.val, K.nbr, (int)K.n, K.width, K.row_len};
    pcg1_smem_body<THREADS, smem_gather_cells(THREADS), smem_update_cells(THREADS), KEEP_P>(K, rows, chunk);
}

// ---------------------------------------------------------------------------
// Shared-memory-resident CG with the direction product updated by recurrence:
// q = A p is formed as q_k = A z_k + beta q_(k-1) (equal to A (z_k + beta
// p_(k-1)) in exact arithmetic), so the stencil gathers z alone and only z
// crosses L2 between blocks.  Each block keeps r, q and p of its cells in
// shared memory and updates its cells of x in place in global memory.  The
// iterates differ from pcg1_smem_body by the rounding of the recurrence.
template <int THREADS, int U, int V, class Rows>
__device__ void pcg1_qrec_body(const gf_krylov_t& K, const Rows& rows, int chunk) {
    __shared__ CgState st;
    extern __shared__ __align__(16) double sm[];
    KCtl* ctl = reinterpret_cast<KCtl*>(K.work);
    barrier_init(K);
    double* partials = K.work + kCtlDoubles;
    double* vec = partials + kPartials;
    const int n = (int)K.n;
    double* z = vec;
    double* inv = vec + n;
    double* x = K.x;
    const int c0 = blockIdx.x * chunk;
    const int c1 = c0 + chunk < n ? c0 + chunk : n;
    const int m = c1 > c0 ? c1 - c0 : 0;
    double* rs = sm;
    double* qs = sm + chunk;
    double* ps = sm + 2 * chunk;
    const bool jac = K.jacobi != 0, linf = K.norm_inf != 0;
    bool ok = true;
    {  // r = b - A x, z = M r, p = q = 0; |r| and r.z
        double loc[2] = {0.0, 0.0};
        auto gx = [&](int i) { return __ldcg(x + i); };
        for (int i = threadIdx.x; i < m; i += THREADS) {
            const int c = c0 + i;
            const double ax = rows.apply(c, __ldg(K.diag + c), gx);
            const double rk = __ldg(K.rhs + c) - ax;
            const double iv = inv_diag(K.diag, c, jac);
            const double zk = iv * rk;
            rs[i] = rk;
            qs[i] = 0.0;
            ps[i] = 0.0;
            inv[c] = iv;
            __stcg(z + c, zk);
            loc[0] = norm_acc(loc[0], rk, linf);
            loc[1] += rk * zk;
        }
        ok = grid_reduce<2, THREADS>(ctl, partials, loc, linf ? 1u : 0u);
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
    // x += alpha p of an iteration runs as side work of the second
    // reduction (the other warps while warp 0 waits for the grid), off the
    // passes; the same additions in the same order, so the same bits.
    for (int it = 1; ok && !st.done && it <= K.max_iter; ++it) {
        {  // w = A z; p = z + beta p; q = w + beta q; p . q
            const double beta = st.beta;
            double loc[1] = {0.0};
            // Plain (L1-cacheable) loads: z is written only before the grid
            // barrier that precedes this pass (see pcg1_smem_body).
            auto gz = [&](int j) { return z[j]; };
            for (int i0 = threadIdx.x; i0 < m; i0 += U * THREADS) {
                double zc[U], w[U];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int i = i0 + u * THREADS;
                    if (i < m) {
                        const int c = c0 + i;
                        zc[u] = z[c];
                        w[u] = rows.apply(c, __ldg(K.diag + c), gz);
                    }
                }
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int i = i0 + u * THREADS;
                    if (i < m) {
                        const double pold = ps[i];
                        const double pk = zc[u] + pold * beta;
                        const double qk = w[u] + qs[i] * beta;
                        ps[i] = pk;
                        qs[i] = qk;
                        loc[0] += pk * qk;
                    }
                }
            }
            ok = grid_reduce<1, THREADS>(ctl, partials, loc, 0u);
            if (!ok) break;
            if (threadIdx.x == 0) st.alpha = st.rz_old / loc[0];
            __syncthreads();
        }
        {  // r -= alpha q; z = M r; |r|, r.z (own cells); x += alpha p during the reduction
            const double alpha = st.alpha;
            double loc[2] = {0.0, 0.0};
            for (int i0 = threadIdx.x; i0 < m; i0 += V * THREADS) {
                double iv[V];
#pragma unroll
                for (int u = 0; u < V; ++u) {
                    const int i = i0 + u * THREADS;
                    if (i < m) iv[u] = inv[c0 + i];
                }
#pragma unroll
                for (int u = 0; u < V; ++u) {
                    const int i = i0 + u * THREADS;
                    if (i < m) {
                        const int c = c0 + i;
                        const double rk = rs[i] - alpha * qs[i];
                        const double zk = iv[u] * rk;
                        rs[i] = rk;
                        __stcg(z + c, zk);
                        loc[0] = norm_acc(loc[0], rk, linf);
                        loc[1] += rk * zk;
                    }
                }
            }
            auto xupd = [&](int t, int nt) {
                for (int i = t; i < m; i += nt) __stcg(x + c0 + i, __ldcg(x + c0 + i) + alpha * ps[i]);
            };
            ok = grid_reduce_side<2, THREADS>(ctl, partials, loc, linf ? 1u : 0u, xupd);
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

template <bool SYM, int THREADS, int U>
__global__ void __launch_bounds__(THREADS, 1) k_pcg1_qrec_box(gf_krylov_t K, int chunk) {
    BoxRows<double, SYM, false, int> rows{K.val, (int)K.n, (int)K.stride_y, (int)K.stride_z};
    pcg1_qrec_body<THREADS, U, 2>(K, rows, chunk);
}

template <int WIDTH, int THREADS, int U>
__global__ void __launch_bounds__(THREADS, 1) k_pcg1_qrec_ell(gf_krylov_t K, int chunk) {
    EllRows<double, WIDTH, int> rows{K.val, K.nbr, (int)K.n, K.width, K.row_len};
    pcg1_qrec_body<THREADS, U, 2>(K, rows, chunk);
}

// ---------------------------------------------------------------------------
// Streaming q-recurrence CG for systems too large for shared memory (octree
// grids of millions of cells).  The recurrences are those of pcg1_qrec_body
// (q_k = A z_k + beta q_(k-1), so the stencil gathers z alone), with every
// vector in the workspace: an iteration reads a cell's row (up to its row
// length), z, p, q and x in the gather pass and r, q and the Jacobi inverse
// in the update pass, about 180 bytes a cell against 230 for pcg1_body,
// whose gather reads z and p at every stencil point.  Each block owns one
// contiguous chunk of cells, so the gathers of a block stay within a short
// window of the cell order (Morton order within each refinement level).
// x += alpha p of iteration k runs in the gather pass of iteration k + 1,
// which reads p anyway (the same additions in the same order), and once
// more after the last iteration.
template <int THREADS, class Rows>
__device__ void pcg1_stream_body(const gf_krylov_t& K, const Rows& rows, int chunk) {
    __shared__ CgState st;
    KCtl* ctl = reinterpret_cast<KCtl*>(K.work);
    barrier_init(K);
    double* partials = K.work + kCtlDoubles;
    double* vec = partials + kPartials;
    const int n = (int)K.n;
    double* z = vec;
    double* inv = vec + n;
    double* r = vec + 2 * (int64_t)n;
    double* p = vec + 3 * (int64_t)n;
    double* q = vec + 4 * (int64_t)n;
    double* x = K.x;
    const int c0 = blockIdx.x * chunk;
    const int c1 = c0 + chunk < n ? c0 + chunk : n;
    const bool jac = K.jacobi != 0, linf = K.norm_inf != 0;
    bool ok = true;
    {  // r = b - A x, z = M r, p = q = 0; |r| and r.z
        double loc[2] = {0.0, 0.0};
        auto gx = [&](int i) { return __ldcg(x + i); };
        for (int c = c0 + threadIdx.x; c < c1; c += THREADS) {
            const double ax = rows.apply(c, __ldg(K.diag + c), gx);
            const double rk = __ldg(K.rhs + c) - ax;
            const double iv = inv_diag(K.diag, c, jac);
            const double zk = iv * rk;
            __stcg(r + c, rk);
            __stcg(q + c, 0.0);
            __stcg(p + c, 0.0);
            __stcg(inv + c, iv);
            __stcg(z + c, zk);
            loc[0] = norm_acc(loc[0], rk, linf);
            loc[1] += rk * zk;
        }
        ok = grid_reduce<2, THREADS>(ctl, partials, loc, linf ? 1u : 0u);
        if (threadIdx.x == 0) {
            const double r0 = norm_fin(loc[0], linf);
            st.r0 = r0;
            st.final = r0;
            st.thresh = fmax(K.atol, K.rtol * r0);
            st.rz_old = loc[1];
            st.beta = 0.0;
            st.alpha = 0.0;
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
    bool pending = false;  // x += alpha p of the last update pass not yet applied
    for (int it = 1; ok && !st.done && it <= K.max_iter; ++it) {
        {  // x += alpha_(k-1) p; w = A z; p = z + beta p; q = w + beta q; p . q
            const double beta = st.beta, alpha_prev = st.alpha;
            double loc[1] = {0.0};
            // Plain (L1-cacheable) loads: z is written only before the grid
            // barrier that precedes this pass (see pcg1_smem_body).
            auto gz = [&](int j) { return z[j]; };
            for (int c = c0 + threadIdx.x; c < c1; c += THREADS) {
                const double zc = z[c];
                const double w = rows.apply(c, __ldg(K.diag + c), gz);
                const double pold = __ldcg(p + c);
                const double qold = __ldcg(q + c);
                if (pending) __stcg(x + c, __ldcg(x + c) + alpha_prev * pold);
                const double pk = zc + pold * beta;
                const double qk = w + qold * beta;
                __stcg(p + c, pk);
                __stcg(q + c, qk);
                loc[0] += pk * qk;
            }
            ok = grid_reduce<1, THREADS>(ctl, partials, loc, 0u);
            if (!ok) break;
            if (threadIdx.x == 0) st.alpha = st.rz_old / loc[0];
            __syncthreads();
        }
        {  // r -= alpha q; z = M r; |r|, r.z
            const double alpha = st.alpha;
            double loc[2] = {0.0, 0.0};
            for (int c = c0 + threadIdx.x; c < c1; c += THREADS) {
                const double rk = __ldcg(r + c) - alpha * __ldcg(q + c);
                const double zk = __ldcg(inv + c) * rk;
                __stcg(r + c, rk);
                __stcg(z + c, zk);
                loc[0] = norm_acc(loc[0], rk, linf);
                loc[1] += rk * zk;
            }
            pending = true;
            ok = grid_reduce<2, THREADS>(ctl, partials, loc, linf ? 1u : 0u);
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
    }
    if (ok && pending) {  // the last iteration's x += alpha p (own cells only)
        const double alpha = st.alpha;
        for (int c = c0 + threadIdx.x; c < c1; c += THREADS) __stcg(x + c, __ldcg(x + c) + alpha * __ldcg(p + c));
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

template <bool SYM, int THREADS, int MINB>
__global__ void __launch_bounds__(THREADS, MINB) k_pcg1_stream_box(gf_krylov_t K, int chunk) {
    BoxRows<double, SYM, false, int> rows{K.val, (int)K.n, (int)K.stride_y, (int)K.stride_z};
    pcg1_stream_body<THREADS>(K, rows, chunk);
}

template <int WIDTH, int THREADS, int MINB>
__global__ void __launch_bounds__(THREADS, MINB) k_pcg1_stream_ell(gf_krylov_t K, int chunk) {
    EllRows<double, WIDTH, int> rows{K.val, K.nbr, (int)K.n, K.width, K.row_len};
    pcg1_stream_body<THREADS>(K, rows, chunk);
}

// ---------------------------------------------------------------------------
// Single-reduction CG with shared-memory-resident vectors and a halo sync.
// The recurrences are those of pcg1_sr_body (Chronopoulos and Gear): with
// z = M r and w = A z, gamma = r.z, delta = w.z, beta = gamma / gamma_old,
// alpha = gamma / (delta - beta gamma / alpha_old), p = z + beta p,
// q = w + beta q (q = A p), x += alpha p, r -= alpha q.  An iteration is two
// passes: gather w = A z and reduce (|r|, gamma, delta) in ONE grid
// reduction (|r| and gamma of the previous update ride along with delta),
// then update the own cells and publish the new z.  The gather of the next
// iteration needs the new z of the neighbouring blocks only, so the second
// synchronisation is point to point: each block waits for the blocks that
// hold the cells its rows read (found once, from the row structure), not
// for the whole grid.  A block cannot overwrite z before every block has
// finished reading it: the overwrite follows the grid reduction, which
// follows every block's gather.  The stopping test sees |r_k| one gather
// later than pcg1_qrec_body; iteration count, statistics and final x are
// those of a PCG run (one extra gather at the end, no extra update).  Each
// block keeps r, p, q and w of its cells in shared memory (4 doubles a
// cell) and updates its cells of x in place in global memory.

// Halo flags: one 64-bit epoch per block, one per 128-byte line (flags of
// neighbouring blocks sharing a line cost ~1.7 us an iteration at 262K
// cells), after z and the Jacobi inverse in the workspace.
constexpr int64_t kHaloFlagStride = 16;
constexpr int64_t kHaloFlagDoubles = kMaxBlocks * kHaloFlagStride;

// Publish epoch ep for this block, then wait (bounded, like grid_reduce)
// until blocks blo..bhi have published it.  The CTA barrier before the
// release makes it cumulative over the whole block's writes; the acquires
// and the CTA barrier after them order every thread's later reads.
__device__ bool halo_sync(KCtl* ctl, unsigned long long* flags, unsigned long long ep, int blo, int bhi) {
    __syncthreads();
    if (threadIdx.x == 0)
        asm volatile("fence.acq_rel.gpu;\n\tst.relaxed.gpu.global.u64 [%0], %1;" ::"l"(
                         flags + kHaloFlagStride * blockIdx.x),
                     "l"(ep)
                     : "memory");
    int err = 0;
    for (int b = blo + (int)threadIdx.x; b <= bhi && !err; b += blockDim.x) {
        if (b == (int)blockIdx.x) continue;
        long long it = 0;
        while (load_acquire(flags + kHaloFlagStride * b) < ep) {
            __nanosleep(20);
            ++it;
            if ((it & 255) == 0 && vload(&ctl->error) != 0) {
                err = 1;
                break;
            }
            if (it > g_spin) {
                atomicExch(&ctl->error, 1);
                err = 1;
                break;
            }
        }
    }
    return __syncthreads_or(err) == 0;
}

template <int THREADS, int U, int V, class Rows>
__device__ void pcg1_halo_body(const gf_krylov_t& K, const Rows& rows, int chunk) {
    __shared__ CgState st;
    __shared__ int s_lo, s_hi;
    extern __shared__ __align__(16) double sm[];
    KCtl* ctl = reinterpret_cast<KCtl*>(K.work);
    barrier_init(K);
    double* partials = K.work + kCtlDoubles;
    double* vec = partials + kPartials;
    const int n = (int)K.n;
    double* z = vec;
    double* inv = vec + n;
    unsigned long long* flags = reinterpret_cast<unsigned long long*>(vec + 2 * (int64_t)n);
    double* x = K.x;
    const int c0 = blockIdx.x * chunk;
    const int c1 = c0 + chunk < n ? c0 + chunk : n;
    const int m = c1 > c0 ? c1 - c0 : 0;
    double* rs = sm;
    double* ps = sm + chunk;
    double* qs = sm + 2 * chunk;
    double* ws = sm + 3 * chunk;
    const bool jac = K.jacobi != 0, linf = K.norm_inf != 0;
    if (threadIdx.x == 0) {
        s_lo = n;
        s_hi = -1;
        // Visible to every block after the first grid reduction below.
        flags[kHaloFlagStride * blockIdx.x] = 0ull;
    }
    __syncthreads();
    bool ok = true;
    {  // r = b - A x, z = M r, p = q = 0; |r| and r.z; the cells the rows read
        double loc[2] = {0.0, 0.0};
        int lo = n, hi = -1;
        auto gx = [&](int i) { return __ldcg(x + i); };
        for (int i = threadIdx.x; i < m; i += THREADS) {
            const int c = c0 + i;
            const double ax = rows.apply(c, __ldg(K.diag + c), gx);
            const double rk = __ldg(K.rhs + c) - ax;
            const double iv = inv_diag(K.diag, c, jac);
            const double zk = iv * rk;
            rows.span(c, lo, hi);
            rs[i] = rk;
            ps[i] = 0.0;
            qs[i] = 0.0;
            inv[c] = iv;
            __stcg(z + c, zk);
            loc[0] = norm_acc(loc[0], rk, linf);
            loc[1] += rk * zk;
        }
        lo = __reduce_min_sync(0xffffffffu, lo);
        hi = __reduce_max_sync(0xffffffffu, hi);
        if ((threadIdx.x & 31) == 0) {
            atomicMin(&s_lo, lo);
            atomicMax(&s_hi, hi);
        }
        ok = grid_reduce<2, THREADS>(ctl, partials, loc, linf ? 1u : 0u);
        if (threadIdx.x == 0) {
            const double r0 = norm_fin(loc[0], linf);
            st.r0 = r0;
            st.final = r0;
            st.thresh = fmax(K.atol, K.rtol * r0);
            st.rz_old = loc[1];
            st.alpha = 1.0;
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
            // Blocks holding the cells this block's rows read (itself when it has none).
            s_lo = m > 0 ? s_lo / chunk : (int)blockIdx.x;
            s_hi = m > 0 ? s_hi / chunk : (int)blockIdx.x;
        }
        __syncthreads();
    }
    double rn = 0.0, gm = 0.0;  // this thread's |r| and r.z of the last update
    // x += alpha p of an update is applied in the next gather pass (as in
    // pcg1_qrec_body): the same additions in the same order.
    bool pending = false;
    for (int it = 1; ok && !st.done && K.max_iter > 0; ++it) {
        {  // x += alpha p; w = A z; delta = w.z; one reduction with |r| and gamma of the last update
            const double alpha_prev = st.alpha;
            const bool upd = pending;
            double loc[3] = {rn, gm, 0.0};
            auto gz = [&](int j) { return z[j]; };
            for (int i0 = threadIdx.x; i0 < m; i0 += U * THREADS) {
                double zc[U], w[U], xo[U];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int i = i0 + u * THREADS;
                    if (i < m) {
                        const int c = c0 + i;
                        if (upd) xo[u] = __ldcg(x + c);
                        zc[u] = z[c];
                        w[u] = rows.apply(c, __ldg(K.diag + c), gz);
                    }
                }
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int i = i0 + u * THREADS;
                    if (i < m) {
                        if (upd) __stcg(x + c0 + i, xo[u] + alpha_prev * ps[i]);
                        ws[i] = w[u];
                        loc[2] += w[u] * zc[u];
                    }
                }
            }
            pending = false;
            // alpha_prev is read above by every thread before this barrier.
            ok = grid_reduce<3, THREADS>(ctl, partials, loc, linf ? 1u : 0u);
            if (!ok) break;
            if (threadIdx.x == 0) {
                if (it > 1) {
                    const double fin = norm_fin(loc[0], linf);
                    st.final = fin;
                    if (fin < st.thresh) {
                        st.done = 1;
                        st.converged = 1;
                        st.its = it - 1;
                        st.status = GF_OK;
                    } else if (!isfinite(fin)) {
                        st.done = 1;
                        st.its = it - 1;
                        st.status = GF_NONFINITE;
                    } else if (it - 1 >= K.max_iter) {
                        st.done = 1;
                        st.its = K.max_iter;
                    }
                }
                if (!st.done) {
                    const double g = it > 1 ? loc[1] : st.rz_old;
                    const double b = it > 1 ? g / st.rz_old : 0.0;
                    st.alpha = g / (it > 1 ? loc[2] - b * g / st.alpha : loc[2]);
                    st.beta = b;
                    st.rz_old = g;
                }
            }
            __syncthreads();
            if (st.done) break;
        }
        {  // p = z + beta p; q = w + beta q; r -= alpha q; z = M r; x follows next pass
            // The own z is recomputed as inv r: the bits it was stored with.
            const double alpha = st.alpha, beta = st.beta;
            pending = true;
            rn = 0.0;
            gm = 0.0;
            for (int i0 = threadIdx.x; i0 < m; i0 += V * THREADS) {
                double iv[V];
#pragma unroll
                for (int u = 0; u < V; ++u) {
                    const int i = i0 + u * THREADS;
                    if (i < m) iv[u] = inv[c0 + i];
                }
#pragma unroll
                for (int u = 0; u < V; ++u) {
                    const int i = i0 + u * THREADS;
                    if (i < m) {
                        const int c = c0 + i;
                        const double pk = iv[u] * rs[i] + ps[i] * beta;
                        const double qk = ws[i] + qs[i] * beta;
                        ps[i] = pk;
                        qs[i] = qk;
                        const double rk = rs[i] - alpha * qk;
                        const double zk = iv[u] * rk;
                        rs[i] = rk;
                        __stcg(z + c, zk);
                        rn = norm_acc(rn, rk, linf);
                        gm += rk * zk;
                    }
                }
            }
            ok = halo_sync(ctl, flags, (unsigned long long)it, s_lo, s_hi);
        }
    }
    if (pending) {
        const double alpha = st.alpha;
        for (int i = threadIdx.x; i < m; i += THREADS) __stcg(x + c0 + i, __ldcg(x + c0 + i) + alpha * ps[i]);
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

template <bool SYM, int U>
__global__ void __launch_bounds__(1024, 1) k_pcg1_halo_box(gf_krylov_t K, int chunk) {
    BoxRows<double, SYM, false, int> rows{K.val, (int)K.n, (int)K.stride_y, (int)K.stride_z};
    pcg1_halo_body<1024, U, 2>(K, rows, chunk);
}

template <int WIDTH, int U>
__global__ void __launch_bounds__(1024, 1) k_pcg1_halo_ell(gf_krylov_t K, int chunk) {
    EllRows<double, WIDTH, int> rows{K.val, K.nbr, (int)K.n, K.width, K.row_len};
    pcg1_halo_body<1024, U, 2>(K, rows, chunk);
}

// ---------------------------------------------------------------------------
// FP32-inner CG in FP64 refinement (the algorithm of pcg1_mixed_body) with
// each block's own-cell FP32 vectors resident in shared memory: r, q, the
// correction d, the Jacobi inverse and (KEEP_P) p, 4-5 floats a cell.  What
// neighbours read goes through global memory as in pcg1_smem_body: FP32
// pairs {z, p} (8 bytes a stencil point) double-buffered by iteration
// parity, plus the FP32 matrix copy and, once per refinement cycle, x (FP64)
// for the true residual.  Per cell the arithmetic is that of
// pcg1_mixed_body, so only the order of the reduction partial sums differs.
//
// Global layout after the header: n doubles (unused), then floats: the two
// pair buffers (4n), the FP32 coefficients (ncoef n) and diagonal (n).
template <int THREADS, int U, int V, bool KEEP_P, class Rows64, class Rows32>
__device__ void pcg1_mixed_smem_body(const gf_krylov_t& K, const Rows64& rows64, Rows32 rows32, int ncoef,
                                     int chunk) {
    __shared__ CgState st;
    __shared__ double s_target;
    __shared__ int s_cycle_done;
    extern __shared__ __align__(16) double sm[];
    KCtl* ctl = reinterpret_cast<KCtl*>(K.work);
    barrier_init(K);
    double* partials = K.work + kCtlDoubles;
    double* base = partials + kPartials;
    const int n = (int)K.n;
    float* f = reinterpret_cast<float*>(base + n);
    float2* zp0 = reinterpret_cast<float2*>(f);
    float2* zp1 = zp0 + n;
    float* val32 = f + 4 * (int64_t)n;
    float* diag32 = val32 + (int64_t)ncoef * n;
    rows32.val = val32;
    const int c0 = blockIdx.x * chunk;
    const int c1 = c0 + chunk < n ? c0 + chunk : n;
    const int m = c1 > c0 ? c1 - c0 : 0;
    float* smf = reinterpret_cast<float*>(sm);
    float* rs = smf;
    float* qs = smf + chunk;
    float* ds = smf + 2 * chunk;
    float* ivs = smf + 3 * chunk;
    float* ps = smf + 4 * chunk;  // only with KEEP_P
    double* x = K.x;
    const bool jac = K.jacobi != 0, linf = K.norm_inf != 0;
    const bool sym_box = K.stride_y > 0 && K.symmetric;
    bool ok = true;
    int its = 0;

    for (int i = threadIdx.x; i < m; i += THREADS) {
        const int c = c0 + i;
        for (int s = 0; s < ncoef; ++s) {
            const int src = sym_box ? (2 * s + 1) : s;
            __stcg(val32 + (int64_t)s * n + c, (float)__ldg(K.val + (int64_t)src * n + c));
        }
        __stcg(diag32 + c, (float)__ldg(K.diag + c));
        ivs[i] = (float)inv_diag(K.diag, c, jac);
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
                for (int i = threadIdx.x; i < m; i += THREADS) x[c0 + i] = x[c0 + i] + (double)ds[i];
                pending = false;
            }
            // The barrier also publishes x and (cycle 0) the FP32 matrix.
            double dummy[1] = {0.0};
            ok = grid_reduce<1, THREADS>(ctl, partials, dummy, 0u);
            if (!ok) break;
            auto gx = [&](int i) { return __ldcg(x + i); };
            for (int i = threadIdx.x; i < m; i += THREADS) {
                const int c = c0 + i;
                const double ax = rows64.apply(c, __ldg(K.diag + c), gx);
                const double rk = __ldg(K.rhs + c) - ax;
                const float r32 = (float)rk;
                const float z32 = ivs[i] * r32;
                rs[i] = r32;
                ds[i] = 0.0f;
                __stcg(zp0 + c, make_float2(z32, 0.0f));
                loc[0] = norm_acc(loc[0], rk, linf);
                loc[1] += (double)r32 * (double)z32;
            }
            ok = grid_reduce<2, THREADS>(ctl, partials, loc, linf ? 1u : 0u);
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
                s_target = fmax(K.inner_eta * nr, (K.inner_margin > 0.0 ? K.inner_margin : 0.5) * st.thresh);
                s_cycle_done = 0;
            }
            __syncthreads();
            if (st.done || cycle == K.max_outer || its >= K.max_iter) break;
        }
        pending = true;
        int k = 0;  // inner iteration of this cycle: pair buffer parity
        while (ok && !s_cycle_done && its < K.max_iter) {
            ++its;
            ++k;
            const float2* cur = (k & 1) ? zp0 : zp1;
            float2* nxt = (k & 1) ? zp1 : zp0;
            {  // p_new = z + p_old beta; q = A p_new; p_new . q
                const float beta = (float)st.beta;
                double loc[1] = {0.0};
                // Plain (L1-cacheable) loads: see pcg1_smem_body.
                auto gp = [&](int j) {
                    const float2 v = cur[j];
                    return v.x + v.y * beta;
                };
                for (int i0 = threadIdx.x; i0 < m; i0 += U * THREADS) {
                    float pc[U], ap[U];
#pragma unroll
                    for (int u = 0; u < U; ++u) {
                        const int i = i0 + u * THREADS;
                        if (i < m) {
                            const int c = c0 + i;
                            pc[u] = gp(c);
                            ap[u] = rows32.apply(c, __ldcg(diag32 + c), gp);
                        }
                    }
#pragma unroll
                    for (int u = 0; u < U; ++u) {
                        const int i = i0 + u * THREADS;
                        if (i < m) {
                            __stcg(&nxt[c0 + i].y, pc[u]);
                            if (KEEP_P) ps[i] = pc[u];
                            qs[i] = ap[u];
                            loc[0] += (double)pc[u] * (double)ap[u];
                        }
                    }
                }
                ok = grid_reduce<1, THREADS>(ctl, partials, loc, 0u);
                if (!ok) break;
                if (threadIdx.x == 0) st.alpha = st.rz_old / loc[0];
                __syncthreads();
            }
            {  // d += alpha p; r -= alpha q; z = M r; |r|, r.z (own cells)
                const float alpha = (float)st.alpha;
                double loc[2] = {0.0, 0.0};
                for (int i0 = threadIdx.x; i0 < m; i0 += V * THREADS) {
                    float pv[V];
#pragma unroll
                    for (int u = 0; u < V; ++u) {
                        const int i = i0 + u * THREADS;
                        if (i < m) pv[u] = KEEP_P ? ps[i] : __ldcg(&nxt[c0 + i].y);
                    }
#pragma unroll
                    for (int u = 0; u < V; ++u) {
                        const int i = i0 + u * THREADS;
                        if (i < m) {
                            ds[i] = ds[i] + alpha * pv[u];
                            const float rk = rs[i] - alpha * qs[i];
                            const float zk = ivs[i] * rk;
                            rs[i] = rk;
                            __stcg(&nxt[c0 + i].x, zk);
                            loc[0] = norm_acc(loc[0], (double)rk, linf);
                            loc[1] += (double)rk * (double)zk;
                        }
                    }
                }
                ok = grid_reduce<2, THREADS>(ctl, partials, loc, linf ? 1u : 0u);
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
        }
    }
    if (ok && pending) {
        // iteration budget spent inside a cycle: keep its correction
        for (int i = threadIdx.x; i < m; i += THREADS) x[c0 + i] = x[c0 + i] + (double)ds[i];
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

template <bool SYM, int THREADS, bool KEEP_P>
__global__ void __launch_bounds__(THREADS, 1) k_pcg1_mixed_smem_box(gf_krylov_t K, int chunk) {
    BoxRows<double, SYM, false, int> rows64{K.val, (int)K.n, (int)K.stride_y, (int)K.stride_z};
    BoxRows<float, SYM, SYM, int> rows32{nullptr, (int)K.n, (int)K.stride_y, (int)K.stride_z};
    pcg1_mixed_smem_body<THREADS, smem_gather_cells(THREADS), smem_update_cells(THREADS), KEEP_P>(
        K, rows64, rows32, SYM ? 3 : 6, chunk);
}

template <int WIDTH, int THREADS, bool KEEP_P>
__global__ void __launch_bounds__(THREADS, 1) k_pcg1_mixed_smem_ell(gf_krylov_t K, int chunk) {
    EllRows<double, WIDTH, int> rows64{K.val, K.nbr, (int)K.n, K.width, K.row_len};
    EllRows<float, WIDTH, int> rows32{nullptr, K.nbr, (int)K.n, K.width, K.row_len};
    pcg1_mixed_smem_body<THREADS, smem_gather_cells(THREADS), smem_update_cells(THREADS), KEEP_P>(
        K, rows64, rows32, K.width, chunk);
}

// ---------------------------------------------------------------------------
// FP32-inner CG in FP64 refinement with shared-memory-resident FP32 vectors
// and q = A p formed by recurrence (q_k = A z_k + beta q_(k-1), as in
// pcg1_qrec_body): the stencil gathers the FP32 z alone.  Each block keeps
// r, q, p, the correction d and the Jacobi inverse of its cells in shared
// memory (5 floats a cell) and folds d into the FP64 x once per refinement
// cycle.  Cycle control, true residuals and stopping rule are those of
// pcg1_mixed_body.
//
// Global layout after the header: n doubles (unused), then floats: z (n),
// the FP32 coefficients (ncoef n) and diagonal (n).
template <int THREADS, int U, int V, class Rows64, class Rows32>
__device__ void pcg1_mixed_qrec_body(const gf_krylov_t& K, const Rows64& rows64, Rows32 rows32, int ncoef,
                                     int chunk) {
    __shared__ CgState st;
    __shared__ double s_target;
    __shared__ int s_cycle_done;
    extern __shared__ __align__(16) double sm[];
    KCtl* ctl = reinterpret_cast<KCtl*>(K.work);
    barrier_init(K);
    double* partials = K.work + kCtlDoubles;
    double* base = partials + kPartials;
    const int n = (int)K.n;
    float* f = reinterpret_cast<float*>(base + n);
    float* z = f;
    float* val32 = f + (int64_t)n;
    float* diag32 = val32 + (int64_t)ncoef * n;
    rows32.val = val32;
    const int c0 = blockIdx.x * chunk;
    const int c1 = c0 + chunk < n ? c0 + chunk : n;
    const int m = c1 > c0 ? c1 - c0 : 0;
    float* smf = reinterpret_cast<float*>(sm);
    float* rs = smf;
    float* qs = smf + chunk;
    float* ds = smf + 2 * chunk;
    float* ivs = smf + 3 * chunk;
    float* ps = smf + 4 * chunk;
    double* x = K.x;
    const bool jac = K.jacobi != 0, linf = K.norm_inf != 0;
    const bool sym_box = K.stride_y > 0 && K.symmetric;
    bool ok = true;
    int its = 0;

    for (int i = threadIdx.x; i < m; i += THREADS) {
        const int c = c0 + i;
        for (int s = 0; s < ncoef; ++s) {
            const int src = sym_box ? (2 * s + 1) : s;
            __stcg(val32 + (int64_t)s * n + c, (float)__ldg(K.val + (int64_t)src * n + c));
        }
        __stcg(diag32 + c, (float)__ldg(K.diag + c));
        ivs[i] = (float)inv_diag(K.diag, c, jac);
    }
    if (threadIdx.x == 0) {
        st.its = 0;
        st.converged = 0;
        st.status = GF_MAX_ITER;
        st.done = 0;
    }
    bool pending = false;
    for (int cycle = 0; ok && cycle <= K.max_outer; ++cycle) {
        {  // fold the pending correction, then the true residual in FP64
            double loc[2] = {0.0, 0.0};
            if (pending) {
                for (int i = threadIdx.x; i < m; i += THREADS) x[c0 + i] = x[c0 + i] + (double)ds[i];
                pending = false;
            }
            // The barrier also publishes x and (cycle 0) the FP32 matrix.
            double dummy[1] = {0.0};
            ok = grid_reduce<1, THREADS>(ctl, partials, dummy, 0u);
            if (!ok) break;
            auto gx = [&](int i) { return __ldcg(x + i); };
            for (int i = threadIdx.x; i < m; i += THREADS) {
                const int c = c0 + i;
                const double ax = rows64.apply(c, __ldg(K.diag + c), gx);
                const double rk = __ldg(K.rhs + c) - ax;
                const float r32 = (float)rk;
                const float z32 = ivs[i] * r32;
                rs[i] = r32;
                ds[i] = 0.0f;
                ps[i] = 0.0f;
                qs[i] = 0.0f;
                __stcg(z + c, z32);
                loc[0] = norm_acc(loc[0], rk, linf);
                loc[1] += (double)r32 * (double)z32;
            }
            ok = grid_reduce<2, THREADS>(ctl, partials, loc, linf ? 1u : 0u);
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
                s_target = fmax(K.inner_eta * nr, (K.inner_margin > 0.0 ? K.inner_margin : 0.5) * st.thresh);
                s_cycle_done = 0;
            }
            __syncthreads();
            if (st.done || cycle == K.max_outer || its >= K.max_iter) break;
        }
        pending = true;
        while (ok && !s_cycle_done && its < K.max_iter) {
            ++its;
            {  // w = A z; p = z + beta p; q = w + beta q; p . q
                const float beta = (float)st.beta;
                double loc[1] = {0.0};
                // Plain (L1-cacheable) loads: see pcg1_smem_body.
                auto gz = [&](int j) { return z[j]; };
                for (int i0 = threadIdx.x; i0 < m; i0 += U * THREADS) {
                    float zc[U], w[U];
#pragma unroll
                    for (int u = 0; u < U; ++u) {
                        const int i = i0 + u * THREADS;
                        if (i < m) {
                            const int c = c0 + i;
                            zc[u] = z[c];
                            w[u] = rows32.apply(c, __ldcg(diag32 + c), gz);
                        }
                    }
#pragma unroll
                    for (int u = 0; u < U; ++u) {
                        const int i = i0 + u * THREADS;
                        if (i < m) {
                            const float pk = zc[u] + ps[i] * beta;
                            const float qk = w[u] + qs[i] * beta;
                            ps[i] = pk;
                            qs[i] = qk;
                            loc[0] += (double)pk * (double)qk;
                        }
                    }
                }
                ok = grid_reduce<1, THREADS>(ctl, partials, loc, 0u);
                if (!ok) break;
                if (threadIdx.x == 0) st.alpha = st.rz_old / loc[0];
                __syncthreads();
            }
            {  // r -= alpha q; z = M r; |r|, r.z (own cells); d += alpha p during the reduction
                const float alpha = (float)st.alpha;
                double loc[2] = {0.0, 0.0};
                for (int i = threadIdx.x; i < m; i += THREADS) {
                    const float rk = rs[i] - alpha * qs[i];
                    const float zk = ivs[i] * rk;
                    rs[i] = rk;
                    __stcg(z + c0 + i, zk);
                    loc[0] = norm_acc(loc[0], (double)rk, linf);
                    loc[1] += (double)rk * (double)zk;
                }
                auto dupd = [&](int t, int nt) {
                    for (int i = t; i < m; i += nt) ds[i] = ds[i] + alpha * ps[i];
                };
                ok = grid_reduce_side<2, THREADS>(ctl, partials, loc, linf ? 1u : 0u, dupd);
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
        }
    }
    if (ok && pending) {
        // iteration budget spent inside a cycle: keep its correction
        for (int i = threadIdx.x; i < m; i += THREADS) x[c0 + i] = x[c0 + i] + (double)ds[i];
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

template <bool SYM, int U>
__global__ void __launch_bounds__(1024, 1) k_pcg1_mixed_qrec_box(gf_krylov_t K, int chunk) {
    BoxRows<double, SYM, false, int> rows64{K.val, (int)K.n, (int)K.stride_y, (int)K.stride_z};
    BoxRows<float, SYM, SYM, int> rows32{nullptr, (int)K.n, (int)K.stride_y, (int)K.stride_z};
    pcg1_mixed_qrec_body<1024, U, 1>(K, rows64, rows32, SYM ? 3 : 6, chunk);
}

template <int WIDTH, int U>
__global__ void __launch_bounds__(1024, 1) k_pcg1_mixed_qrec_ell(gf_krylov_t K, int chunk) {
    EllRows<double, WIDTH, int> rows64{K.val, K.nbr, (int)K.n, K.width, K.row_len};
    EllRows<float, WIDTH, int> rows32{nullptr, K.nbr, (int)K.n, K.width, K.row_len};
    pcg1_mixed_qrec_body<1024, U, 1>(K, rows64, rows32, K.width, chunk);
}

// ---------------------------------------------------------------------------
// FP32-inner CG in FP64 refinement (the cycles of pcg1_mixed_qrec_body) with
// the inner iterations in the single-reduction form of pcg1_halo_body: one
// grid reduction of |r|, gamma = r.z and delta = w.z and one halo sync with
// the neighbouring blocks per inner iteration.  Each block keeps the FP32
// r, q, d, Jacobi inverse, p and w = A z of its cells in shared memory (6
// floats a cell).  The halo flags use the first kHaloFlagDoubles doubles
// of the workspace's vector region, which the FP32-inner forms leave
// unused (n >= kHaloFlagDoubles).  A cycle ends when the FP32 residual of
// the last update is below the cycle target, seen at the next reduction,
// or when the iteration budget is spent; the same updates as
// pcg1_mixed_qrec_body up to the rounding of alpha.
template <int THREADS, class Rows64, class Rows32>
__device__ void pcg1_mixed_halo_body(const gf_krylov_t& K, const Rows64& rows64, Rows32 rows32, int ncoef,
                                     int chunk) {
    __shared__ CgState st;
    __shared__ double s_target;
    __shared__ int s_cycle_done;
    __shared__ int s_lo, s_hi;
    extern __shared__ __align__(16) double sm[];
    KCtl* ctl = reinterpret_cast<KCtl*>(K.work);
    barrier_init(K);
    double* partials = K.work + kCtlDoubles;
    double* base = partials + kPartials;
    unsigned long long* flags = reinterpret_cast<unsigned long long*>(base);
    const int n = (int)K.n;
    float* f = reinterpret_cast<float*>(base + n);
    float* z = f;
    float* val32 = f + (int64_t)n;
    float* diag32 = val32 + (int64_t)ncoef * n;
    rows32.val = val32;
    const int c0 = blockIdx.x * chunk;
    const int c1 = c0 + chunk < n ? c0 + chunk : n;
    const int m = c1 > c0 ? c1 - c0 : 0;
    float* smf = reinterpret_cast<float*>(sm);
    float* rs = smf;
    float* qs = smf + chunk;
    float* ds = smf + 2 * chunk;
    float* ivs = smf + 3 * chunk;
    float* ps = smf + 4 * chunk;
    float* ws = smf + 5 * chunk;
    double* x = K.x;
    const bool jac = K.jacobi != 0, linf = K.norm_inf != 0;
    const bool sym_box = K.stride_y > 0 && K.symmetric;
    bool ok = true;
    int its = 0;

    if (threadIdx.x == 0) {
        st.its = 0;
        st.converged = 0;
        st.status = GF_MAX_ITER;
        st.done = 0;
        s_lo = n;
        s_hi = -1;
        // Visible to every block after the first grid reduction below.
        flags[kHaloFlagStride * blockIdx.x] = 0ull;
    }
    __syncthreads();
    {
        int lo = n, hi = -1;
        for (int i = threadIdx.x; i < m; i += THREADS) {
            const int c = c0 + i;
            for (int sl = 0; sl < ncoef; ++sl) {
                const int src = sym_box ? (2 * sl + 1) : sl;
                __stcg(val32 + (int64_t)sl * n + c, (float)__ldg(K.val + (int64_t)src * n + c));
            }
            __stcg(diag32 + c, (float)__ldg(K.diag + c));
            ivs[i] = (float)inv_diag(K.diag, c, jac);
            rows64.span(c, lo, hi);
        }
        lo = __reduce_min_sync(0xffffffffu, lo);
        hi = __reduce_max_sync(0xffffffffu, hi);
        if ((threadIdx.x & 31) == 0) {
            atomicMin(&s_lo, lo);
            atomicMax(&s_hi, hi);
        }
    }
    unsigned long long hep = 0;
    bool pending = false;
    for (int cycle = 0; ok && cycle <= K.max_outer; ++cycle) {
        {  // fold the pending correction, then the true residual in FP64
            double loc[2] = {0.0, 0.0};
            if (pending) {
                for (int i = threadIdx.x; i < m; i += THREADS) x[c0 + i] = x[c0 + i] + (double)ds[i];
                pending = false;
            }
            // The barrier also publishes x, the halo flags and (cycle 0) the FP32 matrix.
            double dummy[1] = {0.0};
            ok = grid_reduce<1, THREADS>(ctl, partials, dummy, 0u);
            if (!ok) break;
            auto gx = [&](int i) { return __ldcg(x + i); };
            for (int i = threadIdx.x; i < m; i += THREADS) {
                const int c = c0 + i;
                const double ax = rows64.apply(c, __ldg(K.diag + c), gx);
                const double rk = __ldg(K.rhs + c) - ax;
                const float r32 = (float)rk;
                const float z32 = ivs[i] * r32;
                rs[i] = r32;
                ds[i] = 0.0f;
                ps[i] = 0.0f;
                qs[i] = 0.0f;
                __stcg(z + c, z32);
                loc[0] = norm_acc(loc[0], rk, linf);
                loc[1] += (double)r32 * (double)z32;
            }
            ok = grid_reduce<2, THREADS>(ctl, partials, loc, linf ? 1u : 0u);
            if (!ok) break;
            if (threadIdx.x == 0) {
                const double nr = norm_fin(loc[0], linf);
                if (cycle == 0) {
                    st.r0 = nr;
                    st.thresh = fmax(K.atol, K.rtol * nr);
                    // Blocks holding the cells this block's rows read.
                    s_lo = m > 0 ? s_lo / chunk : (int)blockIdx.x;
                    s_hi = m > 0 ? s_hi / chunk : (int)blockIdx.x;
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
                st.alpha = 1.0;
                s_target = fmax(K.inner_eta * nr, (K.inner_margin > 0.0 ? K.inner_margin : 0.5) * st.thresh);
                s_cycle_done = 0;
            }
            __syncthreads();
            if (st.done || cycle == K.max_outer || its >= K.max_iter) break;
        }
        pending = true;
        double rn = 0.0, gm = 0.0;  // this thread's |r| and r.z of the last update
        for (int k = 1; ok; ++k) {
            {  // w = A z; delta = w.z; one reduction with |r| and gamma of the last update
                double loc[3] = {rn, gm, 0.0};
                auto gz = [&](int j) { return z[j]; };
                for (int i = threadIdx.x; i < m; i += THREADS) {
                    const int c = c0 + i;
                    const float zc = z[c];
                    const float w = rows32.apply(c, __ldcg(diag32 + c), gz);
                    ws[i] = w;
                    loc[2] += (double)w * (double)zc;
                }
                ok = grid_reduce<3, THREADS>(ctl, partials, loc, linf ? 1u : 0u);
                if (!ok) break;
                if (threadIdx.x == 0) {
                    if (k > 1) {
                        const double nr = norm_fin(loc[0], linf);
                        if (!(nr >= s_target) || !isfinite(nr)) s_cycle_done = 1;
                    }
                    if (its >= K.max_iter) s_cycle_done = 1;
                    if (!s_cycle_done) {
                        const double g = k > 1 ? loc[1] : st.rz_old;
                        const double b = k > 1 ? g / st.rz_old : 0.0;
                        st.alpha = g / (k > 1 ? loc[2] - b * g / st.alpha : loc[2]);
                        st.beta = b;
                        st.rz_old = g;
                    }
                }
                __syncthreads();
                if (s_cycle_done) break;
            }
            ++its;
            {  // p = z + beta p; q = w + beta q; d += alpha p; r -= alpha q; z = M r
                // The own z is recomputed as inv r: the bits it was stored with.
                const float alpha = (float)st.alpha, beta = (float)st.beta;
                rn = 0.0;
                gm = 0.0;
                for (int i = threadIdx.x; i < m; i += THREADS) {
                    const float pk = ivs[i] * rs[i] + ps[i] * beta;
                    const float qk = ws[i] + qs[i] * beta;
                    ps[i] = pk;
                    qs[i] = qk;
                    ds[i] = ds[i] + alpha * pk;
                    const float rk = rs[i] - alpha * qk;
                    const float zk = ivs[i] * rk;
                    rs[i] = rk;
                    __stcg(z + c0 + i, zk);
                    rn = norm_acc(rn, (double)rk, linf);
                    gm += (double)rk * (double)zk;
                }
                ok = halo_sync(ctl, flags, ++hep, s_lo, s_hi);
            }
        }
    }
    if (ok && pending) {
        // iteration budget spent inside a cycle: keep its correction
        for (int i = threadIdx.x; i < m; i += THREADS) x[c0 + i] = x[c0 + i] + (double)ds[i];
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

template <bool SYM>
__global__ void __launch_bounds__(1024, 1) k_pcg1_mixed_halo_box(gf_krylov_t K, int chunk) {
    BoxRows<double, SYM, false, int> rows64{K.val, (int)K.n, (int)K.stride_y, (int)K.stride_z};
    BoxRows<float, SYM, SYM, int> rows32{nullptr, (int)K.n, (int)K.stride_y, (int)K.stride_z};
    pcg1_mixed_halo_body<1024>(K, rows64, rows32, SYM ? 3 : 6, chunk);
}

template <int WIDTH>
__global__ void __launch_bounds__(1024, 1) k_pcg1_mixed_halo_ell(gf_krylov_t K, int chunk) {
    EllRows<double, WIDTH, int> rows64{K.val, K.nbr, (int)K.n, K.width, K.row_len};
    EllRows<float, WIDTH, int> rows32{nullptr, K.nbr, (int)K.n, K.width, K.row_len};
    pcg1_mixed_halo_body<1024>(K, rows64, rows32, K.width, chunk);
}

// Tile length for the staged kernel (0: the system does not qualify).
static int staged_tile(const gf_krylov_t* k) {
    if (!k->symmetric || k->stride_y < 1 || (k->n & 1)) return 0;
    const void* ptrs[] = {k->diag, k->val, k->x, k->work, k->rhs};
    for (const void* p : ptrs)
        if (reinterpret_cast<uintptr_t>(p) & 15u) return 0;
    for (int T = 1024; T >= 128; T /= 2) {
        const StLayout L(T, k->stride_y);
        if ((size_t)2 * L.stage() * sizeof(double) <= (size_t)kStMaxSmem) return T;
    }
    return 0;
}

// Single-reduction CG on a box: the variant picks the block size only.
template <bool SYM>
static BoxVariant sr_box_kernel(int variant) {
    switch (variant) {
        case 2:
            return {(void*)k_pcg1_sr_box<SYM, 512>, 512, 1};
        case 3:
        case 4:
            return {(void*)k_pcg1_sr_box<SYM, 1024>, 1024, 1};
        default:
            return {(void*)k_pcg1_sr_box<SYM, 256>, 256, 1};
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

// WIDTH: the ELL row width at compile time (6) or 0 (any).  The Jacobi
// inverse of every cell is computed once per solve into the workspace (after
// the six vectors) and gathered from there by the preconditioned SpMVs.
template <int NC, int WIDTH>
__device__ void bicgstab_body(const gf_krylov_t& K, int vb, int vn) {
    __shared__ BiState st[NC];
    __shared__ int s_any;
    KCtl* ctl = reinterpret_cast<KCtl*>(K.work);
    const int bk = vb >= 0 ? vb : (int)blockIdx.x;
    const int nbk = vn >= 0 ? vn : (int)gridDim.x;
    barrier_init_v(K, nbk, bk);
    double* partials = K.work + kCtlDoubles;
    double* vec = partials + kPartials;
    const int64_t n = K.n;
    double* r = vec;
    double* rh = vec + NC * n;
    double* p = vec + 2 * NC * n;
    double* v = vec + 3 * NC * n;
    double* s = vec + 4 * NC * n;
    double* t = vec + 5 * NC * n;
    double* inv = vec + 6 * NC * n;
    double* x = K.x;
    const bool jac = K.jacobi != 0, linf = K.norm_inf != 0;
    const int64_t t0 = bk * (int64_t)blockDim.x + threadIdx.x;
    const int64_t stride = (int64_t)nbk * blockDim.x;
    bool ok = true;

    {  // r = b - A x; r_hat = p = r; |r|, r.r; the Jacobi inverse
        double loc[2 * NC];
#pragma unroll
        for (int j = 0; j < 2 * NC; ++j) loc[j] = 0.0;
        auto gx = [&](int k, int64_t i) { return __ldcg(x + k * n + i); };
        for (int64_t c = t0; c < n; c += stride) {
            __stcg(inv + c, inv_diag(K.diag, c, jac));
            double ax[NC];
            row_apply<NC, WIDTH>(K, c, gx, ax);
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
            auto gy = [&](int k, int64_t i) { return __ldcg(inv + i) * __ldcg(p + k * n + i); };
            for (int64_t c = t0; c < n; c += stride) {
                double av[NC];
                row_apply<NC, WIDTH>(K, c, gy, av);
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
            auto gz = [&](int k, int64_t i) { return __ldcg(inv + i) * __ldcg(s + k * n + i); };
            for (int64_t c = t0; c < n; c += stride) {
                double at[NC];
                row_apply<NC, WIDTH>(K, c, gz, at);
                const double ic = __ldcg(inv + c);
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
                const double ic = __ldcg(inv + c);
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
    if (bk == 0 && threadIdx.x == 0) {
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

// ---------------------------------------------------------------------------
// Mixed precision BiCGStab: FP32 inner BiCGStab cycles inside FP64
// iterative refinement, for all NC components in one launch.  Each cycle
// starts from the true FP64 residual r = b - A x of every component (also
// its stopping test, |r| < max(atol, rtol |r0|) as in FP64), runs the
// reference's right-preconditioned BiCGStab (bicgstab_body, restarts
// included) in FP32 on A e = r with FP64-accumulated dot products until its
// recurrence residual falls below max(eta |r|, margin thresh), and folds
// x += e in FP64.  The FP32 copies of the coefficients (every ELL slot and
// the diagonal) and of the Jacobi inverse are made once per solve.
// Workspace (after the header): (width + 2) n floats of coefficients and 7 NC
// n floats of vectors (r, r_hat, p, v, s, t, e).
template <int NC, int WIDTH, class G>
__device__ __forceinline__ void row_apply32(const gf_krylov_t& K, const float* __restrict__ val32,
                                            const float* __restrict__ diag32, int64_t c, const G& g,
                                            float (&out)[NC]) {
    const int64_t n = K.n;
    const float d = __ldcg(diag32 + c);
#pragma unroll
    for (int k = 0; k < NC; ++k) out[k] = d * g(k, c);
    const int W = WIDTH > 0 ? WIDTH : (K.row_len ? (int)__ldg(K.row_len + c) : K.width);
    for (int s0 = 0; s0 < W; s0 += kSlotGroup) {
        int nb[kSlotGroup];
        float a[kSlotGroup];
#pragma unroll
        for (int j = 0; j < kSlotGroup; ++j) {
            const int s = s0 + j;
            nb[j] = s < W ? __ldg(K.nbr + s * n + c) : (int)c;
            a[j] = s < W ? __ldcg(val32 + s * n + c) : 0.0f;
        }
#pragma unroll
        for (int j = 0; j < kSlotGroup; ++j)
            if (s0 + j < W)
#pragma unroll
                for (int k = 0; k < NC; ++k) out[k] += a[j] * g(k, nb[j]);
    }
}

struct MixBiState {
    double thresh, r0, true_final, target, rho_old, alpha, omega, beta;
    int mode, restarts, its, converged, status, done, ran;
};

template <int NC, int WIDTH>
__global__ void __launch_bounds__(kKThreads) k_bicgstab_mixed(gf_krylov_t K) {
    __shared__ MixBiState st[NC];
    __shared__ int s_any;
    KCtl* ctl = reinterpret_cast<KCtl*>(K.work);
    barrier_init_v(K, (int)gridDim.x, (int)blockIdx.x);
    double* partials = K.work + kCtlDoubles;
    float* f = reinterpret_cast<float*>(partials + kPartials);
    const int64_t n = K.n;
    const int W = K.width;
    float* val32 = f;
    float* diag32 = val32 + (int64_t)W * n;
    float* inv32 = diag32 + n;
    float* r = inv32 + n;
    float* rh = r + NC * n;
    float* p = r + 2 * NC * n;
    float* v = r + 3 * NC * n;
    float* s = r + 4 * NC * n;
    float* t = r + 5 * NC * n;
    float* e = r + 6 * NC * n;
    double* x = K.x;
    const bool jac = K.jacobi != 0, linf = K.norm_inf != 0;
    const int64_t t0 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const double margin = K.inner_margin > 0.0 && K.inner_margin <= 1.0 ? K.inner_margin : 0.5;
    bool ok = true;

    for (int64_t c = t0; c < n; c += stride) {
        for (int sl = 0; sl < W; ++sl) __stcg(val32 + sl * n + c, (float)__ldg(K.val + sl * n + c));
        __stcg(diag32 + c, (float)__ldg(K.diag + c));
        __stcg(inv32 + c, (float)inv_diag(K.diag, c, jac));
    }
    if (threadIdx.x == 0)
        for (int k = 0; k < NC; ++k) {
            st[k].its = 0;
            st[k].converged = 0;
            st[k].status = GF_MAX_ITER;
            st[k].done = 0;
            st[k].ran = 0;
            st[k].r0 = st[k].true_final = 0.0;
        }
    __syncthreads();
    int its_total = 0;
    for (int cycle = 0; ok && cycle <= K.max_outer; ++cycle) {
        {  // fold the corrections, then the true residual in FP64
            for (int64_t c = t0; c < n; c += stride)
#pragma unroll
                for (int k = 0; k < NC; ++k)
                    if (st[k].ran) __stcg(x + k * n + c, __ldcg(x + k * n + c) + (double)__ldcg(e + k * n + c));
            // The barrier also publishes the FP32 coefficients (cycle 0).
            double dummy[1] = {0.0};
            ok = grid_reduce<1>(ctl, partials, dummy, 0u);
            if (!ok) break;
            double loc[2 * NC];
#pragma unroll
            for (int j = 0; j < 2 * NC; ++j) loc[j] = 0.0;
            auto gx = [&](int k, int64_t i) { return __ldcg(x + k * n + i); };
            for (int64_t c = t0; c < n; c += stride) {
                double ax[NC];
                row_apply<NC, WIDTH>(K, c, gx, ax);
#pragma unroll
                for (int k = 0; k < NC; ++k) {
                    const double rk = __ldg(K.rhs + k * n + c) - ax[k];
                    const float r32 = (float)rk;
                    __stcg(r + k * n + c, r32);
                    __stcg(rh + k * n + c, r32);
                    __stcg(p + k * n + c, r32);
                    __stcg(e + k * n + c, 0.0f);
                    loc[k] = norm_acc(loc[k], rk, linf);
                    loc[NC + k] += (double)r32 * (double)r32;
                }
            }
            ok = grid_reduce<2 * NC>(ctl, partials, loc, linf ? ((1u << NC) - 1u) : 0u);
            if (!ok) break;
            if (threadIdx.x == 0) {
                int any = 0;
                for (int k = 0; k < NC; ++k) {
                    MixBiState& b = st[k];
                    b.ran = 0;
                    const double fin = norm_fin(loc[k], linf);
                    if (cycle == 0) {
                        b.r0 = fin;
                        b.thresh = fmax(K.atol, K.rtol * fin);
                    }
                    if (b.done) continue;
                    b.true_final = fin;
                    if (fin < b.thresh) {
                        b.done = 1;
                        b.converged = 1;
                        b.status = GF_OK;
                    } else if (!isfinite(fin)) {
                        b.done = 1;
                        b.status = GF_NONFINITE;
                    } else if (cycle == K.max_outer || its_total >= K.max_iter) {
                        b.done = 1;
                        b.status = GF_MAX_ITER;
                    } else {
                        b.mode = kRun;
                        b.ran = 1;
                        b.restarts = 0;
                        b.target = fmax(K.inner_eta * fin, margin * b.thresh);
                        b.rho_old = loc[NC + k];
                        any = 1;
                    }
                }
                s_any = any;
            }
            __syncthreads();
            if (!s_any) break;
        }
        // Inner FP32 BiCGStab on A e = r (e = 0 to start).
        for (int it = 1; ok && its_total < K.max_iter; ++it) {
            if (threadIdx.x == 0) {
                int any = 0;
                for (int k = 0; k < NC; ++k) {
                    if (st[k].mode == kIdle) st[k].mode = kRun;
                    any |= st[k].ran && (st[k].mode == kRun);
                }
                s_any = any;
            }
            __syncthreads();
            if (!s_any) break;
            ++its_total;
            {  // P1: y = M p, v = A y; r_hat.v, |r_hat|^2, |v|^2
                double loc[3 * NC];
#pragma unroll
                for (int j = 0; j < 3 * NC; ++j) loc[j] = 0.0;
                auto gy = [&](int k, int64_t i) { return __ldcg(inv32 + i) * __ldcg(p + k * n + i); };
                for (int64_t c = t0; c < n; c += stride) {
                    float av[NC];
                    row_apply32<NC, WIDTH>(K, val32, diag32, c, gy, av);
#pragma unroll
                    for (int k = 0; k < NC; ++k) {
                        if (!st[k].ran || st[k].mode != kRun) continue;
                        __stcg(v + k * n + c, av[k]);
                        const double h = __ldcg(rh + k * n + c);
                        loc[k] += h * (double)av[k];
                        loc[NC + k] += h * h;
                        loc[2 * NC + k] += (double)av[k] * (double)av[k];
                    }
                }
                ok = grid_reduce<3 * NC>(ctl, partials, loc, 0u);
                if (!ok) break;
                if (threadIdx.x == 0)
                    for (int k = 0; k < NC; ++k) {
                        MixBiState& b = st[k];
                        if (!b.ran || b.mode != kRun) continue;
                        b.its += 1;
                        const double da = loc[k];
                        if (fabs(da) <= 1e-6 * sqrt(loc[NC + k]) * sqrt(loc[2 * NC + k])) {
                            if (b.restarts >= K.max_restart) b.mode = kDone;
                            else { b.restarts += 1; b.mode = kRestart; }
                        } else {
                            b.alpha = b.rho_old / da;
                        }
                    }
                __syncthreads();
            }
            {  // P2: s = r - alpha v, |s|; restarting systems copy r
                double loc[2 * NC];
#pragma unroll
                for (int j = 0; j < 2 * NC; ++j) loc[j] = 0.0;
                for (int64_t c = t0; c < n; c += stride)
#pragma unroll
                    for (int k = 0; k < NC; ++k) {
                        if (!st[k].ran) continue;
                        const int md = st[k].mode;
                        if (md == kRun) {
                            const float sk = __ldcg(r + k * n + c) - (float)st[k].alpha * __ldcg(v + k * n + c);
                            __stcg(s + k * n + c, sk);
                            loc[k] = norm_acc(loc[k], (double)sk, linf);
                        } else if (md == kRestart) {
                            const float rk = __ldcg(r + k * n + c);
                            __stcg(rh + k * n + c, rk);
                            __stcg(p + k * n + c, rk);
                            loc[NC + k] += (double)rk * (double)rk;
                        }
                    }
                ok = grid_reduce<2 * NC>(ctl, partials, loc, linf ? ((1u << NC) - 1u) : 0u);
                if (!ok) break;
                if (threadIdx.x == 0)
                    for (int k = 0; k < NC; ++k) {
                        MixBiState& b = st[k];
                        if (!b.ran) continue;
                        if (b.mode == kRestart) {
                            b.rho_old = loc[NC + k];
                            b.mode = kIdle;
                        } else if (b.mode == kRun) {
                            const double fin = norm_fin(loc[k], linf);
                            if (fin < b.target) b.mode = kConvS;
                            else if (!isfinite(fin)) b.mode = kDone;
                        }
                    }
                __syncthreads();
            }
            {  // P3: converged-on-s systems take e += alpha y; others z = M s, t = A z
                double loc[2 * NC];
#pragma unroll
                for (int j = 0; j < 2 * NC; ++j) loc[j] = 0.0;
                auto gz = [&](int k, int64_t i) { return __ldcg(inv32 + i) * __ldcg(s + k * n + i); };
                for (int64_t c = t0; c < n; c += stride) {
                    float at[NC];
                    row_apply32<NC, WIDTH>(K, val32, diag32, c, gz, at);
                    const float ic = __ldcg(inv32 + c);
#pragma unroll
                    for (int k = 0; k < NC; ++k) {
                        if (!st[k].ran) continue;
                        const int md = st[k].mode;
                        if (md == kConvS) {
                            __stcg(e + k * n + c, __ldcg(e + k * n + c) + (float)st[k].alpha * ic * __ldcg(p + k * n + c));
                        } else if (md == kRun) {
                            __stcg(t + k * n + c, at[k]);
                            loc[k] += (double)at[k] * (double)at[k];
                            loc[NC + k] += (double)at[k] * (double)__ldcg(s + k * n + c);
                        }
                    }
                }
                ok = grid_reduce<2 * NC>(ctl, partials, loc, 0u);
                if (!ok) break;
                if (threadIdx.x == 0)
                    for (int k = 0; k < NC; ++k) {
                        MixBiState& b = st[k];
                        if (!b.ran) continue;
                        if (b.mode == kConvS) {
                            b.mode = kDone;
                            continue;
                        }
                        if (b.mode != kRun) continue;
                        const double dd = loc[k];
                        if (fabs(dd) <= 1e-6 * dd || (b.omega = loc[NC + k] / dd, fabs(b.omega) <= 1e-6)) {
                            if (b.restarts >= K.max_restart) b.mode = kDone;
                            else { b.restarts += 1; b.mode = kRestart; }
                        }
                    }
                __syncthreads();
            }
            {  // P4: e += alpha y + omega z, r = s - omega t; |r|, r_hat.r, |r_hat|^2, |r|^2
                double loc[4 * NC];
#pragma unroll
                for (int j = 0; j < 4 * NC; ++j) loc[j] = 0.0;
                for (int64_t c = t0; c < n; c += stride) {
                    const float ic = __ldcg(inv32 + c);
#pragma unroll
                    for (int k = 0; k < NC; ++k) {
                        if (!st[k].ran) continue;
                        const int md = st[k].mode;
                        if (md == kRun) {
                            const float sk = __ldcg(s + k * n + c);
                            const float y = ic * __ldcg(p + k * n + c);
                            const float z = ic * sk;
                            __stcg(e + k * n + c,
                                   __ldcg(e + k * n + c) + (float)st[k].alpha * y + (float)st[k].omega * z);
                            const float rk = sk - (float)st[k].omega * __ldcg(t + k * n + c);
                            __stcg(r + k * n + c, rk);
                            const double h = __ldcg(rh + k * n + c);
                            loc[k] = norm_acc(loc[k], (double)rk, linf);
                            loc[NC + k] += h * rk;
                            loc[2 * NC + k] += h * h;
                            loc[3 * NC + k] += (double)rk * (double)rk;
                        } else if (md == kRestart) {
                            const float rk = __ldcg(r + k * n + c);
                            __stcg(rh + k * n + c, rk);
                            __stcg(p + k * n + c, rk);
                            loc[3 * NC + k] += (double)rk * (double)rk;
                        }
                    }
                }
                ok = grid_reduce<4 * NC>(ctl, partials, loc, linf ? ((1u << NC) - 1u) : 0u);
                if (!ok) break;
                if (threadIdx.x == 0)
                    for (int k = 0; k < NC; ++k) {
                        MixBiState& b = st[k];
                        if (!b.ran) continue;
                        if (b.mode == kRestart) {
                            b.rho_old = loc[3 * NC + k];
                            b.mode = kIdle;
                            continue;
                        }
                        if (b.mode != kRun) continue;
                        const double fin = norm_fin(loc[k], linf);
                        if (fin < b.target || !isfinite(fin)) {
                            b.mode = kDone;
                            continue;
                        }
                        const double rho_new = loc[NC + k];
                        if (fabs(rho_new) <= 1e-6 * sqrt(loc[2 * NC + k]) * sqrt(loc[3 * NC + k])) {
                            if (b.restarts >= K.max_restart) b.mode = kDone;
                            else { b.restarts += 1; b.mode = kRestart; }
                            continue;
                        }
                        b.beta = (rho_new / b.rho_old) * (b.alpha / b.omega);
                        b.rho_old = rho_new;
                    }
                __syncthreads();
            }
            {  // P5: p = r + beta (p - omega v); restarting systems copy r
                double loc[NC];
#pragma unroll
                for (int k = 0; k < NC; ++k) loc[k] = 0.0;
                for (int64_t c = t0; c < n; c += stride)
#pragma unroll
                    for (int k = 0; k < NC; ++k) {
                        if (!st[k].ran) continue;
                        const int md = st[k].mode;
                        if (md == kRun) {
                            const float pk = __ldcg(p + k * n + c);
                            __stcg(p + k * n + c, __ldcg(r + k * n + c) +
                                                      (float)st[k].beta * (pk - (float)st[k].omega * __ldcg(v + k * n + c)));
                        } else if (md == kRestart) {
                            const float rk = __ldcg(r + k * n + c);
                            __stcg(rh + k * n + c, rk);
                            __stcg(p + k * n + c, rk);
                            loc[k] += (double)rk * (double)rk;
                        }
                    }
                ok = grid_reduce<NC>(ctl, partials, loc, 0u);
                if (!ok) break;
                if (threadIdx.x == 0)
                    for (int k = 0; k < NC; ++k)
                        if (st[k].ran && st[k].mode == kRestart) {
                            st[k].rho_old = loc[k];
                            st[k].mode = kIdle;
                        }
                __syncthreads();
            }
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0)
        for (int k = 0; k < NC; ++k) {
            double* o = K.stats + 5 * k;
            o[0] = st[k].r0;
            o[1] = st[k].true_final;
            o[2] = st[k].its;
            o[3] = st[k].converged;
            o[4] = ok ? st[k].status : GF_ERR_TIMEOUT;
        }
}

// ---------------------------------------------------------------------------
// Split CG for systems of millions of cells (variant 19): two ordinary
// kernels an iteration instead of one persistent cooperative launch, so each
// pass runs at the occupancy of a plain stream kernel (a standalone SpMV of
// this form reads HBM at ~94 % of the copy rate on a 4M-cell octree; the
// persistent kernel's passes reach ~60 %).  Kernel A: p = z + beta p;
// q = A p and the block partials of p.q.  Kernel B: x += alpha p;
// r -= alpha q; z = M r and the partials of |r| and r.z.  There is no grid
// barrier: each kernel starts by summing the previous kernel's block
// partials in one fixed order (every block gets the same bits), and the
// scalars (threshold, r.z, the done flag) pass between kernels in the
// workspace's control block, written by block 0.  All 2 max_iter + 2
// kernels are enqueued without a host synchronisation; once the stopping
// test has passed the remaining ones return at once.
constexpr int kSplitVariant = 19;
constexpr int kSplitVariants = 13;
constexpr int kSplitThreads = 256;

struct SplitScalars {  // in the control block, after KCtl
    double thresh, r0, fin, rz[2];
    // alpha of the last update (XA forms: written by k_cgs_b, read by the
    // next k_cgs_a, which applies x += alpha p).
    double alpha;
    int done, its, converged, status;
    // Iteration numbers of the graph loop: it_a is read by k_cgs_a and
    // written by k_cgs_b, it_b the other way round, so no kernel reads a
    // counter that one of its own blocks writes.
    int it_a, it_b;
    // XA forms: set by the k_cgs_a that stops the solve; the next k_cgs_b
    // turns it into done (the stopping k_cgs_a still has work to finish in
    // all its blocks, so it must not set the flag its own blocks test).
    int stop;
};
static_assert(2 * sizeof(double) + sizeof(SplitScalars) <= kCtlDoubles * sizeof(double),
              "split CG scalars exceed the control block");

__device__ __forceinline__ SplitScalars* split_scalars(const gf_krylov_t& K) {
    return reinterpret_cast<SplitScalars*>(K.work + 2);
}

// Sum (or max, maxmask bit j) of the NV values of nblk block partials, in
// one fixed order; every thread gets the result.
template <int NV>
__device__ void split_sum(const double* part, int nblk, unsigned maxmask, double (&out)[NV]) {
    __shared__ double sh[NV][kSplitThreads / 32];
    double acc[NV];
#pragma unroll
    for (int j = 0; j < NV; ++j) acc[j] = 0.0;
    for (int b = threadIdx.x; b < nblk; b += blockDim.x)
#pragma unroll
        for (int j = 0; j < NV; ++j) {
            const double y = __ldcg(part + (int64_t)j * nblk + b);
            acc[j] = ((maxmask >> j) & 1u) ? nmax(acc[j], y) : acc[j] + y;
        }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int j = 0; j < NV; ++j) {
        double x = acc[j];
        for (int o = 16; o > 0; o >>= 1) {
            const double y = __shfl_xor_sync(0xffffffffu, x, o);
            x = ((maxmask >> j) & 1u) ? nmax(x, y) : x + y;
        }
        if (lane == 0) sh[j][warp] = x;
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < NV; ++j) {
        double x = sh[j][0];
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) x = ((maxmask >> j) & 1u) ? nmax(x, sh[j][w]) : x + sh[j][w];
        out[j] = x;
    }
    __syncthreads();
}

// Block partials of NV values: one fixed-order block reduction, written by
// thread 0 to part[j * nblk + blockIdx.x].
template <int NV>
__device__ void split_partial(double (&v)[NV], unsigned maxmask, double* part) {
    __shared__ double sh[NV][kSplitThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int j = 0; j < NV; ++j) {
        double x = v[j];
        for (int o = 16; o > 0; o >>= 1) {
            const double y = __shfl_xor_sync(0xffffffffu, x, o);
            x = ((maxmask >> j) & 1u) ? nmax(x, y) : x + y;
        }
        if (lane == 0) sh[j][warp] = x;
    }
    __syncthreads();
    if (threadIdx.x == 0)
#pragma unroll
        for (int j = 0; j < NV; ++j) {
            double x = sh[j][0];
            for (int w = 1; w < (int)(blockDim.x >> 5); ++w)
                x = ((maxmask >> j) & 1u) ? nmax(x, sh[j][w]) : x + sh[j][w];
            __stcg(part + (int64_t)j * gridDim.x + blockIdx.x, x);
        }
}

struct SplitVec {
    double *r, *z, *pa, *pb, *q, *p1, *p2;
};

__device__ __forceinline__ SplitVec split_vec(const gf_krylov_t& K) {
    double* partials = K.work + kCtlDoubles;
    double* vec = partials + kPartials;
    const int64_t n = K.n;
    return {vec, vec + n, vec + 2 * n, vec + 3 * n, vec + 4 * n, partials, partials + kMaxBlocks};
}

// L2 prefetch of one address (a hint: no register result, no fault; every
// address given is inside its array).
__device__ __forceinline__ void pf_l2(const void* p) { asm volatile("prefetch.L2 [%0];" ::"l"(p)); }

// The first slots (up to six) of row c of an ELL operator: what the row
// kernel's first pass reads of the matrix.  Box operators: nothing.
template <class Rows>
__device__ __forceinline__ void split_prefetch_rows(const Rows&, int) {}
template <typename T, int WIDTH, typename I, int GRP>
__device__ __forceinline__ void split_prefetch_rows(const EllRows<T, WIDTH, I, GRP>& r, int c) {
    const int ws = WIDTH > 0 ? WIDTH : (r.w < 6 ? r.w : 6);
    for (int s = 0; s < ws; ++s) {
        pf_l2(r.val + (int64_t)s * r.n + c);
        pf_l2(r.nbr + (int64_t)s * r.n + c);
    }
}

template <class Rows, int MINB>
__global__ void __launch_bounds__(kSplitThreads, MINB) k_cgs_init(gf_krylov_t K, Rows rows) {
    const SplitVec v = split_vec(K);
    const int n = (int)K.n;
    const bool jac = K.jacobi != 0, linf = K.norm_inf != 0;
    double loc[2] = {0.0, 0.0};
    auto gx = [&](int i) { return __ldcg(K.x + i); };
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        const double ax = rows.apply(c, __ldg(K.diag + c), gx);
        const double rk = __ldg(K.rhs + c) - ax;
        const double zk = inv_diag(K.diag, c, jac) * rk;
        __stcg(v.r + c, rk);
        __stcg(v.z + c, zk);
        __stcg(v.pa + c, 0.0);
        loc[0] = norm_acc(loc[0], rk, linf);
        loc[1] += rk * zk;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) split_scalars(K)->it_a = 1;
    split_partial<2>(loc, linf ? 1u : 0u, v.p2);
}

// Iteration it: the stopping test on the previous update's |r| (it > 1; the
// initial residual at it = 1), then p = z + beta p, q = A p, partials of p.q.
// it = max_iter + 1 only finishes the statistics.  LOOP: the body of a
// CUDA graph while-loop; it comes from the control block and the kernel that
// ends the solve sets the loop's condition to 0.  XA: this kernel also
// applies the previous iteration's x += alpha p (it reads p_old anyway), so
// the update kernel reads neither x nor p; x gets the same values in the
// same order as in the other forms.
// PF: before summing the previous kernel's partials (a chain of dependent
// L2 reads during which HBM would idle), each thread prefetches into L2 what
// its first PF cells will read, so the streaming starts with the kernel.
// EARLY: in the graph loop, the prefetches that do not depend on the
// iteration number go out before the loop's control reads, and the scalars
// of the previous kernels (threshold, r.z, alpha) are read before the
// partial sums instead of after them (the same values).
template <class Rows, int MINB, bool LOOP, bool QREC = false, bool XA = false, int PF = 0, bool EARLY = false>
__global__ void __launch_bounds__(kSplitThreads, MINB) k_cgs_a(gf_krylov_t K, Rows rows, int it, int pa_old,
                                                              cudaGraphConditionalHandle loop) {
    SplitScalars* S = split_scalars(K);
    const SplitVec v = split_vec(K);
    const int n = (int)K.n;
    // early prefetch: what does not depend on the iteration number (in the
    // graph loop this kernel never runs after the solve has stopped)
    constexpr bool early_pf = EARLY && LOOP && PF > 0;
    if (early_pf) {
        const int c = blockIdx.x * blockDim.x + threadIdx.x;
        if (c < n) {
            pf_l2(v.z + c);
            if (QREC) pf_l2(v.q + c);
            if (XA) pf_l2(K.x + c);
            pf_l2(K.diag + c);
            split_prefetch_rows(rows, c);
        }
    }
    if (*(volatile int*)&S->done) {
        if (LOOP && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(loop, 0);
        return;
    }
    if (LOOP) {
        it = *(volatile int*)&S->it_a;
        pa_old = it & 1;
    }
    const bool linf = K.norm_inf != 0;
    if (early_pf) {
        const int c = blockIdx.x * blockDim.x + threadIdx.x;
        if (c < n && it > 1) pf_l2((pa_old ? v.pa : v.pb) + c);
    } else if (PF > 0) {
        const int step = gridDim.x * blockDim.x;
        int c = blockIdx.x * blockDim.x + threadIdx.x;
        for (int k = 0; k < PF && c < n; ++k, c += step) {
            pf_l2(v.z + c);
            if (it > 1) pf_l2((pa_old ? v.pa : v.pb) + c);
            if (QREC && it > 1) pf_l2(v.q + c);
            if (XA && it > 1) pf_l2(K.x + c);
            pf_l2(K.diag + c);
            split_prefetch_rows(rows, c);
        }
    }
    double e_thresh = 0.0, e_rz = 0.0, e_alpha = 0.0;
    if (EARLY && it > 1) {
        e_alpha = S->alpha;
        if (threadIdx.x == 0) {
            e_thresh = S->thresh;
            e_rz = S->rz[(it - 1) & 1];
        }
    }
    __shared__ double s_beta;
    __shared__ int s_stop;
    double red[2];
    split_sum<2>(v.p2, gridDim.x, linf ? 1u : 0u, red);
    if (threadIdx.x == 0) {
        const double fin = norm_fin(red[0], linf);
        double thresh;
        if (it == 1) {
            thresh = fmax(K.atol, K.rtol * fin);
            if (blockIdx.x == 0) {
                S->r0 = fin;
                S->thresh = thresh;
            }
        } else {
            thresh = EARLY ? e_thresh : S->thresh;
        }
        int status = -1;
        if (fin < thresh) status = GF_OK;
        else if (!isfinite(fin)) status = GF_NONFINITE;
        else if (it > K.max_iter || it < 1) status = GF_MAX_ITER;
        s_stop = status >= 0;
        s_beta = it == 1 ? 0.0 : red[1] / (EARLY ? e_rz : S->rz[(it - 1) & 1]);
        if (blockIdx.x == 0) {
            S->fin = fin;
            if (status >= 0) {
                const int its = status == GF_MAX_ITER ? K.max_iter : it - 1;
                double* o = K.stats;
                o[0] = it == 1 ? fin : S->r0;
                o[1] = fin;
                o[2] = its;
                o[3] = status == GF_OK;
                o[4] = status;
                S->its = its;
                S->status = status;
                S->converged = status == GF_OK;
                __threadfence();
                if (XA) S->stop = 1;
                else S->done = 1;
                if (LOOP) cudaGraphSetConditional(loop, 0);
            } else {
                S->rz[it & 1] = red[1];
                if (LOOP) S->it_b = it;
            }
        }
    }
    __syncthreads();
    const double* p_old = pa_old ? v.pa : v.pb;
    // XA: x += alpha p of the previous iteration (none before the first).
    const bool upd = XA && it > 1;
    const double alpha = upd ? (EARLY ? e_alpha : S->alpha) : 0.0;
    if (s_stop) {
        if (upd)
            for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
                __stcg(K.x + c, __ldcg(K.x + c) + alpha * __ldcg(p_old + c));
        return;
    }
    const double beta = s_beta;
    double* p_new = pa_old ? v.pb : v.pa;
    double loc[1] = {0.0};
    if (QREC) {
        // q = A p by recurrence, q = A z + beta q: the rows gather z alone
        // (one vector instead of two), q of the own cell is read back.
        const bool first = it == 1;
        auto gz = [&](int i) { return v.z[i]; };
        for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
            const double zc = v.z[c];
            const double po = first ? 0.0 : p_old[c];
            if (upd) __stcg(K.x + c, __ldcg(K.x + c) + alpha * po);
            const double pc = first ? zc : zc + po * beta;
            const double az = rows.apply(c, __ldg(K.diag + c), gz);
            const double qc = first ? az : az + __ldcg(v.q + c) * beta;
            __stcg(p_new + c, pc);
            __stcg(v.q + c, qc);
            loc[0] += pc * qc;
        }
    } else {
        auto gp = [&](int i) { return v.z[i] + p_old[i] * beta; };
        for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
            const double po = p_old[c];
            if (upd) __stcg(K.x + c, __ldcg(K.x + c) + alpha * po);
            const double pc = v.z[c] + po * beta;
            const double ap = rows.apply(c, __ldg(K.diag + c), gp);
            __stcg(p_new + c, pc);
            __stcg(v.q + c, ap);
            loc[0] += pc * ap;
        }
    }
    split_partial<1>(loc, 0u, v.p1);
}

// x += alpha p (not in the XA forms, whose k_cgs_a applies it); r -= alpha q;
// z = M r; partials of |r| and r.z.
template <int MINB, bool LOOP, bool PAIRS, bool XA = false, int PF = 0, bool EARLY = false>
__global__ void __launch_bounds__(kSplitThreads, MINB) k_cgs_b(gf_krylov_t K, int it, int p_is_b) {
    SplitScalars* S = split_scalars(K);
    const SplitVec v = split_vec(K);
    const int n = (int)K.n;
    // the first 2 PF cells (pairs) of this thread's grid-stride loop; with
    // EARLY in the graph loop (XA: nothing here depends on the iteration
    // number) before the loop's control reads
    auto prefetch = [&](int pb) {
        const int64_t step = (int64_t)gridDim.x * blockDim.x * (PAIRS ? 2 : 1);
        for (int64_t c = (int64_t)(blockIdx.x * blockDim.x + threadIdx.x) * (PAIRS ? 2 : 1), k = 0; k < 2 * PF && c < n;
             ++k, c += step) {
            pf_l2(v.r + c);
            pf_l2(v.q + c);
            pf_l2(K.diag + c);
            if (!XA) {
                pf_l2(K.x + c);
                pf_l2((pb ? v.pb : v.pa) + c);
            }
        }
    };
    constexpr bool early_pf = EARLY && LOOP && XA && PF > 0;
    if (early_pf) prefetch(0);
    if (*(volatile int*)&S->done) return;
    if (XA && *(volatile int*)&S->stop) {
        if (blockIdx.x == 0 && threadIdx.x == 0) S->done = 1;
        return;
    }
    if (LOOP) {
        it = *(volatile int*)&S->it_b;
        p_is_b = it & 1;
        if (blockIdx.x == 0 && threadIdx.x == 0) S->it_a = it + 1;
    }
    const bool jac = K.jacobi != 0, linf = K.norm_inf != 0;
    if (PF > 0 && !early_pf) prefetch(p_is_b);
    const double rz = EARLY ? S->rz[it & 1] : 0.0;
    double red[1];
    split_sum<1>(v.p1, gridDim.x, 0u, red);
    const double alpha = (EARLY ? rz : S->rz[it & 1]) / red[0];
    if (XA && blockIdx.x == 0 && threadIdx.x == 0) S->alpha = alpha;
    const double* p = p_is_b ? v.pb : v.pa;
    double loc[2] = {0.0, 0.0};
    // Pairs of cells with 16-byte loads and stores where every vector is
    // 16-byte aligned (the workspace vectors are when n is even): half the
    // memory instructions of the streaming update.
    const bool pairs = PAIRS && (n & 1) == 0 &&
                       ((reinterpret_cast<uintptr_t>(K.x) | reinterpret_cast<uintptr_t>(K.diag)) & 15u) == 0;
    if (pairs) {
        const int n2 = n >> 1;
        double2* x2 = reinterpret_cast<double2*>(K.x);
        const double2* p2 = reinterpret_cast<const double2*>(p);
        double2* r2 = reinterpret_cast<double2*>(v.r);
        const double2* q2 = reinterpret_cast<const double2*>(v.q);
        double2* z2 = reinterpret_cast<double2*>(v.z);
        const double2* d2 = reinterpret_cast<const double2*>(K.diag);
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n2; i += gridDim.x * blockDim.x) {
            double2 xv = make_double2(0.0, 0.0), pv = xv;
            if (!XA) {
                xv = __ldcg(x2 + i);
                pv = __ldcg(p2 + i);
            }
            const double2 rv = __ldcg(r2 + i), qv = __ldcg(q2 + i);
            const double2 dv = __ldg(d2 + i);
            const double r0 = rv.x - alpha * qv.x, r1 = rv.y - alpha * qv.y;
            double i0 = 1.0, i1 = 1.0;
            if (jac) {
                i0 = fabs(dv.x) < 2.220446049250313e-16 ? 1.0 : 1.0 / dv.x;
                i1 = fabs(dv.y) < 2.220446049250313e-16 ? 1.0 : 1.0 / dv.y;
            }
            const double z0 = i0 * r0, z1 = i1 * r1;
            if (!XA) __stcg(x2 + i, make_double2(xv.x + alpha * pv.x, xv.y + alpha * pv.y));
            __stcg(r2 + i, make_double2(r0, r1));
            __stcg(z2 + i, make_double2(z0, z1));
            loc[0] = norm_acc(norm_acc(loc[0], r0, linf), r1, linf);
            loc[1] += r0 * z0 + r1 * z1;
        }
    } else {
        for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
            if (!XA) __stcg(K.x + c, __ldcg(K.x + c) + alpha * __ldcg(p + c));
            const double rk = __ldcg(v.r + c) - alpha * __ldcg(v.q + c);
            const double zk = inv_diag(K.diag, c, jac) * rk;
            __stcg(v.r + c, rk);
            __stcg(v.z + c, zk);
            loc[0] = norm_acc(loc[0], rk, linf);
            loc[1] += rk * zk;
        }
    }
    split_partial<2>(loc, linf ? 1u : 0u, v.p2);
}

// Graph while-loops of the split CG, cached by everything their kernel
// nodes hold (the descriptor, the row operator, the grid size and the
// device), so the repeated solves of an algorithm reuse one instantiated
// graph; the least recently used of kSplitLoops entries is replaced.
constexpr int kSplitLoops = 64;

struct SplitLoop {
    int dev = -1;
    const void* fa = nullptr;
    const void* fb = nullptr;
    unsigned grid = 0;
    unsigned char kbytes[sizeof(gf_krylov_t)] = {};
    unsigned char rbytes[64] = {};
    size_t rlen = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    uint64_t used = 0;
};

static std::mutex g_split_mu;
static SplitLoop g_split_loops[kSplitLoops];
static uint64_t g_split_clock = 0;

static bool split_graph_enabled() {
    static const bool on = [] {
        const char* v = getenv("GF_SPLIT_GRAPH");
        return v == nullptr || v[0] != '0';
    }();
    return on;
}

static int split_loop_exec(const void* fa, const void* fb, const gf_krylov_t& K, const void* rows, size_t rlen,
                           unsigned grid, cudaGraphExec_t* out) {
    if (rlen > sizeof(SplitLoop::rbytes)) {
        set_error("gf_pcg_solve: split CG row operator too large for the graph cache");
        return GF_ERR_INVALID;
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        set_error("gf_pcg_solve: %s", cudaGetErrorString(e));
        return GF_ERR_CUDA;
    }
    std::lock_guard<std::mutex> lock(g_split_mu);
    SplitLoop* victim = &g_split_loops[0];
    for (SplitLoop& L : g_split_loops) {
        if (L.exec != nullptr && L.dev == dev && L.fa == fa && L.fb == fb && L.grid == grid && L.rlen == rlen &&
            memcmp(L.kbytes, &K, sizeof(gf_krylov_t)) == 0 && memcmp(L.rbytes, rows, rlen) == 0) {
            L.used = ++g_split_clock;
            *out = L.exec;
            return GF_OK;
        }
        if (L.used < victim->used) victim = &L;
    }
    // Build: graph { while (cond) { k_cgs_a -> k_cgs_b } }, cond = 1 at launch.
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaGraphConditionalHandle handle = 0;
    e = cudaGraphCreate(&graph, 0);
    if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&handle, graph, 1, cudaGraphCondAssignDefault);
    cudaGraphNodeParams cp = {};
    cudaGraphNode_t cond = nullptr, na = nullptr, nb = nullptr;
    if (e == cudaSuccess) {
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = handle;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        e = cudaGraphAddNode(&cond, graph, nullptr, 0, &cp);
    }
    gf_krylov_t kcopy = K;
    alignas(16) unsigned char rcopy[sizeof(SplitLoop::rbytes)];
    memcpy(rcopy, rows, rlen);
    int it0 = 0, par0 = 0;
    if (e == cudaSuccess) {
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        void* a_args[] = {&kcopy, rcopy, &it0, &par0, &handle};
        cudaKernelNodeParams ka = {};
        ka.func = const_cast<void*>(fa);
        ka.gridDim = dim3(grid);
        ka.blockDim = dim3(kSplitThreads);
        ka.kernelParams = a_args;
        e = cudaGraphAddKernelNode(&na, body, nullptr, 0, &ka);
        if (e == cudaSuccess) {
            void* b_args[] = {&kcopy, &it0, &par0};
            cudaKernelNodeParams kb = {};
            kb.func = const_cast<void*>(fb);
            kb.gridDim = dim3(grid);
            kb.blockDim = dim3(kSplitThreads);
            kb.kernelParams = b_args;
            e = cudaGraphAddKernelNode(&nb, body, &na, 1, &kb);
        }
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
    if (e != cudaSuccess) {
        if (graph != nullptr) cudaGraphDestroy(graph);
        set_error("gf_pcg_solve: split CG graph set-up failed: %s", cudaGetErrorString(e));
        return GF_ERR_CUDA;
    }
    // An in-flight executable graph is released when its launch completes.
    if (victim->exec != nullptr) cudaGraphExecDestroy(victim->exec);
    if (victim->graph != nullptr) cudaGraphDestroy(victim->graph);
    victim->dev = dev;
    victim->fa = fa;
    victim->fb = fb;
    victim->grid = grid;
    memcpy(victim->kbytes, &K, sizeof(gf_krylov_t));
    memset(victim->rbytes, 0, sizeof(victim->rbytes));
    memcpy(victim->rbytes, rows, rlen);
    victim->rlen = rlen;
    victim->graph = graph;
    victim->exec = exec;
    victim->used = ++g_split_clock;
    *out = exec;
    return GF_OK;
}

template <class Rows, int MINB, bool PAIRS, bool QREC = false, bool XA = false, int PF = 0, bool EARLY = false>
static int launch_split_rows(const gf_krylov_t* k, const Rows& rows, cudaStream_t st) {
    int dev = 0, sms = 0, per_sm = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess)
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_cgs_a<Rows, MINB, false, QREC, XA, PF, EARLY>, kSplitThreads, 0);
    if (e != cudaSuccess || per_sm < 1) {
        set_error("gf_pcg_solve: split CG set-up failed: %s", cudaGetErrorString(e));
        return GF_ERR_CUDA;
    }
    int64_t grid = (int64_t)per_sm * sms;
    const int64_t want = (k->n + kSplitThreads - 1) / kSplitThreads;
    if (grid > want) grid = want;
    if (grid > kMaxBlocks) grid = kMaxBlocks;
    if (k->block_cap > 0 && grid > k->block_cap) grid = k->block_cap;
    if (grid < 1) grid = 1;
    e = cudaMemsetAsync(k->work, 0, sizeof(double) * kCtlDoubles, st);
    if (e != cudaSuccess) {
        set_error("gf_pcg_solve: %s", cudaGetErrorString(e));
        return GF_ERR_CUDA;
    }
    const gf_krylov_t K = *k;
    const unsigned g = (unsigned)grid;
    k_cgs_init<Rows, MINB><<<g, kSplitThreads, 0, st>>>(K, rows);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error("gf_pcg_solve: split CG launch failed: %s", cudaGetErrorString(e));
        return GF_ERR_CUDA;
    }
    // Outside stream capture the iterations run as a CUDA graph while-loop
    // (one graph launch, the loop ends on the device when the solve stops);
    // inside a capture every permitted iteration is enqueued and those
    // after the stop return at once.
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (split_graph_enabled() && cudaStreamIsCapturing(st, &cap) == cudaSuccess &&
        cap == cudaStreamCaptureStatusNone) {
        cudaGraphExec_t exec = nullptr;
        const int rc = split_loop_exec((const void*)k_cgs_a<Rows, MINB, true, QREC, XA, PF, EARLY>,
                                       (const void*)k_cgs_b<MINB, true, PAIRS, XA, PF, EARLY>, K,
                                       &rows, sizeof(Rows), g, &exec);
        if (rc != GF_OK) return rc;
        e = cudaGraphLaunch(exec, st);
        if (e != cudaSuccess) {
            set_error("gf_pcg_solve: split CG graph launch failed: %s", cudaGetErrorString(e));
            return GF_ERR_CUDA;
        }
        return GF_OK;
    }
    for (int it = 1; it <= k->max_iter; ++it) {
        // p_old is pa at odd iterations (p_new then goes to pb), pb at even.
        k_cgs_a<Rows, MINB, false, QREC, XA, PF, EARLY><<<g, kSplitThreads, 0, st>>>(K, rows, it, it & 1, 0);
        k_cgs_b<MINB, false, PAIRS, XA, PF, EARLY><<<g, kSplitThreads, 0, st>>>(K, it, it & 1);
    }
    k_cgs_a<Rows, MINB, false, QREC, XA, PF, EARLY><<<g, kSplitThreads, 0, st>>>(K, rows, k->max_iter + 1, (k->max_iter + 1) & 1, 0);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error("gf_pcg_solve: split CG launch failed: %s", cudaGetErrorString(e));
        return GF_ERR_CUDA;
    }
    return GF_OK;
}

template <int MINB, bool PAIRS, int GRP = 1, bool QREC = false, bool XA = false, int PF = 0, bool EARLY = false>
static int launch_split_m(const gf_krylov_t* k, void* stream) {
    const int64_t row_span = (int64_t)(k->stride_y > 0 ? 6 : (k->width > 6 ? k->width : 6)) * k->n;
    if (row_span >= ((int64_t)1 << 31)) {
        set_error("gf_pcg_solve: system not eligible for the split CG");
        return GF_ERR_INVALID;
    }
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    if (k->stride_y > 0) {
        if (k->symmetric)
            return launch_split_rows<BoxRows<double, true, false, int>, MINB, PAIRS, QREC, XA, PF, EARLY>(
                k, BoxRows<double, true, false, int>{k->val, (int)k->n, (int)k->stride_y, (int)k->stride_z}, st);
        return launch_split_rows<BoxRows<double, false, false, int>, MINB, PAIRS, QREC, XA, PF, EARLY>(
            k, BoxRows<double, false, false, int>{k->val, (int)k->n, (int)k->stride_y, (int)k->stride_z}, st);
    }
    // One slot at a time (the loop of a plain SpMV): the occupancy, not the
    // loads of one thread, keeps the memory system busy.
    if (k->width == 6)
        return launch_split_rows<EllRows<double, 6, int, 1>, MINB, PAIRS, QREC, XA, PF, EARLY>(
            k, EllRows<double, 6, int, 1>{k->val, k->nbr, (int)k->n, k->width, k->row_len}, st);
    return launch_split_rows<EllRows<double, 0, int, GRP>, MINB, PAIRS, QREC, XA, PF, EARLY>(
        k, EllRows<double, 0, int, GRP>{k->val, k->nbr, (int)k->n, k->width, k->row_len}, st);
}

// Variant 19: 8 blocks of 256 threads an SM; 20: 6 (more registers);
// 21: 8 with the update kernel on pairs of cells; 22: 7, pairs; 23: 7,
// pairs, ELL slots loaded two at a time; 24: 6, pairs, four at a time;
// 25: 8, pairs, q = A p by recurrence (the rows gather z alone); 26: 8,
// q by recurrence, update one cell at a time; 27: 25 with x += alpha p in
// the row kernel (the update kernel reads neither x nor p); 28: 21 with the
// same; 29: 27 with the first cell's data prefetched into L2 while each
// kernel sums the previous kernel's partials; 30: the same for the first two
// cells (four of the update kernel); 31: 29 with the prefetches and the
// scalar reads moved ahead of the loop's control reads and partial sums.
static int launch_split(const gf_krylov_t* k, void* stream, int which) {
    switch (which) {
        case 1: return launch_split_m<6, false>(k, stream);
        case 2: return launch_split_m<8, true>(k, stream);
        case 3: return launch_split_m<7, true>(k, stream);
        case 4: return launch_split_m<7, true, 2>(k, stream);
        case 5: return launch_split_m<6, true, 4>(k, stream);
        case 6: return launch_split_m<8, true, 1, true>(k, stream);
        case 7: return launch_split_m<8, false, 1, true>(k, stream);
        case 8: return launch_split_m<8, true, 1, true, true>(k, stream);
        case 9: return launch_split_m<8, true, 1, false, true>(k, stream);
        case 10: return launch_split_m<8, true, 1, true, true, 1>(k, stream);
        case 11: return launch_split_m<8, true, 1, true, true, 2>(k, stream);
        case 12: return launch_split_m<8, true, 1, true, true, 1, true>(k, stream);
        default: return launch_split_m<8, false>(k, stream);
    }
}

// ---------------------------------------------------------------------------
// Batched solves: the systems of several independent cases (the solve
// server's same-phase solves) in ONE cooperative launch.  System i owns the
// blocks [blk0[i], blk0[i+1]) and runs the single-system kernel's body on
// them with its own barrier counter and partials (its workspace), so its
// iterates do not depend on which other systems share the launch.
constexpr int kMaxBatch = 16;

struct KBatch {
    int count;
    int blk0[kMaxBatch + 1];
    gf_krylov_t sys[kMaxBatch];
};

__device__ __forceinline__ int batch_system(const KBatch& B) {
    int s = 0;
    while (s + 1 < B.count && (int)blockIdx.x >= B.blk0[s + 1]) ++s;
    return s;
}

// Zeroes every system's barrier control block (one launch for the batch).
__global__ void k_batch_reset(const KBatch B) {
    for (int i = threadIdx.x; i < B.count; i += blockDim.x) {
        KCtl* ctl = reinterpret_cast<KCtl*>(B.sys[i].work);
        ctl->count = 0ull;
        ctl->error = 0;
        ctl->pad = 0;
    }
}

__global__ void __launch_bounds__(kCgThreads, 4) k_pcg1_batched(const KBatch B) {
    const int s = batch_system(B);
    const gf_krylov_t& K = B.sys[s];
    const int bid = (int)blockIdx.x - B.blk0[s], nb = B.blk0[s + 1] - B.blk0[s];
    if (K.mixed) {
        // FP32 inner iterations inside FP64 refinement (pcg1_mixed_body).
        if (K.stride_y > 0) {
            if (K.symmetric) {
                BoxRows<double, true, false> rows64{K.val, K.n, K.stride_y, K.stride_z};
                BoxRows<float, true, true> rows32{nullptr, K.n, K.stride_y, K.stride_z};
                pcg1_mixed_body<kCgThreads, 1>(K, rows64, rows32, 3, bid, nb);
            } else {
                BoxRows<double, false, false> rows64{K.val, K.n, K.stride_y, K.stride_z};
                BoxRows<float, false, false> rows32{nullptr, K.n, K.stride_y, K.stride_z};
                pcg1_mixed_body<kCgThreads, 1>(K, rows64, rows32, 6, bid, nb);
            }
        } else {
            EllRows<double, 0> rows64{K.val, K.nbr, K.n, K.width, K.row_len};
            EllRows<float, 0> rows32{nullptr, K.nbr, K.n, K.width, K.row_len};
            pcg1_mixed_body<kCgThreads, 1>(K, rows64, rows32, K.width, bid, nb);
        }
        return;
    }
    if (K.stride_y > 0) {
        if (K.symmetric) {
            BoxRows<double, true, false> rows{K.val, K.n, K.stride_y, K.stride_z};
            pcg1_body<kCgThreads, 1>(K, rows, bid, nb);
        } else {
            BoxRows<double, false, false> rows{K.val, K.n, K.stride_y, K.stride_z};
            pcg1_body<kCgThreads, 1>(K, rows, bid, nb);
        }
    } else if (K.width == 6) {
        EllRows<double, 6> rows{K.val, K.nbr, K.n, K.width, K.row_len};
        pcg1_body<kCgThreads, 1>(K, rows, bid, nb);
    } else {
        EllRows<double, 0> rows{K.val, K.nbr, K.n, K.width, K.row_len};
        pcg1_body<kCgThreads, 1>(K, rows, bid, nb);
    }
}

template <int NC>
__global__ void __launch_bounds__(kKThreads) k_bicgstab_batched(const KBatch B) {
    const int s = batch_system(B);
    const gf_krylov_t& K = B.sys[s];
    const int bid = (int)blockIdx.x - B.blk0[s], nb = B.blk0[s + 1] - B.blk0[s];
    if (K.width == 6)
        bicgstab_body<NC, 6>(K, bid, nb);
    else
        bicgstab_body<NC, 0>(K, bid, nb);
}

template <int NC, int WIDTH>
__global__ void __launch_bounds__(kKThreads) k_bicgstab(gf_krylov_t K) {
    bicgstab_body<NC, WIDTH>(K, -1, -1);
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

// Cooperative launch of the staged box CG: one block per SM, two stages of
// dynamic shared memory.
static int launch_staged(const gf_krylov_t* k, int T, void* stream) {
    const char* what = "gf_pcg_solve";
    const void* kern = (const void*)k_pcg1_box_staged<kStThreads>;
    const size_t smem = (size_t)2 * StLayout(T, k->stride_y).stage() * sizeof(double);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int dev = 0, sms = 0, per_sm = 0;
    if (e == cudaSuccess) e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kStThreads, smem);
    if (e != cudaSuccess || per_sm < 1) {
        set_error("%s: staged kernel set-up failed: %s", what, cudaGetErrorString(e));
        return GF_ERR_CUDA;
    }
    const int64_t ntiles = (k->n + T - 1) / T;
    int64_t cap = (int64_t)per_sm * sms;
    if (cap > kMaxBlocks) cap = kMaxBlocks;
    if (k->block_cap > 0 && k->block_cap < cap) cap = k->block_cap;
    const int grid = (int)(ntiles < cap ? ntiles : cap);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    e = cudaMemsetAsync(k->work, 0, sizeof(KCtl), s);
    if (e != cudaSuccess) {
        set_error("%s: %s", what, cudaGetErrorString(e));
        return GF_ERR_CUDA;
    }
    gf_krylov_t arg = *k;
    int targ = T;
    void* args[] = {&arg, &targ};
    e = cudaLaunchCooperativeKernel(kern, dim3(grid), dim3(kStThreads), args, smem, s);
    if (e != cudaSuccess) {
        set_error("%s: cooperative launch failed: %s", what, cudaGetErrorString(e));
        return GF_ERR_CUDA;
    }
    return GF_OK;
}

// Cooperative launch of the shared-memory-resident CG: 1, 2 or 4 blocks per
// SM, whichever most gives each block a chunk whose four vectors fit its
// shared memory; GF_ERR_INVALID (no launch) when none fits.
template <int THREADS, bool KEEP_P>
static const void* smem_kernel(const gf_krylov_t* k) {
    if (k->stride_y > 0)
        return k->symmetric ? (const void*)k_pcg1_smem_box<true, THREADS, KEEP_P>
                            : (const void*)k_pcg1_smem_box<false, THREADS, KEEP_P>;
    return k->width == 6 ? (const void*)k_pcg1_smem_ell<6, THREADS, KEEP_P>
                         : (const void*)k_pcg1_smem_ell<0, THREADS, KEEP_P>;
}

template <int THREADS, bool KEEP_P>
static const void* mixed_smem_kernel(const gf_krylov_t* k) {
    if (k->stride_y > 0)
        return k->symmetric ? (const void*)k_pcg1_mixed_smem_box<true, THREADS, KEEP_P>
                            : (const void*)k_pcg1_mixed_smem_box<false, THREADS, KEEP_P>;
    return k->width == 6 ? (const void*)k_pcg1_mixed_smem_ell<6, THREADS, KEEP_P>
                         : (const void*)k_pcg1_mixed_smem_ell<0, THREADS, KEEP_P>;
}

template <int U>
static const void* qrec_kernel(const gf_krylov_t* k) {
    if (k->stride_y > 0)
        return k->symmetric ? (const void*)k_pcg1_qrec_box<true, 1024, U> : (const void*)k_pcg1_qrec_box<false, 1024, U>;
    return k->width == 6 ? (const void*)k_pcg1_qrec_ell<6, 1024, U> : (const void*)k_pcg1_qrec_ell<0, 1024, U>;
}

static int launch_smem_arrays(const gf_krylov_t* k, void* stream, int threads, int narr, size_t elem,
                              const void* kern);

template <int THREADS, int MINB>
static const void* stream_kernel(const gf_krylov_t* k) {
    if (k->stride_y > 0)
        return k->symmetric ? (const void*)k_pcg1_stream_box<true, THREADS, MINB>
                            : (const void*)k_pcg1_stream_box<false, THREADS, MINB>;
    return k->width == 6 ? (const void*)k_pcg1_stream_ell<6, THREADS, MINB>
                         : (const void*)k_pcg1_stream_ell<0, THREADS, MINB>;
}

// Streaming CG (variants 12-14): every co-resident block owns one contiguous
// chunk of cells.  GF_ERR_INVALID (no launch) where 32-bit cell indices do
// not reach every coefficient slot.
static int launch_stream(const gf_krylov_t* k, void* stream, int which) {
    const char* what = "gf_pcg_solve";
    const int64_t row_span = (int64_t)(k->stride_y > 0 ? 6 : (k->width > 6 ? k->width : 6)) * k->n;
    if (row_span >= ((int64_t)1 << 31)) {
        set_error("%s: system not eligible for the streaming CG", what);
        return GF_ERR_INVALID;
    }
    const void* kern = which == 1 ? stream_kernel<1024, 1>(k) : which == 2 ? stream_kernel<256, 4>(k)
                                                                           : stream_kernel<512, 2>(k);
    const int threads = which == 1 ? 1024 : which == 2 ? 256 : 512;
    int dev = 0, sms = 0, coop = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
    int per_sm = 0;
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, 0);
    if (e != cudaSuccess || !coop || per_sm < 1) {
        set_error("%s: streaming CG set-up failed: %s", what, cudaGetErrorString(e));
        return GF_ERR_CUDA;
    }
    int64_t grid = (int64_t)per_sm * sms;
    const int64_t want = (k->n + threads - 1) / threads;
    if (grid > want) grid = want;
    if (grid > kMaxBlocks) grid = kMaxBlocks;
    if (k->block_cap > 0 && grid > k->block_cap) grid = k->block_cap;
    if (grid < 1) grid = 1;
    const int64_t chunk = (k->n + grid - 1) / grid;
    grid = (k->n + chunk - 1) / chunk;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    e = cudaMemsetAsync(k->work, 0, sizeof(KCtl), st);
    if (e != cudaSuccess) {
        set_error("%s: %s", what, cudaGetErrorString(e));
        return GF_ERR_CUDA;
    }
    gf_krylov_t arg = *k;
    int ch = (int)chunk;
    void* args[] = {&arg, &ch};
    e = cudaLaunchCooperativeKernel(kern, dim3((unsigned)grid), dim3(threads), args, 0, st);
    if (e != cudaSuccess) {
        set_error("%s: cooperative launch failed: %s", what, cudaGetErrorString(e));
        return GF_ERR_CUDA;
    }
    return GF_OK;
}

// FP64: 4 doubles a cell with p kept, else 3.  Mixed: 5 floats, else 4.
static int launch_smem(const gf_krylov_t* k, void* stream, int threads) {
    const bool mixed = k->mixed != 0;
    const size_t elem = mixed ? sizeof(float) : sizeof(double);
    for (int keep = 1; keep >= 0; --keep) {
        const void* kern;
        if (mixed)
            kern = threads == 1024 ? (keep ? mixed_smem_kernel<1024, true>(k) : mixed_smem_kernel<1024, false>(k))
                                   : (keep ? mixed_smem_kernel<512, true>(k) : mixed_smem_kernel<512, false>(k));
        else
            kern = threads == 1024 ? (keep ? smem_kernel<1024, true>(k) : smem_kernel<1024, false>(k))
                                   : (keep ? smem_kernel<512, true>(k) : smem_kernel<512, false>(k));
        const int narr = (mixed ? 4 : 3) + keep;
        const int st = launch_smem_arrays(k, stream, threads, narr, elem, kern);
        if (st != GF_ERR_INVALID) return st;
    }
    return GF_ERR_INVALID;
}

template <int U>
static const void* mixed_qrec_kernel(const gf_krylov_t* k) {
    if (k->stride_y > 0)
        return k->symmetric ? (const void*)k_pcg1_mixed_qrec_box<true, U> : (const void*)k_pcg1_mixed_qrec_box<false, U>;
    return k->width == 6 ? (const void*)k_pcg1_mixed_qrec_ell<6, U> : (const void*)k_pcg1_mixed_qrec_ell<0, U>;
}

// The q-recurrence forms (1024 threads): FP64 keeps r, q and p in shared
// memory (3 doubles a cell), FP32-inner r, q, p, d and the inverse (5 floats).
static int launch_qrec(const gf_krylov_t* k, void* stream, int unroll) {
    if (k->mixed) {
        const void* kern = unroll == 2 ? mixed_qrec_kernel<2>(k) : mixed_qrec_kernel<1>(k);
        return launch_smem_arrays(k, stream, 1024, 5, sizeof(float), kern);
    }
    const void* kern = unroll == 2 ? qrec_kernel<2>(k) : qrec_kernel<1>(k);
    return launch_smem_arrays(k, stream, 1024, 3, sizeof(double), kern);
}

template <int U>
static const void* halo_kernel(const gf_krylov_t* k) {
    if (k->stride_y > 0)
        return k->symmetric ? (const void*)k_pcg1_halo_box<true, U> : (const void*)k_pcg1_halo_box<false, U>;
    return k->width == 6 ? (const void*)k_pcg1_halo_ell<6, U> : (const void*)k_pcg1_halo_ell<0, U>;
}

// FP64 single-reduction form: r, p, q and w in shared memory (4 doubles a
// cell), the halo flags after z and the inverse in the workspace; the
// q-recurrence form (variant 8) when either does not fit.
static int launch_halo(const gf_krylov_t* k, void* stream, int unroll) {
    if (k->work_len >= kHeader + 2 * k->n + kHaloFlagDoubles) {
        const void* kern = unroll == 2 ? halo_kernel<2>(k) : halo_kernel<1>(k);
        const int st = launch_smem_arrays(k, stream, 1024, 4, sizeof(double), kern);
        if (st != GF_ERR_INVALID) return st;
    }
    return launch_qrec(k, stream, 1);
}

// FP32-inner single-reduction form (variants 10/11): r, q, d, inverse, p and
// w in shared memory (6 floats a cell), the halo flags at the start of the
// workspace's vector region; GF_ERR_INVALID (no launch) when n is too small
// for the flags or the arrays do not fit.
static int launch_mixed_halo(const gf_krylov_t* k, void* stream) {
    if (k->n < kHaloFlagDoubles) return GF_ERR_INVALID;
    const void* kern;
    if (k->stride_y > 0)
        kern = k->symmetric ? (const void*)k_pcg1_mixed_halo_box<true> : (const void*)k_pcg1_mixed_halo_box<false>;
    else
        kern = k->width == 6 ? (const void*)k_pcg1_mixed_halo_ell<6> : (const void*)k_pcg1_mixed_halo_ell<0>;
    return launch_smem_arrays(k, stream, 1024, 6, sizeof(float), kern);
}

static int launch_smem_arrays(const gf_krylov_t* k, void* stream, int threads, int narr, size_t elem,
                              const void* kern) {
    const char* what = "gf_pcg_solve";
    const int kSmemThreads = threads;
    int dev = 0, sms = 0, optin = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (e != cudaSuccess) {
        set_error("%s: %s", what, cudaGetErrorString(e));
        return GF_ERR_CUDA;
    }
    cudaFuncAttributes fa;
    e = cudaFuncGetAttributes(&fa, kern);
    if (e != cudaSuccess) {
        set_error("%s: %s", what, cudaGetErrorString(e));
        return GF_ERR_CUDA;
    }
    const int64_t static_smem = (int64_t)fa.sharedSizeBytes;  // CgState and the reduction scratch
    // 32-bit cell indices (coefficient slot x n included) and 16-byte pair
    // buffers in the workspace.
    const int64_t row_span = (int64_t)(k->stride_y > 0 ? 6 : (k->width > 6 ? k->width : 6)) * k->n;
    if (row_span >= ((int64_t)1 << 31) || (reinterpret_cast<uintptr_t>(k->work) & 15u)) {
        set_error("%s: system not eligible for shared-memory-resident CG", what);
        return GF_ERR_INVALID;
    }
    for (int per_sm : {4, 2, 1}) {
        int64_t grid = (int64_t)sms * per_sm;
        const int64_t want = (k->n + kSmemThreads - 1) / kSmemThreads;
        if (grid > want) grid = want;
        if (grid > kMaxBlocks) grid = kMaxBlocks;
        if (k->block_cap > 0 && grid > k->block_cap) grid = k->block_cap;
        if (grid < 1) grid = 1;
        int64_t chunk = (k->n + grid - 1) / grid;
        chunk = (chunk + 1) & ~1LL;
        const size_t smem = (size_t)(narr * chunk) * elem;
        if ((int64_t)smem + static_smem > optin) continue;
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        int occ = 0;
        if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kSmemThreads, smem);
        if (e != cudaSuccess) {
            set_error("%s: shared-memory CG set-up failed: %s", what, cudaGetErrorString(e));
            return GF_ERR_CUDA;
        }
        if ((int64_t)occ * sms < grid) continue;
        // The chunks must cover n with these many blocks.
        grid = (k->n + chunk - 1) / chunk;
        cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
        e = cudaMemsetAsync(k->work, 0, sizeof(KCtl), s);
        if (e != cudaSuccess) {
            set_error("%s: %s", what, cudaGetErrorString(e));
            return GF_ERR_CUDA;
        }
        gf_krylov_t arg = *k;
        int carg = (int)chunk;
        void* args[] = {&arg, &carg};
        e = cudaLaunchCooperativeKernel(kern, dim3((unsigned)grid), dim3(kSmemThreads), args, smem, s);
        if (e != cudaSuccess) {
            set_error("%s: cooperative launch failed: %s", what, cudaGetErrorString(e));
            return GF_ERR_CUDA;
        }
        return GF_OK;
    }
    set_error("%s: system too large for shared-memory-resident CG", what);
    return GF_ERR_INVALID;
}

// nvec vectors of ncomp x n doubles plus `extra` doubles after the header.
static bool valid_krylov(const gf_krylov_t* k, int nvec, const char* what, int64_t extra = 0) {
    if (k == nullptr || k->n <= 0 || k->width <= 0 || k->ncomp < 1 || k->ncomp > 3 || k->nbr == nullptr ||
        k->diag == nullptr || k->val == nullptr || k->rhs == nullptr || k->x == nullptr || k->work == nullptr ||
        k->stats == nullptr || k->max_iter < 0) {
        set_error("%s: invalid arguments", what);
        return false;
    }
    const int64_t need = kHeader + (int64_t)nvec * k->ncomp * k->n + extra;
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
    // kind 3 + 100 * width: mixed-precision BiCGStab (ncomp components):
    // (width + 2) n coefficient floats and 7 ncomp n vector floats.
    if (kind >= 3 && kind % 100 == 3) {
        const int64_t width = (kind - 3) / 100 > 0 ? (kind - 3) / 100 : kMaxEll;
        const int64_t floats = (width + 2 + 7 * (int64_t)ncomp) * n;
        return kHeader + (floats + 1) / 2 + 1;
    }
    // kind 2 + 100 * width: mixed-precision CG for an ELL of that width.
    if (kind >= 2) {
        const int64_t width = (kind - 2) / 100 > 0 ? (kind - 2) / 100 : kMaxEll;
        const int64_t floats = (width + 8) * n;
        return kHeader + n + (floats + 1) / 2 + 1;
    }
    const int bicgstab = kind == 1;
    const int nvec = bicgstab ? 6 : (ncomp == 1 ? 7 : 3);
    // BiCGStab keeps the Jacobi inverse (n doubles) after its six vectors.
    return kHeader + (int64_t)nvec * ncomp * n + (bicgstab ? n : 0);
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
        if (k->variant == kSmemVariant || k->variant == kSmemVariant + 1) {
            const int st = launch_smem(k, stream, k->variant == kSmemVariant ? 512 : 1024);
            if (st != GF_ERR_INVALID) return st;
        }
        if (k->variant >= kQrecVariant && k->variant <= kHaloVariant + 1) {
            int st = GF_ERR_INVALID;
            if (k->variant >= kHaloVariant) st = launch_mixed_halo(k, stream);
            if (st == GF_ERR_INVALID) st = launch_qrec(k, stream, (k->variant - kQrecVariant) % 2 == 0 ? 1 : 2);
            if (st != GF_ERR_INVALID) return st;
        }
        if (box) {
            // Variants 5-9 that do not qualify fall back to 512-thread blocks.
            const int v = (k->variant >= 0 && k->variant < kBoxVariants) ? k->variant
                          : (k->variant >= kStagedVariant ? 2 : 0);
            const BoxVariant bv = k->symmetric ? box_kernel<true, true>(v) : box_kernel<true, false>(v);
            return launch_persistent(bv.kern, k, stream, "gf_pcg_solve", bv.threads, bv.unroll);
        }
        if (k->width == 6) return launch_persistent(k_pcg1_mixed<6>, k, stream, "gf_pcg_solve", kCgThreads);
        return launch_persistent(k_pcg1_mixed<0>, k, stream, "gf_pcg_solve", kCgThreads);
    }
    if (!valid_krylov(k, k->ncomp == 1 ? (k->single_reduction ? 7 : 5) : 3, "gf_pcg_solve")) return GF_ERR_INVALID;
    switch (k->ncomp) {
        case 1:
            if (k->single_reduction) {
                if (box) {
                    const int v = (k->variant >= 0 && k->variant < kBoxVariants) ? k->variant : 0;
                    const BoxVariant bv = k->symmetric ? sr_box_kernel<true>(v) : sr_box_kernel<false>(v);
                    return launch_persistent(bv.kern, k, stream, "gf_pcg_solve", bv.threads, 1);
                }
                if (k->width == 6) return launch_persistent(k_pcg1_sr<6>, k, stream, "gf_pcg_solve", kCgThreads);
                return launch_persistent(k_pcg1_sr<0>, k, stream, "gf_pcg_solve", kCgThreads);
            }
            if (k->variant == kSmemVariant || k->variant == kSmemVariant + 1) {
                const int st = launch_smem(k, stream, k->variant == kSmemVariant ? 512 : 1024);
                if (st != GF_ERR_INVALID) return st;
            }
            if (k->variant == kQrecVariant || k->variant == kQrecVariant + 1) {
                const int st = launch_qrec(k, stream, k->variant == kQrecVariant ? 1 : 2);
                if (st != GF_ERR_INVALID) return st;
            }
            if (k->variant == kHaloVariant || k->variant == kHaloVariant + 1) {
                const int st = launch_halo(k, stream, k->variant == kHaloVariant ? 1 : 2);
                if (st != GF_ERR_INVALID) return st;
            }
            if (k->variant >= kStreamVariant && k->variant < kStreamVariant + kStreamVariants) {
                const int st = launch_stream(k, stream, k->variant - kStreamVariant);
                if (st != GF_ERR_INVALID) return st;
            }
            if (k->variant >= kSplitVariant && k->variant < kSplitVariant + kSplitVariants) {
                const int st = launch_split(k, stream, k->variant - kSplitVariant);
                if (st != GF_ERR_INVALID) return st;
            }
            if (box && k->variant == kStagedVariant) {
                const int T = staged_tile(k);
                if (T > 0) return launch_staged(k, T, stream);
            }
            if (box) {
                // Variants 5-7 that do not qualify fall back to 512-thread blocks.
                const int v = (k->variant >= 0 && k->variant < kBoxVariants) ? k->variant
                              : (k->variant >= kStagedVariant ? 2 : 0);
                const BoxVariant bv = k->symmetric ? box_kernel<false, true>(v) : box_kernel<false, false>(v);
                return launch_persistent(bv.kern, k, stream, "gf_pcg_solve", bv.threads, bv.unroll);
            }
            if (k->variant >= kOccVariant && k->variant < kOccVariant + kOccVariants &&
                (int64_t)(k->width > 6 ? k->width : 6) * k->n < ((int64_t)1 << 31)) {
                const int w = k->variant - kOccVariant;
                const BoxVariant ev = k->width == 6 ? ell_occ_kernel<6>(w) : ell_occ_kernel<0>(w);
                return launch_persistent(ev.kern, k, stream, "gf_pcg_solve", ev.threads, 1);
            }
            {
                // Variants beyond the five launch shapes fall back to 256 x 1.
                const int v = (k->variant >= 0 && k->variant < kBoxVariants) ? k->variant : 0;
                const BoxVariant ev = k->width == 6 ? ell_kernel<6>(v) : ell_kernel<0>(v);
                return launch_persistent(ev.kern, k, stream, "gf_pcg_solve", ev.threads, ev.unroll);
            }
        case 2:
            return launch_persistent(k_pcg<2>, k, stream, "gf_pcg_solve");
        default:
            return launch_persistent(k_pcg<3>, k, stream, "gf_pcg_solve");
    }
}

int gf_bicgstab_solve(const gf_krylov_t* k, void* stream) {
    if (k != nullptr && k->mixed) {
        // FP32 inner cycles in FP64 refinement (k_bicgstab_mixed).
        if (!valid_krylov(k, 0, "gf_bicgstab_solve") || k->max_outer < 1 || k->width > kMaxEll ||
            k->work_len < gf_krylov_workspace_size(k->n, k->ncomp, 3 + 100 * k->width)) {
            set_error("gf_bicgstab_solve: mixed precision needs max_outer >= 1, width <= %d and the mixed "
                      "BiCGStab workspace", kMaxEll);
            return GF_ERR_INVALID;
        }
        const bool m6 = k->width == 6;
        switch (k->ncomp) {
            case 1:
                return m6 ? launch_persistent(k_bicgstab_mixed<1, 6>, k, stream, "gf_bicgstab_solve")
                          : launch_persistent(k_bicgstab_mixed<1, 0>, k, stream, "gf_bicgstab_solve");
            case 2:
                return m6 ? launch_persistent(k_bicgstab_mixed<2, 6>, k, stream, "gf_bicgstab_solve")
                          : launch_persistent(k_bicgstab_mixed<2, 0>, k, stream, "gf_bicgstab_solve");
            default:
                return m6 ? launch_persistent(k_bicgstab_mixed<3, 6>, k, stream, "gf_bicgstab_solve")
                          : launch_persistent(k_bicgstab_mixed<3, 0>, k, stream, "gf_bicgstab_solve");
        }
    }
    if (!valid_krylov(k, 6, "gf_bicgstab_solve", k ? k->n : 0)) return GF_ERR_INVALID;
    const bool w6 = k->width == 6;
    switch (k->ncomp) {
        case 1:
            return w6 ? launch_persistent(k_bicgstab<1, 6>, k, stream, "gf_bicgstab_solve")
                      : launch_persistent(k_bicgstab<1, 0>, k, stream, "gf_bicgstab_solve");
        case 2:
            return w6 ? launch_persistent(k_bicgstab<2, 6>, k, stream, "gf_bicgstab_solve")
                      : launch_persistent(k_bicgstab<2, 0>, k, stream, "gf_bicgstab_solve");
        default:
            return w6 ? launch_persistent(k_bicgstab<3, 6>, k, stream, "gf_bicgstab_solve")
                      : launch_persistent(k_bicgstab<3, 0>, k, stream, "gf_bicgstab_solve");
    }
}

}  // extern "C"

// Batched launch of count systems (gf_pcg_solve_batched /
// gf_bicgstab_solve_batched).  blocks[i] persistent blocks for system i;
// their sum must be co-resident.
static int launch_batched(const gf_krylov_t* sys, int32_t count, const int32_t* blocks, void* stream, bool bicg) {
    const char* what = bicg ? "gf_bicgstab_solve_batched" : "gf_pcg_solve_batched";
    if (sys == nullptr || blocks == nullptr || count < 1 || count > kMaxBatch) {
        set_error("%s: need 1..%d systems and their block counts", what, kMaxBatch);
        return GF_ERR_INVALID;
    }
    KBatch B;
    memset(&B, 0, sizeof(B));
    B.count = count;
    int total = 0;
    for (int i = 0; i < count; ++i) {
        const gf_krylov_t& k = sys[i];
        if (k.mixed && bicg) {
            set_error("%s: system %d: the batched BiCGStab has no FP32-inner form", what, i);
            return GF_ERR_INVALID;
        }
        if (k.mixed && !bicg) {
            // FP32-inner CG: one system and the mixed workspace.
            if (!valid_krylov(&k, 0, what) || k.ncomp != 1 || k.max_outer < 1 || k.width > kMaxEll ||
                k.work_len < gf_krylov_workspace_size(k.n, 1, 2 + 100 * k.width)) {
                set_error("%s: system %d: mixed precision needs one system, max_outer >= 1 and the mixed "
                          "workspace", what, i);
                return GF_ERR_INVALID;
            }
        } else {
            const int nvec = bicg ? 6 : (k.ncomp == 1 ? 5 : 3);
            if (!valid_krylov(&k, nvec, what, bicg ? k.n : 0)) return GF_ERR_INVALID;
        }
        if ((bicg && k.mixed) || k.single_reduction || (!bicg && k.ncomp != 1) ||
            (bicg && k.ncomp != sys[0].ncomp)) {
            set_error("%s: system %d: one system for CG, FP64 and the same component count for BiCGStab", what, i);
            return GF_ERR_INVALID;
        }
        if (k.stride_y > 0 && (k.width != 6 || k.stride_z < k.stride_y || k.stride_y < 1)) {
            set_error("%s: system %d: a box layout needs width 6 and strides 1 <= stride_y <= stride_z", what, i);
            return GF_ERR_INVALID;
        }
        if (blocks[i] < 1 || blocks[i] > kMaxBlocks) {
            set_error("%s: system %d: block count %d outside 1..%d", what, i, blocks[i], kMaxBlocks);
            return GF_ERR_INVALID;
        }
        B.sys[i] = k;
        B.blk0[i] = total;
        total += blocks[i];
    }
    B.blk0[count] = total;
    const void* kern = !bicg ? (const void*)k_pcg1_batched
                             : (sys[0].ncomp == 1 ? (const void*)k_bicgstab_batched<1>
                                                  : sys[0].ncomp == 2 ? (const void*)k_bicgstab_batched<2>
                                                                      : (const void*)k_bicgstab_batched<3>);
    const int threads = bicg ? kKThreads : kCgThreads;
    int dev = 0, sms = 0, coop = 0, per_sm = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, 0);
    if (e != cudaSuccess || !coop) {
        set_error("%s: set-up failed: %s", what, cudaGetErrorString(e));
        return GF_ERR_CUDA;
    }
    if (total > per_sm * sms) {
        set_error("%s: %d blocks requested, %d co-resident at most", what, total, per_sm * sms);
        return GF_ERR_INVALID;
    }
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    k_batch_reset<<<1, 32, 0, st>>>(B);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error("%s: %s", what, cudaGetErrorString(e));
        return GF_ERR_CUDA;
    }
    void* args[] = {&B};
    e = cudaLaunchCooperativeKernel(kern, dim3(total), dim3(threads), args, 0, st);
    if (e != cudaSuccess) {
        set_error("%s: cooperative launch failed: %s", what, cudaGetErrorString(e));
        return GF_ERR_CUDA;
    }
    return GF_OK;
}

extern "C" {

int gf_pcg_solve_batched(const gf_krylov_t* systems, int32_t count, const int32_t* blocks, void* stream) {
    return launch_batched(systems, count, blocks, stream, false);
}

int gf_bicgstab_solve_batched(const gf_krylov_t* systems, int32_t count, const int32_t* blocks, void* stream) {
    return launch_batched(systems, count, blocks, stream, true);
}

int gf_batch_max_blocks(int32_t bicgstab) {
    const void* kern = bicgstab ? (const void*)k_bicgstab_batched<3> : (const void*)k_pcg1_batched;
    int dev = 0, sms = 0, per_sm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) !=
        cudaSuccess || cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, bicgstab ? kKThreads : kCgThreads,
                                                                      0) != cudaSuccess) {
        set_error("gf_batch_max_blocks: device query failed");
        return -1;
    }
    return per_sm * sms;
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

// One FP64 system of up to 262,144 cells (14.3 MiB).
constexpr int64_t kStaticScratchCells = 262144;
constexpr int64_t kStaticScratchDoubles = kHeader + 7 * kStaticScratchCells;

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
    // The system's own workspace size, not the whole array: the launch
    // shape depends on work_len, and this keeps it the one gf_pcg_solve
    // picks for a workspace sized by gf_krylov_workspace_size.
    local.work_len = need;
    // gf_pcg_solve clears the barrier control block before its launch; the
    // partials and vectors are written before they are read.
    return gf_pcg_solve(&local, stream);
}

}  // extern "C"
