/*
 * CPU oracle: Jacobi-preconditioned CG and right-preconditioned BiCGStab
 * with breakdown restarts, multi-threaded with OpenMP.
 *
 * Test and baseline infrastructure only: the same algorithms as
 * oracle/solvers.py (cg_single, bicgstab_single), which restate the
 * reference's solvers/cg.py:237-336 and solvers/bicgstab.py:76-272
 * (paths inside the reference's src/gridfoam), written in C so that the
 * CPU baseline of a multi-million-cell case runs on every host core.
 *
 * The matrix is given by rows (CSR of the off-diagonal LDU coefficients,
 * coef[e] the coefficient of x[col[e]] in row r, rowptr[r] <= e <
 * rowptr[r+1]) plus the diagonal.  Dot products and norms sum fixed chunks
 * in parallel and then the chunk partials in order, so results do not
 * depend on the thread count.
 */
#include <math.h>
#ifdef _OPENMP
#include <omp.h>
#endif
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define CHUNK 4096

static void spmv(int64_t n, const int64_t* rowptr, const int32_t* col, const double* coef,
                 const double* diag, const double* x, double* y) {
#pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < n; ++r) {
        double s = diag[r] * x[r];
        for (int64_t e = rowptr[r]; e < rowptr[r + 1]; ++e) s += coef[e] * x[col[e]];
        y[r] = s;
    }
}

/* sum_i a[i] * b[i] in fixed chunks; part holds ceil(n / CHUNK) doubles. */
static double dot(int64_t n, const double* a, const double* b, double* part) {
    const int64_t nc = (n + CHUNK - 1) / CHUNK;
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < nc; ++c) {
        const int64_t lo = c * CHUNK, hi = lo + CHUNK < n ? lo + CHUNK : n;
        double s = 0.0;
        for (int64_t i = lo; i < hi; ++i) s += a[i] * b[i];
        part[c] = s;
    }
    double s = 0.0;
    for (int64_t c = 0; c < nc; ++c) s += part[c];
    return s;
}

static double amax(int64_t n, const double* a, double* part) {
    const int64_t nc = (n + CHUNK - 1) / CHUNK;
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < nc; ++c) {
        const int64_t lo = c * CHUNK, hi = lo + CHUNK < n ? lo + CHUNK : n;
        double s = 0.0;
        for (int64_t i = lo; i < hi; ++i) {
            const double v = fabs(a[i]);
            if (v > s || v != v) s = v;
        }
        part[c] = s;
    }
    double s = 0.0;
    for (int64_t c = 0; c < nc; ++c)
        if (part[c] > s || part[c] != part[c]) s = part[c];
    return s;
}

static double norm(int64_t n, const double* a, int norm_inf, double* part) {
    if (norm_inf) return n ? amax(n, a, part) : 0.0;
    return sqrt(dot(n, a, a, part));
}

/* z = inv * r (inv NULL: identity) */
static void precond(int64_t n, const double* inv, const double* r, double* z) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) z[i] = inv ? inv[i] * r[i] : r[i];
}

/* One parallel pass over fixed chunks of rows: q = A p and the chunk
 * partials of p.q (summed in chunk order by the caller). */
static double spmv_dot(int64_t n, const int64_t* rowptr, const int32_t* col, const double* coef,
                       const double* diag, const double* p, double* q, double* part) {
    const int64_t nc = (n + CHUNK - 1) / CHUNK;
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < nc; ++c) {
        const int64_t lo = c * CHUNK, hi = lo + CHUNK < n ? lo + CHUNK : n;
        double s = 0.0;
        for (int64_t r = lo; r < hi; ++r) {
            double y = diag[r] * p[r];
            for (int64_t e = rowptr[r]; e < rowptr[r + 1]; ++e) y += coef[e] * p[col[e]];
            q[r] = y;
            s += p[r] * y;
        }
        part[c] = s;
    }
    double s = 0.0;
    for (int64_t c = 0; c < nc; ++c) s += part[c];
    return s;
}

/* stats: initial residual, final residual, iterations, converged.  Each
 * iteration is three passes: q = A p with p.q; x += alpha p, r -= alpha q,
 * z = M r with |r| and r.z; p = z + beta p.  The sums are those of the
 * separate loops (rows in slot order, dot products by chunks in order). */
int oracle_cg(int64_t n, const int64_t* rowptr, const int32_t* col, const double* coef, const double* diag,
              const double* b, double* x, const double* inv, double atol, double rtol, int norm_inf,
              int max_iter, double* stats) {
    const int64_t nch = (n + CHUNK - 1) / CHUNK;
    const int64_t nc = 2 * nch + 2;
    double* buf = (double*)malloc(sizeof(double) * (4 * n + nc));
    if (!buf) return 1;
    double *r = buf, *z = buf + n, *p = buf + 2 * n, *q = buf + 3 * n, *part = buf + 4 * n,
           *part2 = buf + 4 * n + nch + 1;
    spmv(n, rowptr, col, coef, diag, x, q);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) r[i] = b[i] - q[i];
    const double r0 = norm(n, r, norm_inf, part);
    const double thresh = atol > rtol * r0 ? atol : rtol * r0;
    if (r0 < thresh) {
        stats[0] = r0, stats[1] = r0, stats[2] = 0, stats[3] = 1;
        free(buf);
        return 0;
    }
    precond(n, inv, r, z);
    memcpy(p, z, sizeof(double) * n);
    double rz = dot(n, r, z, part);
    int converged = 0, it = 0;
    double fin = r0;
    for (it = 1; it <= max_iter; ++it) {
        const double alpha = rz / spmv_dot(n, rowptr, col, coef, diag, p, q, part);
#pragma omp parallel for schedule(static)
        for (int64_t c = 0; c < nch; ++c) {
            const int64_t lo = c * CHUNK, hi = lo + CHUNK < n ? lo + CHUNK : n;
            double s = 0.0, t = 0.0;
            for (int64_t i = lo; i < hi; ++i) {
                x[i] = x[i] + alpha * p[i];
                const double ri = r[i] - alpha * q[i];
                r[i] = ri;
                const double zi = inv ? inv[i] * ri : ri;
                z[i] = zi;
                if (norm_inf) {
                    const double v = fabs(ri);
                    if (v > s || v != v) s = v;
                } else {
                    s += ri * ri;
                }
                t += ri * zi;
            }
            part[c] = s;
            part2[c] = t;
        }
        double s = 0.0, rz_new = 0.0;
        for (int64_t c = 0; c < nch; ++c) {
            if (norm_inf) {
                if (part[c] > s || part[c] != part[c]) s = part[c];
            } else {
                s += part[c];
            }
            rz_new += part2[c];
        }
        fin = norm_inf ? s : sqrt(s);
        if (fin < thresh) {
            converged = 1;
            break;
        }
        const double beta = rz_new / rz;
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; ++i) p[i] = z[i] + p[i] * beta;
        rz = rz_new;
    }
    if (it > max_iter) it = max_iter;
    stats[0] = r0, stats[1] = fin, stats[2] = it, stats[3] = converged;
    free(buf);
    return 0;
}

/* bicgstab.py:262-272: eps * |x| * |y| (2-norms; NULL counts as 1). */
static double btol(int64_t n, const double* x, const double* y, double* part) {
    const double xn = x ? sqrt(dot(n, x, x, part)) : 1.0;
    const double yn = y ? sqrt(dot(n, y, y, part)) : 1.0;
    return 1e-6 * xn * yn;
}

int oracle_bicgstab(int64_t n, const int64_t* rowptr, const int32_t* col, const double* coef,
                    const double* diag, const double* b, double* x, const double* inv, double atol, double rtol,
                    int norm_inf, int max_iter, int max_restart, double* stats) {
    const int64_t nc = (n + CHUNK - 1) / CHUNK + 1;
    double* buf = (double*)malloc(sizeof(double) * (8 * n + nc));
    if (!buf) return 1;
    double *r = buf, *rh = buf + n, *p = buf + 2 * n, *v = buf + 3 * n, *y = buf + 4 * n, *s = buf + 5 * n,
           *zz = buf + 6 * n, *t = buf + 7 * n, *part = buf + 8 * n;
    spmv(n, rowptr, col, coef, diag, x, v);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) r[i] = b[i] - v[i];
    const double r0 = norm(n, r, norm_inf, part);
    const double thresh = atol > rtol * r0 ? atol : rtol * r0;
    if (r0 < thresh) {
        stats[0] = r0, stats[1] = r0, stats[2] = 0, stats[3] = 1;
        free(buf);
        return 0;
    }
    int restarts = 0, converged = 0, it = 0;
    double fin = r0;
    memcpy(rh, r, sizeof(double) * n);
    memcpy(p, r, sizeof(double) * n);
    double rho_old = dot(n, r, r, part);
#define RESTART()                                   \
    do {                                            \
        if (restarts >= max_restart) goto done;     \
        ++restarts;                                 \
        memcpy(rh, r, sizeof(double) * n);          \
        memcpy(p, r, sizeof(double) * n);           \
        rho_old = dot(n, r, r, part);               \
    } while (0)
    for (it = 1; it <= max_iter; ++it) {
        precond(n, inv, p, y);
        spmv(n, rowptr, col, coef, diag, y, v);
        const double da = dot(n, rh, v, part);
        if (fabs(da) <= btol(n, rh, v, part)) {
            RESTART();
            continue;
        }
        const double alpha = rho_old / da;
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; ++i) s[i] = r[i] - alpha * v[i];
        fin = norm(n, s, norm_inf, part);
        if (fin < thresh) {
#pragma omp parallel for schedule(static)
            for (int64_t i = 0; i < n; ++i) x[i] = x[i] + alpha * y[i];
            converged = 1;
            break;
        }
        precond(n, inv, s, zz);
        spmv(n, rowptr, col, coef, diag, zz, t);
        const double dd = dot(n, t, t, part);
        if (fabs(dd) <= btol(n, t, t, part)) {
            RESTART();
            continue;
        }
        const double omega = dot(n, t, s, part) / dd;
        if (fabs(omega) <= btol(n, NULL, NULL, part)) {
            RESTART();
            continue;
        }
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; ++i) {
            x[i] = x[i] + alpha * y[i] + omega * zz[i];
            r[i] = s[i] - omega * t[i];
        }
        fin = norm(n, r, norm_inf, part);
        if (fin < thresh) {
            converged = 1;
            break;
        }
        const double rho_new = dot(n, rh, r, part);
        if (fabs(rho_new) <= btol(n, rh, r, part)) {
            RESTART();
            continue;
        }
        const double beta = (rho_new / rho_old) * (alpha / omega);
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; ++i) p[i] = r[i] + beta * (p[i] - omega * v[i]);
        rho_old = rho_new;
    }
#undef RESTART
done:
    if (it > max_iter) it = max_iter;
    stats[0] = r0, stats[1] = fin, stats[2] = it, stats[3] = converged;
    free(buf);
    return 0;
}

int oracle_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* out[c, k] = sum of values[i, k] over the i with index[i] == c, summed in
 * increasing i: rows of a stable sort of the index (perm, rowptr).  The
 * order of every sum is that of numpy's bincount, so the result is the same
 * bit for bit (oracle/case.py scatter_add). */
void oracle_segment_sum(int64_t n, const int64_t* rowptr, const int64_t* perm, int64_t ncomp,
                        const double* values, double* out) {
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < n; ++c) {
        for (int64_t k = 0; k < ncomp; ++k) {
            double s = 0.0;
            for (int64_t e = rowptr[c]; e < rowptr[c + 1]; ++e) s += values[perm[e] * ncomp + k];
            out[c * ncomp + k] = s;
        }
    }
}
