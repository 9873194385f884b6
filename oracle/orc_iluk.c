/*
 * orc_iluk.c -- TEST INFRASTRUCTURE ONLY.  CPU FP64 conjugate gradients preconditioned by an
 * incomplete LU factorisation with k levels of fill, ILU(k): the preconditioner of the
 * reference's serial PETSc solver (KSPCG with PCILU, -pc_factor_levels 3, src/la/solve.cc:370).
 * PETSc is a third-party dependency (>= 3.4.0, CMakeLists.txt:279) that is not vendored with
 * the reference, so this restates the published algorithm: the level-of-fill rule of Saad,
 * "Iterative Methods for Sparse Linear Systems" (2nd ed., section 10.3.3, algorithm 10.5):
 * an entry of the original pattern has level 0, an update a_ij -= a_ik a_kj creates level
 * lev_ik + lev_kj + 1, and entries above level k are dropped; the numeric factorisation is the
 * IKJ elimination restricted to that pattern.  Used by bench.py's CPU baseline and pinned by
 * tests/test_oracle_golden.py (ILU(0) equals orc_ilu0; enough levels give the exact LU).
 * It is never linked into or called by the product.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* Pattern (rows sorted, diagonal included) of ILU(p) of a CSR matrix with sorted rows.
 * Returns nnz and fills frp [n+1] and fcol [nnz] when nnz <= cap (else only returns nnz);
 * -1 for a missing diagonal or more than 2^31-1 entries. */
static int64_t iluk_pattern(int64_t n, const int32_t *rp, const int32_t *col, int p, int32_t *frp, int32_t *fcol,
                            int64_t cap) {
    /* next[]: sorted linked list of the current row's columns, head at index n, -1 ends it;
     * lev[j]: level of column j in the current row, INT32_MAX when absent.  Finished rows are
     * kept (columns and levels) in growing buffers. */
    int32_t *next = (int32_t *)malloc((size_t)(n + 1) * sizeof(int32_t));
    int32_t *lev = (int32_t *)malloc((size_t)n * sizeof(int32_t));
    int64_t *ufirst = (int64_t *)malloc((size_t)n * sizeof(int64_t));
    int64_t *start = (int64_t *)malloc((size_t)(n + 1) * sizeof(int64_t));
    int64_t bcap = (int64_t)rp[n] * 2 + 16, nnz = 0, result = 0;
    int32_t *bcol = (int32_t *)malloc((size_t)bcap * sizeof(int32_t));
    int32_t *blev = (int32_t *)malloc((size_t)bcap * sizeof(int32_t));
    const int32_t head = (int32_t)n;
    for (int64_t j = 0; j < n; ++j) lev[j] = INT32_MAX;
    start[0] = 0;
    for (int64_t i = 0; i < n; ++i) {
        next[head] = -1;
        int32_t tail = head, has_diag = 0;
        for (int32_t k = rp[i]; k < rp[i + 1]; ++k) {
            const int32_t c = col[k];
            next[tail] = c;
            next[c] = -1;
            tail = c;
            lev[c] = 0;
            if (c == i) has_diag = 1;
        }
        if (!has_diag) {
            result = -1;
            break;
        }
        /* eliminate with the finished rows k < i in increasing order; a column j > k that an
         * update creates is linked in behind k, so the walk also reaches new columns below i */
        for (int32_t k = next[head]; k >= 0 && k < i; k = next[k]) {
            const int32_t lk = lev[k];
            int32_t prev = k;
            for (int64_t q = ufirst[k]; q < start[k + 1]; ++q) {
                const int32_t j = bcol[q];
                const int32_t nl = lk + blev[q] + 1;
                if (lev[j] == INT32_MAX) {
                    if (nl > p) continue;
                    while (next[prev] >= 0 && next[prev] < j) prev = next[prev];
                    next[j] = next[prev];
                    next[prev] = j;
                    lev[j] = nl;
                } else if (nl < lev[j]) {
                    lev[j] = nl;
                }
                prev = j;
            }
        }
        int64_t cnt = 0;
        for (int32_t c = next[head]; c >= 0; c = next[c]) ++cnt;
        if (nnz + cnt > bcap) {
            bcap = (nnz + cnt) * 2;
            bcol = (int32_t *)realloc(bcol, (size_t)bcap * sizeof(int32_t));
            blev = (int32_t *)realloc(blev, (size_t)bcap * sizeof(int32_t));
        }
        ufirst[i] = -1;
        for (int32_t c = next[head]; c >= 0; c = next[c]) {
            if (c > i && ufirst[i] < 0) ufirst[i] = nnz;
            bcol[nnz] = c;
            blev[nnz] = lev[c];
            lev[c] = INT32_MAX;
            ++nnz;
        }
        if (ufirst[i] < 0) ufirst[i] = nnz;
        start[i + 1] = nnz;
        if (nnz > INT32_MAX) {
            result = -1;
            break;
        }
    }
    if (result == 0) {
        result = nnz;
        if (nnz <= cap && frp && fcol) {
            for (int64_t i = 0; i <= n; ++i) frp[i] = (int32_t)start[i];
            memcpy(fcol, bcol, (size_t)nnz * sizeof(int32_t));
        }
    }
    free(next); free(lev); free(ufirst); free(start); free(bcol); free(blev);
    return result;
}

/* ILU(p) of a CSR matrix (sorted rows with a diagonal entry): pattern and values of L (unit
 * lower, strictly below the diagonal) and U in one CSR (frp [n+1], fcol/fval [nnz]) with the
 * diagonal positions dpos [n].  Returns nnz when it fits cap (the arrays are filled), nnz
 * without filling anything when it does not, -1 for a missing diagonal, -2 for a zero pivot. */
int64_t orc_iluk(int64_t n, const int32_t *rp, const int32_t *col, const double *val, int p, int32_t *frp,
                 int32_t *fcol, double *fval, int32_t *dpos, int64_t cap) {
    int64_t nnz = iluk_pattern(n, rp, col, p, frp, fcol, cap);
    if (nnz < 0 || nnz > cap || !fval) return nnz;
    /* numeric IKJ elimination inside the pattern; mark[j] = position of column j in row i */
    int32_t *mark = (int32_t *)malloc((size_t)n * sizeof(int32_t));
    for (int64_t j = 0; j < n; ++j) mark[j] = -1;
    int64_t rc = nnz;
    for (int64_t i = 0; i < n && rc >= 0; ++i) {
        dpos[i] = -1;
        for (int32_t q = frp[i]; q < frp[i + 1]; ++q) {
            mark[fcol[q]] = q;
            fval[q] = 0.0;
            if (fcol[q] == i) dpos[i] = q;
        }
        for (int32_t k = rp[i]; k < rp[i + 1]; ++k) fval[mark[col[k]]] = val[k];
        for (int32_t q = frp[i]; q < dpos[i]; ++q) {
            const int32_t c = fcol[q];
            const double f = (fval[q] /= fval[dpos[c]]);
            for (int32_t t = dpos[c] + 1; t < frp[c + 1]; ++t) {
                const int32_t m = mark[fcol[t]];
                if (m >= 0) fval[m] -= f * fval[t];
            }
        }
        if (fval[dpos[i]] == 0.0) rc = -2;
        for (int32_t q = frp[i]; q < frp[i + 1]; ++q) mark[fcol[q]] = -1;
    }
    free(mark);
    return rc;
}

static void iluk_apply(int64_t n, const int32_t *frp, const int32_t *fcol, const double *fval, const int32_t *dpos,
                       const double *r, double *z) {
    for (int64_t i = 0; i < n; ++i) {
        double s = r[i];
        for (int32_t q = frp[i]; q < dpos[i]; ++q) s -= fval[q] * z[fcol[q]];
        z[i] = s;
    }
    for (int64_t i = n - 1; i >= 0; --i) {
        double s = z[i];
        for (int32_t q = dpos[i] + 1; q < frp[i + 1]; ++q) s -= fval[q] * z[fcol[q]];
        z[i] = s / fval[dpos[i]];
    }
}

static void iluk_mv(int64_t n, const int32_t *rp, const int32_t *col, const double *val, const double *x, double *y) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        double s = 0.0;
        for (int32_t k = rp[i]; k < rp[i + 1]; ++k) s += val[k] * x[col[k]];
        y[i] = s;
    }
}

/* CG preconditioned by ILU(p) on a CSR SPD matrix, FP64: SpMV and vector updates threaded
 * (OpenMP), the triangular solves sequential.  The stopping rule of orc_pcg_jacobi: the
 * recursively updated residual satisfies |D^-1/2 r| <= rtol |D^-1/2 b| and |r| <= rtol |b|.
 * Returns iterations, -1 if max_it was reached, -2 if the factorisation failed (or its memory
 * could not be allocated).  res_out gets
 * the true Jacobi-scaled relative residual, t_factor_out the factorisation's seconds (pattern
 * and values) and fill_out the factor's nonzeros divided by the matrix's. */
int orc_pcg_iluk(int64_t n, const int32_t *rp, const int32_t *col, const double *val, const double *b, double *x,
                 int p, double rtol, int max_it, double *res_out, double *t_factor_out, double *fill_out) {
    extern double omp_get_wtime(void);
    const double t0 = omp_get_wtime();
    /* a first guess of the fill (p + 2 times the matrix's entries, at most 8); a second pass
     * with the exact size when the factor is larger */
    int64_t cap = (int64_t)rp[n] * (p < 6 ? p + 2 : 8);
    int32_t *frp = (int32_t *)malloc((size_t)(n + 1) * sizeof(int32_t));
    int32_t *fcol = (int32_t *)malloc((size_t)cap * sizeof(int32_t));
    double *fval = (double *)malloc((size_t)cap * sizeof(double));
    int32_t *dpos = (int32_t *)malloc((size_t)n * sizeof(int32_t));
    int64_t nnz = frp && fcol && fval && dpos ? orc_iluk(n, rp, col, val, p, frp, fcol, fval, dpos, cap) : -3;
    if (nnz > cap) {
        cap = nnz;
        int32_t *c2 = (int32_t *)realloc(fcol, (size_t)cap * sizeof(int32_t));
        double *v2 = c2 ? (double *)realloc(fval, (size_t)cap * sizeof(double)) : NULL;
        if (c2) fcol = c2;
        if (v2) fval = v2;
        nnz = c2 && v2 ? orc_iluk(n, rp, col, val, p, frp, fcol, fval, dpos, cap) : -3;
    }
    if (nnz < 0) {
        free(frp); free(fcol); free(fval); free(dpos);
        return -2;
    }
    if (t_factor_out) *t_factor_out = omp_get_wtime() - t0;
    if (fill_out) *fill_out = (double)nnz / (double)rp[n];
    double *r = (double *)malloc(n * sizeof(double)), *z = (double *)malloc(n * sizeof(double));
    double *pp = (double *)malloc(n * sizeof(double)), *q = (double *)malloc(n * sizeof(double));
    double *dinv = (double *)malloc(n * sizeof(double));
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        double d = 1.0;
        for (int32_t k = rp[i]; k < rp[i + 1]; ++k)
            if (col[k] == i) d = val[k];
        dinv[i] = 1.0 / d;
    }
    iluk_mv(n, rp, col, val, x, q);
    double bb = 0.0, bdb = 0.0, rr = 0.0, rdr = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : bb, bdb, rr, rdr)
    for (int64_t i = 0; i < n; ++i) {
        r[i] = b[i] - q[i];
        bb += b[i] * b[i];
        bdb += b[i] * dinv[i] * b[i];
        rr += r[i] * r[i];
        rdr += r[i] * dinv[i] * r[i];
    }
    iluk_apply(n, frp, fcol, fval, dpos, r, z);
    double rz = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : rz)
    for (int64_t i = 0; i < n; ++i) {
        pp[i] = z[i];
        rz += r[i] * z[i];
    }
    const double tol2 = rtol * rtol * bb, tol2s = rtol * rtol * bdb;
    int it = 0;
    while ((rr > tol2 || rdr > tol2s) && it < max_it) {
        iluk_mv(n, rp, col, val, pp, q);
        double pq = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : pq)
        for (int64_t i = 0; i < n; ++i) pq += pp[i] * q[i];
        const double alpha = rz / pq;
        rr = 0.0;
        rdr = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : rr, rdr)
        for (int64_t i = 0; i < n; ++i) {
            x[i] += alpha * pp[i];
            r[i] -= alpha * q[i];
            rr += r[i] * r[i];
            rdr += r[i] * dinv[i] * r[i];
        }
        iluk_apply(n, frp, fcol, fval, dpos, r, z);
        double rz_new = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : rz_new)
        for (int64_t i = 0; i < n; ++i) rz_new += r[i] * z[i];
        const double beta = rz_new / rz;
        rz = rz_new;
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; ++i) pp[i] = z[i] + beta * pp[i];
        ++it;
    }
    iluk_mv(n, rp, col, val, x, q);
    double res = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : res)
    for (int64_t i = 0; i < n; ++i) res += (b[i] - q[i]) * dinv[i] * (b[i] - q[i]);
    if (res_out) *res_out = bdb > 0.0 ? sqrt(res / bdb) : 0.0;
    free(r); free(z); free(pp); free(q); free(dinv); free(frp); free(fcol); free(fval); free(dpos);
    return (rr > tol2 || rdr > tol2s) ? -1 : it;
}
