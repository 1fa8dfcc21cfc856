/*
 * Plain-C FP64 restatement of the AIR Tools II hot path (TEST ORACLE).
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA path and the timed CPU
 * baseline of bench.py; the product never links it.  Parity status vs MATLAB:
 * unpinned (no MATLAB/Octave here, no golden vectors in the reference); the
 * ray tracer below is cross-checked against the independent NumPy
 * restatement in oracle/airt_oracle.py.
 *
 * Build: gcc -O2 -fopenmp -ffp-contract=off -shared -fPIC (no FMA contraction,
 * so every multiply and add rounds separately, as in the MATLAB code).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct { double t; int idx; } tkey;

/* MATLAB sort(t): ascending, stable, NaN last (testprobs/paralleltomo.m:230). */
static int cmp_tkey(const void *pa, const void *pb) {
    const tkey *a = (const tkey *)pa, *b = (const tkey *)pb;
    int na = isnan(a->t), nb = isnan(b->t);
    if (na != nb) return na - nb;
    if (!na) {
        if (a->t < b->t) return -1;
        if (a->t > b->t) return 1;
    }
    return (a->idx > b->idx) - (a->idx < b->idx);
}

/* One ray of testprobs/paralleltomo.m:207-263 (fanlineartomo.m:271-318 with
 * exclude=0).  Writes 0-based column-major pixel indices and lengths;
 * returns the count.  Work buffers hold 2(N+1) entries. */
static int trace_one(int N, double x0t, double y0t, double a, double b, int exclude,
                     tkey *key, double *px, double *py, int64_t *cols, double *vals) {
    const int G = N + 1;
    const double h = N / 2.0;
    for (int i = 0; i < G; ++i) {
        double g = -h + (double)i;
        double tx = (g - x0t) / a;
        double ty = (g - y0t) / b;
        key[i].t = tx; key[i].idx = i;
        key[G + i].t = ty; key[G + i].idx = G + i;
    }
    qsort(key, 2 * G, sizeof(tkey), cmp_tkey);
    int np_ = 0;
    for (int s = 0; s < 2 * G; ++s) {
        int id = key[s].idx;
        double xx, yy;
        if (id < G) { xx = -h + (double)id; yy = b * key[s].t + y0t; }
        else { yy = -h + (double)(id - G); xx = a * key[s].t + x0t; }
        if (xx >= -h && xx <= h && yy >= -h && yy <= h) { px[np_] = xx; py[np_] = yy; ++np_; }
    }
    /* drop a point whose successor lies within 1e-10 in both coordinates */
    int nk = 0;
    for (int s = 0; s < np_; ++s) {
        if (s + 1 < np_ && fabs(px[s + 1] - px[s]) <= 1e-10 && fabs(py[s + 1] - py[s]) <= 1e-10)
            continue;
        px[nk] = px[s]; py[nk] = py[s]; ++nk;
    }
    if (nk < 2) return 0;
    if (exclude && ((b == 0 && fabs(y0t - h) < 1e-15) || (a == 0 && fabs(x0t - h) < 1e-15)))
        return 0;
    for (int s = 0; s + 1 < nk; ++s) {
        double dx = px[s + 1] - px[s], dy = py[s + 1] - py[s];
        vals[s] = sqrt(dx * dx + dy * dy);
        double xm = 0.5 * (px[s] + px[s + 1]) + h;
        double ym = 0.5 * (py[s] + py[s + 1]) + h;
        cols[s] = (int64_t)(floor(xm) * N + (N - floor(ym))) - 1;
    }
    return nk - 1;
}

/* Count pass: counts[r] = entries of ray r (before duplicate summing). */
int oracle_trace_count(int N, int64_t nrays, const double *x0t, const double *y0t,
                       const double *a, const double *b, int exclude, int64_t *counts) {
#pragma omp parallel
    {
        int G2 = 2 * (N + 1);
        tkey *key = malloc(sizeof(tkey) * G2);
        double *px = malloc(sizeof(double) * G2), *py = malloc(sizeof(double) * G2);
        int64_t *cols = malloc(sizeof(int64_t) * G2);
        double *vals = malloc(sizeof(double) * G2);
#pragma omp for schedule(dynamic, 64)
        for (int64_t r = 0; r < nrays; ++r)
            counts[r] = trace_one(N, x0t[r], y0t[r], a[r], b[r], exclude, key, px, py, cols, vals);
        free(key); free(px); free(py); free(cols); free(vals);
    }
    return 0;
}

/* Fill pass: ray r's entries at [offs[r], offs[r+1]). */
int oracle_trace_fill(int N, int64_t nrays, const double *x0t, const double *y0t,
                      const double *a, const double *b, int exclude, const int64_t *offs,
                      int64_t *cols_out, double *vals_out) {
#pragma omp parallel
    {
        int G2 = 2 * (N + 1);
        tkey *key = malloc(sizeof(tkey) * G2);
        double *px = malloc(sizeof(double) * G2), *py = malloc(sizeof(double) * G2);
#pragma omp for schedule(dynamic, 64)
        for (int64_t r = 0; r < nrays; ++r)
            trace_one(N, x0t[r], y0t[r], a[r], b[r], exclude, key, px, py,
                      cols_out + offs[r], vals_out + offs[r]);
        free(key); free(px); free(py);
    }
    return 0;
}

/* ------------------------------------------------------------------------
 * FP64 SIRT loop of sirt/sirt.m:198-261 with constant relaxpar, diagonal M
 * and D, box bounds (scalars; NaN = absent) and the DP rule
 * (auxil/check_stoprules.m:56-72; taudelta < 0 = rule NONE).  A is given as
 * CSR (forward) and CSC (transpose) in double.  Returns finaliter; writes the
 * final iterate to x and the residual norms to resn[0..finaliter].
 * ---------------------------------------------------------------------- */
int oracle_sirt_csr(int64_t m, int64_t n, const int64_t *rp, const int64_t *ci, const double *rv,
                    const int64_t *cp, const int64_t *ri, const double *cv,
                    const double *b, const double *M, const double *D, double lambda,
                    double lb, double ub, double taudelta, int kmax, double *x, double *resn) {
    double *r = malloc(sizeof(double) * m), *Mr = malloc(sizeof(double) * m);
    double nrm2 = 0.0;
#pragma omp parallel for reduction(+ : nrm2) schedule(static)
    for (int64_t i = 0; i < m; ++i) {
        double s = 0.0;
        for (int64_t q = rp[i]; q < rp[i + 1]; ++q) s += rv[q] * x[ci[q]];
        r[i] = b[i] - s;
        nrm2 += r[i] * r[i];
    }
    resn[0] = sqrt(nrm2);
    int k = 0;
    if (taudelta >= 0 && resn[0] <= taudelta) { free(r); free(Mr); return 0; }
    while (k < kmax) {
        ++k;
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < m; ++i) Mr[i] = M[i] * r[i];
#pragma omp parallel for schedule(static)
        for (int64_t j = 0; j < n; ++j) {
            double g = 0.0;
            for (int64_t q = cp[j]; q < cp[j + 1]; ++q) g += cv[q] * Mr[ri[q]];
            double xj = x[j] + lambda * (D[j] * g);
            if (!isnan(lb)) xj = xj < lb ? lb : xj;
            if (!isnan(ub)) xj = xj > ub ? ub : xj;
            x[j] = xj;
        }
        nrm2 = 0.0;
#pragma omp parallel for reduction(+ : nrm2) schedule(static)
        for (int64_t i = 0; i < m; ++i) {
            double s = 0.0;
            for (int64_t q = rp[i]; q < rp[i + 1]; ++q) s += rv[q] * x[ci[q]];
            r[i] = b[i] - s;
            nrm2 += r[i] * r[i];
        }
        resn[k] = sqrt(nrm2);
        if (taudelta >= 0 && resn[k] <= taudelta) break;
    }
    free(r); free(Mr);
    return k;
}

/* ------------------------------------------------------------------------
 * FP64 Kaczmarz sweeps of art/art.m:227-309 in a fixed row order (0-based
 * rows[], nrows per sweep), constant relaxpar, damped squared row norms
 * nrm[], scalar bounds (NaN = absent).  art.m:279-284 clamps the whole x
 * after every row; once x is feasible (after the first row step) only the
 * row's support can leave the box, so the whole-vector clamp is done once,
 * after the first step, and the support afterwards -- the same iterates.
 * Runs `sweeps` sweeps; x is updated in place.
 * ---------------------------------------------------------------------- */
int oracle_kaczmarz(int64_t m, int64_t n, const int64_t *rp, const int64_t *ci, const double *rv,
                    const double *b, const double *nrm, const int64_t *rows, int64_t nrows,
                    double lambda, double lb, double ub, int sweeps, double *x) {
    (void)m;
    int bounded = !isnan(lb) || !isnan(ub);
    int first = 1;
    for (int k = 0; k < sweeps; ++k) {
        for (int64_t t = 0; t < nrows; ++t) {
            int64_t i = rows[t];
            double s = 0.0;
            for (int64_t q = rp[i]; q < rp[i + 1]; ++q) s += rv[q] * x[ci[q]];
            double c = lambda * (b[i] - s) / nrm[i];
            for (int64_t q = rp[i]; q < rp[i + 1]; ++q) x[ci[q]] = x[ci[q]] + c * rv[q];
            if (!bounded) continue;
            if (first) {
                for (int64_t j = 0; j < n; ++j) {
                    double v = x[j];
                    if (!isnan(lb)) v = v < lb ? lb : v;
                    if (!isnan(ub)) v = v > ub ? ub : v;
                    x[j] = v;
                }
                first = 0;
            } else {
                for (int64_t q = rp[i]; q < rp[i + 1]; ++q) {
                    double v = x[ci[q]];
                    if (!isnan(lb)) v = v < lb ? lb : v;
                    if (!isnan(ub)) v = v > ub ? ub : v;
                    x[ci[q]] = v;
                }
            }
        }
    }
    return 0;
}

int oracle_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
