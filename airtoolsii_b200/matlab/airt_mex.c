/*
 * airt_mex.c -- MATLAB / GNU Octave MEX gateway to libairt (include/airt.h).
 *
 * One MEX function, dispatched on a command string, carries every entry
 * point of the C-ABI to the toolbox's host code; the .m shims beside this
 * file keep the AIR Tools II signatures (sirt.m, art.m, cart.m,
 * paralleltomo.m, fanlineartomo.m, fbp.m) and call it.
 *
 * Build (MATLAB R2018a or later, interleaved complex API):
 *   mex -R2018a -I<repo>/include airt_mex.c -L<repo>/airtoolsii_b200 -lairt
 * with gpuArray commands (batch_backproject, unet_forward; Parallel
 * Computing Toolbox):
 *   mex -R2018a -DAIRT_MEX_GPUARRAY -I<repo>/include airt_mex.c \
 *       -L<repo>/airtoolsii_b200 -lairt -lmwgpu
 * GNU Octave 7 or later:  mkoctfile --mex -I<repo>/include airt_mex.c -L... -lairt
 *
 * Handles (problem, batch, network) travel to MATLAB as uint64 scalars.
 * Every non-zero status becomes mexErrMsgIdAndTxt("AIRT:<code>", message)
 * with the library's airt_last_error() text.
 *
 * Commands (outputs = airt_mex(cmd, inputs...)):
 *   v            = airt_mex('version')
 *   h            = airt_mex('matrix', A)                       sparse double m x n
 *   h            = airt_mex('parallel', N, cosd(th), sind(th), offsets, isMF)
 *   h            = airt_mex('fan', N, cosd(th), sind(th), cosd(om), sind(om), R, isMF)
 *   h            = airt_mex('seismic', N, x0, y0, xp, yp, isMF)
 *   h            = airt_mex('spherical', N, cosd(ang), sind(ang), radii, int64(nPhi), ck, sk, isMF)
 *   mn           = airt_mex('size', h)                         [m n]
 *   A            = airt_mex('export', h)                       the stored matrix, sparse
 *   y            = airt_mex('apply', h, v, transp)             A*v or A'*v
 *   [M, D]       = airt_mex('weights', h, method)              get_mfun_dfun.m diagonals
 *   rho          = airt_mex('rho', h, opts)                    calc_relaxpar.m:91-103
 *   [X, info]    = airt_mex('sirt', h, opts, b, x0, K)         sirt.m:198-261
 *   [X, info]    = airt_mex('art', h, opts, b, x0, K)          art.m:227-309
 *   [X, info]    = airt_mex('cart', h, opts, b, x0, K)         cart.m:211-309
 *   x            = airt_mex('fbp', h, b, na, kernel)           fbp.m:74-79
 *                  airt_mex('destroy', h)
 *   bh           = airt_mex('batch', int32(N), int32(nA), int32(p), cos_t, sin_t, offsets)
 *   [ro, co, nz] = airt_mex('batch_layout', bh, ninst)
 *   rho          = airt_mex('batch_rho', bh, ninst, method)
 *   [x, it, sr, ms] = airt_mex('batch_sirt', bh, ninst, opts, b, x0)    per-instance rule
 *   [x, ms]      = airt_mex('batch_kaczmarz', bh, ninst, b, sweeps, relaxpar, lbound, ubound)
 *   x            = airt_mex('batch_backproject', bh, ninst, method, b)   b, x: gpuArray
 *   [X, it, sr]  = airt_mex('sirt_multi', h, opts, B, X0, taudelta)     B, X0, X: gpuArray
 *                  airt_mex('batch_destroy', bh)
 *   uh           = airt_mex('unet', H, W, base, levels, max_batch, seed)
 *   w            = airt_mex('unet_params', uh)                 single vector
 *                  airt_mex('unet_set_params', uh, w)
 *   y            = airt_mex('unet_forward', uh, x, B)          x, y: gpuArray double
 *                  airt_mex('unet_destroy', uh)
 *
 * Method codes in opts.method and the method arguments: 0 landweber,
 * 1 cimmino, 2 cav, 3 drop, 4 sart, 5 custom (opts.M, opts.D: diagonal
 * vectors, or full matrices -- the Mflag/Dflag = 2 case).  Stopping rules
 * in opts.stoprule: 0 NONE, 1 DP, 2 ME, 3 NCP.  Bounds in opts.lbound /
 * opts.ubound: empty (none), a scalar, or an n-vector.  Row, column and
 * iteration lists are 1-based doubles as MATLAB has them.
 */
#include <stdint.h>
#include <string.h>

#include "mex.h"
#ifdef AIRT_MEX_GPUARRAY
#include "gpu/mxGPUArray.h"
#endif

#include "airt.h"

/* ------------------------------------------------------------------ helpers */
static void chk(int st) {
    if (st != AIRT_OK) {
        static const char *ids[] = {"AIRT:ok", "AIRT:arg", "AIRT:oom", "AIRT:cuda", "AIRT:timeout",
                                    "AIRT:unsupported"};
        const char *id = (st >= 0 && st <= AIRT_ERR_UNSUPPORTED) ? ids[st] : "AIRT:status";
        mexErrMsgIdAndTxt(id, "%s", airt_last_error());
    }
}

static void need(int cond, const char *msg) {
    if (!cond) mexErrMsgIdAndTxt("AIRT:usage", "%s", msg);
}

static mxArray *handle_out(const void *p) {
    mxArray *a = mxCreateNumericMatrix(1, 1, mxUINT64_CLASS, mxREAL);
    *(uint64_t *)mxGetData(a) = (uint64_t)(uintptr_t)p;
    return a;
}

static void *handle_in(const mxArray *a) {
    need(a && mxIsUint64(a) && mxGetNumberOfElements(a) == 1, "expected a uint64 handle");
    return (void *)(uintptr_t)(*(const uint64_t *)mxGetData(a));
}

static const double *dvec(const mxArray *a, int64_t *count) {
    need(a && mxIsDouble(a) && !mxIsComplex(a) && !mxIsSparse(a), "expected a real double array");
    if (count) *count = (int64_t)mxGetNumberOfElements(a);
    return mxGetDoubles(a);
}

static double scalar(const mxArray *a) {
    need(a && mxIsNumeric(a) && mxGetNumberOfElements(a) == 1, "expected a numeric scalar");
    return mxGetScalar(a);
}

static const mxArray *field(const mxArray *s, const char *name) {
    if (!s || !mxIsStruct(s)) return NULL;
    const mxArray *f = mxGetField(s, 0, name);
    return (f && !mxIsEmpty(f)) ? f : NULL;
}

static double dfield(const mxArray *s, const char *name, double dflt) {
    const mxArray *f = field(s, name);
    return f ? scalar(f) : dflt;
}

static const double *vfield(const mxArray *s, const char *name, int64_t *count) {
    const mxArray *f = field(s, name);
    if (!f) {
        if (count) *count = 0;
        return NULL;
    }
    return dvec(f, count);
}

/* lbound / ubound: absent or empty -> none, 1 element -> scalar, n -> vector */
static void bound(const mxArray *s, const char *name, int64_t n, int *kind, double *val,
                  const double **vec) {
    int64_t c = 0;
    const double *v = vfield(s, name, &c);
    *val = 0.0;
    *vec = NULL;
    if (!v) {
        *kind = AIRT_BOUND_NONE;
    } else if (c == 1) {
        *kind = AIRT_BOUND_SCALAR;
        *val = v[0];
    } else {
        need(c == n, "a bound must be a scalar or have one entry per unknown");
        *kind = AIRT_BOUND_VECTOR;
        *vec = v;
    }
}

/* 1-based double index list -> 0-based int64 (mxMalloc'd) */
static int64_t *index_list(const mxArray *a, int64_t *count) {
    int64_t c = 0;
    const double *v = dvec(a, &c);
    int64_t *out = (int64_t *)mxMalloc((size_t)(c > 0 ? c : 1) * sizeof(int64_t));
    for (int64_t i = 0; i < c; ++i) out[i] = (int64_t)v[i] - 1;
    *count = c;
    return out;
}

/* iteration list K (1-based iteration numbers, kept as numbers) */
static int64_t *iter_list(const mxArray *a, int64_t *count) {
    int64_t c = 0;
    const double *v = dvec(a, &c);
    need(c >= 1, "Max no. of iterations must ALWAYS be specified.");
    int64_t *out = (int64_t *)mxMalloc((size_t)c * sizeof(int64_t));
    for (int64_t i = 0; i < c; ++i) out[i] = (int64_t)v[i];
    *count = c;
    return out;
}

static void problem_size(airt_problem *h, int64_t *m, int64_t *n) {
    int64_t nnz = 0;
    chk(airt_problem_size(h, m, n, &nnz));
}

/* NCP fields shared by the three solvers: res_dims ([rows cols] or [rows]) and ncp_smooth */
static void ncp_fields(const mxArray *o, int *rows, int *cols, int *smooth) {
    int64_t c = 0;
    const double *rd = vfield(o, "res_dims", &c);
    *rows = c >= 1 ? (int)rd[0] : 0;
    *cols = c >= 2 ? (int)rd[1] : 1;
    *smooth = (int)dfield(o, "ncp_smooth", 2);
}

static mxArray *info_struct(const airt_info *info, const double *resn) {
    static const char *names[] = {"stoprule", "finaliter", "relaxpar", "nsaved", "gpu_ms",
                                  "resnorms"};
    mxArray *s = mxCreateStructMatrix(1, 1, 6, names);
    mxSetField(s, 0, "stoprule", mxCreateDoubleScalar((double)info->stoprule));
    mxSetField(s, 0, "finaliter", mxCreateDoubleScalar((double)info->finaliter));
    mxSetField(s, 0, "relaxpar", mxCreateDoubleScalar(info->relaxpar));
    mxSetField(s, 0, "nsaved", mxCreateDoubleScalar((double)info->nsaved));
    mxSetField(s, 0, "gpu_ms", mxCreateDoubleScalar(info->gpu_ms));
    mxArray *r = mxCreateDoubleMatrix((mwSize)(info->finaliter + 1), 1, mxREAL);
    memcpy(mxGetDoubles(r), resn, (size_t)(info->finaliter + 1) * sizeof(double));
    mxSetField(s, 0, "resnorms", r);
    return s;
}

/* X is allocated n x nK and trimmed to the saved columns (sirt.m:270) */
static void trim_columns(mxArray *X, int64_t nsaved) { mxSetN(X, (mwSize)nsaved); }

/* ------------------------------------------------------------------ commands */
static void cmd_matrix(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
    need(nrhs == 2 && mxIsSparse(prhs[1]) && mxIsDouble(prhs[1]) && !mxIsComplex(prhs[1]),
         "airt_mex('matrix', A): A must be a real sparse double matrix");
    const mxArray *A = prhs[1];
    airt_problem *h = NULL;
    chk(airt_problem_from_csc((int64_t)mxGetM(A), (int64_t)mxGetN(A),
                              (const uint64_t *)mxGetJc(A), (const uint64_t *)mxGetIr(A),
                              mxGetDoubles(A), &h));
    plhs[0] = handle_out(h);
    (void)nlhs;
}

static void cmd_parallel(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
    need(nrhs == 6, "airt_mex('parallel', N, cos_t, sin_t, offsets, isMF)");
    int64_t nA = 0, nA2 = 0, p = 0;
    const double *ct = dvec(prhs[2], &nA), *st = dvec(prhs[3], &nA2), *off = dvec(prhs[4], &p);
    need(nA == nA2, "cos_t and sin_t differ in length");
    airt_problem *h = NULL;
    chk(airt_problem_parallel((int)scalar(prhs[1]), (int)nA, ct, st, (int)p, off,
                              scalar(prhs[5]) != 0, &h));
    plhs[0] = handle_out(h);
    (void)nlhs;
}

static void cmd_fan(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
    need(nrhs == 8, "airt_mex('fan', N, cos_t, sin_t, cos_w, sin_w, R, isMF)");
    int64_t nA = 0, nA2 = 0, p = 0, p2 = 0;
    const double *ct = dvec(prhs[2], &nA), *st = dvec(prhs[3], &nA2);
    const double *cw = dvec(prhs[4], &p), *sw = dvec(prhs[5], &p2);
    need(nA == nA2 && p == p2, "angle tables differ in length");
    airt_problem *h = NULL;
    chk(airt_problem_fan((int)scalar(prhs[1]), (int)nA, ct, st, (int)p, cw, sw, scalar(prhs[6]),
                         scalar(prhs[7]) != 0, &h));
    plhs[0] = handle_out(h);
    (void)nlhs;
}

static void cmd_seismic(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
    need(nrhs == 7, "airt_mex('seismic', N, x0, y0, xp, yp, isMF)");
    int64_t s = 0, s2 = 0, p = 0, p2 = 0;
    const double *sx = dvec(prhs[2], &s), *sy = dvec(prhs[3], &s2);
    const double *rx = dvec(prhs[4], &p), *ry = dvec(prhs[5], &p2);
    need(s == s2 && p == p2, "source or receiver tables differ in length");
    airt_problem *h = NULL;
    chk(airt_problem_seismic((int)scalar(prhs[1]), (int)s, sx, sy, (int)p, rx, ry,
                             scalar(prhs[6]) != 0, &h));
    plhs[0] = handle_out(h);
    (void)nlhs;
}

static void cmd_spherical(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
    need(nrhs == 9, "airt_mex('spherical', N, cos_t, sin_t, radii, int64(nPhi), ck, sk, isMF)");
    int64_t nA = 0, nA2 = 0, nc = 0, nk = 0, nk2 = 0;
    const double *ct = dvec(prhs[2], &nA), *st = dvec(prhs[3], &nA2), *rad = dvec(prhs[4], &nc);
    need(mxIsInt64(prhs[5]) && (int64_t)mxGetNumberOfElements(prhs[5]) == nc,
         "nPhi must be an int64 vector with one entry per circle");
    const double *ck = dvec(prhs[6], &nk), *sk = dvec(prhs[7], &nk2);
    need(nA == nA2 && nk == nk2, "angle tables differ in length");
    airt_problem *h = NULL;
    chk(airt_problem_spherical((int)scalar(prhs[1]), (int)nA, ct, st, (int)nc, rad,
                               (const int64_t *)mxGetInt64s(prhs[5]), ck, sk,
                               scalar(prhs[8]) != 0, &h));
    plhs[0] = handle_out(h);
    (void)nlhs;
}

static void cmd_size(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
    need(nrhs == 2, "airt_mex('size', h)");
    int64_t m = 0, n = 0;
    problem_size((airt_problem *)handle_in(prhs[1]), &m, &n);
    plhs[0] = mxCreateDoubleMatrix(1, 2, mxREAL);
    mxGetDoubles(plhs[0])[0] = (double)m;
    mxGetDoubles(plhs[0])[1] = (double)n;
    (void)nlhs;
}

static void cmd_export(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
    need(nrhs == 2, "airt_mex('export', h)");
    airt_problem *h = (airt_problem *)handle_in(prhs[1]);
    int64_t m = 0, n = 0, nnz = 0;
    chk(airt_problem_size(h, &m, &n, &nnz));
    plhs[0] = mxCreateSparse((mwSize)m, (mwSize)n, (mwSize)(nnz > 0 ? nnz : 1), mxREAL);
    chk(airt_problem_export_csc(h, (uint64_t *)mxGetJc(plhs[0]), (uint64_t *)mxGetIr(plhs[0]),
                                mxGetDoubles(plhs[0])));
    (void)nlhs;
}

static void cmd_apply(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
    need(nrhs == 4, "airt_mex('apply', h, v, transp)");
    airt_problem *h = (airt_problem *)handle_in(prhs[1]);
    const int tr = scalar(prhs[3]) != 0;
    int64_t m = 0, n = 0, c = 0;
    problem_size(h, &m, &n);
    const double *v = dvec(prhs[2], &c);
    need(c == (tr ? m : n), "the vector length does not match the operator");
    plhs[0] = mxCreateDoubleMatrix((mwSize)(tr ? n : m), 1, mxREAL);
    chk(airt_apply(h, v, mxGetDoubles(plhs[0]), tr));
    (void)nlhs;
}

static void cmd_weights(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
    need(nrhs == 3, "airt_mex('weights', h, method)");
    airt_problem *h = (airt_problem *)handle_in(prhs[1]);
    int64_t m = 0, n = 0;
    problem_size(h, &m, &n);
    plhs[0] = mxCreateDoubleMatrix((mwSize)m, 1, mxREAL);
    mxArray *D = mxCreateDoubleMatrix((mwSize)n, 1, mxREAL);
    chk(airt_weights(h, (int)scalar(prhs[2]), mxGetDoubles(plhs[0]), mxGetDoubles(D)));
    if (nlhs > 1) plhs[1] = D;
    else mxDestroyArray(D);
}

/* opts.M / opts.D of a custom method: vector (diagonal) or full square matrix */
static const double *custom_weight(const mxArray *o, const char *name, int64_t len, int *full) {
    const mxArray *f = field(o, name);
    *full = 0;
    if (!f) return NULL;
    need(mxIsDouble(f) && !mxIsSparse(f) && !mxIsComplex(f),
         "custom M and D must be full real double arrays (vectors or matrices)");
    const int64_t r = (int64_t)mxGetM(f), c = (int64_t)mxGetN(f);
    if (r == 1 || c == 1) {
        need(r * c == len, "custom weight vector has the wrong length");
    } else {
        need(r == len && c == len, "custom weight matrix has the wrong size");
        *full = 1;
    }
    return mxGetDoubles(f);
}

static void cmd_rho(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
    need(nrhs == 3 && mxIsStruct(prhs[2]), "airt_mex('rho', h, opts)");
    airt_problem *h = (airt_problem *)handle_in(prhs[1]);
    const mxArray *o = prhs[2];
    int64_t m = 0, n = 0;
    problem_size(h, &m, &n);
    const int method = (int)dfield(o, "method", AIRT_SART);
    const double tol = dfield(o, "tol", 1e-7);
    const int maxit = (int)dfield(o, "maxit", 200);
    double rho = 0.0;
    if (method == AIRT_CUSTOM) {
        int mf = 0, df = 0;
        const double *M = custom_weight(o, "M", m, &mf), *D = custom_weight(o, "D", n, &df);
        if (mf || df) chk(airt_rho_custom(h, M, mf, D, df, tol, maxit > 1000 ? maxit : 1000, &rho));
        else chk(airt_rho(h, method, M, D, tol, maxit, &rho));
    } else {
        chk(airt_rho(h, method, NULL, NULL, tol, maxit, &rho));
    }
    plhs[0] = mxCreateDoubleScalar(rho);
    (void)nlhs;
}

static void cmd_sirt(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
    need(nrhs == 6 && mxIsStruct(prhs[2]), "airt_mex('sirt', h, opts, b, x0, K)");
    airt_problem *h = (airt_problem *)handle_in(prhs[1]);
    const mxArray *o = prhs[2];
    int64_t m = 0, n = 0, nb = 0, nx = 0, nK = 0, ntab = 0;
    problem_size(h, &m, &n);
    const double *b = dvec(prhs[3], &nb);
    need(nb == m, "The size of A and b do not match.");
    const double *x0 = mxIsEmpty(prhs[4]) ? NULL : dvec(prhs[4], &nx);
    need(!x0 || nx == n, "The size of x0 does not match the problem.");
    int64_t *K = iter_list(prhs[5], &nK);

    airt_sirt_opts so;
    memset(&so, 0, sizeof so);
    so.method = (int)dfield(o, "method", AIRT_SART);
    if (so.method == AIRT_CUSTOM) {
        so.M = custom_weight(o, "M", m, &so.M_full);
        so.D = custom_weight(o, "D", n, &so.D_full);
    }
    so.relax_kind = (int)dfield(o, "relax_kind", AIRT_RELAX_CONST);
    so.relaxpar = dfield(o, "relaxpar", 1.0);
    so.relax_table = vfield(o, "relax_table", &ntab);
    need(so.relax_kind != AIRT_RELAX_TABLE || ntab >= K[nK - 1], "relax_table needs kmax entries");
    so.stoprule = (int)dfield(o, "stoprule", AIRT_STOP_NONE);
    so.taudelta = dfield(o, "taudelta", 0.0);
    bound(o, "lbound", n, &so.lb_kind, &so.lb, &so.lbv);
    bound(o, "ubound", n, &so.ub_kind, &so.ub, &so.ubv);
    so.kmax = K[nK - 1];
    ncp_fields(o, &so.ncp_rows, &so.ncp_cols, &so.ncp_smooth);

    airt_info info;
    double *resn = (double *)mxMalloc((size_t)(so.kmax + 1) * sizeof(double));
    plhs[0] = mxCreateDoubleMatrix((mwSize)n, (mwSize)nK, mxREAL);
    chk(airt_sirt(h, &so, b, x0, K, nK, mxGetDoubles(plhs[0]), resn, &info));
    trim_columns(plhs[0], info.nsaved);
    if (nlhs > 1) plhs[1] = info_struct(&info, resn);
    mxFree(resn);
    mxFree(K);
}

static void cmd_art(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
    need(nrhs == 6 && mxIsStruct(prhs[2]), "airt_mex('art', h, opts, b, x0, K)");
    airt_problem *h = (airt_problem *)handle_in(prhs[1]);
    const mxArray *o = prhs[2];
    int64_t m = 0, n = 0, nb = 0, nx = 0, nK = 0, ntab = 0;
    problem_size(h, &m, &n);
    const double *b = dvec(prhs[3], &nb);
    need(nb == m, "The size of A and b do not match.");
    const double *x0 = mxIsEmpty(prhs[4]) ? NULL : dvec(prhs[4], &nx);
    need(!x0 || nx == n, "The size of x0 does not match the problem.");
    int64_t *K = iter_list(prhs[5], &nK);

    airt_art_opts ao;
    memset(&ao, 0, sizeof ao);
    ao.order_kind = (int)dfield(o, "order_kind", 0);
    int64_t *rows = NULL;
    if (ao.order_kind == 2) {
        const mxArray *r = field(o, "rows");
        need(r != NULL, "opts.rows is required for a caller row order");
        rows = index_list(r, &ao.nrows);
        ao.rows_stride = (int64_t)dfield(o, "rows_stride", 0);
        if (ao.rows_stride > 0) ao.nrows = ao.rows_stride;
        ao.rows = rows;
    }
    ao.relaxpar = dfield(o, "relaxpar", 1.0);
    ao.relax_table = vfield(o, "relax_table", &ntab);
    ao.damp = dfield(o, "damp", 0.0);
    ao.stoprule = (int)dfield(o, "stoprule", AIRT_STOP_NONE);
    ao.taudelta = dfield(o, "taudelta", 0.0);
    bound(o, "lbound", n, &ao.lb_kind, &ao.lb, &ao.lbv);
    bound(o, "ubound", n, &ao.ub_kind, &ao.ub, &ao.ubv);
    ao.kmax = K[nK - 1];
    ncp_fields(o, &ao.ncp_rows, &ao.ncp_cols, &ao.ncp_smooth);

    airt_info info;
    double *resn = (double *)mxMalloc((size_t)(ao.kmax + 1) * sizeof(double));
    plhs[0] = mxCreateDoubleMatrix((mwSize)n, (mwSize)nK, mxREAL);
    chk(airt_art(h, &ao, b, x0, K, nK, mxGetDoubles(plhs[0]), resn, &info));
    trim_columns(plhs[0], info.nsaved);
    if (nlhs > 1) plhs[1] = info_struct(&info, resn);
    mxFree(resn);
    if (rows) mxFree(rows);
    mxFree(K);
}

static void cmd_cart(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
    need(nrhs == 6 && mxIsStruct(prhs[2]), "airt_mex('cart', h, opts, b, x0, K)");
    airt_problem *h = (airt_problem *)handle_in(prhs[1]);
    const mxArray *o = prhs[2];
    int64_t m = 0, n = 0, nb = 0, nx = 0, nK = 0;
    problem_size(h, &m, &n);
    const double *b = dvec(prhs[3], &nb);
    need(nb == m, "The size of A and b do not match.");
    const double *x0 = mxIsEmpty(prhs[4]) ? NULL : dvec(prhs[4], &nx);
    need(!x0 || nx == n, "The size of x0 does not match the problem.");
    int64_t *K = iter_list(prhs[5], &nK);

    airt_cart_opts co;
    memset(&co, 0, sizeof co);
    co.order_kind = (int)dfield(o, "order_kind", 0);
    int64_t *cols = NULL;
    if (co.order_kind == 2) {
        const mxArray *c = field(o, "cols");
        need(c != NULL, "opts.cols is required for a caller column order");
        cols = index_list(c, &co.ncols);
        co.cols = cols;
    }
    co.relaxpar = dfield(o, "relaxpar", 0.25);
    co.damp = dfield(o, "damp", 0.0);
    co.stoprule = (int)dfield(o, "stoprule", AIRT_STOP_NONE);
    co.taudelta = dfield(o, "taudelta", 0.0);
    bound(o, "lbound", n, &co.lb_kind, &co.lb, &co.lbv);
    bound(o, "ubound", n, &co.ub_kind, &co.ub, &co.ubv);
    co.kmax = K[nK - 1];
    ncp_fields(o, &co.ncp_rows, &co.ncp_cols, &co.ncp_smooth);
    co.thr = dfield(o, "THR", 1e-4);
    co.kbegin = (int64_t)dfield(o, "Kbegin", 10);
    co.nunflag = (int64_t)dfield(o, "Nunflag", (double)((co.kmax + 2) / 4));  /* round(kmax/4) */
    co.seed = (uint64_t)dfield(o, "seed", 0);

    airt_info info;
    double *resn = (double *)mxMalloc((size_t)(co.kmax + 1) * sizeof(double));
    plhs[0] = mxCreateDoubleMatrix((mwSize)n, (mwSize)nK, mxREAL);
    chk(airt_cart(h, &co, b, x0, K, nK, mxGetDoubles(plhs[0]), resn, &info));
    trim_columns(plhs[0], info.nsaved);
    if (nlhs > 1) plhs[1] = info_struct(&info, resn);
    mxFree(resn);
    if (cols) mxFree(cols);
    mxFree(K);
}

static void cmd_fbp(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
    need(nrhs == 5, "airt_mex('fbp', h, b, na, kernel)");
    airt_problem *h = (airt_problem *)handle_in(prhs[1]);
    int64_t m = 0, n = 0, nb = 0, order = 0;
    problem_size(h, &m, &n);
    const double *b = dvec(prhs[2], &nb);
    need(nb == m, "The size of A and b do not match.");
    const double *kern = dvec(prhs[4], &order);
    plhs[0] = mxCreateDoubleMatrix((mwSize)n, 1, mxREAL);
    chk(airt_fbp(h, b, (int)scalar(prhs[3]), kern, (int)order, mxGetDoubles(plhs[0])));
    (void)nlhs;
}

static void cmd_destroy(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
    need(nrhs == 2, "airt_mex('destroy', h)");
    chk(airt_destroy((airt_problem *)handle_in(prhs[1])));
    (void)nlhs;
    (void)plhs;
}

/* ---- batches: a batch travels as its handle plus its instance count */
static const int *ivec(const mxArray *a, int64_t *count) {
    need(a && mxIsInt32(a), "expected an int32 array");
    *count = (int64_t)mxGetNumberOfElements(a);
    return (const int *)mxGetInt32s(a);
}

/* rows m and columns n of the whole block-diagonal batch of k instances */
static void batch_dims(airt_batch *bh, int64_t k, int64_t *m, int64_t *n) {
    need(k >= 1, "the instance count must be positive");
    int64_t *ro = (int64_t *)mxMalloc((size_t)(k + 1) * sizeof(int64_t));
    int64_t *co = (int64_t *)mxMalloc((size_t)(k + 1) * sizeof(int64_t));
    chk(airt_batch_layout(bh, ro, co, NULL));
    *m = ro[k];
    *n = co[k];
    mxFree(ro);
    mxFree(co);
}

static void cmd_batch(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
    need(nrhs == 7, "airt_mex('batch', int32(N), int32(nA), int32(p), cos_t, sin_t, offsets)");
    int64_t k = 0, k2 = 0, k3 = 0, nc = 0, ns = 0, no = 0;
    const int *N = ivec(prhs[1], &k), *nA = ivec(prhs[2], &k2), *p = ivec(prhs[3], &k3);
    need(k == k2 && k == k3 && k >= 1, "one N, nA and p per instance");
    int64_t sa = 0, sp = 0;
    for (int64_t i = 0; i < k; ++i) {
        sa += nA[i];
        sp += p[i];
    }
    const double *ct = dvec(prhs[4], &nc), *st = dvec(prhs[5], &ns), *off = dvec(prhs[6], &no);
    need(nc == sa && ns == sa && no == sp, "angle and offset tables must concatenate the instances'");
    airt_batch *bh = NULL;
    chk(airt_batch_parallel((int)k, N, nA, p, ct, st, off, &bh));
    plhs[0] = handle_out(bh);
    (void)nlhs;
}

static void cmd_batch_layout(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
    need(nrhs == 3, "airt_mex('batch_layout', bh, ninst)");
    airt_batch *bh = (airt_batch *)handle_in(prhs[1]);
    const int64_t k = (int64_t)scalar(prhs[2]);
    need(k >= 1, "the instance count must be positive");
    mxArray *ro = mxCreateNumericMatrix((mwSize)(k + 1), 1, mxINT64_CLASS, mxREAL);
    mxArray *co = mxCreateNumericMatrix((mwSize)(k + 1), 1, mxINT64_CLASS, mxREAL);
    int64_t nnz = 0;
    chk(airt_batch_layout(bh, (int64_t *)mxGetInt64s(ro), (int64_t *)mxGetInt64s(co), &nnz));
    plhs[0] = ro;
    if (nlhs > 1) plhs[1] = co;
    else mxDestroyArray(co);
    if (nlhs > 2) plhs[2] = mxCreateDoubleScalar((double)nnz);
}

static void cmd_batch_rho(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
    need(nrhs == 4, "airt_mex('batch_rho', bh, ninst, method)");
    airt_batch *bh = (airt_batch *)handle_in(prhs[1]);
    const int64_t k = (int64_t)scalar(prhs[2]);
    need(k >= 1, "the instance count must be positive");
    plhs[0] = mxCreateDoubleMatrix((mwSize)k, 1, mxREAL);
    chk(airt_batch_rho(bh, (int)scalar(prhs[3]), 1e-7, 200, mxGetDoubles(plhs[0])));
    (void)nlhs;
}

static void cmd_batch_sirt(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
    need(nrhs == 6 && mxIsStruct(prhs[3]), "airt_mex('batch_sirt', bh, ninst, opts, b, x0)");
    airt_batch *bh = (airt_batch *)handle_in(prhs[1]);
    const int64_t k = (int64_t)scalar(prhs[2]);
    const mxArray *o = prhs[3];
    int64_t m = 0, n = 0, nl = 0, ntd = 0, nb = 0, nx = 0;
    batch_dims(bh, k, &m, &n);
    const double *lam = vfield(o, "relaxpar", &nl);
    need(lam && nl == k, "opts.relaxpar: one relaxation parameter per instance");
    const double *td = vfield(o, "taudelta", &ntd);
    need(!td || ntd == k, "opts.taudelta: one threshold per instance");
    const double *b = dvec(prhs[4], &nb);
    need(nb == m, "b must concatenate the instances' right-hand sides");
    const double *x0 = mxIsEmpty(prhs[5]) ? NULL : dvec(prhs[5], &nx);
    need(!x0 || nx == n, "x0 must concatenate the instances' starting vectors");
    int lbk, ubk;
    double lb, ub;
    const double *lbv, *ubv;
    bound(o, "lbound", 1, &lbk, &lb, &lbv);
    bound(o, "ubound", 1, &ubk, &ub, &ubv);
    plhs[0] = mxCreateDoubleMatrix((mwSize)n, 1, mxREAL);
    mxArray *it = mxCreateNumericMatrix((mwSize)k, 1, mxINT64_CLASS, mxREAL);
    mxArray *sr = mxCreateNumericMatrix((mwSize)k, 1, mxINT32_CLASS, mxREAL);
    double ms = 0.0;
    /* opts.stoprule (0 NONE, 1 DP, 2 ME, 3 NCP) applies per instance; without it, DP when
       taudelta is given */
    const int rule = (int)dfield(o, "stoprule", td ? AIRT_STOP_DP : AIRT_STOP_NONE);
    chk(airt_batch_sirt_rule(bh, (int)dfield(o, "method", AIRT_CIMMINO), lam, b, rule, td,
                             (int)dfield(o, "ncp_smooth", 2), (int64_t)dfield(o, "kmax", 100),
                             lbk, lb, ubk, ub, x0, mxGetDoubles(plhs[0]),
                             (int64_t *)mxGetInt64s(it), (int *)mxGetInt32s(sr), &ms));
    if (nlhs > 1) plhs[1] = it;
    else mxDestroyArray(it);
    if (nlhs > 2) plhs[2] = sr;
    else mxDestroyArray(sr);
    if (nlhs > 3) plhs[3] = mxCreateDoubleScalar(ms);
}

static void cmd_batch_kaczmarz(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
    need(nrhs == 8, "airt_mex('batch_kaczmarz', bh, ninst, b, sweeps, relaxpar, lbound, ubound)");
    airt_batch *bh = (airt_batch *)handle_in(prhs[1]);
    const int64_t k = (int64_t)scalar(prhs[2]);
    int64_t m = 0, n = 0, nb = 0;
    batch_dims(bh, k, &m, &n);
    const double *b = dvec(prhs[3], &nb);
    need(nb == m, "b must concatenate the instances' right-hand sides");
    const int lbk = mxIsEmpty(prhs[6]) ? AIRT_BOUND_NONE : AIRT_BOUND_SCALAR;
    const int ubk = mxIsEmpty(prhs[7]) ? AIRT_BOUND_NONE : AIRT_BOUND_SCALAR;
    const double lb = lbk ? scalar(prhs[6]) : 0.0, ub = ubk ? scalar(prhs[7]) : 0.0;
    plhs[0] = mxCreateDoubleMatrix((mwSize)n, 1, mxREAL);
    double ms = 0.0;
    chk(airt_batch_kaczmarz(bh, b, (int64_t)scalar(prhs[4]), scalar(prhs[5]), lbk, lb, ubk, ub,
                            mxGetDoubles(plhs[0]), &ms));
    if (nlhs > 1) plhs[1] = mxCreateDoubleScalar(ms);
}

static void cmd_batch_destroy(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
    need(nrhs == 2, "airt_mex('batch_destroy', bh)");
    chk(airt_batch_destroy((airt_batch *)handle_in(prhs[1])));
    (void)nlhs;
    (void)plhs;
}

/* ---- learned warm start */
static void cmd_unet(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
    need(nrhs == 7, "airt_mex('unet', H, W, base, levels, max_batch, seed)");
    airt_unet *uh = NULL;
    chk(airt_unet_create((int)scalar(prhs[1]), (int)scalar(prhs[2]), (int)scalar(prhs[3]),
                         (int)scalar(prhs[4]), (int)scalar(prhs[5]), (uint64_t)scalar(prhs[6]),
                         &uh));
    plhs[0] = handle_out(uh);
    (void)nlhs;
}

static void cmd_unet_params(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
    need(nrhs == 2, "airt_mex('unet_params', uh)");
    airt_unet *uh = (airt_unet *)handle_in(prhs[1]);
    int64_t np = 0;
    chk(airt_unet_num_params(uh, &np));
    plhs[0] = mxCreateNumericMatrix((mwSize)np, 1, mxSINGLE_CLASS, mxREAL);
    chk(airt_unet_get_params(uh, (float *)mxGetSingles(plhs[0])));
    (void)nlhs;
}

static void cmd_unet_set_params(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
    need(nrhs == 3 && mxIsSingle(prhs[2]), "airt_mex('unet_set_params', uh, single(w))");
    airt_unet *uh = (airt_unet *)handle_in(prhs[1]);
    int64_t np = 0;
    chk(airt_unet_num_params(uh, &np));
    need((int64_t)mxGetNumberOfElements(prhs[2]) == np, "wrong number of network parameters");
    chk(airt_unet_set_params(uh, (const float *)mxGetSingles(prhs[2])));
    (void)nlhs;
    (void)plhs;
}

static void cmd_unet_destroy(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
    need(nrhs == 2, "airt_mex('unet_destroy', uh)");
    chk(airt_unet_destroy((airt_unet *)handle_in(prhs[1])));
    (void)nlhs;
    (void)plhs;
}

#ifdef AIRT_MEX_GPUARRAY
/* Device-vector commands: the operands are gpuArrays, so the data stay on
 * the device between the network, the back projection and the solver. */
static mxGPUArray *gpu_double_vector(mwSize len) {
    const mwSize dims[2] = {len, 1};
    return mxGPUCreateGPUArray(2, dims, mxDOUBLE_CLASS, mxREAL, MX_GPU_DO_NOT_INITIALIZE);
}

static void cmd_batch_backproject(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
    need(nrhs == 5 && mxIsGPUArray(prhs[4]),
         "airt_mex('batch_backproject', bh, ninst, method, gpuArray b)");
    airt_batch *bh = (airt_batch *)handle_in(prhs[1]);
    int64_t m = 0, n = 0;
    batch_dims(bh, (int64_t)scalar(prhs[2]), &m, &n);
    const mxGPUArray *b = mxGPUCreateFromMxArray(prhs[4]);
    need(mxGPUGetClassID(b) == mxDOUBLE_CLASS && (int64_t)mxGPUGetNumberOfElements(b) == m,
         "b must be a double gpuArray with one entry per batch row");
    mxGPUArray *x = gpu_double_vector((mwSize)n);
    double ms = 0.0;
    const int st = airt_batch_backproject(bh, (int)scalar(prhs[3]),
                                          (const double *)mxGPUGetDataReadOnly(b),
                                          (double *)mxGPUGetData(x), &ms);
    mxGPUDestroyGPUArray(b);
    if (st != AIRT_OK) mxGPUDestroyGPUArray(x);
    chk(st);
    plhs[0] = mxGPUCreateMxArrayOnGPU(x);
    mxGPUDestroyGPUArray(x);
    (void)nlhs;
}

/* [X, it, sr] = airt_mex('sirt_multi', h, opts, gpuArray B, X0, taudelta): SIRT on the K
   columns of B (m x K) at once; X0 (n x K gpuArray) or empty; taudelta K values or empty. */
static void cmd_sirt_multi(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
    need(nrhs == 6 && mxIsStruct(prhs[2]) && mxIsGPUArray(prhs[3]),
         "airt_mex('sirt_multi', h, opts, gpuArray B, X0, taudelta)");
    airt_problem *h = (airt_problem *)handle_in(prhs[1]);
    const mxArray *o = prhs[2];
    int64_t m = 0, n = 0, ntd = 0;
    problem_size(h, &m, &n);
    const mxGPUArray *B = mxGPUCreateFromMxArray(prhs[3]);
    need(mxGPUGetClassID(B) == mxDOUBLE_CLASS && mxGPUGetNumberOfElements(B) % (mwSize)m == 0,
         "B must be a double gpuArray with m rows");
    const int K = (int)(mxGPUGetNumberOfElements(B) / (mwSize)m);
    const mxGPUArray *X0 = NULL;
    if (!mxIsEmpty(prhs[4])) {
        need(mxIsGPUArray(prhs[4]), "X0 must be a gpuArray or empty");
        X0 = mxGPUCreateFromMxArray(prhs[4]);
        need(mxGPUGetNumberOfElements(X0) == (mwSize)(n * K), "X0 must be n x K");
    }
    const double *td = mxIsEmpty(prhs[5]) ? NULL : dvec(prhs[5], &ntd);
    need(!td || ntd == K, "taudelta: one threshold per column of B");
    airt_sirt_opts so;
    memset(&so, 0, sizeof so);
    so.method = (int)dfield(o, "method", AIRT_CIMMINO);
    so.relax_kind = AIRT_RELAX_CONST;
    so.relaxpar = dfield(o, "relaxpar", 1.0);
    so.stoprule = td ? AIRT_STOP_DP : AIRT_STOP_NONE;
    bound(o, "lbound", 1, &so.lb_kind, &so.lb, &so.lbv);
    bound(o, "ubound", 1, &so.ub_kind, &so.ub, &so.ubv);
    so.kmax = (int64_t)dfield(o, "kmax", 100);
    const mwSize dims[2] = {(mwSize)n, (mwSize)K};
    mxGPUArray *X = mxGPUCreateGPUArray(2, dims, mxDOUBLE_CLASS, mxREAL, MX_GPU_DO_NOT_INITIALIZE);
    mxArray *it = mxCreateNumericMatrix((mwSize)K, 1, mxINT64_CLASS, mxREAL);
    mxArray *sr = mxCreateNumericMatrix((mwSize)K, 1, mxINT32_CLASS, mxREAL);
    double ms = 0.0;
    const int st = airt_sirt_multi_device(
        h, &so, K, (const double *)mxGPUGetDataReadOnly(B),
        X0 ? (const double *)mxGPUGetDataReadOnly(X0) : NULL, td, NULL, NULL, 0, NULL,
        (double *)mxGPUGetData(X), (int64_t *)mxGetInt64s(it), (int *)mxGetInt32s(sr), &ms);
    mxGPUDestroyGPUArray(B);
    if (X0) mxGPUDestroyGPUArray(X0);
    if (st != AIRT_OK) {
        mxGPUDestroyGPUArray(X);
        mxDestroyArray(it);
        mxDestroyArray(sr);
    }
    chk(st);
    plhs[0] = mxGPUCreateMxArrayOnGPU(X);
    mxGPUDestroyGPUArray(X);
    if (nlhs > 1) plhs[1] = it;
    else mxDestroyArray(it);
    if (nlhs > 2) plhs[2] = sr;
    else mxDestroyArray(sr);
}

static void cmd_unet_forward(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
    need(nrhs == 4 && mxIsGPUArray(prhs[2]), "airt_mex('unet_forward', uh, gpuArray x, B)");
    airt_unet *uh = (airt_unet *)handle_in(prhs[1]);
    const int B = (int)scalar(prhs[3]);
    const mxGPUArray *x = mxGPUCreateFromMxArray(prhs[2]);
    need(mxGPUGetClassID(x) == mxDOUBLE_CLASS && B >= 1 && mxGPUGetNumberOfElements(x) % B == 0,
         "x must be a double gpuArray of B images");
    mxGPUArray *y = gpu_double_vector(mxGPUGetNumberOfElements(x));
    const int st = airt_unet_forward_f64(uh, (const double *)mxGPUGetDataReadOnly(x),
                                         (double *)mxGPUGetData(y), B, NULL);
    mxGPUDestroyGPUArray(x);
    if (st != AIRT_OK) mxGPUDestroyGPUArray(y);
    chk(st);
    plhs[0] = mxGPUCreateMxArrayOnGPU(y);
    mxGPUDestroyGPUArray(y);
    (void)nlhs;
}
#endif

/* ------------------------------------------------------------------ dispatch */
typedef void (*command_fn)(int, mxArray **, int, const mxArray **);
struct command {
    const char *name;
    command_fn fn;
};

static const struct command commands[] = {
    {"matrix", cmd_matrix},
    {"parallel", cmd_parallel},
    {"fan", cmd_fan},
    {"seismic", cmd_seismic},
    {"spherical", cmd_spherical},
    {"size", cmd_size},
    {"export", cmd_export},
    {"apply", cmd_apply},
    {"weights", cmd_weights},
    {"rho", cmd_rho},
    {"sirt", cmd_sirt},
    {"art", cmd_art},
    {"cart", cmd_cart},
    {"fbp", cmd_fbp},
    {"destroy", cmd_destroy},
    {"batch", cmd_batch},
    {"batch_layout", cmd_batch_layout},
    {"batch_rho", cmd_batch_rho},
    {"batch_sirt", cmd_batch_sirt},
    {"batch_kaczmarz", cmd_batch_kaczmarz},
    {"batch_destroy", cmd_batch_destroy},
    {"unet", cmd_unet},
    {"unet_params", cmd_unet_params},
    {"unet_set_params", cmd_unet_set_params},
    {"unet_destroy", cmd_unet_destroy},
#ifdef AIRT_MEX_GPUARRAY
    {"batch_backproject", cmd_batch_backproject},
    {"sirt_multi", cmd_sirt_multi},
    {"unet_forward", cmd_unet_forward},
#endif
};

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
    char cmd[64];
    need(nrhs >= 1 && mxIsChar(prhs[0]) && mxGetString(prhs[0], cmd, sizeof cmd) == 0,
         "airt_mex: the first argument is the command name");
#ifdef AIRT_MEX_GPUARRAY
    mxInitGPU();
#endif
    if (!strcmp(cmd, "version")) {
        plhs[0] = mxCreateDoubleScalar((double)airt_version());
        return;
    }
    for (size_t i = 0; i < sizeof commands / sizeof commands[0]; ++i)
        if (!strcmp(cmd, commands[i].name)) {
            commands[i].fn(nlhs, plhs, nrhs, prhs);
            return;
        }
    mexErrMsgIdAndTxt("AIRT:cmd", "airt_mex: unknown command '%s'", cmd);
}
