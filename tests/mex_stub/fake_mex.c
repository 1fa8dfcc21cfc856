/* A minimal stand-in for the MATLAB MEX runtime (test infrastructure): just
 * enough of the documented mx / mex C API, with the declarations of
 * tests/mex_stub/mex.h, to run airt_mex.c's mexFunction from Python through
 * ctypes where MATLAB is not installed.  Arrays are column-major; struct
 * arrays are 1x1; errors raised with mexErrMsgIdAndTxt return to fm_call
 * through longjmp with the identifier and message kept for the caller. */
#include <setjmp.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "mex.h"
#include "gpu/mxGPUArray.h"

struct mxArray_tag {
    mxClassID cls;
    size_t m, n;
    int sparse;
    void *data;          /* numeric / char data, or values of a sparse matrix */
    mwIndex *jc, *ir;    /* sparse */
    size_t nzmax;
    int nfields;         /* struct */
    char **names;
    mxArray **values;
};

static jmp_buf g_jmp;

static char *dup_string(const char *s) {
    const size_t n = strlen(s) + 1;
    char *d = (char *)malloc(n);
    memcpy(d, s, n);
    return d;
}
static char g_err_id[128], g_err_msg[1024];

static size_t elsize(mxClassID c) {
    switch (c) {
        case mxDOUBLE_CLASS: case mxINT64_CLASS: case mxUINT64_CLASS: return 8;
        case mxSINGLE_CLASS: case mxINT32_CLASS: case mxUINT32_CLASS: return 4;
        case mxCHAR_CLASS: return 1;
        default: return 8;
    }
}

static mxArray *alloc_array(mxClassID c, size_t m, size_t n) {
    mxArray *a = (mxArray *)calloc(1, sizeof(mxArray));
    a->cls = c;
    a->m = m;
    a->n = n;
    a->data = calloc(m * n > 0 ? m * n : 1, elsize(c));
    return a;
}

void mexErrMsgIdAndTxt(const char *id, const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    snprintf(g_err_id, sizeof g_err_id, "%s", id);
    vsnprintf(g_err_msg, sizeof g_err_msg, fmt, ap);
    va_end(ap);
    longjmp(g_jmp, 1);
}
void mexWarnMsgIdAndTxt(const char *id, const char *fmt, ...) { (void)id; (void)fmt; }
size_t mxGetM(const mxArray *a) { return a->m; }
size_t mxGetN(const mxArray *a) { return a->n; }
void mxSetN(mxArray *a, mwSize n) { a->n = n; }
size_t mxGetNumberOfElements(const mxArray *a) { return a->m * a->n; }
bool mxIsEmpty(const mxArray *a) { return a->m * a->n == 0; }
bool mxIsSparse(const mxArray *a) { return a->sparse != 0; }
bool mxIsDouble(const mxArray *a) { return a->cls == mxDOUBLE_CLASS; }
bool mxIsSingle(const mxArray *a) { return a->cls == mxSINGLE_CLASS; }
bool mxIsComplex(const mxArray *a) { (void)a; return false; }
bool mxIsNumeric(const mxArray *a) {
    return a->cls >= mxDOUBLE_CLASS && a->cls <= mxUINT64_CLASS;
}
bool mxIsChar(const mxArray *a) { return a->cls == mxCHAR_CLASS; }
bool mxIsStruct(const mxArray *a) { return a->cls == mxSTRUCT_CLASS; }
bool mxIsInt32(const mxArray *a) { return a->cls == mxINT32_CLASS; }
bool mxIsInt64(const mxArray *a) { return a->cls == mxINT64_CLASS; }
bool mxIsUint64(const mxArray *a) { return a->cls == mxUINT64_CLASS; }
double mxGetScalar(const mxArray *a) {
    switch (a->cls) {
        case mxDOUBLE_CLASS: return ((double *)a->data)[0];
        case mxSINGLE_CLASS: return ((float *)a->data)[0];
        case mxINT32_CLASS: return ((int32_t *)a->data)[0];
        case mxINT64_CLASS: return (double)((int64_t *)a->data)[0];
        case mxUINT64_CLASS: return (double)((uint64_t *)a->data)[0];
        default: return 0.0;
    }
}
void *mxGetData(const mxArray *a) { return a->data; }
mxDouble *mxGetDoubles(const mxArray *a) { return a->cls == mxDOUBLE_CLASS ? (double *)a->data : NULL; }
mxSingle *mxGetSingles(const mxArray *a) { return a->cls == mxSINGLE_CLASS ? (float *)a->data : NULL; }
mxInt32 *mxGetInt32s(const mxArray *a) { return a->cls == mxINT32_CLASS ? (int32_t *)a->data : NULL; }
mxInt64 *mxGetInt64s(const mxArray *a) { return a->cls == mxINT64_CLASS ? (int64_t *)a->data : NULL; }
mwIndex *mxGetJc(const mxArray *a) { return a->jc; }
mwIndex *mxGetIr(const mxArray *a) { return a->ir; }
int mxGetString(const mxArray *a, char *buf, mwSize buflen) {
    if (a->cls != mxCHAR_CLASS || a->m * a->n + 1 > buflen) return 1;
    memcpy(buf, a->data, a->m * a->n);
    buf[a->m * a->n] = 0;
    return 0;
}
mxArray *mxGetField(const mxArray *s, mwIndex i, const char *name) {
    (void)i;
    for (int k = 0; k < s->nfields; ++k)
        if (!strcmp(s->names[k], name)) return s->values[k];
    return NULL;
}
void mxSetField(mxArray *s, mwIndex i, const char *name, mxArray *value) {
    (void)i;
    for (int k = 0; k < s->nfields; ++k)
        if (!strcmp(s->names[k], name)) {
            s->values[k] = value;
            return;
        }
}
mxArray *mxCreateStructMatrix(mwSize m, mwSize n, int nfields, const char **names) {
    mxArray *a = alloc_array(mxSTRUCT_CLASS, m, n);
    a->nfields = nfields;
    a->names = (char **)calloc((size_t)nfields, sizeof(char *));
    a->values = (mxArray **)calloc((size_t)nfields, sizeof(mxArray *));
    for (int k = 0; k < nfields; ++k) a->names[k] = dup_string(names[k]);
    return a;
}
mxArray *mxCreateDoubleMatrix(mwSize m, mwSize n, mxComplexity c) {
    (void)c;
    return alloc_array(mxDOUBLE_CLASS, m, n);
}
mxArray *mxCreateDoubleScalar(double v) {
    mxArray *a = alloc_array(mxDOUBLE_CLASS, 1, 1);
    ((double *)a->data)[0] = v;
    return a;
}
mxArray *mxCreateNumericMatrix(mwSize m, mwSize n, mxClassID cls, mxComplexity c) {
    (void)c;
    return alloc_array(cls, m, n);
}
mxArray *mxCreateSparse(mwSize m, mwSize n, mwSize nzmax, mxComplexity c) {
    (void)c;
    mxArray *a = alloc_array(mxDOUBLE_CLASS, 0, 0);
    free(a->data);
    a->m = m;
    a->n = n;
    a->sparse = 1;
    a->nzmax = nzmax;
    a->data = calloc(nzmax ? nzmax : 1, sizeof(double));
    a->ir = (mwIndex *)calloc(nzmax ? nzmax : 1, sizeof(mwIndex));
    a->jc = (mwIndex *)calloc(n + 1, sizeof(mwIndex));
    return a;
}
void mxDestroyArray(mxArray *a) {
    if (!a) return;
    for (int k = 0; k < a->nfields; ++k) {
        free(a->names[k]);
        mxDestroyArray(a->values[k]);
    }
    free(a->names);
    free(a->values);
    free(a->data);
    free(a->jc);
    free(a->ir);
    free(a);
}
void *mxMalloc(size_t n) { return malloc(n ? n : 1); }
void mxFree(void *p) { free(p); }

/* mxGPUArray entry points are not provided: the gateway is built without
 * AIRT_MEX_GPUARRAY for this runtime. */

/* ---- the Python side */
mxArray *fm_numeric(int cls, size_t m, size_t n, const void *src) {
    mxArray *a = alloc_array((mxClassID)cls, m, n);
    if (src) memcpy(a->data, src, m * n * elsize((mxClassID)cls));
    return a;
}
mxArray *fm_char(const char *s) {
    mxArray *a = alloc_array(mxCHAR_CLASS, 1, strlen(s));
    memcpy(a->data, s, strlen(s));
    return a;
}
mxArray *fm_sparse(size_t m, size_t n, size_t nnz, const uint64_t *jc, const uint64_t *ir,
                   const double *pr) {
    mxArray *a = mxCreateSparse(m, n, nnz, mxREAL);
    memcpy(a->jc, jc, (n + 1) * sizeof(mwIndex));
    memcpy(a->ir, ir, nnz * sizeof(mwIndex));
    memcpy(a->data, pr, nnz * sizeof(double));
    return a;
}
mxArray *fm_struct(int nfields, const char **names) {
    return mxCreateStructMatrix(1, 1, nfields, names);
}
void fm_set_field(mxArray *s, const char *name, mxArray *v) { mxSetField(s, 0, name, v); }
mxArray *fm_get_field(const mxArray *s, const char *name) { return mxGetField(s, 0, name); }
int fm_class(const mxArray *a) { return (int)a->cls; }
size_t fm_m(const mxArray *a) { return a->m; }
size_t fm_n(const mxArray *a) { return a->n; }
int fm_is_sparse(const mxArray *a) { return a->sparse; }
void *fm_data(const mxArray *a) { return a->data; }
mwIndex *fm_jc(const mxArray *a) { return a->jc; }
mwIndex *fm_ir(const mxArray *a) { return a->ir; }
void fm_destroy(mxArray *a) { mxDestroyArray(a); }
const char *fm_err_id(void) { return g_err_id; }
const char *fm_err_msg(void) { return g_err_msg; }

/* Runs mexFunction; returns 0, or 1 after mexErrMsgIdAndTxt (see fm_err_*). */
int fm_call(int nlhs, mxArray **plhs, int nrhs, const mxArray **prhs) {
    g_err_id[0] = g_err_msg[0] = 0;
    if (setjmp(g_jmp)) return 1;
    mexFunction(nlhs, plhs, nrhs, prhs);
    return 0;
}
