/* Declarations of the documented MATLAB MEX / matrix C API functions the
 * gateway uses, for a syntax and type check of airt_mex.c with gcc where
 * MATLAB is not installed (test infrastructure; not MathWorks' header). */
#ifndef AIRT_TEST_MEX_STUB_H
#define AIRT_TEST_MEX_STUB_H
#include <stddef.h>
#include <stdbool.h>
#include <stdint.h>

typedef struct mxArray_tag mxArray;
typedef size_t mwSize;
typedef size_t mwIndex;
typedef double mxDouble;
typedef float mxSingle;
typedef int32_t mxInt32;
typedef int64_t mxInt64;
typedef enum {
    mxUNKNOWN_CLASS, mxCELL_CLASS, mxSTRUCT_CLASS, mxLOGICAL_CLASS, mxCHAR_CLASS, mxVOID_CLASS,
    mxDOUBLE_CLASS, mxSINGLE_CLASS, mxINT8_CLASS, mxUINT8_CLASS, mxINT16_CLASS, mxUINT16_CLASS,
    mxINT32_CLASS, mxUINT32_CLASS, mxINT64_CLASS, mxUINT64_CLASS, mxFUNCTION_CLASS
} mxClassID;
typedef enum { mxREAL, mxCOMPLEX } mxComplexity;

void mexErrMsgIdAndTxt(const char *id, const char *fmt, ...);
void mexWarnMsgIdAndTxt(const char *id, const char *fmt, ...);
size_t mxGetM(const mxArray *a);
size_t mxGetN(const mxArray *a);
void mxSetN(mxArray *a, mwSize n);
size_t mxGetNumberOfElements(const mxArray *a);
bool mxIsEmpty(const mxArray *a);
bool mxIsSparse(const mxArray *a);
bool mxIsDouble(const mxArray *a);
bool mxIsSingle(const mxArray *a);
bool mxIsComplex(const mxArray *a);
bool mxIsNumeric(const mxArray *a);
bool mxIsChar(const mxArray *a);
bool mxIsStruct(const mxArray *a);
bool mxIsInt32(const mxArray *a);
bool mxIsInt64(const mxArray *a);
bool mxIsUint64(const mxArray *a);
double mxGetScalar(const mxArray *a);
void *mxGetData(const mxArray *a);
mxDouble *mxGetDoubles(const mxArray *a);
mxSingle *mxGetSingles(const mxArray *a);
mxInt32 *mxGetInt32s(const mxArray *a);
mxInt64 *mxGetInt64s(const mxArray *a);
mwIndex *mxGetJc(const mxArray *a);
mwIndex *mxGetIr(const mxArray *a);
int mxGetString(const mxArray *a, char *buf, mwSize buflen);
mxArray *mxGetField(const mxArray *s, mwIndex i, const char *name);
void mxSetField(mxArray *s, mwIndex i, const char *name, mxArray *value);
mxArray *mxCreateStructMatrix(mwSize m, mwSize n, int nfields, const char **names);
mxArray *mxCreateDoubleMatrix(mwSize m, mwSize n, mxComplexity c);
mxArray *mxCreateDoubleScalar(double v);
mxArray *mxCreateNumericMatrix(mwSize m, mwSize n, mxClassID cls, mxComplexity c);
mxArray *mxCreateSparse(mwSize m, mwSize n, mwSize nzmax, mxComplexity c);
void mxDestroyArray(mxArray *a);
void *mxMalloc(size_t n);
void mxFree(void *p);
void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]);
#endif
