/* Declarations of the documented mxGPUArray C API functions the gateway's
 * gpuArray commands use (test infrastructure for a syntax check; not
 * MathWorks' header). */
#ifndef AIRT_TEST_MXGPUARRAY_STUB_H
#define AIRT_TEST_MXGPUARRAY_STUB_H
#include "../mex.h"
typedef struct mxGPUArray_tag mxGPUArray;
typedef enum { MX_GPU_INITIALIZE_VALUES, MX_GPU_DO_NOT_INITIALIZE } mxGPUInitialize;
int mxInitGPU(void);
int mxIsGPUArray(const mxArray *a);
const mxGPUArray *mxGPUCreateFromMxArray(const mxArray *a);
mxGPUArray *mxGPUCreateGPUArray(mwSize ndims, const mwSize *dims, mxClassID cls,
                                mxComplexity c, mxGPUInitialize init);
mxClassID mxGPUGetClassID(const mxGPUArray *g);
mwSize mxGPUGetNumberOfElements(const mxGPUArray *g);
const void *mxGPUGetDataReadOnly(const mxGPUArray *g);
void *mxGPUGetData(mxGPUArray *g);
mxArray *mxGPUCreateMxArrayOnGPU(const mxGPUArray *g);
void mxGPUDestroyGPUArray(const mxGPUArray *g);
#endif
