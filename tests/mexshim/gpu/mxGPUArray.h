/* A stand-in for MATLAB's gpu/mxGPUArray.h (the subset gasatt_mex.c uses);
 * test infrastructure only. */
#ifndef GASATT_FAKE_MXGPUARRAY_H
#define GASATT_FAKE_MXGPUARRAY_H
#include "../mex.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct mxGPUArray_tag mxGPUArray;
typedef enum { MX_GPU_INITIALIZE_VALUES = 0, MX_GPU_DO_NOT_INITIALIZE } mxGPUInitialize;

int mxInitGPU(void);
int mxIsGPUArray(const mxArray *a);
mxGPUArray *mxGPUCopyFromMxArray(const mxArray *a);
mxClassID mxGPUGetClassID(const mxGPUArray *g);
mxComplexity mxGPUGetComplexity(const mxGPUArray *g);
const mwSize *mxGPUGetDimensions(const mxGPUArray *g);
mwSize mxGPUGetNumberOfDimensions(const mxGPUArray *g);
void *mxGPUGetData(mxGPUArray *g);
mxGPUArray *mxGPUCreateGPUArray(mwSize ndim, const mwSize *dims, mxClassID cls, mxComplexity c,
                                mxGPUInitialize init);
mxArray *mxGPUCreateMxArrayOnGPU(const mxGPUArray *g);
void mxGPUDestroyGPUArray(const mxGPUArray *g);

#ifdef __cplusplus
}
#endif
#endif
