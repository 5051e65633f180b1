/* A stand-in for MATLAB's mex.h with the subset of the MEX/MX API that
 * gasatt_mex.c uses, so the gateway compiles and runs without MATLAB (test
 * infrastructure only; a real build includes MATLAB's own header). */
#ifndef GASATT_FAKE_MEX_H
#define GASATT_FAKE_MEX_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct mxArray_tag mxArray;
typedef size_t mwSize;
typedef size_t mwIndex;
typedef enum {
  mxUNKNOWN_CLASS = 0, mxCELL_CLASS, mxSTRUCT_CLASS, mxLOGICAL_CLASS, mxCHAR_CLASS,
  mxVOID_CLASS, mxDOUBLE_CLASS, mxSINGLE_CLASS, mxINT8_CLASS, mxUINT8_CLASS, mxINT16_CLASS,
  mxUINT16_CLASS, mxINT32_CLASS, mxUINT32_CLASS, mxINT64_CLASS, mxUINT64_CLASS
} mxClassID;
typedef enum { mxREAL = 0, mxCOMPLEX } mxComplexity;

void mexErrMsgIdAndTxt(const char *id, const char *fmt, ...);
int mexAtExit(void (*fn)(void));
void mexMakeMemoryPersistent(void *p);

void *mxMalloc(size_t n);
void mxFree(void *p);
int mxIsChar(const mxArray *a);
int mxIsDouble(const mxArray *a);
int mxIsComplex(const mxArray *a);
int mxIsUint64(const mxArray *a);
int mxIsStruct(const mxArray *a);
int mxGetString(const mxArray *a, char *buf, mwSize len);
size_t mxGetM(const mxArray *a);
size_t mxGetN(const mxArray *a);
size_t mxGetNumberOfElements(const mxArray *a);
double mxGetScalar(const mxArray *a);
double *mxGetDoubles(const mxArray *a);
void *mxGetData(const mxArray *a);
mxArray *mxCreateDoubleMatrix(mwSize m, mwSize n, mxComplexity c);
mxArray *mxCreateDoubleScalar(double v);
mxArray *mxCreateNumericMatrix(mwSize m, mwSize n, mxClassID cls, mxComplexity c);
mxArray *mxCreateStructMatrix(mwSize m, mwSize n, int nfields, const char **names);
mxArray *mxGetField(const mxArray *s, mwIndex i, const char *name);
void mxSetField(mxArray *s, mwIndex i, const char *name, mxArray *v);
void mxDestroyArray(mxArray *a);

#ifdef __cplusplus
}
#endif
#endif
