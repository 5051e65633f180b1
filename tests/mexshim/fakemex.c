/*
 * fakemex.c - a minimal MATLAB MEX/MX/mxGPUArray runtime for running the
 * gateway gas-atenuator_b200/mex/gasatt_mex.c without MATLAB (test
 * infrastructure only).  Host arrays live in malloc'd memory, gpuArrays in
 * cudaMalloc'd buffers shared by reference count between an mxGPUArray and
 * the mxArray made from it (MATLAB's ownership rule: the mxArray keeps the
 * data after the mxGPUArray is destroyed).  mexErrMsgIdAndTxt returns to
 * fx_call through longjmp.  The fx_* functions are the harness the Python
 * tests drive through ctypes.
 */
#include <setjmp.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <cuda_runtime.h>

#include "mex.h"
#include "gpu/mxGPUArray.h"

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]);

typedef struct devbuf {
  void *p;
  int refs;
} devbuf;

struct mxArray_tag {
  mxClassID cls;
  size_t m, n;
  void *data;          /* host data (double, uint64 or char) */
  devbuf *dev;         /* gpuArray data */
  int nfields;
  char **names;
  mxArray **values;
};

struct mxGPUArray_tag {
  mxClassID cls;
  mwSize dims[2];
  devbuf *dev;
};

static jmp_buf g_jmp;
static int g_in_call = 0;
static char g_err[1024];
static void (*g_exit_fn)(void) = NULL;

static devbuf *devbuf_new(size_t bytes) {
  devbuf *b = (devbuf *)calloc(1, sizeof *b);
  b->refs = 1;
  if (bytes && cudaMalloc(&b->p, bytes) != cudaSuccess) {
    free(b);
    mexErrMsgIdAndTxt("fake:cuda", "cudaMalloc of %zu bytes failed", bytes);
  }
  return b;
}
static void devbuf_drop(devbuf *b) {
  if (b && --b->refs == 0) {
    if (b->p) cudaFree(b->p);
    free(b);
  }
}

/* ------------------------------------------------------------ mex / mx */
void mexErrMsgIdAndTxt(const char *id, const char *fmt, ...) {
  va_list ap;
  int k = snprintf(g_err, sizeof g_err, "%s: ", id);
  va_start(ap, fmt);
  vsnprintf(g_err + k, sizeof g_err - (size_t)k, fmt, ap);
  va_end(ap);
  if (g_in_call) longjmp(g_jmp, 1);
  fprintf(stderr, "mex error outside a call: %s\n", g_err);
  abort();
}
int mexAtExit(void (*fn)(void)) { g_exit_fn = fn; return 0; }
void mexMakeMemoryPersistent(void *p) { (void)p; }
void *mxMalloc(size_t n) { return malloc(n ? n : 1); }
void mxFree(void *p) { free(p); }

static mxArray *mk(mxClassID cls, size_t m, size_t n, size_t elem) {
  mxArray *a = (mxArray *)calloc(1, sizeof *a);
  a->cls = cls; a->m = m; a->n = n;
  if (elem) a->data = calloc((m * n) != 0 ? m * n : 1, elem);
  return a;
}
int mxIsChar(const mxArray *a) { return a && a->cls == mxCHAR_CLASS; }
int mxIsDouble(const mxArray *a) { return a && a->cls == mxDOUBLE_CLASS; }
int mxIsComplex(const mxArray *a) { (void)a; return 0; }
int mxIsUint64(const mxArray *a) { return a && a->cls == mxUINT64_CLASS; }
int mxIsStruct(const mxArray *a) { return a && a->cls == mxSTRUCT_CLASS; }
int mxGetString(const mxArray *a, char *buf, mwSize len) {
  if (!mxIsChar(a) || len == 0) return 1;
  strncpy(buf, (const char *)a->data, len - 1);
  buf[len - 1] = 0;
  return strlen((const char *)a->data) >= len ? 1 : 0;
}
size_t mxGetM(const mxArray *a) { return a->m; }
size_t mxGetN(const mxArray *a) { return a->n; }
size_t mxGetNumberOfElements(const mxArray *a) { return a->m * a->n; }
double mxGetScalar(const mxArray *a) {
  if (a->cls == mxDOUBLE_CLASS && a->data) return ((double *)a->data)[0];
  if (a->cls == mxUINT64_CLASS) return (double)((uint64_t *)a->data)[0];
  return 0;
}
double *mxGetDoubles(const mxArray *a) { return a->cls == mxDOUBLE_CLASS ? (double *)a->data : NULL; }
void *mxGetData(const mxArray *a) { return a->data; }
mxArray *mxCreateDoubleMatrix(mwSize m, mwSize n, mxComplexity c) { (void)c; return mk(mxDOUBLE_CLASS, m, n, 8); }
mxArray *mxCreateDoubleScalar(double v) {
  mxArray *a = mk(mxDOUBLE_CLASS, 1, 1, 8);
  ((double *)a->data)[0] = v;
  return a;
}
mxArray *mxCreateNumericMatrix(mwSize m, mwSize n, mxClassID cls, mxComplexity c) {
  (void)c;
  return mk(cls, m, n, cls == mxUINT64_CLASS || cls == mxDOUBLE_CLASS ? 8 : 4);
}
mxArray *mxCreateStructMatrix(mwSize m, mwSize n, int nfields, const char **names) {
  mxArray *a = mk(mxSTRUCT_CLASS, m, n, 0);
  int k;
  a->nfields = nfields;
  a->names = (char **)calloc((size_t)nfields, sizeof(char *));
  a->values = (mxArray **)calloc((size_t)nfields, sizeof(mxArray *));
  for (k = 0; k < nfields; ++k) a->names[k] = strdup(names[k]);
  return a;
}
mxArray *mxGetField(const mxArray *s, mwIndex i, const char *name) {
  int k;
  (void)i;
  for (k = 0; k < s->nfields; ++k)
    if (!strcmp(s->names[k], name)) return s->values[k];
  return NULL;
}
void mxSetField(mxArray *s, mwIndex i, const char *name, mxArray *v) {
  int k;
  (void)i;
  for (k = 0; k < s->nfields; ++k)
    if (!strcmp(s->names[k], name)) { s->values[k] = v; return; }
}
void mxDestroyArray(mxArray *a) {
  int k;
  if (!a) return;
  free(a->data);
  devbuf_drop(a->dev);
  for (k = 0; k < a->nfields; ++k) { free(a->names[k]); mxDestroyArray(a->values[k]); }
  free(a->names);
  free(a->values);
  free(a);
}

/* ---------------------------------------------------------------- gpu */
int mxInitGPU(void) { return 0; }
int mxIsGPUArray(const mxArray *a) { return a && a->dev != NULL; }
mxGPUArray *mxGPUCopyFromMxArray(const mxArray *a) {
  mxGPUArray *g = (mxGPUArray *)calloc(1, sizeof *g);
  const size_t bytes = a->m * a->n * 8;
  g->cls = a->cls; g->dims[0] = a->m; g->dims[1] = a->n;
  g->dev = devbuf_new(bytes);
  if (bytes) cudaMemcpy(g->dev->p, a->dev->p, bytes, cudaMemcpyDeviceToDevice);
  return g;
}
mxClassID mxGPUGetClassID(const mxGPUArray *g) { return g->cls; }
mxComplexity mxGPUGetComplexity(const mxGPUArray *g) { (void)g; return mxREAL; }
const mwSize *mxGPUGetDimensions(const mxGPUArray *g) {
  mwSize *d = (mwSize *)mxMalloc(2 * sizeof(mwSize));
  d[0] = g->dims[0]; d[1] = g->dims[1];
  return d;
}
mwSize mxGPUGetNumberOfDimensions(const mxGPUArray *g) { (void)g; return 2; }
void *mxGPUGetData(mxGPUArray *g) { return g->dev->p; }
mxGPUArray *mxGPUCreateGPUArray(mwSize ndim, const mwSize *dims, mxClassID cls, mxComplexity c,
                                mxGPUInitialize init) {
  mxGPUArray *g = (mxGPUArray *)calloc(1, sizeof *g);
  size_t bytes;
  (void)c;
  g->cls = cls; g->dims[0] = dims[0]; g->dims[1] = ndim > 1 ? dims[1] : 1;
  bytes = g->dims[0] * g->dims[1] * 8;
  g->dev = devbuf_new(bytes);
  if (init == MX_GPU_INITIALIZE_VALUES && bytes) cudaMemset(g->dev->p, 0, bytes);
  else if (bytes) cudaMemset(g->dev->p, 0xFF, bytes);   /* NaN: "not initialised" shows */
  return g;
}
mxArray *mxGPUCreateMxArrayOnGPU(const mxGPUArray *g) {
  mxArray *a = mk(g->cls, g->dims[0], g->dims[1], 0);
  a->dev = g->dev;
  a->dev->refs++;
  return a;
}
void mxGPUDestroyGPUArray(const mxGPUArray *g) {
  if (!g) return;
  devbuf_drop(g->dev);
  free((void *)g);
}

/* ------------------------------------------------------------ harness */
mxArray *fx_double(size_t m, size_t n, const double *v) {
  mxArray *a = mk(mxDOUBLE_CLASS, m, n, 8);
  if (v) memcpy(a->data, v, m * n * 8);
  return a;
}
mxArray *fx_uint64(size_t m, size_t n, const uint64_t *v) {
  mxArray *a = mk(mxUINT64_CLASS, m, n, 8);
  if (v) memcpy(a->data, v, m * n * 8);
  return a;
}
mxArray *fx_string(const char *s) {
  mxArray *a = mk(mxCHAR_CLASS, 1, strlen(s), 0);
  a->data = strdup(s);
  return a;
}
/* a gpuArray with a copy of host data; NULL on a failed allocation */
mxArray *fx_gpu(size_t m, size_t n, const double *v) {
  mxArray *a = mk(mxDOUBLE_CLASS, m, n, 0);
  devbuf *b = (devbuf *)calloc(1, sizeof *b);
  b->refs = 1;
  if ((m * n) != 0 && cudaMalloc(&b->p, m * n * 8) != cudaSuccess) { free(b); free(a); return NULL; }
  if ((m * n) != 0) cudaMemcpy(b->p, v, m * n * 8, cudaMemcpyHostToDevice);
  a->dev = b;
  return a;
}
mxArray *fx_struct(int nfields, const char **names, mxArray **values) {
  mxArray *s = mxCreateStructMatrix(1, 1, nfields, names);
  int k;
  for (k = 0; k < nfields; ++k) s->values[k] = values[k];
  return s;
}
int fx_call(int nlhs, mxArray **plhs, int nrhs, mxArray **prhs) {
  int k;
  for (k = 0; k < nlhs; ++k) plhs[k] = NULL;
  g_err[0] = 0;
  g_in_call = 1;
  if (setjmp(g_jmp)) {
    g_in_call = 0;
    return 1;
  }
  mexFunction(nlhs, plhs, nrhs, (const mxArray **)prhs);
  g_in_call = 0;
  return 0;
}
const char *fx_error(void) { return g_err; }
size_t fx_rows(const mxArray *a) { return a->m; }
size_t fx_cols(const mxArray *a) { return a->n; }
int fx_is_gpu(const mxArray *a) { return a->dev != NULL; }
int fx_class(const mxArray *a) { return (int)a->cls; }
/* the values of a (host or gpu) into out, m * n elements of 8 bytes */
int fx_read(const mxArray *a, void *out) {
  const size_t bytes = a->m * a->n * 8;
  if (a->dev) return bytes ? (int)cudaMemcpy(out, a->dev->p, bytes, cudaMemcpyDeviceToHost) : 0;
  memcpy(out, a->data, bytes);
  return 0;
}
mxArray *fx_field(const mxArray *s, const char *name) { return mxGetField(s, 0, name); }
void fx_destroy(mxArray *a) { mxDestroyArray(a); }
void fx_exit(void) {
  if (g_exit_fn) g_exit_fn();
  g_exit_fn = NULL;
}
