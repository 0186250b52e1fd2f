/* A host-memory implementation of the MEX API subset declared in mex.h, so that
 * MEX gateways (the library's own and the reference's) can be built and run
 * without MATLAB.  Arrays are column-major blocks of host memory with
 * interleaved complex values, as in the R2018a API.  mexErrMsgIdAndTxt unwinds
 * to mxstub_call with longjmp, like MATLAB's error return.  Test
 * infrastructure only. */
#include <setjmp.h>
#include <stdarg.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "mex.h"

struct mxArray_tag {
  mxClassID cls;
  int cplx;
  mwSize ndim;
  mwSize dims[8];
  size_t n;
  void* data;
};

static __thread jmp_buf* g_jb = NULL;
static __thread char g_err[1024];
static void (*g_atexit[16])(void);
static int g_natexit = 0;

static size_t elem_size(mxClassID c, int cplx) {
  size_t s;
  switch (c) {
    case mxDOUBLE_CLASS: case mxINT64_CLASS: case mxUINT64_CLASS: s = 8; break;
    case mxSINGLE_CLASS: case mxINT32_CLASS: case mxUINT32_CLASS: s = 4; break;
    case mxINT16_CLASS: case mxUINT16_CLASS: s = 2; break;
    case mxCELL_CLASS: s = sizeof(mxArray*); break;
    default: s = 1; break;   /* logical, char (one byte per character here), int8, uint8 */
  }
  return cplx ? 2 * s : s;
}

mxArray* mxstub_new(int cls, int cplx, int ndim, const size_t* dims) {
  mxArray* a = (mxArray*)calloc(1, sizeof(mxArray));
  if (!a || ndim < 1 || ndim > 8) { free(a); return NULL; }
  a->cls = (mxClassID)cls;
  a->cplx = cplx;
  a->ndim = (mwSize)(ndim < 2 ? 2 : ndim);
  a->dims[0] = dims[0];
  a->dims[1] = ndim >= 2 ? dims[1] : 1;
  a->n = 1;
  for (int i = 0; i < (int)a->ndim; ++i) {
    if (i >= 2) a->dims[i] = dims[i];
    a->n *= a->dims[i];
  }
  a->data = calloc(a->n ? a->n : 1, elem_size(a->cls, cplx));
  if (!a->data) { free(a); return NULL; }
  return a;
}

mxArray* mxstub_string(const char* s) {
  const size_t d[2] = {1, strlen(s)};
  mxArray* a = mxstub_new(mxCHAR_CLASS, 0, 2, d);
  if (a) memcpy(a->data, s, d[1]);
  return a;
}

void mxstub_free(mxArray* a) {
  if (!a) return;
  if (a->cls == mxCELL_CLASS) {
    mxArray** c = (mxArray**)a->data;
    for (size_t i = 0; i < a->n; ++i) mxstub_free(c[i]);
  }
  free(a->data);
  free(a);
}

void* mxstub_data(const mxArray* a) { return a ? a->data : NULL; }
int mxstub_class(const mxArray* a) { return a ? (int)a->cls : -1; }
int mxstub_is_complex(const mxArray* a) { return a ? a->cplx : 0; }
int mxstub_ndim(const mxArray* a) { return a ? (int)a->ndim : 0; }
size_t mxstub_dim(const mxArray* a, int i) { return (a && i < (int)a->ndim) ? a->dims[i] : 1; }
const char* mxstub_last_error(void) { return g_err; }

/* Runs fn(nlhs, plhs, nrhs, prhs); 0 on return, 1 when the gateway raised an
 * error (message in mxstub_last_error). */
int mxstub_call(void (*fn)(int, mxArray**, int, const mxArray**), int nlhs, mxArray** plhs, int nrhs,
                const mxArray** prhs) {
  jmp_buf jb;
  jmp_buf* prev = g_jb;
  g_err[0] = 0;
  if (setjmp(jb)) {
    g_jb = prev;
    return 1;
  }
  g_jb = &jb;
  fn(nlhs, plhs, nrhs, prhs);
  g_jb = prev;
  return 0;
}

/* Runs (and forgets) the functions registered with mexAtExit, as MATLAB does
 * when a MEX file is cleared. */
void mxstub_run_atexit(void) {
  while (g_natexit > 0) g_atexit[--g_natexit]();
}

void mexErrMsgIdAndTxt(const char* id, const char* fmt, ...) {
  va_list ap;
  int k = snprintf(g_err, sizeof g_err, "%s: ", id ? id : "");
  va_start(ap, fmt);
  if (k >= 0 && k < (int)sizeof g_err) vsnprintf(g_err + k, sizeof g_err - (size_t)k, fmt, ap);
  va_end(ap);
  if (g_jb) longjmp(*g_jb, 1);
  fprintf(stderr, "mex error outside mxstub_call: %s\n", g_err);
  abort();
}

int mexAtExit(void (*fn)(void)) {
  for (int i = 0; i < g_natexit; ++i)
    if (g_atexit[i] == fn) return 0;
  if (g_natexit < 16) g_atexit[g_natexit++] = fn;
  return 0;
}

int mxGetString(const mxArray* a, char* buf, mwSize len) {
  if (!a || a->cls != mxCHAR_CLASS || len == 0) return 1;
  const size_t n = a->n < len - 1 ? a->n : len - 1;
  memcpy(buf, a->data, n);
  buf[n] = 0;
  return n < a->n ? 1 : 0;
}

char* mxArrayToString(const mxArray* a) {
  if (!a || a->cls != mxCHAR_CLASS) return NULL;
  char* s = (char*)malloc(a->n + 1);
  if (!s) return NULL;
  memcpy(s, a->data, a->n);
  s[a->n] = 0;
  return s;
}

mxComplexDouble* mxGetComplexDoubles(const mxArray* a) {
  return (a && a->cls == mxDOUBLE_CLASS && a->cplx) ? (mxComplexDouble*)a->data : NULL;
}
double* mxGetDoubles(const mxArray* a) { return (a && a->cls == mxDOUBLE_CLASS && !a->cplx) ? (double*)a->data : NULL; }
int* mxGetInt32s(const mxArray* a) { return (a && a->cls == mxINT32_CLASS && !a->cplx) ? (int*)a->data : NULL; }
short* mxGetInt16s(const mxArray* a) { return (a && a->cls == mxINT16_CLASS && !a->cplx) ? (short*)a->data : NULL; }
mxLogical* mxGetLogicals(const mxArray* a) { return (a && a->cls == mxLOGICAL_CLASS) ? (mxLogical*)a->data : NULL; }
mwSize mxGetNumberOfDimensions(const mxArray* a) { return a ? a->ndim : 0; }
const mwSize* mxGetDimensions(const mxArray* a) { return a ? a->dims : NULL; }
size_t mxGetNumberOfElements(const mxArray* a) { return a ? a->n : 0; }
int mxIsComplex(const mxArray* a) { return a ? a->cplx : 0; }
int mxIsDouble(const mxArray* a) { return a ? a->cls == mxDOUBLE_CLASS : 0; }
mxClassID mxGetClassID(const mxArray* a) { return a ? a->cls : mxUNKNOWN_CLASS; }

mxArray* mxCreateNumericArray(mwSize ndim, const mwSize* dims, mxClassID cls, mxComplexity cplx) {
  return mxstub_new((int)cls, cplx == mxCOMPLEX, (int)ndim, dims);
}
mxArray* mxCreateUninitNumericArray(mwSize ndim, size_t* dims, mxClassID cls, mxComplexity cplx) {
  return mxstub_new((int)cls, cplx == mxCOMPLEX, (int)ndim, dims);
}
mxArray* mxCreateCellArray(mwSize ndim, const mwSize* dims) { return mxstub_new(mxCELL_CLASS, 0, (int)ndim, dims); }
void mxSetCell(mxArray* a, mwIndex i, mxArray* v) {
  if (a && a->cls == mxCELL_CLASS && i < a->n) ((mxArray**)a->data)[i] = v;
}
mxArray* mxGetCell(const mxArray* a, mwIndex i) {
  return (a && a->cls == mxCELL_CLASS && i < a->n) ? ((mxArray**)a->data)[i] : NULL;
}

double mxGetScalar(const mxArray* a) {
  if (!a || a->n == 0) return 0.0;
  switch (a->cls) {
    case mxDOUBLE_CLASS: return ((double*)a->data)[0];
    case mxSINGLE_CLASS: return ((float*)a->data)[0];
    case mxINT32_CLASS: return ((int32_t*)a->data)[0];
    case mxUINT32_CLASS: return ((uint32_t*)a->data)[0];
    case mxINT16_CLASS: return ((int16_t*)a->data)[0];
    case mxINT64_CLASS: return (double)((int64_t*)a->data)[0];
    case mxLOGICAL_CLASS: return ((mxLogical*)a->data)[0] ? 1.0 : 0.0;
    default: return ((unsigned char*)a->data)[0];
  }
}

void* mxMalloc(size_t n) { return malloc(n ? n : 1); }
void* mxCalloc(size_t n, size_t size) { return calloc(n ? n : 1, size ? size : 1); }
void mxFree(void* p) { free(p); }
