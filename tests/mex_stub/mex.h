/* The part of the MATLAB MEX C API (R2018a interleaved-complex API) that the
 * gateways in hybridpendulum-up_b200/mex/hp_mex.c and the reference's MEX
 * sources use, written from the public API reference.  MATLAB is not installed
 * on the build or GPU machines, so tests/mex_stub/mx_runtime.c implements these
 * functions over plain host memory: tests build a gateway against it, call its
 * mexFunction through ctypes and read the outputs back.  Test infrastructure
 * only; nothing in the library links it. */
#ifndef HP_TEST_MEX_STUB_H
#define HP_TEST_MEX_STUB_H
#include <stddef.h>
#ifndef __cplusplus
#include <stdbool.h>
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef struct mxArray_tag mxArray;
typedef size_t mwSize;
typedef size_t mwIndex;
typedef bool mxLogical;
typedef struct { double real, imag; } mxComplexDouble;
/* class ids of the public matrix.h */
typedef enum {
  mxUNKNOWN_CLASS = 0, mxCELL_CLASS = 1, mxSTRUCT_CLASS = 2, mxLOGICAL_CLASS = 3, mxCHAR_CLASS = 4,
  mxVOID_CLASS = 5, mxDOUBLE_CLASS = 6, mxSINGLE_CLASS = 7, mxINT8_CLASS = 8, mxUINT8_CLASS = 9,
  mxINT16_CLASS = 10, mxUINT16_CLASS = 11, mxINT32_CLASS = 12, mxUINT32_CLASS = 13, mxINT64_CLASS = 14,
  mxUINT64_CLASS = 15
} mxClassID;
typedef enum { mxREAL = 0, mxCOMPLEX = 1 } mxComplexity;

/* the gateway every MEX file defines (C linkage, as MATLAB looks it up by name) */
void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]);
void mexErrMsgIdAndTxt(const char* id, const char* fmt, ...);
int mexAtExit(void (*fn)(void));
int mxGetString(const mxArray* a, char* buf, mwSize len);
char* mxArrayToString(const mxArray* a);
mxComplexDouble* mxGetComplexDoubles(const mxArray* a);
double* mxGetDoubles(const mxArray* a);
int* mxGetInt32s(const mxArray* a);
short* mxGetInt16s(const mxArray* a);
mxLogical* mxGetLogicals(const mxArray* a);
mwSize mxGetNumberOfDimensions(const mxArray* a);
const mwSize* mxGetDimensions(const mxArray* a);
size_t mxGetNumberOfElements(const mxArray* a);
int mxIsComplex(const mxArray* a);
int mxIsDouble(const mxArray* a);
mxClassID mxGetClassID(const mxArray* a);
mxArray* mxCreateUninitNumericArray(mwSize ndim, size_t* dims, mxClassID cls, mxComplexity cplx);
mxArray* mxCreateNumericArray(mwSize ndim, const mwSize* dims, mxClassID cls, mxComplexity cplx);
mxArray* mxCreateCellArray(mwSize ndim, const mwSize* dims);
void mxSetCell(mxArray* a, mwIndex i, mxArray* v);
mxArray* mxGetCell(const mxArray* a, mwIndex i);
double mxGetScalar(const mxArray* a);
void* mxMalloc(size_t n);
void* mxCalloc(size_t n, size_t size);
void mxFree(void* p);

#ifdef __cplusplus
}
#endif
#endif
