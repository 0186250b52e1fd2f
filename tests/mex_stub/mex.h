/* Declarations of the MATLAB MEX C API (R2018a interleaved-complex API) that
 * the gateway in hybridpendulum-up_b200/mex/hp_mex.c uses, written from the
 * public API reference so the gateway can be compile-checked where MATLAB is
 * not installed.  Declarations only: nothing here is linked or run. */
#ifndef HP_TEST_MEX_STUB_H
#define HP_TEST_MEX_STUB_H
#include <stddef.h>

typedef struct mxArray_tag mxArray;
typedef size_t mwSize;
typedef struct { double real, imag; } mxComplexDouble;
typedef enum { mxUNKNOWN_CLASS = 0, mxDOUBLE_CLASS = 6 } mxClassID;
typedef enum { mxREAL = 0, mxCOMPLEX = 1 } mxComplexity;

void mexErrMsgIdAndTxt(const char* id, const char* fmt, ...);
int mexAtExit(void (*fn)(void));
int mxGetString(const mxArray* a, char* buf, mwSize len);
mxComplexDouble* mxGetComplexDoubles(const mxArray* a);
double* mxGetDoubles(const mxArray* a);
mwSize mxGetNumberOfDimensions(const mxArray* a);
const mwSize* mxGetDimensions(const mxArray* a);
int mxIsComplex(const mxArray* a);
int mxIsDouble(const mxArray* a);
mxArray* mxCreateUninitNumericArray(mwSize ndim, size_t* dims, mxClassID cls, mxComplexity cplx);
double mxGetScalar(const mxArray* a);
void* mxMalloc(size_t n);
void mxFree(void* p);
#endif
