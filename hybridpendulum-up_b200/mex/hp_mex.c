/*
 * MEX gateways that put libhp.so in place of the reference's CUDA MEX files.
 * Compile once per gateway (MATLAB resolves a MEX by file name):
 *
 *   mex -R2018a -DHP_MEX_PROPAGATE3 -output pendulum_propagate         hp_mex.c -I<repo>/include -L<pkg> -lhp
 *   mex -R2018a -DHP_MEX_PROPAGATE3 -DHP_MEX_MIXED -output pendulum_propagate32 hp_mex.c ...
 *   mex -R2018a -DHP_MEX_PROPAGATE2 -output pendulum_propagate_reduced hp_mex.c ...
 *   mex -R2018a -DHP_MEX_FFTSO3R    -output fftSO3R_mex                hp_mex.c ...
 *   mex -R2018a -DHP_MEX_GYROBIAS   -output gyrobias_propagate         hp_mex.c ...
 *
 * Signatures (unchanged from the reference):
 *   Fnew = pendulum_propagate(F,X,OJO,MR,bt,G,dt,L,u,CG,method)
 *          (propagation/mex/sources/pendulum_propagate/kernel.cu:16-76)
 *   Fnew = pendulum_propagate_reduced(F,X,MR,bt,G,dt,L,u,CG,method)
 *          (propagation/mex/sources/pendulum_propagate_reduced/kernel.cu:16-74)
 *   F = fftSO3R_mex('forward',f,d,w) ; f = fftSO3R_mex('backward',F,d)
 *          (propagation/mex/sources/fftSO3R/kernel.cu:8-19, 197-202)
 *   Fnew = gyrobias_propagate(F,X,dt,u,G1,G2)
 *          (propagation/mex/sources/gyrobias_propagate/kernel.cu:8-130)
 * u, CG, d and w are accepted and ignored: the library builds the same tables on
 * the device.  X is taken as fftn of the uniform grid of period L; OJO is reduced
 * to the diagonal-J coefficients (g1 x2 x3, g2 x1 x3, g3 x1 x2) by an inverse
 * DFT and a least-squares fit.  Plans are cached across calls and destroyed at exit.
 */
#include <math.h>
#include <string.h>
#include "mex.h"
#include "hp.h"

#ifndef M_PI   /* not in strict ISO C */
#define M_PI 3.14159265358979323846
#endif

#ifdef HP_MEX_MIXED
#define HP_MEX_PRECISION HP_MIXED
#else
#define HP_MEX_PRECISION HP_FP64
#endif

static hp_plan* g_plan = NULL;
static int g_key[5] = {0, 0, 0, 0, -1};

static void cleanup(void) {
  if (g_plan) hp_plan_destroy(g_plan);
  g_plan = NULL;
}

static void check(int st) {
  if (st != HP_OK) mexErrMsgIdAndTxt("hp:error", "libhp error %d: %s", st, hp_last_error());
}

static hp_plan* plan_for(int B, int Bx, int ndim, int precision, int symmetry) {
  const int key[5] = {B, Bx, ndim, precision, symmetry};
  if (g_plan && memcmp(key, g_key, sizeof key) == 0) return g_plan;
  cleanup();
  check(hp_plan_create(&g_plan, B, Bx, ndim, precision, symmetry));
  memcpy(g_key, key, sizeof key);
  mexAtExit(cleanup);
  return g_plan;
}

static int method_code(const mxArray* a) {
  char buf[16];
  if (mxGetString(a, buf, sizeof buf)) mexErrMsgIdAndTxt("hp:method", "method must be a string");
  for (char* c = buf; *c; ++c) if (*c >= 'A' && *c <= 'Z') *c += 32;
  if (!strcmp(buf, "euler")) return HP_EULER;
  if (!strcmp(buf, "midpoint")) return HP_MIDPOINT;
  if (!strcmp(buf, "rk2")) return HP_RK2;
  if (!strcmp(buf, "rk4")) return HP_RK4;
  mexErrMsgIdAndTxt("hp:method", "'method' must be one of 'euler','midpoint','RK2','RK4'");
  return -1;
}

#if defined(HP_MEX_PROPAGATE3) || defined(HP_MEX_PROPAGATE2) || defined(HP_MEX_GYROBIAS)
/* ifftn of one N^3 component by separable 1-D inverse DFTs (real part kept). */
static void ifft3_real(const mxComplexDouble* X, int N, double* out) {
  const size_t n3 = (size_t)N * N * N;
  double* re = mxMalloc(sizeof(double) * n3);
  double* im = mxMalloc(sizeof(double) * n3);
  double* tr = mxMalloc(sizeof(double) * N);
  double* ti = mxMalloc(sizeof(double) * N);
  for (size_t i = 0; i < n3; ++i) { re[i] = X[i].real; im[i] = X[i].imag; }
  size_t stride = 1;
  for (int axis = 0; axis < 3; ++axis, stride *= N) {
    for (size_t base = 0; base < n3; ++base) {
      if ((base / stride) % N) continue;                /* first element of each line */
      for (int k = 0; k < N; ++k) {
        double sr = 0, si = 0;
        for (int j = 0; j < N; ++j) {
          const double a = 2 * M_PI * (double)j * k / N, c = cos(a), s = sin(a);
          const size_t o = base + (size_t)j * stride;
          sr += re[o] * c - im[o] * s;
          si += re[o] * s + im[o] * c;
        }
        tr[k] = sr / N;
        ti[k] = si / N;
      }
      for (int k = 0; k < N; ++k) { re[base + (size_t)k * stride] = tr[k]; im[base + (size_t)k * stride] = ti[k]; }
    }
  }
  memcpy(out, re, sizeof(double) * n3);
  mxFree(re); mxFree(im); mxFree(tr); mxFree(ti);
}

#endif

#if defined(HP_MEX_PROPAGATE3) || defined(HP_MEX_PROPAGATE2)
/* (g1, g2, g3) with ifftn(OJO_i) = g_i * x_j * x_k on the grid x = -L/2 + L*idx/N. */
static void fit_gyro(const mxArray* OJO, int N, double L, double g[3]) {
  const size_t n3 = (size_t)N * N * N;
  const mxComplexDouble* O = mxGetComplexDoubles(OJO);
  if (!O) mexErrMsgIdAndTxt("hp:OJO", "OJO must be complex double");
  double* v = mxMalloc(sizeof(double) * n3);
  const int pj[3] = {1, 0, 0}, pk[3] = {2, 2, 1};
  for (int i = 0; i < 3; ++i) {
    ifft3_real(O + i * n3, N, v);
    double num = 0, den = 0, mx = 0;
    for (size_t e = 0; e < n3; ++e) {
      const int id[3] = {(int)(e % N), (int)((e / N) % N), (int)(e / N / N)};
      const double b = (-L / 2 + L * id[pj[i]] / N) * (-L / 2 + L * id[pk[i]] / N);
      num += v[e] * b;
      den += b * b;
      if (fabs(v[e]) > mx) mx = fabs(v[e]);
    }
    g[i] = den > 0 ? num / den : 0.0;
    for (size_t e = 0; e < n3; ++e) {
      const int id[3] = {(int)(e % N), (int)((e / N) % N), (int)(e / N / N)};
      const double b = (-L / 2 + L * id[pj[i]] / N) * (-L / 2 + L * id[pk[i]] / N);
      if (fabs(v[e] - g[i] * b) > 1e-8 * (mx > 1 ? mx : 1))
        mexErrMsgIdAndTxt("hp:OJO", "OJO is not of the diagonal-J form supported by libhp");
    }
  }
  mxFree(v);
}

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
#ifdef HP_MEX_PROPAGATE3
  const int ndim = 3, nexp = 11, iMR = 3, ib = 4, iG = 5, idt = 6, iL = 7, imeth = 10;
#else
  const int ndim = 2, nexp = 10, iMR = 2, ib = 3, iG = 4, idt = 5, iL = 6, imeth = 9;
#endif
  if (nrhs != nexp) mexErrMsgIdAndTxt("hp:nrhs", "expected %d inputs", nexp);
  const mxArray* F = prhs[0];
  if (!mxIsComplex(F) || !mxIsDouble(F)) mexErrMsgIdAndTxt("hp:F", "F must be complex double");
  const mwSize* dims = mxGetDimensions(F);
  if (mxGetNumberOfDimensions(F) != (mwSize)(3 + ndim)) mexErrMsgIdAndTxt("hp:F", "F has the wrong rank");
  const int B = (int)dims[2], Bx = (int)dims[3] / 2;
  hp_plan* p = plan_for(B, Bx, ndim, HP_MEX_PRECISION, HP_REAL);
  hp_model m;
  memset(&m, 0, sizeof m);
  m.L = mxGetScalar(prhs[iL]);
  const double* b = mxGetDoubles(prhs[ib]);
  const double* G = mxGetDoubles(prhs[iG]);
  for (int i = 0; i < ndim; ++i) {
    m.b[i] = b[i];
    for (int j = 0; j < ndim; ++j) m.G[i * 3 + j] = G[i + ndim * j];   /* column-major in MATLAB */
  }
#ifdef HP_MEX_PROPAGATE3
  fit_gyro(prhs[2], 2 * Bx, m.L, m.gyro);
#endif
  check(hp_plan_set_model(p, &m, (const double*)mxGetComplexDoubles(prhs[iMR]), HP_HOST));
  plhs[0] = mxCreateUninitNumericArray(mxGetNumberOfDimensions(F), (size_t*)dims, mxDOUBLE_CLASS, mxCOMPLEX);
  check(hp_pendulum_propagate(p, (const double*)mxGetComplexDoubles(F),
                              (double*)mxGetComplexDoubles(plhs[0]), mxGetScalar(prhs[idt]),
                              method_code(prhs[imeth]), HP_HOST));
  (void)nlhs;
}
#endif

#ifdef HP_MEX_FFTSO3R
void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  char dir[16];
  if (nrhs < 2 || mxGetString(prhs[0], dir, sizeof dir)) mexErrMsgIdAndTxt("hp:args", "fftSO3R_mex(direction, A, ...)");
  const mxArray* A = prhs[1];
  const mwSize nd = mxGetNumberOfDimensions(A);
  const mwSize* dims = mxGetDimensions(A);
  const int ndim = (int)nd - 3;
  if (!strcmp(dir, "forward")) {
    const int B = (int)dims[0] / 2, Bx = (int)dims[3] / 2;
    hp_plan* p = plan_for(B, Bx, ndim, HP_FP64, HP_REAL);
    mwSize od[6];
    od[0] = od[1] = 2 * B - 1; od[2] = B;
    for (int a = 0; a < ndim; ++a) od[3 + a] = 2 * Bx;
    plhs[0] = mxCreateUninitNumericArray(nd, od, mxDOUBLE_CLASS, mxCOMPLEX);
    check(hp_fftSO3R_forward(p, mxGetDoubles(A), (double*)mxGetComplexDoubles(plhs[0]), HP_HOST));
  } else if (!strcmp(dir, "backward")) {
    const int B = (int)dims[2], Bx = (int)dims[3] / 2;
    hp_plan* p = plan_for(B, Bx, ndim, HP_FP64, HP_REAL);
    mwSize od[6];
    od[0] = od[1] = od[2] = 2 * B;
    for (int a = 0; a < ndim; ++a) od[3 + a] = 2 * Bx;
    plhs[0] = mxCreateUninitNumericArray(nd, od, mxDOUBLE_CLASS, mxREAL);
    check(hp_fftSO3R_backward(p, (const double*)mxGetComplexDoubles(A), mxGetDoubles(plhs[0]), HP_HOST));
  } else {
    mexErrMsgIdAndTxt("hp:direction", "direction must be 'forward' or 'backward'");
  }
  (void)nlhs;
}
#endif

#ifdef HP_MEX_GYROBIAS
/* The bias grid period L is read off X = fftn(x) (gyro_bias.m:68-99): x_1 at
 * the first grid point is -L/2. */
void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  if (nrhs != 6) mexErrMsgIdAndTxt("hp:nrhs", "expected 6 inputs (F,X,dt,u,G1,G2)");
  const mxArray* F = prhs[0];
  if (!mxIsComplex(F) || !mxIsDouble(F)) mexErrMsgIdAndTxt("hp:F", "F must be complex double");
  if (mxGetNumberOfDimensions(F) != 6) mexErrMsgIdAndTxt("hp:F", "F has the wrong rank");
  const mwSize* dims = mxGetDimensions(F);
  const int B = (int)dims[2], Bx = (int)dims[3] / 2, N = 2 * Bx;
  const mxComplexDouble* X = mxGetComplexDoubles(prhs[1]);
  if (!X) mexErrMsgIdAndTxt("hp:X", "X must be complex double");
  double* x1 = mxMalloc(sizeof(double) * (size_t)N * N * N);
  ifft3_real(X, N, x1);
  const double L = -2.0 * x1[0];
  mxFree(x1);
  const double* G1 = mxGetDoubles(prhs[4]);
  const double* G2 = mxGetDoubles(prhs[5]);
  double g1[9], g2[9];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) { g1[i * 3 + j] = G1[i + 3 * j]; g2[i * 3 + j] = G2[i + 3 * j]; }
  hp_plan* p = plan_for(B, Bx, 3, HP_MEX_PRECISION, HP_REAL);
  check(hp_plan_set_gyro_bias_model(p, L, g1, g2));
  plhs[0] = mxCreateUninitNumericArray(6, (size_t*)dims, mxDOUBLE_CLASS, mxCOMPLEX);
  check(hp_gyrobias_propagate(p, (const double*)mxGetComplexDoubles(F), (double*)mxGetComplexDoubles(plhs[0]),
                              mxGetScalar(prhs[2]), HP_HOST));
  (void)nlhs;
}
#endif
