/*
 * MEX gateways that put libhp.so in place of the reference's CUDA MEX files.
 * Compile once per gateway (MATLAB resolves a MEX by file name):
 *
 *   mex -R2018a -DHP_MEX_PROPAGATE3 -output pendulum_propagate         hp_mex.c -I<repo>/include -L<pkg> -lhp
 *   mex -R2018a -DHP_MEX_PROPAGATE3 -DHP_MEX_MIXED -output pendulum_propagate32 hp_mex.c ...
 *   mex -R2018a -DHP_MEX_PROPAGATE2 -output pendulum_propagate_reduced hp_mex.c ...
 *   mex -R2018a -DHP_MEX_FFTSO3R    -output fftSO3R_mex                hp_mex.c ...
 *   mex -R2018a -DHP_MEX_GYROBIAS   -output gyrobias_propagate         hp_mex.c ...
 *   mex -R2018a -DHP_MEX_PROPAGATE_DEN -output pendulum_propagate_reduced_den hp_mex.c ...
 *   mex -R2018a -DHP_MEX_DISCRETE   -output pendulum_reduced_discrete_propagate hp_mex.c ...
 *   mex -R2018a -DHP_MEX_GETLAMBDA  -output getLambda_mex              hp_mex.c ...
 *   mex -R2018a -DHP_MEX_GETOMEGA   -output getOmega_mex               hp_mex.c ...
 *   mex -R2018a -DHP_MEX_GETFCL     -output getFcL_mex                 hp_mex.c ...
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
 *   Fnew = pendulum_propagate_reduced_den(F,f,X,mR,bt,G,dt,L,u,d,w,method)
 *          (propagation/mex/sources/pendulum_propagate_reduced_den/kernel.cu:8-77)
 *   df = pendulum_reduced_discrete_propagate(true,f,lambda,indR,fcL,fcL_indx)
 *   [lambda,indR,PC] = getLambda_mex(R,x,d,h,r,theta_t,lambda_max,false)
 *   Omega_new = getOmega_mex(R,x,indR,epsilon,PC,'new')
 *   [fcL,fcL_indx] = getFcL_mex(x,Omega_new,lambda,Gd,nD)
 *          (propagation/discrete/mex/sources/pendulum_reduced_collision/src/
 *           mexPropagate.cpp:6-77, mexLambda.cpp:7-99, mexOmega.cpp:5-34,
 *           mexFcL.cpp:6-35; callers pendulum_reduced_hybrid.m:130-141, 228-232)
 * u, CG, d and w are accepted and ignored: the library builds the same tables on
 * the device.  X is taken as fftn of the uniform grid of period L; OJO is reduced
 * to the diagonal-J coefficients (g1 x2 x3, g2 x1 x3, g3 x1 x2) by an inverse
 * DFT and a least-squares fit.  Plans are cached across calls and destroyed at exit.
 * The collision gateways read B from R (or f) and the omega grid (Bx, period L =
 * -2 x(1,1,1)) from x, and check that R is the Euler-angle grid of
 * fftSO3R.m:26-47 and x the uniform grid of pendulum_reduced_hybrid.m:60-68,
 * since the library rebuilds both on the device.  The noise-free forms
 * (getLambda_mex(...,true), getOmega_mex(...,'old'),
 * pendulum_reduced_discrete_propagate(false,...)) of the discrete-only study
 * pendulum_reduced_collision.m are not provided.
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

#if defined(HP_MEX_PROPAGATE3) || defined(HP_MEX_PROPAGATE2) || defined(HP_MEX_PROPAGATE_DEN)
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
#endif

#if defined(HP_MEX_PROPAGATE3) || defined(HP_MEX_GYROBIAS)
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

#if defined(HP_MEX_PROPAGATE3)
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
#endif

#if defined(HP_MEX_PROPAGATE3) || defined(HP_MEX_PROPAGATE2)
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

#if defined(HP_MEX_GETLAMBDA) || defined(HP_MEX_GETOMEGA) || defined(HP_MEX_GETFCL)
/* Omega grid (n components, 2Bx points per axis) from x(n, 2Bx, 2Bx[, 2Bx]):
 * returns ndim and sets Bx and L; errors unless x is the uniform grid. */
static int grid_of(const mxArray* xa, int* Bx, double* L) {
  const mwSize nd = mxGetNumberOfDimensions(xa);
  const mwSize* dims = mxGetDimensions(xa);
  const double* x = mxGetDoubles(xa);
  if (!x || nd < 3 || (int)dims[0] != (int)nd - 1 || (dims[0] != 2 && dims[0] != 3))
    mexErrMsgIdAndTxt("hp:x", "x must be a real (n, 2Bx, 2Bx[, 2Bx]) grid with n = 2 or 3");
  const int n = (int)dims[0], N = (int)dims[1];
  *Bx = N / 2;
  *L = -2.0 * x[0];
  size_t tot = 1;
  for (int a = 1; a <= n; ++a) tot *= (size_t)N;
  for (size_t e = 0; e < tot; ++e) {
    size_t r = e;
    for (int a = 0; a < n; ++a, r /= (size_t)N) {
      const double want = -*L / 2 + *L * (double)(r % (size_t)N) / N;
      if (fabs(x[e * n + a] - want) > 1e-9 * (*L > 1 ? *L : 1))
        mexErrMsgIdAndTxt("hp:x", "x must be the uniform grid -L/2 + L*(0:2Bx-1)/(2Bx) on every axis");
    }
  }
  return n;
}
#endif

#if defined(HP_MEX_GETLAMBDA) || defined(HP_MEX_GETOMEGA)
/* B from R(3, 3, 2B, 2B, 2B); errors unless R(:,:,a,b,c) = Rz(pi a/B) Ry(pi (2b+1)/(4B)) Rz(pi c/B). */
static int bandlimit_of_R(const mxArray* Ra) {
  const mwSize* dims = mxGetDimensions(Ra);
  const double* R = mxGetDoubles(Ra);
  if (!R || mxGetNumberOfDimensions(Ra) != 5 || dims[0] != 3 || dims[1] != 3 || dims[2] != dims[3] || dims[2] != dims[4])
    mexErrMsgIdAndTxt("hp:R", "R must be a real (3, 3, 2B, 2B, 2B) array of rotations");
  const int n = (int)dims[2], B = n / 2;
  for (int c = 0; c < n; ++c)
    for (int b = 0; b < n; ++b)
      for (int a = 0; a < n; ++a) {
        const double al = M_PI / B * a, be = M_PI / (4.0 * B) * (2 * b + 1), ga = M_PI / B * c;
        const double ca = cos(al), sa = sin(al), cb = cos(be), sb = sin(be), cg = cos(ga), sg = sin(ga);
        const double T[3][3] = {{ca * cb, -sa, ca * sb}, {sa * cb, ca, sa * sb}, {-sb, 0, cb}};
        const double* r = R + 9 * ((size_t)a + (size_t)n * ((size_t)b + (size_t)n * c));
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j) {
            const double want = T[i][0] * (j == 0 ? cg : (j == 1 ? -sg : 0)) +
                                T[i][1] * (j == 0 ? sg : (j == 1 ? cg : 0)) + T[i][2] * (j == 2 ? 1 : 0);
            if (fabs(r[i + 3 * j] - want) > 1e-9)
              mexErrMsgIdAndTxt("hp:R", "R must be the Euler-angle grid of fftSO3R.m (Rz(alpha) Ry(beta) Rz(gamma))");
          }
      }
  return B;
}
#endif

#ifdef HP_MEX_GETLAMBDA
void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  if (nrhs != 8) mexErrMsgIdAndTxt("hp:nrhs", "expected 8 inputs (R,x,d,h,r,theta_t,lambda_max,compact)");
  const int B = bandlimit_of_R(prhs[0]);
  int Bx;
  hp_collision_params prm;
  memset(&prm, 0, sizeof prm);
  const int ndim = grid_of(prhs[1], &Bx, &prm.L);
  prm.d = mxGetScalar(prhs[2]);
  prm.h = mxGetScalar(prhs[3]);
  prm.r = mxGetScalar(prhs[4]);
  prm.theta_t = mxGetScalar(prhs[5]);
  prm.lambda_max = mxGetScalar(prhs[6]);
  prm.nD = 1;
  if (mxGetScalar(prhs[7]) != 0.0)
    mexErrMsgIdAndTxt("hp:compact", "the compact form (lambda_indx cells of the noise-free model) is not provided");
  hp_plan* p = plan_for(B, Bx, ndim, HP_FP64, HP_REAL);
  int numR = 0;
  check(hp_collision_lambda(p, &prm, &numR, NULL, NULL, NULL, HP_HOST));
  size_t ld[4] = {(size_t)numR, (size_t)(2 * Bx), (size_t)(2 * Bx), (size_t)(2 * Bx)};
  size_t id[2] = {(size_t)numR, 1};
  size_t pd[4] = {3, (size_t)(2 * B), (size_t)(2 * B), (size_t)(2 * B)};
  plhs[0] = mxCreateUninitNumericArray((mwSize)(1 + ndim), ld, mxDOUBLE_CLASS, mxREAL);
  plhs[1] = mxCreateUninitNumericArray(2, id, mxINT32_CLASS, mxREAL);
  plhs[2] = mxCreateUninitNumericArray(4, pd, mxDOUBLE_CLASS, mxREAL);
  int numR2 = 0;
  check(hp_collision_lambda(p, &prm, &numR2, mxGetDoubles(plhs[0]), mxGetInt32s(plhs[1]), mxGetDoubles(plhs[2]),
                            HP_HOST));
  if (numR2 != numR) mexErrMsgIdAndTxt("hp:lambda", "colliding attitudes changed between calls");
  (void)nlhs;
}
#endif

#ifdef HP_MEX_GETOMEGA
void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  char dir[8];
  if (nrhs != 6) mexErrMsgIdAndTxt("hp:nrhs", "expected 6 inputs (R,x,indR,epsilon,PC,direction)");
  if (mxGetString(prhs[5], dir, sizeof dir)) mexErrMsgIdAndTxt("hp:direction", "direction must be a string");
  for (char* c = dir; *c; ++c) if (*c >= 'A' && *c <= 'Z') *c += 32;
  if (strcmp(dir, "new"))
    mexErrMsgIdAndTxt("hp:direction", "only the 'new' direction (the reset map of the hybrid model) is provided");
  const int B = bandlimit_of_R(prhs[0]);
  int Bx;
  hp_collision_params prm;
  memset(&prm, 0, sizeof prm);
  const int ndim = grid_of(prhs[1], &Bx, &prm.L);
  const int* indR = mxGetInt32s(prhs[2]);
  if (!indR) mexErrMsgIdAndTxt("hp:indR", "indR must be int32");
  const int numR = (int)mxGetNumberOfElements(prhs[2]);
  prm.epsilon = mxGetScalar(prhs[3]);
  hp_plan* p = plan_for(B, Bx, ndim, HP_FP64, HP_REAL);
  size_t od[5] = {(size_t)ndim, (size_t)numR, (size_t)(2 * Bx), (size_t)(2 * Bx), (size_t)(2 * Bx)};
  plhs[0] = mxCreateUninitNumericArray((mwSize)(2 + ndim), od, mxDOUBLE_CLASS, mxREAL);
  check(hp_collision_omega(p, &prm, numR, indR, mxGetDoubles(plhs[0]), HP_HOST));
  (void)nlhs;
}
#endif

#ifdef HP_MEX_GETFCL
void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  if (nrhs != 5) mexErrMsgIdAndTxt("hp:nrhs", "expected 5 inputs (x,Omega,lambda,Gd,nD)");
  int Bx;
  hp_collision_params prm;
  memset(&prm, 0, sizeof prm);
  const int ndim = grid_of(prhs[0], &Bx, &prm.L);
  const mxArray* Om = prhs[1];
  const mwSize* odims = mxGetDimensions(Om);
  if (!mxGetDoubles(Om) || mxGetNumberOfDimensions(Om) != (mwSize)(2 + ndim) || (int)odims[0] != ndim)
    mexErrMsgIdAndTxt("hp:Omega", "Omega must be a real (n, numR, 2Bx, 2Bx[, 2Bx]) array");
  const int numR = (int)odims[1];
  if (!mxGetDoubles(prhs[2]) || mxGetNumberOfElements(prhs[2]) != mxGetNumberOfElements(Om) / (size_t)ndim)
    mexErrMsgIdAndTxt("hp:lambda", "lambda must be a real (numR, 2Bx, 2Bx[, 2Bx]) array");
  const double* Gd = mxGetDoubles(prhs[3]);
  if (!Gd || mxGetNumberOfElements(prhs[3]) != (size_t)(ndim * ndim)) mexErrMsgIdAndTxt("hp:Gd", "Gd must be n x n");
  for (int i = 0; i < ndim * ndim; ++i) prm.Gd[i] = Gd[i];
  prm.nD = (int)mxGetScalar(prhs[4]);
  /* the taps do not depend on the SO(3) grid: the smallest plan carries the omega grid */
  hp_plan* p = plan_for(2, Bx, ndim, HP_FP64, HP_REAL);
  size_t fd[5] = {(size_t)prm.nD, (size_t)numR, (size_t)(2 * Bx), (size_t)(2 * Bx), (size_t)(2 * Bx)};
  plhs[0] = mxCreateUninitNumericArray((mwSize)(2 + ndim), fd, mxDOUBLE_CLASS, mxREAL);
  plhs[1] = mxCreateUninitNumericArray((mwSize)(2 + ndim), fd, mxINT16_CLASS, mxREAL);
  check(hp_collision_fcL(p, &prm, numR, mxGetDoubles(Om), mxGetDoubles(prhs[2]), mxGetDoubles(plhs[0]),
                         mxGetInt16s(plhs[1]), HP_HOST));
  (void)nlhs;
}
#endif

#ifdef HP_MEX_DISCRETE
/* The tables are copied to the device on every call, as the reference MEX
 * does; hp_state_hybrid_step keeps them resident instead. */
void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  if (nrhs != 6) mexErrMsgIdAndTxt("hp:nrhs", "expected 6 inputs (true,f,lambda,indR,fcL,fcL_indx)");
  if (mxGetScalar(prhs[0]) == 0.0)
    mexErrMsgIdAndTxt("hp:noise", "only the noisy form (true, ..., fcL, fcL_indx) of the hybrid model is provided");
  const mxArray* f = prhs[1];
  const mwSize nd = mxGetNumberOfDimensions(f);
  const mwSize* dims = mxGetDimensions(f);
  if (!mxGetDoubles(f) || (nd != 5 && nd != 6)) mexErrMsgIdAndTxt("hp:f", "f must be a real (2B,2B,2B,2Bx,2Bx[,2Bx]) array");
  const int B = (int)dims[0] / 2, Bx = (int)dims[3] / 2, ndim = (int)nd - 3;
  const int numR = (int)mxGetDimensions(prhs[2])[0];
  const mwSize* fdims = mxGetDimensions(prhs[4]);
  const int nD = (int)fdims[0];
  if (!mxGetDoubles(prhs[2]) || !mxGetInt32s(prhs[3]) || !mxGetDoubles(prhs[4]) || !mxGetInt16s(prhs[5]) ||
      (int)mxGetNumberOfElements(prhs[3]) != numR ||
      mxGetNumberOfElements(prhs[5]) != mxGetNumberOfElements(prhs[4]) ||
      mxGetNumberOfElements(prhs[4]) != (size_t)nD * mxGetNumberOfElements(prhs[2]))
    mexErrMsgIdAndTxt("hp:tables", "lambda (double), indR (int32), fcL (double), fcL_indx (int16) disagree in size");
  hp_plan* p = plan_for(B, Bx, ndim, HP_FP64, HP_REAL);
  hp_collision* c = NULL;
  check(hp_collision_create_from_tables(p, numR, nD, mxGetInt32s(prhs[3]), mxGetDoubles(prhs[2]),
                                        mxGetDoubles(prhs[4]), mxGetInt16s(prhs[5]), HP_HOST, &c));
  plhs[0] = mxCreateUninitNumericArray(nd, (size_t*)dims, mxDOUBLE_CLASS, mxREAL);
  const int st = hp_collision_df(c, mxGetDoubles(f), mxGetDoubles(plhs[0]), HP_HOST);
  hp_collision_destroy(c);
  check(st);
  (void)nlhs;
}
#endif

#ifdef HP_MEX_PROPAGATE_DEN
void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  if (nrhs != 12) mexErrMsgIdAndTxt("hp:nrhs", "expected 12 inputs (F,f,X,mR,bt,G,dt,L,u,d,w,method)");
  const mxArray* F = prhs[0];
  if (!mxIsComplex(F) || !mxIsDouble(F) || mxGetNumberOfDimensions(F) != 5)
    mexErrMsgIdAndTxt("hp:F", "F must be complex double (2lmax+1,2lmax+1,lmax+1,2Bx,2Bx)");
  const mwSize* dims = mxGetDimensions(F);
  const int B = (int)dims[2], Bx = (int)dims[3] / 2;
  const double* f = mxGetDoubles(prhs[1]);
  if (!f || mxGetNumberOfElements(prhs[1]) != (size_t)8 * B * B * B * 4 * Bx * Bx)
    mexErrMsgIdAndTxt("hp:f", "f must be the real (2B,2B,2B,2Bx,2Bx) density of F");
  const double* mR = mxGetDoubles(prhs[3]);
  if (!mR || mxGetNumberOfElements(prhs[3]) != (size_t)2 * 8 * B * B * B)
    mexErrMsgIdAndTxt("hp:mR", "mR must be a real (2,2B,2B,2B) array");
  hp_plan* p = plan_for(B, Bx, 2, HP_MEX_PRECISION, HP_REAL);
  hp_model m;
  memset(&m, 0, sizeof m);
  m.L = mxGetScalar(prhs[7]);
  const double* b = mxGetDoubles(prhs[4]);
  const double* G = mxGetDoubles(prhs[5]);
  if (!b || !G) mexErrMsgIdAndTxt("hp:model", "bt and G must be real");
  for (int i = 0; i < 2; ++i) {
    m.b[i] = b[i];
    for (int j = 0; j < 2; ++j) m.G[i * 3 + j] = G[i + 2 * j];   /* column-major in MATLAB */
  }
  check(hp_plan_set_den_model(p, &m, mR, HP_HOST));
  plhs[0] = mxCreateUninitNumericArray(5, (size_t*)dims, mxDOUBLE_CLASS, mxCOMPLEX);
  check(hp_pendulum_propagate_den(p, (const double*)mxGetComplexDoubles(F), f, (double*)mxGetComplexDoubles(plhs[0]),
                                  mxGetScalar(prhs[6]), method_code(prhs[11]), HP_HOST));
  (void)nlhs;
}
#endif
