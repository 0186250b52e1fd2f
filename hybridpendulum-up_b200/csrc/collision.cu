// Hybrid collision operator of pendulum_reduced_hybrid (2-D reduced Omega,
// and its extension to a 3-D Omega grid):
// switching rate lambda(R, x), reset map Omega+, truncated Gaussian kernel fcL
// and the per-step update df = sum_d fcL f(R, idx) - lambda f (FP64, as the
// reference).  Follows propagation/discrete/mex/sources/pendulum_reduced_collision:
// getLambda.cu:8-85,192-267, getOmega.cu:64-103, getFcL.cu:11-166,
// propagate.cu:6-121,181-231.
//
// 3-D Omega (no reference counterpart: the reference builds the 2-D reduced
// model only, getOmega.cu:86-96 takes Omega = [x1, x2, 0]): the same
// kinematics with all three components, omega = R Omega, the reset acting on
// the (2, 3) components of omega as in 2-D, Omega+ = R^T omega+ in R^3 and a
// 3-D Gaussian of covariance Gd (3x3) for the landing kernel.
//
// Layouts (those of the reference MEX):
//   f, df         [ix][iR]      ix = i + 2Bx j (+ 4Bx^2 k), iR = a + 2B b + 4B^2 c
//   lambda        [ix][k]       k indexes the colliding attitudes indR
//   fcL, fcL_idx  [ix][k][d]    d < nD
#include <cmath>
#include <vector>
#include "common.cuh"
#include "plan.hpp"

using namespace hp;

struct CollisionTables {
  int numR = 0, nD = 0;
  int* indR = nullptr;        // [numR]
  double* lambda = nullptr;   // [nx][numR]
  double* omega = nullptr;    // [nx][numR][ndim]
  double* fcL = nullptr;      // [nx][numR][nD]
  short* idx = nullptr;       // [nx][numR][nD]
  double* PC = nullptr;       // [nR][3]
};

static CollisionTables g_dummy;

// R(:,:,a,b,c) = Rz(alpha_a) Ry(beta_b) Rz(gamma_c) as in fftSO3R.m:30-47.
__device__ __forceinline__ void rot_of(int iR, int B, double R[3][3]) {
  const int n = 2 * B;
  const int a = iR % n, b = (iR / n) % n, c = iR / (n * n);
  const double al = M_PI / B * a, be = M_PI / (4.0 * B) * (2 * b + 1), ga = M_PI / B * c;
  const double ca = cos(al), sa = sin(al), cb = cos(be), sb = sin(be), cg = cos(ga), sg = sin(ga);
  const double Ra[3][3] = {{ca, -sa, 0}, {sa, ca, 0}, {0, 0, 1}};
  const double Rb[3][3] = {{cb, 0, sb}, {0, 1, 0}, {-sb, 0, cb}};
  const double Rg[3][3] = {{cg, -sg, 0}, {sg, cg, 0}, {0, 0, 1}};
  double T[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) T[i][j] = Ra[i][0] * Rb[0][j] + Ra[i][1] * Rb[1][j] + Ra[i][2] * Rb[2][j];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) R[i][j] = T[i][0] * Rg[0][j] + T[i][1] * Rg[1][j] + T[i][2] * Rg[2][j];
}

// Category (0: none, 1: ramp, 2: full), theta = asin(R13) and PC per attitude.
__global__ void k_coll_theta(int B, int nR, double theta0, double thetat, double h, double r, char* cat,
                             double* theta, double* PC) {
  const int iR = blockIdx.x * blockDim.x + threadIdx.x;
  if (iR >= nR) return;
  double R[3][3];
  rot_of(iR, B, R);
  const double th = asin(R[0][2]);
  theta[iR] = th;
  cat[iR] = th < theta0 - thetat ? 0 : (th > theta0 + thetat ? 2 : 1);
  const double lr3 = h - r * tan(th);
  PC[3 * iR] = lr3 * R[0][2] + r / cos(th);
  PC[3 * iR + 1] = lr3 * R[1][2];
  PC[3 * iR + 2] = lr3 * R[2][2];
}

// lambda(ix, k) and Omega+(ix, k) for the colliding attitudes.
template <int NDIM>
__global__ void k_coll_lambda_omega(int B, int N, double L, int numR, const int* __restrict__ indR,
                                    const char* __restrict__ cat, const double* __restrict__ theta,
                                    const double* __restrict__ PC, double theta0, double thetat, double lmax,
                                    double eps, double* __restrict__ lambda, double* __restrict__ omega) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const int nx = NDIM == 3 ? N * N * N : N * N;
  if (t >= (long long)nx * numR) return;
  const int k = (int)(t % numR), ix = (int)(t / numR);
  const int iR = indR[k];
  double R[3][3];
  rot_of(iR, B, R);
  const double x1 = -L / 2 + L / N * (ix % N), x2 = -L / 2 + L / N * ((ix / N) % N);
  const double x3 = NDIM == 3 ? -L / 2 + L / N * (ix / (N * N)) : 0.0;
  double lam = cat[iR] == 2 ? lmax : lmax / 2 * sin(M_PI / (2 * thetat) * (theta[iR] - theta0)) + lmax / 2;
  if (cat[iR] == 0) lam = 0.0;
  // omega = R Omega (spatial angular velocity); contact-point velocity along
  // the wall normal, (omega x PC)_1.  PC's (2, 3) components are lr3 R e3's, so
  // the spin x3 R e3 about the pendulum axis drops out exactly: the velocity
  // is formed from x1, x2 alone, as in the 2-D model (with x3 it would be
  // rounding noise at x1 = x2 = 0, whose sign would pick lambda).
  const double v1 = R[1][0] * x1 + R[1][1] * x2, v2 = R[2][0] * x1 + R[2][1] * x2;
  const double vC = v1 * PC[3 * iR + 2] - v2 * PC[3 * iR + 1];
  lambda[t] = vC < 0.0 ? 0.0 : lam;
  const double w0 = R[0][0] * x1 + R[0][1] * x2 + R[0][2] * x3;
  double w1 = v1 + R[1][2] * x3;
  double w2 = v2 + R[2][2] * x3;
  // reset map
  const double nt = sqrt(R[1][2] * R[1][2] + R[2][2] * R[2][2]);
  const double t1 = R[2][2] / nt, t2 = -R[1][2] / nt;
  const double ot = (1.0 + eps) * (w1 * t1 + w2 * t2);
  w1 -= ot * t1;
  w2 -= ot * t2;
#pragma unroll
  for (int c = 0; c < NDIM; ++c) omega[NDIM * t + c] = R[0][c] * w0 + R[1][c] * w1 + R[2][c] * w2;
}

// inverse covariance (symmetric part) and normaliser of the landing Gaussian
struct GaussQ { double i00, i01, i02, i11, i12, i22, cn; };

// Largest nD Gaussian taps per (landing point ix1, attitude k), ties keeping the
// lower source index first (the stable descending sort of getFcL.cu:76).
template <int MAXD, int NDIM>
__global__ void k_coll_topd(int N, double L, int numR, int nD, const double* __restrict__ omega, GaussQ g,
                            double* __restrict__ fcL, short* __restrict__ idx) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const int nx = NDIM == 3 ? N * N * N : N * N;
  if (t >= (long long)nx * numR) return;
  const int k = (int)(t % numR), ix1 = (int)(t / numR);
  const double x1 = -L / 2 + L / N * (ix1 % N), x2 = -L / 2 + L / N * ((ix1 / N) % N);
  const double x3 = NDIM == 3 ? -L / 2 + L / N * (ix1 / (N * N)) : 0.0;
  double v[MAXD];
  int id[MAXD];
  int cnt = 0;
  for (int ix2 = 0; ix2 < nx; ++ix2) {
    const double* o = omega + NDIM * ((long long)ix2 * numR + k);
    const double d0 = x1 - o[0];
    const double d1 = x2 - o[1];
    double q = g.i00 * d0 * d0 + g.i01 * d0 * d1 + g.i11 * d1 * d1;
    if (NDIM == 3) {
      const double d2 = x3 - o[2];
      q += g.i02 * d0 * d2 + g.i12 * d1 * d2 + g.i22 * d2 * d2;
    }
    const double fc = exp(-0.5 * q) * g.cn;
    if (cnt < nD || fc > v[nD - 1]) {
      int p = cnt < nD ? cnt++ : nD - 1;      // insertion position from the end
      while (p > 0 && v[p - 1] < fc) {         // strict: equal values keep the earlier index first
        v[p] = v[p - 1];
        id[p] = id[p - 1];
        --p;
      }
      v[p] = fc;
      id[p] = ix2;
    }
  }
  for (int d = 0; d < nD; ++d) {
    fcL[t * nD + d] = d < cnt ? v[d] : 0.0;
    idx[t * nD + d] = (short)(d < cnt ? id[d] : 0);
  }
}

__global__ void k_coll_norm(int nx, int numR, int nD, const double* __restrict__ fcL, const short* __restrict__ idx,
                            double* __restrict__ norm) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)nx * numR * nD) return;
  const int k = (int)((t / nD) % numR);
  atomicAdd(&norm[(long long)idx[t] * numR + k], fcL[t]);
}

__global__ void k_coll_scale(int nx, int numR, int nD, double dxn, const double* __restrict__ norm,
                             const double* __restrict__ lambda, double* __restrict__ fcL, const short* __restrict__ idx) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)nx * numR * nD) return;
  const int k = (int)((t / nD) % numR);
  const long long src = (long long)idx[t] * numR + k;
  // a source whose every kept tap underflowed to 0 has norm 0: its taps stay 0
  // (the reference divides unguarded; its 2-D setups never reach 0/0)
  fcL[t] = norm[src] > 0.0 ? fcL[t] / (norm[src] * dxn) * (lambda[src] * dxn) : 0.0;
}

// df(R_k, x) = sum_d fcL f(R_k, idx) - lambda f(R_k, x); rows of non-colliding
// attitudes are left as the caller set them (zero).
template <typename T>
__global__ void k_coll_df(int nx, int nR, int numR, int nD, const int* __restrict__ indR,
                          const double* __restrict__ lambda, const double* __restrict__ fcL,
                          const short* __restrict__ idx, const T* __restrict__ f, T* __restrict__ df) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)nx * numR) return;
  const int k = (int)(t % numR), ix = (int)(t / numR);
  const int iR = indR[k];
  double s = 0.0;
  for (int d = 0; d < nD; ++d) s += fcL[t * nD + d] * (double)f[(long long)idx[t * nD + d] * nR + iR];
  df[(long long)ix * nR + iR] = (T)(s - lambda[t] * (double)f[(long long)ix * nR + iR]);
}

// f += dt * df(f) in place (pendulum_reduced_hybrid.m:232-233): the colliding
// columns are first gathered into fk[k][ix] so that every tap reads the
// pre-update density (k_coll_gather_t / k_coll_update_t below).

// --------------------------------------------------------------- C ABI ----
struct hp_collision {
  hp_plan* plan = nullptr;
  CollisionTables t;
  double L = 0;
  // the tables transposed to [k][d][ix] / [k][ix] in the plan's compute
  // precision, for the in-place update of the hybrid step (built on first use)
  void* fcLT = nullptr;
  short* idxT = nullptr;
  void* lamT = nullptr;
};

extern "C" int hp_collision_create(hp_plan* p, const hp_collision_params* prm, hp_collision** out, int* numR) {
  if (!p || !prm || !out) { hp_set_error("null argument"); return HP_ERR_INVALID; }
  *out = nullptr;
  if (prm->nD < 1 || prm->nD > 32) { hp_set_error("nD must be in 1..32"); return HP_ERR_INVALID; }
  if (!(prm->L > 0) || !(prm->theta_t > 0)) { hp_set_error("bad collision parameters"); return HP_ERR_INVALID; }
  const int B = p->B, N = p->N, nR = 8 * B * B * B, nx = (int)p->nx, nd = p->ndim;
  if (nx > 32768) { hp_set_error("the tap indices are 16-bit: at most 32768 omega points"); return HP_ERR_UNSUPPORTED; }
  cudaStream_t s = p->stream;
  const double hr = std::sqrt(prm->h * prm->h + prm->r * prm->r);
  const double theta0 = std::asin(prm->d / hr) - std::asin(prm->r / hr);
  char* cat = nullptr;
  double* theta = nullptr;
  hp_collision* c = new hp_collision();
  c->plan = p;
  c->L = prm->L;
  auto fail = [&](int code) { hp_collision_destroy(c); cudaFree(cat); cudaFree(theta); return code; };
  if (cudaMalloc(&cat, nR) != cudaSuccess || cudaMalloc(&theta, sizeof(double) * nR) != cudaSuccess ||
      cudaMalloc(&c->t.PC, sizeof(double) * 3 * nR) != cudaSuccess) {
    cudaGetLastError();
    hp_set_error("device allocation failed");
    return fail(HP_ERR_ALLOC);
  }
  {
    ProfScope _ps(p, "coll.setup", s);
    k_coll_theta<<<(nR + 127) / 128, 128, 0, s>>>(B, nR, theta0, prm->theta_t, prm->h, prm->r, cat, theta, c->t.PC);
  }
  std::vector<char> hc(nR);
  if (cudaMemcpyAsync(hc.data(), cat, nR, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess) {
    hp_set_error(cudaGetErrorString(cudaGetLastError()));
    return fail(HP_ERR_CUDA);
  }
  std::vector<int> hind;
  for (int i = 0; i < nR; ++i) if (hc[i] != 0) hind.push_back(i);
  const int nk = (int)hind.size();
  c->t.numR = nk;
  c->t.nD = prm->nD;
  if (numR) *numR = nk;
  if (nk == 0) { cudaFree(cat); cudaFree(theta); *out = c; return HP_OK; }
  const size_t nxk = (size_t)nx * nk;
  double* norm = nullptr;
  if (cudaMalloc(&c->t.indR, sizeof(int) * nk) != cudaSuccess ||
      cudaMalloc(&c->t.lambda, sizeof(double) * nxk) != cudaSuccess ||
      cudaMalloc(&c->t.omega, sizeof(double) * nd * nxk) != cudaSuccess ||
      cudaMalloc(&c->t.fcL, sizeof(double) * nxk * prm->nD) != cudaSuccess ||
      cudaMalloc(&c->t.idx, sizeof(short) * nxk * prm->nD) != cudaSuccess ||
      cudaMalloc(&norm, sizeof(double) * nxk) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(norm);
    hp_set_error("device allocation failed");
    return fail(HP_ERR_ALLOC);
  }
  HP_CUDA_TRY(cudaMemcpyAsync(c->t.indR, hind.data(), sizeof(int) * nk, cudaMemcpyHostToDevice, s));
  const unsigned g1 = (unsigned)((nxk + 127) / 128);
  {
    ProfScope _ps(p, "coll.setup", s);
    if (nd == 3)
      k_coll_lambda_omega<3><<<g1, 128, 0, s>>>(B, N, prm->L, nk, c->t.indR, cat, theta, c->t.PC, theta0, prm->theta_t,
                                                prm->lambda_max, prm->epsilon, c->t.lambda, c->t.omega);
    else
      k_coll_lambda_omega<2><<<g1, 128, 0, s>>>(B, N, prm->L, nk, c->t.indR, cat, theta, c->t.PC, theta0, prm->theta_t,
                                                prm->lambda_max, prm->epsilon, c->t.lambda, c->t.omega);
  }
  // Gaussian of covariance Gd (column-major nd x nd): q = d^T Gd^-1 d with the
  // cross terms of the symmetric part folded (i01 = (inv01 + inv10), ...)
  GaussQ g{};
  {
    const double* G = prm->Gd;
    double inv[3][3] = {}, det = 0;
    if (nd == 2) {
      const double g00 = G[0], g10 = G[1], g01 = G[2], g11 = G[3];
      det = g00 * g11 - g01 * g10;
      inv[0][0] = g11 / det; inv[0][1] = -g01 / det; inv[1][0] = -g10 / det; inv[1][1] = g00 / det;
    } else {
      auto at = [&](int i, int j) { return G[i + 3 * j]; };
      const double c00 = at(1, 1) * at(2, 2) - at(1, 2) * at(2, 1), c01 = at(1, 2) * at(2, 0) - at(1, 0) * at(2, 2),
                   c02 = at(1, 0) * at(2, 1) - at(1, 1) * at(2, 0);
      det = at(0, 0) * c00 + at(0, 1) * c01 + at(0, 2) * c02;
      // inverse = adjugate / det (adj[j][i] = cofactor[i][j])
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
          const int a0 = (j + 1) % 3, a1 = (j + 2) % 3, b0 = (i + 1) % 3, b1 = (i + 2) % 3;
          inv[i][j] = (at(a0, b0) * at(a1, b1) - at(a0, b1) * at(a1, b0)) / det;
        }
    }
    if (!(det > 0) || !std::isfinite(det)) { cudaFree(norm); hp_set_error("Gd must be positive definite"); return fail(HP_ERR_INVALID); }
    g.i00 = inv[0][0]; g.i01 = inv[0][1] + inv[1][0]; g.i11 = inv[1][1];
    g.i02 = inv[0][2] + inv[2][0]; g.i12 = inv[1][2] + inv[2][1]; g.i22 = inv[2][2];
    g.cn = 1.0 / (std::pow(2 * M_PI, 0.5 * nd) * std::sqrt(det));
  }
  {
    ProfScope _ps(p, "coll.setup", s);
    if (nd == 3) k_coll_topd<32, 3><<<g1, 128, 0, s>>>(N, prm->L, nk, prm->nD, c->t.omega, g, c->t.fcL, c->t.idx);
    else k_coll_topd<32, 2><<<g1, 128, 0, s>>>(N, prm->L, nk, prm->nD, c->t.omega, g, c->t.fcL, c->t.idx);
  }
  const double dx = prm->L / N, dx2 = nd == 3 ? dx * dx * dx : dx * dx;
  HP_CUDA_TRY(cudaMemsetAsync(norm, 0, sizeof(double) * nxk, s));
  const unsigned g2 = (unsigned)((nxk * prm->nD + 127) / 128);
  {
    ProfScope _ps(p, "coll.setup", s);
    k_coll_norm<<<g2, 128, 0, s>>>(nx, nk, prm->nD, c->t.fcL, c->t.idx, norm);
    k_coll_scale<<<g2, 128, 0, s>>>(nx, nk, prm->nD, dx2, norm, c->t.lambda, c->t.fcL, c->t.idx);
  }
  HP_CUDA_TRY(cudaGetLastError());
  HP_CUDA_TRY(cudaStreamSynchronize(s));
  cudaFree(norm);
  cudaFree(cat);
  cudaFree(theta);
  *out = c;
  return HP_OK;
}

extern "C" int hp_collision_destroy(hp_collision* c) {
  if (!c) return HP_OK;
  cudaFree(c->t.indR); cudaFree(c->t.lambda); cudaFree(c->t.omega); cudaFree(c->t.fcL);
  cudaFree(c->t.idx); cudaFree(c->t.PC);
  cudaFree(c->fcLT); cudaFree(c->idxT); cudaFree(c->lamT);
  delete c;
  return HP_OK;
}

extern "C" int hp_collision_tables(hp_collision* c, double* lambda, int* indR, double* omega, double* fcL,
                                   short* fcL_indx, double* PC, int mem) {
  if (!c) { hp_set_error("null argument"); return HP_ERR_INVALID; }
  if (mem != HP_DEVICE && mem != HP_HOST) { hp_set_error("bad mem"); return HP_ERR_INVALID; }
  hp_plan* p = c->plan;
  const cudaMemcpyKind kind = mem == HP_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
  const size_t nxk = (size_t)p->nx * c->t.numR;
  const int nR = 8 * p->B * p->B * p->B;
  if (lambda && nxk) HP_CUDA_TRY(cudaMemcpy(lambda, c->t.lambda, sizeof(double) * nxk, kind));
  if (indR && c->t.numR) HP_CUDA_TRY(cudaMemcpy(indR, c->t.indR, sizeof(int) * c->t.numR, kind));
  if (omega && nxk) HP_CUDA_TRY(cudaMemcpy(omega, c->t.omega, sizeof(double) * p->ndim * nxk, kind));
  if (fcL && nxk) HP_CUDA_TRY(cudaMemcpy(fcL, c->t.fcL, sizeof(double) * nxk * c->t.nD, kind));
  if (fcL_indx && nxk) HP_CUDA_TRY(cudaMemcpy(fcL_indx, c->t.idx, sizeof(short) * nxk * c->t.nD, kind));
  if (PC) HP_CUDA_TRY(cudaMemcpy(PC, c->t.PC, sizeof(double) * 3 * nR, kind));
  return HP_OK;
}

extern "C" int hp_collision_df(hp_collision* c, const double* f, double* df, int mem) {
  if (!c || !f || !df) { hp_set_error("null argument"); return HP_ERR_INVALID; }
  if (mem != HP_DEVICE && mem != HP_HOST) { hp_set_error("bad mem"); return HP_ERR_INVALID; }
  hp_plan* p = c->plan;
  const long long nR = 8LL * p->B * p->B * p->B, nx = p->nx, n = nR * nx;
  int st = HP_OK;
  const double* fd = f;
  double* dd = df;
  if (mem == HP_HOST) {
    double* a = (double*)p->ws_get("coll.f", sizeof(double) * n, &st);
    if (st) return st;
    double* b = (double*)p->ws_get("coll.df", sizeof(double) * n, &st);
    if (st) return st;
    HP_CUDA_TRY(cudaMemcpyAsync(a, f, sizeof(double) * n, cudaMemcpyHostToDevice, p->stream));
    fd = a;
    dd = b;
  }
  HP_CUDA_TRY(cudaMemsetAsync(dd, 0, sizeof(double) * n, p->stream));
  if (c->t.numR > 0) {
    const long long nt = nx * c->t.numR;
    ProfScope _ps(p, "coll.df", p->stream);
    k_coll_df<double><<<(unsigned)((nt + 255) / 256), 256, 0, p->stream>>>(
        (int)nx, (int)nR, c->t.numR, c->t.nD, c->t.indR, c->t.lambda, c->t.fcL, c->t.idx, fd, dd);
  }
  HP_CUDA_TRY(cudaGetLastError());
  if (mem == HP_HOST) HP_CUDA_TRY(cudaMemcpyAsync(df, dd, sizeof(double) * n, cudaMemcpyDeviceToHost, p->stream));
  HP_CUDA_TRY(cudaStreamSynchronize(p->stream));
  return HP_OK;
}

// [ix][k][d] -> [k][d][ix] (and [ix][k] -> [k][ix] for lambda)
template <typename T>
__global__ void k_coll_transpose(int nx, int numR, int nD, const double* __restrict__ lambda,
                                 const double* __restrict__ fcL, const short* __restrict__ idx,
                                 T* __restrict__ lamT, T* __restrict__ fcLT, short* __restrict__ idxT) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;   // output index, ix fastest
  const long long n = (long long)nx * numR * (nD + 1);
  if (t >= n) return;
  const int ix = (int)(t % nx);
  const long long r = t / nx;                        // k * (nD + 1) + slot
  const int k = (int)(r / (nD + 1)), slot = (int)(r % (nD + 1));
  const long long src = (long long)ix * numR + k;
  if (slot == nD) {
    lamT[(long long)k * nx + ix] = (T)lambda[src];
  } else {
    fcLT[((long long)k * nD + slot) * nx + ix] = (T)fcL[src * nD + slot];
    idxT[((long long)k * nD + slot) * nx + ix] = idx[src * nD + slot];
  }
}

// fk[k][ix] = f[ix][indR[k]] through a 32 x 32 tile: reads run along k
// (indR ascending), writes along ix
template <typename T>
__global__ void k_coll_gather_t(int nx, long long nR, int numR, const int* __restrict__ indR, const T* __restrict__ f,
                                T* __restrict__ fk) {
  __shared__ T tile[32][33];
  const int k0 = blockIdx.x * 32, x0 = blockIdx.y * 32;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int ix = x0 + r, k = k0 + threadIdx.x;
    tile[r][threadIdx.x] = (ix < nx && k < numR) ? f[(long long)ix * nR + indR[k]] : (T)0;
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int k = k0 + r, ix = x0 + threadIdx.x;
    if (k < numR && ix < nx) fk[(long long)k * nx + ix] = tile[threadIdx.x][r];
  }
}

// f[ix][indR[k]] = fk + dt (sum_d fcL fk[k][idx] - lambda fk), computed with ix
// along lanes (coalesced tables, gathers within one row of fk) and written
// back through a tile with k along lanes.  Per (k, ix) the nD table entries
// are loaded together, then the nD gathers, so each thread waits twice per row
// instead of once per tap (NDMAX >= nD, a compile-time bound for the unrolling).
template <typename T, int NDMAX>
__global__ void k_coll_update_t(int nx, long long nR, int numR, int nD, const int* __restrict__ indR,
                                const T* __restrict__ lamT, const T* __restrict__ fcLT,
                                const short* __restrict__ idxT, const T* __restrict__ fk, T* __restrict__ f,
                                double dt) {
  __shared__ T tile[32][33];
  const int k0 = blockIdx.x * 32, x0 = blockIdx.y * 32;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int k = k0 + r, ix = x0 + threadIdx.x;
    T v = (T)0;
    if (k < numR && ix < nx) {
      const T* row = fk + (long long)k * nx;
      T w[NDMAX];
      int id[NDMAX];
#pragma unroll
      for (int d = 0; d < NDMAX; ++d) {
        const long long o = ((long long)k * nD + d) * nx + ix;
        w[d] = d < nD ? fcLT[o] : (T)0;
        id[d] = d < nD ? (int)idxT[o] : 0;
      }
      const T lam = lamT[(long long)k * nx + ix];
      T g[NDMAX];
#pragma unroll
      for (int d = 0; d < NDMAX; ++d) g[d] = d < nD ? row[id[d]] : (T)0;
      double s = 0.0;
#pragma unroll
      for (int d = 0; d < NDMAX; ++d) s += (double)w[d] * (double)g[d];
      const double f0 = (double)row[ix];
      v = (T)(f0 + dt * (s - (double)lam * f0));
    }
    tile[r][threadIdx.x] = v;
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int ix = x0 + r, k = k0 + threadIdx.x;
    if (k < numR && ix < nx) f[(long long)ix * nR + indR[k]] = tile[threadIdx.x][r];
  }
}

template <typename T>
static int coll_apply_T(hp_collision* c, T* f, double dt, cudaStream_t s) {
  hp_plan* p = c->plan;
  if (c->t.numR == 0) return HP_OK;
  const long long nR = 8LL * p->B * p->B * p->B, nx = p->nx, nt = nx * c->t.numR;
  const int nD = c->t.nD;
  int st = HP_OK;
  if (!c->fcLT) {
    if (cudaMalloc(&c->fcLT, sizeof(T) * nt * nD) != cudaSuccess ||
        cudaMalloc(&c->idxT, sizeof(short) * nt * nD) != cudaSuccess ||
        cudaMalloc(&c->lamT, sizeof(T) * nt) != cudaSuccess) {
      cudaGetLastError();
      cudaFree(c->fcLT); cudaFree(c->idxT); cudaFree(c->lamT);
      c->fcLT = c->lamT = nullptr;
      c->idxT = nullptr;
      hp_set_error("device allocation failed");
      return HP_ERR_ALLOC;
    }
    const long long n = nt * (nD + 1);
    k_coll_transpose<T><<<(unsigned)((n + 255) / 256), 256, 0, s>>>((int)nx, c->t.numR, nD, c->t.lambda, c->t.fcL,
                                                                     c->t.idx, (T*)c->lamT, (T*)c->fcLT, c->idxT);
    HP_CUDA_TRY(cudaGetLastError());
  }
  T* fk = (T*)p->ws_get("coll.fk", sizeof(T) * nt, &st);
  if (st) return st;
  ProfScope _ps(p, "coll.df", s);
  // attitude tiles fastest (omega tiles fastest measured 2.2x as long at B=30, 60x60)
  if ((nx + 31) / 32 > 65535) { hp_set_error("omega grid too large for one launch"); return HP_ERR_UNSUPPORTED; }
  dim3 grid((unsigned)((c->t.numR + 31) / 32), (unsigned)((nx + 31) / 32));
  k_coll_gather_t<T><<<grid, dim3(32, 8), 0, s>>>((int)nx, nR, c->t.numR, c->t.indR, f, fk);
  const T* lam = (const T*)c->lamT;
  const T* fcl = (const T*)c->fcLT;
  if (nD <= 8)
    k_coll_update_t<T, 8><<<grid, dim3(32, 8), 0, s>>>((int)nx, nR, c->t.numR, nD, c->t.indR, lam, fcl, c->idxT, fk, f, dt);
  else if (nD <= 16)
    k_coll_update_t<T, 16><<<grid, dim3(32, 8), 0, s>>>((int)nx, nR, c->t.numR, nD, c->t.indR, lam, fcl, c->idxT, fk, f, dt);
  else
    k_coll_update_t<T, 32><<<grid, dim3(32, 8), 0, s>>>((int)nx, nR, c->t.numR, nD, c->t.indR, lam, fcl, c->idxT, fk, f, dt);
  HP_CUDA_TRY(cudaGetLastError());
  return HP_OK;
}

int hp_collision_apply(hp_collision* c, void* f, double dt, cudaStream_t s) {
  if (c->plan->precision == HP_FP64) return coll_apply_T<double>(c, (double*)f, dt, s);
  return coll_apply_T<float>(c, (float*)f, dt, s);
}

hp_plan* hp_collision_plan(const hp_collision* c) { return c->plan; }
