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
#include <algorithm>
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

// Omega+ = R^T omega+ of the reset map (getOmega.cu:73-92): omega = R Omega,
// its component along t = (R33, -R23)/|.| in the (2, 3) plane reflected with
// restitution eps.  2-D: Omega = (x1, x2, 0), the first two components kept.
template <int NDIM>
__device__ __forceinline__ void reset_map(const double R[3][3], double x1, double x2, double x3, double eps,
                                          double* out) {
  const double w0 = R[0][0] * x1 + R[0][1] * x2 + R[0][2] * x3;
  double w1 = R[1][0] * x1 + R[1][1] * x2 + R[1][2] * x3;
  double w2 = R[2][0] * x1 + R[2][1] * x2 + R[2][2] * x3;
  const double nt = sqrt(R[1][2] * R[1][2] + R[2][2] * R[2][2]);
  const double t1 = R[2][2] / nt, t2 = -R[1][2] / nt;
  const double ot = (1.0 + eps) * (w1 * t1 + w2 * t2);
  w1 -= ot * t1;
  w2 -= ot * t2;
#pragma unroll
  for (int c = 0; c < NDIM; ++c) out[c] = R[0][c] * w0 + R[1][c] * w1 + R[2][c] * w2;
}

// lambda(ix, k) and (omega != NULL) Omega+(ix, k) for the colliding attitudes.
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
  if (omega) reset_map<NDIM>(R, x1, x2, x3, eps, omega + NDIM * t);
}

// Omega+ of the colliding attitudes indR (getOmega.cu:73-92, the 'new'
// direction) without the switching rate.
template <int NDIM>
__global__ void k_coll_omega(int B, int N, double L, int numR, const int* __restrict__ indR, double eps,
                             double* __restrict__ omega) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const int nx = NDIM == 3 ? N * N * N : N * N;
  if (t >= (long long)nx * numR) return;
  const int k = (int)(t % numR), ix = (int)(t / numR);
  double R[3][3];
  rot_of(indR[k], B, R);
  const double x1 = -L / 2 + L / N * (ix % N), x2 = -L / 2 + L / N * ((ix / N) % N);
  const double x3 = NDIM == 3 ? -L / 2 + L / N * (ix / (N * N)) : 0.0;
  reset_map<NDIM>(R, x1, x2, x3, eps, omega + NDIM * t);
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

// Gaussian of covariance Gd (column-major nd x nd): q = d^T Gd^-1 d with the
// cross terms of the symmetric part folded (i01 = inv01 + inv10, ...)
// (getFcL.cu:13-22 for nd = 2).
static int gauss_of(const double* G, int nd, GaussQ* g) {
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
  if (!(det > 0) || !std::isfinite(det)) { hp_set_error("Gd must be positive definite"); return HP_ERR_INVALID; }
  g->i00 = inv[0][0]; g->i01 = inv[0][1] + inv[1][0]; g->i11 = inv[1][1];
  g->i02 = inv[0][2] + inv[2][0]; g->i12 = inv[1][2] + inv[2][1]; g->i22 = inv[2][2];
  g->cn = 1.0 / (std::pow(2 * M_PI, 0.5 * nd) * std::sqrt(det));
  return HP_OK;
}

// fcL / fcL_indx [ix][k][d] of getFcL.cu:11-166 from Omega+ [ix][k][nd] and
// lambda [ix][k] (device): the nD largest Gaussian taps per landing point,
// normalised per source point over the taps that reach it, times lambda dx^n.
// norm: device scratch of nx * numR doubles.  Enqueued on s.
static int build_fcL(hp_plan* p, const hp_collision_params* prm, int numR, const double* omega, const double* lambda,
                     double* fcL, short* idx, double* norm, cudaStream_t s) {
  const int nd = p->ndim, N = p->N, nx = (int)p->nx;
  GaussQ g{};
  const int st = gauss_of(prm->Gd, nd, &g);
  if (st) return st;
  const size_t nxk = (size_t)nx * numR;
  const unsigned g1 = (unsigned)((nxk + 127) / 128);
  {
    ProfScope _ps(p, "coll.setup", s);
    if (nd == 3) k_coll_topd<32, 3><<<g1, 128, 0, s>>>(N, prm->L, numR, prm->nD, omega, g, fcL, idx);
    else k_coll_topd<32, 2><<<g1, 128, 0, s>>>(N, prm->L, numR, prm->nD, omega, g, fcL, idx);
  }
  const double dx = prm->L / N, dx2 = nd == 3 ? dx * dx * dx : dx * dx;
  HP_CUDA_TRY(cudaMemsetAsync(norm, 0, sizeof(double) * nxk, s));
  const unsigned g2 = (unsigned)((nxk * prm->nD + 127) / 128);
  {
    ProfScope _ps(p, "coll.setup", s);
    k_coll_norm<<<g2, 128, 0, s>>>(nx, numR, prm->nD, fcL, idx, norm);
    k_coll_scale<<<g2, 128, 0, s>>>(nx, numR, prm->nD, dx2, norm, lambda, fcL, idx);
  }
  HP_CUDA_TRY(cudaGetLastError());
  return HP_OK;
}

// Category, theta and contact point per attitude (getLambda.cu:8-40,
// 202-226) and the colliding attitudes, ascending (getLambda.cu:33-39).
static int attitude_stage(hp_plan* p, const hp_collision_params* prm, double theta0, char* cat, double* theta,
                          double* PC, std::vector<int>& hind) {
  const int B = p->B, nR = 8 * B * B * B;
  cudaStream_t s = p->stream;
  {
    ProfScope _ps(p, "coll.setup", s);
    k_coll_theta<<<(nR + 127) / 128, 128, 0, s>>>(B, nR, theta0, prm->theta_t, prm->h, prm->r, cat, theta, PC);
  }
  std::vector<char> hc(nR);
  if (cudaMemcpyAsync(hc.data(), cat, nR, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess) {
    hp_set_error(cudaGetErrorString(cudaGetLastError()));
    return HP_ERR_CUDA;
  }
  hind.clear();
  for (int i = 0; i < nR; ++i) if (hc[i] != 0) hind.push_back(i);
  return HP_OK;
}

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
  auto fail = [&](int code) { hp_collision_destroy(c); hp_dev_free(cat); hp_dev_free(theta); return code; };
  if (hp_dev_alloc(&cat, nR) != cudaSuccess || hp_dev_alloc(&theta, sizeof(double) * nR) != cudaSuccess ||
      hp_dev_alloc(&c->t.PC, sizeof(double) * 3 * nR) != cudaSuccess) {
    cudaGetLastError();
    hp_set_error("device allocation failed");
    return fail(HP_ERR_ALLOC);
  }
  std::vector<int> hind;
  {
    const int st = attitude_stage(p, prm, theta0, cat, theta, c->t.PC, hind);
    if (st) return fail(st);
  }
  const int nk = (int)hind.size();
  c->t.numR = nk;
  c->t.nD = prm->nD;
  if (numR) *numR = nk;
  if (nk == 0) { hp_dev_free(cat); hp_dev_free(theta); *out = c; return HP_OK; }
  const size_t nxk = (size_t)nx * nk;
  double* norm = nullptr;
  if (hp_dev_alloc(&c->t.indR, sizeof(int) * nk) != cudaSuccess ||
      hp_dev_alloc(&c->t.lambda, sizeof(double) * nxk) != cudaSuccess ||
      hp_dev_alloc(&c->t.omega, sizeof(double) * nd * nxk) != cudaSuccess ||
      hp_dev_alloc(&c->t.fcL, sizeof(double) * nxk * prm->nD) != cudaSuccess ||
      hp_dev_alloc(&c->t.idx, sizeof(short) * nxk * prm->nD) != cudaSuccess ||
      hp_dev_alloc(&norm, sizeof(double) * nxk) != cudaSuccess) {
    cudaGetLastError();
    hp_dev_free(norm);
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
  {
    const int st = build_fcL(p, prm, nk, c->t.omega, c->t.lambda, c->t.fcL, c->t.idx, norm, s);
    if (st) { hp_dev_free(norm); return fail(st); }
  }
  HP_CUDA_TRY(cudaGetLastError());
  HP_CUDA_TRY(cudaStreamSynchronize(s));
  hp_dev_free(norm);
  hp_dev_free(cat);
  hp_dev_free(theta);
  *out = c;
  return HP_OK;
}

extern "C" int hp_collision_destroy(hp_collision* c) {
  if (!c) return HP_OK;
  hp_dev_free(c->t.indR); hp_dev_free(c->t.lambda); hp_dev_free(c->t.omega); hp_dev_free(c->t.fcL);
  hp_dev_free(c->t.idx); hp_dev_free(c->t.PC);
  hp_dev_free(c->fcLT); hp_dev_free(c->idxT); hp_dev_free(c->lamT);
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
  if ((omega && nxk && !c->t.omega) || (PC && !c->t.PC)) {
    hp_set_error("an operator made from given tables holds no Omega+ or contact-point table");
    return HP_ERR_INVALID;
  }
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

// ---- the table builders one stage at a time (the separate MEX calls of
// pendulum_reduced_hybrid.m:130-141) and an operator from given tables ----

namespace {
// device copy of a caller array (host or device) of n elements of T
template <typename T>
struct DevIn {
  const T* ptr = nullptr;
  T* own = nullptr;
  int load(const T* src, size_t n, int mem, cudaStream_t s) {
    if (mem == HP_DEVICE || n == 0) { ptr = src; return HP_OK; }
    if (hp_dev_alloc(&own, sizeof(T) * n) != cudaSuccess) { cudaGetLastError(); hp_set_error("device allocation failed"); return HP_ERR_ALLOC; }
    HP_CUDA_TRY(cudaMemcpyAsync(own, src, sizeof(T) * n, cudaMemcpyHostToDevice, s));
    ptr = own;
    return HP_OK;
  }
  ~DevIn() { hp_dev_free(own); }
};
struct DevBuf {
  void* p = nullptr;
  ~DevBuf() { hp_dev_free(p); }
  int alloc(size_t bytes) {
    if (bytes && hp_dev_alloc(&p, bytes) != cudaSuccess) { cudaGetLastError(); hp_set_error("device allocation failed"); return HP_ERR_ALLOC; }
    return HP_OK;
  }
};
}  // namespace

// entries of idx (n) outside [0, lim) and of indR outside [0, nR) or not
// ascending count into *bad
__global__ void k_coll_check(const short* __restrict__ idx, long long n, int lim, const int* __restrict__ indR,
                             int numR, int nR, int* bad) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t < n && (idx[t] < 0 || idx[t] >= lim)) atomicAdd(bad, 1);
  if (t < numR && (indR[t] < 0 || indR[t] >= nR || (t > 0 && indR[t] <= indR[t - 1]))) atomicAdd(bad, 1);
}

extern "C" int hp_collision_lambda(hp_plan* p, const hp_collision_params* prm, int* numR, double* lambda, int* indR,
                                   double* PC, int mem) {
  if (!p || !prm || !numR) { hp_set_error("null argument"); return HP_ERR_INVALID; }
  if (mem != HP_DEVICE && mem != HP_HOST) { hp_set_error("bad mem"); return HP_ERR_INVALID; }
  if (!(prm->L > 0) || !(prm->theta_t > 0)) { hp_set_error("bad collision parameters"); return HP_ERR_INVALID; }
  const int B = p->B, N = p->N, nR = 8 * B * B * B, nx = (int)p->nx;
  cudaStream_t s = p->stream;
  const double hr = std::sqrt(prm->h * prm->h + prm->r * prm->r);
  const double theta0 = std::asin(prm->d / hr) - std::asin(prm->r / hr);
  DevBuf cat, theta, pc;
  int st = cat.alloc(nR);
  if (!st) st = theta.alloc(sizeof(double) * nR);
  if (!st) st = pc.alloc(sizeof(double) * 3 * nR);
  if (st) return st;
  std::vector<int> hind;
  st = attitude_stage(p, prm, theta0, (char*)cat.p, (double*)theta.p, (double*)pc.p, hind);
  if (st) return st;
  const int nk = (int)hind.size();
  *numR = nk;
  const cudaMemcpyKind kind = mem == HP_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
  if (PC) HP_CUDA_TRY(cudaMemcpyAsync(PC, pc.p, sizeof(double) * 3 * nR, kind, s));
  if (indR && nk) {
    if (mem == HP_HOST) std::copy(hind.begin(), hind.end(), indR);
    else HP_CUDA_TRY(cudaMemcpyAsync(indR, hind.data(), sizeof(int) * nk, cudaMemcpyHostToDevice, s));
  }
  if (lambda && nk) {
    const size_t nxk = (size_t)nx * nk;
    DevBuf ind, lam;
    st = ind.alloc(sizeof(int) * nk);
    if (!st) st = lam.alloc(sizeof(double) * nxk);
    if (st) return st;
    HP_CUDA_TRY(cudaMemcpyAsync(ind.p, hind.data(), sizeof(int) * nk, cudaMemcpyHostToDevice, s));
    const unsigned g1 = (unsigned)((nxk + 127) / 128);
    {
      ProfScope _ps(p, "coll.setup", s);
      if (p->ndim == 3)
        k_coll_lambda_omega<3><<<g1, 128, 0, s>>>(B, N, prm->L, nk, (const int*)ind.p, (const char*)cat.p,
                                                  (const double*)theta.p, (const double*)pc.p, theta0, prm->theta_t,
                                                  prm->lambda_max, 0.0, (double*)lam.p, nullptr);
      else
        k_coll_lambda_omega<2><<<g1, 128, 0, s>>>(B, N, prm->L, nk, (const int*)ind.p, (const char*)cat.p,
                                                  (const double*)theta.p, (const double*)pc.p, theta0, prm->theta_t,
                                                  prm->lambda_max, 0.0, (double*)lam.p, nullptr);
    }
    HP_CUDA_TRY(cudaGetLastError());
    HP_CUDA_TRY(cudaMemcpyAsync(lambda, lam.p, sizeof(double) * nxk, kind, s));
    HP_CUDA_TRY(cudaStreamSynchronize(s));   // before the scratch is freed
  }
  HP_CUDA_TRY(cudaStreamSynchronize(s));
  return HP_OK;
}

extern "C" int hp_collision_omega(hp_plan* p, const hp_collision_params* prm, int numR, const int* indR,
                                  double* omega, int mem) {
  if (!p || !prm || (numR > 0 && (!indR || !omega)) || numR < 0) { hp_set_error("null argument"); return HP_ERR_INVALID; }
  if (mem != HP_DEVICE && mem != HP_HOST) { hp_set_error("bad mem"); return HP_ERR_INVALID; }
  if (!(prm->L > 0)) { hp_set_error("L must be positive"); return HP_ERR_INVALID; }
  if (numR == 0) return HP_OK;
  const int B = p->B, N = p->N, nR = 8 * B * B * B, nd = p->ndim;
  const size_t nxk = (size_t)p->nx * numR;
  cudaStream_t s = p->stream;
  DevIn<int> ind;
  int st = ind.load(indR, numR, mem, s);
  if (st) return st;
  DevBuf bad;
  if ((st = bad.alloc(sizeof(int)))) return st;
  HP_CUDA_TRY(cudaMemsetAsync(bad.p, 0, sizeof(int), s));
  k_coll_check<<<(numR + 255) / 256, 256, 0, s>>>(nullptr, 0, 1, ind.ptr, numR, nR, (int*)bad.p);
  int hbad = 0;
  HP_CUDA_TRY(cudaMemcpyAsync(&hbad, bad.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  HP_CUDA_TRY(cudaStreamSynchronize(s));
  if (hbad) { hp_set_error("indR must be ascending attitude indices in [0, (2B)^3)"); return HP_ERR_INVALID; }
  DevBuf out;
  double* od = omega;
  if (mem == HP_HOST) {
    if ((st = out.alloc(sizeof(double) * nd * nxk))) return st;
    od = (double*)out.p;
  }
  {
    ProfScope _ps(p, "coll.setup", s);
    const unsigned g1 = (unsigned)((nxk + 127) / 128);
    if (nd == 3) k_coll_omega<3><<<g1, 128, 0, s>>>(B, N, prm->L, numR, ind.ptr, prm->epsilon, od);
    else k_coll_omega<2><<<g1, 128, 0, s>>>(B, N, prm->L, numR, ind.ptr, prm->epsilon, od);
  }
  HP_CUDA_TRY(cudaGetLastError());
  if (mem == HP_HOST) HP_CUDA_TRY(cudaMemcpyAsync(omega, od, sizeof(double) * nd * nxk, cudaMemcpyDeviceToHost, s));
  HP_CUDA_TRY(cudaStreamSynchronize(s));
  return HP_OK;
}

extern "C" int hp_collision_fcL(hp_plan* p, const hp_collision_params* prm, int numR, const double* omega,
                                const double* lambda, double* fcL, short* fcL_indx, int mem) {
  if (!p || !prm || numR < 0 || (numR > 0 && (!omega || !lambda || !fcL || !fcL_indx))) {
    hp_set_error("null argument");
    return HP_ERR_INVALID;
  }
  if (mem != HP_DEVICE && mem != HP_HOST) { hp_set_error("bad mem"); return HP_ERR_INVALID; }
  if (prm->nD < 1 || prm->nD > 32) { hp_set_error("nD must be in 1..32"); return HP_ERR_INVALID; }
  if (!(prm->L > 0)) { hp_set_error("L must be positive"); return HP_ERR_INVALID; }
  if (p->nx > 32768) { hp_set_error("the tap indices are 16-bit: at most 32768 omega points"); return HP_ERR_UNSUPPORTED; }
  if (numR == 0) return HP_OK;
  const int nd = p->ndim;
  const size_t nxk = (size_t)p->nx * numR, nt = nxk * prm->nD;
  cudaStream_t s = p->stream;
  DevIn<double> om, lam;
  int st = om.load(omega, nd * nxk, mem, s);
  if (!st) st = lam.load(lambda, nxk, mem, s);
  if (st) return st;
  DevBuf norm, fo, io;
  if ((st = norm.alloc(sizeof(double) * nxk))) return st;
  double* fd = fcL;
  short* id = fcL_indx;
  if (mem == HP_HOST) {
    if ((st = fo.alloc(sizeof(double) * nt)) || (st = io.alloc(sizeof(short) * nt))) return st;
    fd = (double*)fo.p;
    id = (short*)io.p;
  }
  st = build_fcL(p, prm, numR, om.ptr, lam.ptr, fd, id, (double*)norm.p, s);
  if (st) return st;
  if (mem == HP_HOST) {
    HP_CUDA_TRY(cudaMemcpyAsync(fcL, fd, sizeof(double) * nt, cudaMemcpyDeviceToHost, s));
    HP_CUDA_TRY(cudaMemcpyAsync(fcL_indx, id, sizeof(short) * nt, cudaMemcpyDeviceToHost, s));
  }
  HP_CUDA_TRY(cudaStreamSynchronize(s));
  return HP_OK;
}

extern "C" int hp_collision_create_from_tables(hp_plan* p, int numR, int nD, const int* indR, const double* lambda,
                                               const double* fcL, const short* fcL_indx, int mem,
                                               hp_collision** out) {
  if (!p || !out || numR < 0 || (numR > 0 && (!indR || !lambda || !fcL || !fcL_indx))) {
    hp_set_error("null argument");
    return HP_ERR_INVALID;
  }
  *out = nullptr;
  if (mem != HP_DEVICE && mem != HP_HOST) { hp_set_error("bad mem"); return HP_ERR_INVALID; }
  if (nD < 1 || nD > 32) { hp_set_error("nD must be in 1..32"); return HP_ERR_INVALID; }
  if (p->nx > 32768) { hp_set_error("the tap indices are 16-bit: at most 32768 omega points"); return HP_ERR_UNSUPPORTED; }
  const int nR = 8 * p->B * p->B * p->B;
  if (numR > nR) { hp_set_error("numR exceeds the number of attitudes"); return HP_ERR_SHAPE; }
  cudaStream_t s = p->stream;
  hp_collision* c = new hp_collision();
  c->plan = p;
  c->t.numR = numR;
  c->t.nD = nD;
  if (numR == 0) { *out = c; return HP_OK; }
  const size_t nxk = (size_t)p->nx * numR, nt = nxk * nD;
  const cudaMemcpyKind kind = mem == HP_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
  if (hp_dev_alloc(&c->t.indR, sizeof(int) * numR) != cudaSuccess ||
      hp_dev_alloc(&c->t.lambda, sizeof(double) * nxk) != cudaSuccess ||
      hp_dev_alloc(&c->t.fcL, sizeof(double) * nt) != cudaSuccess ||
      hp_dev_alloc(&c->t.idx, sizeof(short) * nt) != cudaSuccess) {
    cudaGetLastError();
    hp_collision_destroy(c);
    hp_set_error("device allocation failed");
    return HP_ERR_ALLOC;
  }
  int st = HP_OK;
  DevBuf bad;
  if (cudaMemcpyAsync(c->t.indR, indR, sizeof(int) * numR, kind, s) != cudaSuccess ||
      cudaMemcpyAsync(c->t.lambda, lambda, sizeof(double) * nxk, kind, s) != cudaSuccess ||
      cudaMemcpyAsync(c->t.fcL, fcL, sizeof(double) * nt, kind, s) != cudaSuccess ||
      cudaMemcpyAsync(c->t.idx, fcL_indx, sizeof(short) * nt, kind, s) != cudaSuccess) {
    hp_set_error(cudaGetErrorString(cudaGetLastError()));
    st = HP_ERR_CUDA;
  }
  // every tap must read an omega point of the grid and every attitude a row of
  // f: out-of-range tables are rejected before any kernel dereferences them
  if (!st) st = bad.alloc(sizeof(int));
  int hbad = 0;
  if (!st && (cudaMemsetAsync(bad.p, 0, sizeof(int), s) != cudaSuccess)) st = HP_ERR_CUDA;
  if (!st) {
    const long long n = (long long)std::max<size_t>(nt, (size_t)numR);
    k_coll_check<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(c->t.idx, (long long)nt, (int)p->nx, c->t.indR, numR, nR,
                                                             (int*)bad.p);
    if (cudaMemcpyAsync(&hbad, bad.p, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess) {
      hp_set_error(cudaGetErrorString(cudaGetLastError()));
      st = HP_ERR_CUDA;
    }
  }
  if (!st && hbad) {
    hp_set_error("tables out of range: fcL_indx must lie in [0, nx) and indR be ascending in [0, (2B)^3)");
    st = HP_ERR_INVALID;
  }
  if (st) { hp_collision_destroy(c); return st; }
  *out = c;
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
    if (hp_dev_alloc(&c->fcLT, sizeof(T) * nt * nD) != cudaSuccess ||
        hp_dev_alloc(&c->idxT, sizeof(short) * nt * nD) != cudaSuccess ||
        hp_dev_alloc(&c->lamT, sizeof(T) * nt) != cudaSuccess) {
      cudaGetLastError();
      hp_dev_free(c->fcLT); hp_dev_free(c->idxT); hp_dev_free(c->lamT);
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
