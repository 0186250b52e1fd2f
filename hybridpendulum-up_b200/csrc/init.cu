// Initial densities on the GPU: matrix Fisher on SO(3) times a Gaussian in
// omega, the initial condition of propagation/pendulum.m:210-220,
// pendulum_reduced.m and pendulum_reduced_hybrid.m:167-180:
//   f(R, x) = exp(tr(F^T R)) / c(s) * exp(-(x-mu)^T Sigma^-1 (x-mu) / 2) / sqrt((2 pi)^n det Sigma)
// with F = U diag(s) V^T and c(s) the matrix Fisher normalising constant
// ('matrix Fisher/pdf_MF_normal.m:38', Kunze's integral).  The density is the
// outer product of an SO(3) factor and an omega factor, written by one pass.
#include <cmath>
#include <vector>

#include "common.cuh"
#include "plan.hpp"

using namespace hp;

namespace {

// c(s) = int_{-1}^{1} 1/2 exp(s3 u) I0((s1-s2)(1-u)/2) I0((s1+s2)(1+u)/2) du by
// composite Gauss-Legendre (16 panels x 8 nodes; the integrand is entire).
double mf_normaliser(const double s[3]) {
  static const double xg[8] = {-0.9602898564975363, -0.7966664774136267, -0.5255324099163290, -0.1834346424956498,
                               0.1834346424956498,  0.5255324099163290,  0.7966664774136267,  0.9602898564975363};
  static const double wg[8] = {0.1012285362903763, 0.2223810344533745, 0.3137066458778873, 0.3626837833783620,
                               0.3626837833783620, 0.3137066458778873, 0.2223810344533745, 0.1012285362903763};
  const int panels = 16;
  double c = 0.0;
  for (int k = 0; k < panels; ++k) {
    const double a = -1.0 + 2.0 * k / panels, h = 1.0 / panels;
    for (int j = 0; j < 8; ++j) {
      const double u = a + h * (xg[j] + 1.0);
      c += h * wg[j] * 0.5 * std::exp(s[2] * u) * std::cyl_bessel_i(0.0, std::fabs(0.5 * (s[0] - s[1]) * (1 - u))) *
           std::cyl_bessel_i(0.0, std::fabs(0.5 * (s[0] + s[1]) * (1 + u)));
    }
  }
  return c;
}

// fR[a + 2B (b + 2B c)] = exp(tr(F^T R_abc)) / c, R = Rz(alpha) Ry(beta) Rz(gamma)
__global__ void k_mf_factor(int B, const double* __restrict__ Fm, double cinv, double* __restrict__ fR) {
  const int n = 2 * B;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n * n * n) return;
  const int a = t % n, b = (t / n) % n, c = t / (n * n);
  const double al = M_PI / B * a, be = M_PI / (4.0 * B) * (2 * b + 1), ga = M_PI / B * c;
  double sa, ca, sb, cb, sg, cg;
  sincos(al, &sa, &ca);
  sincos(be, &sb, &cb);
  sincos(ga, &sg, &cg);
  // R = Rz(al) Ry(be) Rz(ga)
  const double R[3][3] = {{ca * cb * cg - sa * sg, -ca * cb * sg - sa * cg, ca * sb},
                          {sa * cb * cg + ca * sg, -sa * cb * sg + ca * cg, sa * sb},
                          {-sb * cg, sb * sg, cb}};
  double tr = 0.0;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) tr += Fm[i * 3 + j] * R[i][j];
  fR[t] = exp(tr) * cinv;
}

// fx[w] = N(x(w); mu, Sigma), x_i = -L/2 + L k_i / N, w = k1 + N k2 (+ N^2 k3)
__global__ void k_gauss_factor(int N, int nd, double L, const double* __restrict__ mu, const double* __restrict__ Si,
                               double norm, long long nx, double* __restrict__ fx) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= nx) return;
  double d[3] = {0, 0, 0};
  long long w = t;
  for (int i = 0; i < nd; ++i) {
    d[i] = -L / 2 + L * (double)(w % N) / N - mu[i];
    w /= N;
  }
  double q = 0.0;
  for (int i = 0; i < nd; ++i)
    for (int j = 0; j < nd; ++j) q += d[i] * Si[i * 3 + j] * d[j];
  fx[t] = exp(-0.5 * q) * norm;
}

template <typename T>
__global__ void k_outer(const double* __restrict__ fR, const double* __restrict__ fx, long long nR, long long n,
                        T* __restrict__ f) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
    f[t] = (T)(fR[t % nR] * fx[t / nR]);
}

int inv_det(const double* S, int nd, double* Si, double* det) {
  if (nd == 2) {
    const double a = S[0], b = S[1], c = S[3], d = S[4];
    *det = a * d - b * c;
    if (!(*det > 0)) return HP_ERR_INVALID;
    Si[0] = d / *det; Si[1] = -b / *det; Si[3] = -c / *det; Si[4] = a / *det;
    return HP_OK;
  }
  const double* m = S;
  const double c00 = m[4] * m[8] - m[5] * m[7], c01 = m[5] * m[6] - m[3] * m[8], c02 = m[3] * m[7] - m[4] * m[6];
  *det = m[0] * c00 + m[1] * c01 + m[2] * c02;
  if (!(*det > 0)) return HP_ERR_INVALID;
  const double id = 1.0 / *det;
  Si[0] = c00 * id; Si[1] = (m[2] * m[7] - m[1] * m[8]) * id; Si[2] = (m[1] * m[5] - m[2] * m[4]) * id;
  Si[3] = c01 * id; Si[4] = (m[0] * m[8] - m[2] * m[6]) * id; Si[5] = (m[2] * m[3] - m[0] * m[5]) * id;
  Si[6] = c02 * id; Si[7] = (m[1] * m[6] - m[0] * m[7]) * id; Si[8] = (m[0] * m[4] - m[1] * m[3]) * id;
  return HP_OK;
}

// f (FP64, device) of the plan's grid
int density_mfg(hp_plan* p, const double* U, const double* s, const double* V, const double* mu,
                const double* Sigma, double* f, cudaStream_t st) {
  const int nd = p->ndim;
  double Fm[9] = {}, Si[9] = {}, det = 0;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      for (int k = 0; k < 3; ++k) Fm[i * 3 + j] += U[i * 3 + k] * s[k] * V[j * 3 + k];
  if (inv_det(Sigma, nd, Si, &det) != HP_OK) { hp_set_error("Sigma must be positive definite"); return HP_ERR_INVALID; }
  const double c = mf_normaliser(s);
  if (!(c > 0) || !std::isfinite(c)) { hp_set_error("matrix Fisher normalising constant out of range"); return HP_ERR_NONFINITE; }
  const double gnorm = 1.0 / std::sqrt(std::pow(2.0 * M_PI, nd) * det);
  int stt = HP_OK;
  const long long nR = 8LL * p->B * p->B * p->B;
  double* fR = (double*)p->ws_get("init.fR", sizeof(double) * nR, &stt);
  if (stt) return stt;
  double* fx = (double*)p->ws_get("init.fx", sizeof(double) * p->nx, &stt);
  if (stt) return stt;
  double* par = (double*)p->ws_get("init.par", sizeof(double) * 21, &stt);
  if (stt) return stt;
  double h[21] = {};
  for (int i = 0; i < 9; ++i) { h[i] = Fm[i]; h[12 + i] = Si[i]; }
  for (int i = 0; i < nd; ++i) h[9 + i] = mu[i];
  HP_CUDA_TRY(cudaMemcpyAsync(par, h, sizeof(h), cudaMemcpyHostToDevice, st));
  ProfScope _ps(p, "init.density", st);
  k_mf_factor<<<(unsigned)((nR + 255) / 256), 256, 0, st>>>(p->B, par, 1.0 / c, fR);
  k_gauss_factor<<<(unsigned)((p->nx + 255) / 256), 256, 0, st>>>(p->N, nd, p->model.L, par + 9, par + 12, gnorm,
                                                                   p->nx, fx);
  const long long n = nR * p->nx;
  k_outer<double><<<148 * 8, 256, 0, st>>>(fR, fx, nR, n, f);
  HP_CUDA_TRY(cudaGetLastError());
  HP_CUDA_TRY(cudaStreamSynchronize(st));   // keeps the host parameter block alive until used
  return HP_OK;
}

int check_args(hp_plan* p, const double* U, const double* s, const double* V, const double* mu, const double* Sigma) {
  if (!p || !U || !s || !V || !mu || !Sigma) { hp_set_error("null argument"); return HP_ERR_INVALID; }
  if (!p->has_model) { hp_set_error("no model: the omega period L comes from hp_plan_set_model"); return HP_ERR_NO_MODEL; }
  for (int i = 0; i < 9; ++i)
    if (!std::isfinite(U[i]) || !std::isfinite(V[i])) { hp_set_error("U, V must be finite"); return HP_ERR_NONFINITE; }
  return HP_OK;
}

}  // namespace

extern "C" int hp_density_mf_gauss(hp_plan* p, const double* U, const double* s, const double* V, const double* mu,
                                   const double* Sigma, double* f, int mem) {
  int st = check_args(p, U, s, V, mu, Sigma);
  if (st) return st;
  if (!f) { hp_set_error("null argument"); return HP_ERR_INVALID; }
  if (mem != HP_DEVICE && mem != HP_HOST) { hp_set_error("mem must be HP_DEVICE or HP_HOST"); return HP_ERR_INVALID; }
  const size_t fb = sizeof(double) * (size_t)p->n_grid();
  double* d = f;
  if (mem == HP_HOST) {
    d = (double*)p->ws_get("init.f", fb, &st);
    if (st) return st;
  }
  st = density_mfg(p, U, s, V, mu, Sigma, d, p->stream);
  if (st) return st;
  if (mem == HP_HOST) {
    HP_CUDA_TRY(cudaMemcpyAsync(f, d, fb, cudaMemcpyDeviceToHost, p->stream));
    HP_CUDA_TRY(cudaStreamSynchronize(p->stream));
  }
  return HP_OK;
}

extern "C" int hp_state_init_mf_gauss(hp_state* sta, const double* U, const double* s, const double* V,
                                      const double* mu, const double* Sigma) {
  if (!sta) { hp_set_error("null argument"); return HP_ERR_INVALID; }
  hp_plan* p = sta->plan;
  int st = check_args(p, U, s, V, mu, Sigma);
  if (st) return st;
  if (p->symmetry != HP_REAL) { hp_set_error("initial densities need an HP_REAL plan"); return HP_ERR_UNSUPPORTED; }
  double* f = (double*)p->ws_get("init.f", sizeof(double) * (size_t)p->n_grid(), &st);
  if (st) return st;
  st = density_mfg(p, U, s, V, mu, Sigma, f, p->stream);
  if (st) return st;
  st = hp_forward_internal64(p, f, sta->F, p->stream);
  if (st) return st;
  sta->fg_valid = false;
  sta->f32_valid = false;
  HP_CUDA_TRY(cudaStreamSynchronize(p->stream));
  // the FP64 grid density and transform buffers are only needed here
  for (const char* k : {"init.f", "tf.t1", "tf.t2"}) p->ws_release(k);
  return HP_OK;
}
