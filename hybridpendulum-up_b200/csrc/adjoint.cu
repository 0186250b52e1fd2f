// Adjoint of the propagation step and the parameter gradients of a
// trajectory (reverse mode through forward-Euler steps with checkpoints).
//
// With the plain coefficient inner product <X, Y> = Re sum conj(X) Y and
// W = diag(2l+1), the derivative A = Lie + Damp + Gyro + Grav + Noise of
// pendulum.m:388-527 has the exact discrete adjoint
//   A^H = -W (Lie + Gyro + Grav - Noise) W^-1 - sum_i b_i M_i D_i
// because
//   * u^l_i is anti-Hermitian and M_i (multiply by x_i on the omega grid) is
//     self-adjoint, so the Lie term and the gyroscopic term D_i M_j M_k are
//     anti-self-adjoint and commute with W;
//   * the gravity term -D_i Grav_i is a Galerkin product with a real
//     function of R, self-adjoint in the (2l+1)-weighted inner product, so
//     Grav_i^H = W Grav_i W^-1;
//   * the noise multiplier is real and diagonal;
//   * (b_i D_i M_i)^H = -b_i M_i D_i (D_i = 2 pi i kappa / L is imaginary);
//     M_i and D_i do not commute on the grid, so this term is applied as its
//     own pass (multiply by D_i, inverse FFT, times x_i, FFT).
// The first bracket is the forward derivative kernel with b = 0 and G -> -G.
#include <algorithm>
#include <cmath>
#include <vector>

#include "common.cuh"
#include "plan.hpp"

using namespace hp;

#define ADJ_CHECK(expr)         \
  do {                          \
    int _s = (expr);            \
    if (_s != HP_OK) return _s; \
  } while (0)

namespace {

constexpr int kDotThreads = 256;
constexpr int kDotBlocks = 592;  // 4 per SM

// out = (add ? lam : 0) - a * (2l+1) * d1
__global__ void k_adj_combine(RowLayout L, const double2* __restrict__ lam, const double2* __restrict__ d1,
                              double2* __restrict__ out, double a, int add) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= L.nrows * L.nx) return;
  const int l = L.rows[t / L.nx].x;
  const double s = a * (2 * l + 1);
  const double2 v = d1[t];
  double2 o = add ? lam[t] : make_double2(0.0, 0.0);
  o.x -= s * v.x;
  o.y -= s * v.y;
  out[t] = o;
}

// out = in / (2l+1)
__global__ void k_row_unweight(RowLayout L, const double2* __restrict__ in, double2* __restrict__ out) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= L.nrows * L.nx) return;
  const double s = 1.0 / (2 * L.rows[t / L.nx].x + 1);
  const double2 v = in[t];
  out[t] = make_double2(s * v.x, s * v.y);
}

// out += coef * M_axis (D_axis in): one thread per line of N points along
// `axis` (stride N^axis inside a row).
template <int N>
__global__ void __launch_bounds__(128) k_axis_md(RowLayout L, const double2* __restrict__ in,
                                                 double2* __restrict__ out, int axis, double coef, double Llen) {
  const long long nlines = L.nx / N;
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= L.nrows * nlines) return;
  const long long row = t / nlines, q = t % nlines;
  long long stride = 1;
  for (int a = 0; a < axis; ++a) stride *= N;
  const long long lo = q % stride, hi = q / stride;
  const long long base = row * L.nx + hi * stride * N + lo;
  const double tp = 2.0 * M_PI / Llen;
  double2 x[N];
#pragma unroll
  for (int j = 0; j < N; ++j) {
    const double2 v = in[base + j * stride];
    const double dk = tp * kappa_first(j, N);
    x[j] = make_double2(-dk * v.y, dk * v.x);  // D v = i dk v
  }
  fft<N, true>(x);
#pragma unroll
  for (int j = 0; j < N; ++j) {
    const double xc = (-Llen / 2 + Llen * j / N) / N;
    x[j] = xc * x[j];
  }
  fft<N, false>(x);
#pragma unroll
  for (int j = 0; j < N; ++j) {
    double2 o = out[base + j * stride];
    o.x += coef * x[j].x;
    o.y += coef * x[j].y;
    out[base + j * stride] = o;
  }
}

// out (=, or += with acc) coef * D_daxis (M_axis in): one thread per line of N
// points along `axis`; M_axis multiplies by x_axis on the omega grid
// (inverse FFT, times x, FFT), D_daxis by 2 pi i kappa / L along axis daxis
// (any axis, applied per point after M; daxis < 0: none).
template <int N>
__global__ void __launch_bounds__(128) k_line_dm(RowLayout L, const double2* __restrict__ in,
                                                 double2* __restrict__ out, int axis, int daxis, double coef,
                                                 double Llen, int acc) {
  const long long nlines = L.nx / N;
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= L.nrows * nlines) return;
  const long long row = t / nlines, q = t % nlines;
  long long stride = 1, dstride = 1;
  for (int a = 0; a < axis; ++a) stride *= N;
  for (int a = 0; a < daxis; ++a) dstride *= N;
  const long long lo = q % stride, hi = q / stride;
  const long long w0 = hi * stride * N + lo;   // omega index of the line's first point
  const long long base = row * L.nx + w0;
  const double tp = 2.0 * M_PI / Llen;
  double2 x[N];
#pragma unroll
  for (int j = 0; j < N; ++j) x[j] = in[base + j * stride];
  fft<N, true>(x);
#pragma unroll
  for (int j = 0; j < N; ++j) {
    const double xc = (-Llen / 2 + Llen * j / N) / N;
    x[j] = xc * x[j];
  }
  fft<N, false>(x);
#pragma unroll
  for (int j = 0; j < N; ++j) {
    double2 v = x[j];
    if (daxis >= 0) {   // i dk v
      const long long w = w0 + j * stride;
      const double dk = tp * kappa_first((int)((w / dstride) % N), N);
      v = make_double2(-dk * v.y, dk * v.x);
    }
    double2 o = acc ? out[base + j * stride] : make_double2(0.0, 0.0);
    o.x += coef * v.x;
    o.y += coef * v.y;
    out[base + j * stride] = o;
  }
}

__device__ __forceinline__ double row_weight(const RowLayout& L, long long row, int half) {
  return (half && L.rows[row].y > 0) ? 2.0 : 1.0;
}

// acc[slot * gridDim.x + block] += scale * sum w Re(conj(a) b); one slot per call.
__global__ void __launch_bounds__(kDotThreads) k_dot(RowLayout L, const double2* __restrict__ a,
                                                     const double2* __restrict__ b, double* __restrict__ acc,
                                                     int slot, double scale, int half) {
  __shared__ double red[kDotThreads];
  double s = 0.0;
  const long long n = L.nrows * L.nx;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    const double2 u = a[t], v = b[t];
    s += row_weight(L, t / L.nx, half) * (u.x * v.x + u.y * v.y);
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int k = kDotThreads / 2; k > 0; k >>= 1) {
    if (threadIdx.x < k) red[threadIdx.x] += red[threadIdx.x + k];
    __syncthreads();
  }
  if (threadIdx.x == 0) acc[(long long)slot * gridDim.x + blockIdx.x] += scale * red[0];
}

// The noise-term gradients: slots slot0 + (i, j) pair index (i <= j) get
// scale * sum w c_ij(k) Re(conj(a) b), c_ii = -(2 pi kd_i / L)^2 with the
// Nyquist bin kept, c_ij = -(2 pi k_i / L)(2 pi k_j / L) with it zeroed
// (pendulum.m:510-523).
__global__ void __launch_bounds__(kDotThreads) k_dot_noise(RowLayout L, const double2* __restrict__ a,
                                                           const double2* __restrict__ b, double* __restrict__ acc,
                                                           int slot0, double scale, int half, double Llen) {
  __shared__ double red[6][kDotThreads];
  double s[6] = {0, 0, 0, 0, 0, 0};
  const long long n = L.nrows * L.nx;
  const int N = L.N, nd = L.ndim;
  const double tp = 2.0 * M_PI / Llen;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    const double2 u = a[t], v = b[t];
    const double r = row_weight(L, t / L.nx, half) * (u.x * v.x + u.y * v.y);
    long long w = t % L.nx;
    double d1[3] = {0, 0, 0}, dd[3] = {0, 0, 0};
    for (int i = 0; i < nd; ++i) {
      const int k = (int)(w % N);
      w /= N;
      d1[i] = tp * kappa_first(k, N);
      dd[i] = tp * kappa_diag(k, N);
    }
    int q = 0;
    for (int i = 0; i < 3; ++i)
      for (int j = i; j < 3; ++j, ++q) {
        if (i >= nd || j >= nd) continue;
        s[q] -= r * (i == j ? dd[i] * dd[i] : d1[i] * d1[j]);
      }
  }
  for (int q = 0; q < 6; ++q) red[q][threadIdx.x] = s[q];
  __syncthreads();
  for (int k = kDotThreads / 2; k > 0; k >>= 1) {
    if (threadIdx.x < k)
      for (int q = 0; q < 6; ++q) red[q][threadIdx.x] += red[q][threadIdx.x + k];
    __syncthreads();
  }
  if (threadIdx.x < 6) acc[(long long)(slot0 + threadIdx.x) * gridDim.x + blockIdx.x] += scale * red[threadIdx.x][0];
}

// out = (in + C in) / 2 on the full layout, C the real-density mirror
// F^l_{mn}[k] -> (-1)^(m-n) conj F^l_{-m,-n}[-k].
__global__ void k_sym_full(int lmax, int N, int ndim, long long nx, const double2* __restrict__ in,
                           double2* __restrict__ out) {
  const int D = 2 * lmax + 1;
  const long long Dfull = (long long)D * D * (lmax + 1);
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= Dfull * nx) return;
  const long long fi = t % Dfull, w = t / Dfull;
  const int m = (int)(fi % D) - lmax, n = (int)((fi / D) % D) - lmax, l = (int)(fi / ((long long)D * D));
  long long wm = 0, mul = 1, ww = w;
  for (int a = 0; a < ndim; ++a) {
    const int k = (int)(ww % N);
    ww /= N;
    wm += mul * ((N - k) % N);
    mul *= N;
  }
  const long long fm = (-m + lmax) + (long long)D * (-n + lmax) + (long long)D * D * l;
  const double2 a = in[t], b = in[fm + Dfull * wm];
  const double sg = ((m - n) & 1) ? -1.0 : 1.0;
  out[t] = make_double2(0.5 * (a.x + sg * b.x), 0.5 * (a.y - sg * b.y));
}

template <int N>
int axis_md_launch(hp_plan* p, const double2* in, double2* out, int axis, double coef, cudaStream_t s) {
  const long long nl = p->nrows * (p->nx / N);
  ProfScope _ps(p, "adj.axis", s);
  k_axis_md<N><<<(unsigned)((nl + 127) / 128), 128, 0, s>>>(p->layout(), in, out, axis, coef, p->model.L);
  HP_CUDA_TRY(cudaGetLastError());
  return HP_OK;
}

template <int N>
int line_dm_launch(hp_plan* p, const double2* in, double2* out, int axis, int daxis, double coef, int acc,
                   cudaStream_t s) {
  const long long nl = p->nrows * (p->nx / N);
  ProfScope _ps(p, "adj.axis", s);
  k_line_dm<N><<<(unsigned)((nl + 127) / 128), 128, 0, s>>>(p->layout(), in, out, axis, daxis, coef, p->model.L, acc);
  HP_CUDA_TRY(cudaGetLastError());
  return HP_OK;
}

// out = coef D_daxis M_axis in (acc: out += ...)
int line_dm(hp_plan* p, const double2* in, double2* out, int axis, int daxis, double coef, int acc,
            cudaStream_t s) {
  switch (p->N) {
#define X(n) case n: return line_dm_launch<n>(p, in, out, axis, daxis, coef, acc, s);
    HP_FOR_EACH_N(X)
#undef X
    default:
      hp_set_error("omega grid size 2Bx not supported (even, 4..64)");
      return HP_ERR_UNSUPPORTED;
  }
}

int axis_md(hp_plan* p, const double2* in, double2* out, int axis, double coef, cudaStream_t s) {
  switch (p->N) {
#define X(n) case n: return axis_md_launch<n>(p, in, out, axis, coef, s);
    HP_FOR_EACH_N(X)
#undef X
    default:
      hp_set_error("omega grid size 2Bx not supported (even, 4..64)");
      return HP_ERR_UNSUPPORTED;
  }
}

// out = (add ? lam : 0) + a * A^H lam   (internal layout, FP64 buffers)
int adjoint_apply(hp_plan* p, const double2* lam, double2* out, double a, int add, cudaStream_t s) {
  const DerivParams base = hp_model_params(p);
  DerivParams q = base;
  for (int i = 0; i < 3; ++i) q.b[i] = 0.0;
  for (int i = 0; i < 9; ++i) q.G[i] = -base.G[i];
  int st = HP_OK;
  const size_t ib = 16 * (size_t)p->nrows * p->nx;
  double2* t = (double2*)p->ws_get("adj.t", ib, &st);
  if (st) return st;
  double2* d1 = (double2*)p->ws_get("adj.d1", ib, &st);
  if (st) return st;
  const long long n = p->nrows * p->nx;
  const unsigned g = (unsigned)((n + 255) / 256);
  {
    ProfScope _ps(p, "adj.weight", s);
    k_row_unweight<<<g, 256, 0, s>>>(p->layout(), lam, t);
    HP_CUDA_TRY(cudaGetLastError());
  }
  ADJ_CHECK(hp_derivative_eval_prm(p, q, t, nullptr, 1.0, d1, nullptr, 0.0, s));
  {
    ProfScope _ps(p, "adj.weight", s);
    k_adj_combine<<<g, 256, 0, s>>>(p->layout(), lam, d1, out, a, add);
    HP_CUDA_TRY(cudaGetLastError());
  }
  for (int i = 0; i < p->ndim; ++i)
    if (base.b[i] != 0.0) ADJ_CHECK(axis_md(p, lam, out, i, -a * base.b[i], s));
  return HP_OK;
}

// Gradient slots: b[0..2], gyro[3..5], gscale[6..8], G pairs [9..14]
// ((0,0),(0,1),(0,2),(1,1),(1,2),(2,2)).
constexpr int kSlots = 15;

// acc += dt * Re<lam, dA/dtheta F> for every parameter theta.  The terms of
// the derivative are linear in their parameters, so dA/dtheta F is the term
// itself with unit coefficient, each formed by the passes it needs alone:
//   damping   dA/db_i F    =  D_i M_i F            (one line pass)
//   gyroscope dA/dgyro_i F = -D_i M_j M_k F        (two line passes; j, k the other axes)
//   gravity   dA/dgs_i F   =  the gravity pass with component i alone
// (the forms of the plane pass's Y0, Y1, Y2 products and the axis-3 pass).
int grad_terms(hp_plan* p, const double2* lam, const double2* F, double dt, double* acc, cudaStream_t s) {
  const DerivParams base = hp_model_params(p);
  int st = HP_OK;
  const size_t ib = 16 * (size_t)p->nrows * p->nx;
  double2* y = (double2*)p->ws_get("adj.y", ib, &st);
  if (st) return st;
  const int half = p->symmetry == HP_REAL;
  auto dot = [&](int slot) -> int {
    ProfScope _ps(p, "adj.dot", s);
    k_dot<<<kDotBlocks, kDotThreads, 0, s>>>(p->layout(), lam, y, acc, slot, dt, half);
    HP_CUDA_TRY(cudaGetLastError());
    return HP_OK;
  };
  for (int i = 0; i < p->ndim; ++i) {
    ADJ_CHECK(line_dm(p, F, y, i, i, 1.0, 0, s));
    ADJ_CHECK(dot(i));
  }
  if (p->ndim == 3) {
    double2* t = (double2*)p->ws_get("adj.t", ib, &st);
    if (st) return st;
    for (int i = 0; i < 3; ++i) {
      const int j = (i + 1) % 3, k = (i + 2) % 3;
      ADJ_CHECK(line_dm(p, F, t, j, -1, 1.0, 0, s));
      ADJ_CHECK(line_dm(p, t, y, k, i, -1.0, 0, s));
      ADJ_CHECK(dot(3 + i));
    }
  }
  for (int i = 0; i < p->ndim; ++i) {
    DerivParams z = base;
    for (int a = 0; a < 3; ++a) { z.b[a] = 0; z.gyro[a] = 0; z.gs[a] = 0; }
    for (int a = 0; a < 9; ++a) z.G[a] = 0;
    z.lie = 0;
    z.gs[i] = 1.0;
    ADJ_CHECK(hp_gravity_noise_eval64(p, z, F, y, s));
    ADJ_CHECK(dot(6 + i));
  }
  ProfScope _ps(p, "adj.dot", s);
  k_dot_noise<<<kDotBlocks, kDotThreads, 0, s>>>(p->layout(), lam, F, acc, 9, dt, half, p->model.L);
  HP_CUDA_TRY(cudaGetLastError());
  return HP_OK;
}

int check_mem(int mem) {
  if (mem != HP_DEVICE && mem != HP_HOST) { hp_set_error("mem must be HP_DEVICE or HP_HOST"); return HP_ERR_INVALID; }
  return HP_OK;
}

// full-layout (mem) -> internal FP64, symmetrised for HP_REAL plans
int load_full(hp_plan* p, const double* src, int mem, double2* dst, cudaStream_t s) {
  int st = HP_OK;
  const size_t fb = 16 * (size_t)p->n_full();
  double2* a = (double2*)p->ws_get("adj.full_a", fb, &st);
  if (st) return st;
  const double2* in = (const double2*)src;
  if (mem == HP_HOST) {
    HP_CUDA_TRY(cudaMemcpyAsync(a, src, fb, cudaMemcpyHostToDevice, s));
    in = a;
  }
  if (p->symmetry == HP_REAL) {
    double2* b = (double2*)p->ws_get("adj.full_b", fb, &st);
    if (st) return st;
    const long long n = p->n_full();
    {
      ProfScope _ps(p, "layout", s);
      k_sym_full<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(p->lmax, p->N, p->ndim, p->nx, in, b);
      HP_CUDA_TRY(cudaGetLastError());
    }
    in = b;
  }
  return hp_full_to_internal(p, in, dst, s);
}

int store_full(hp_plan* p, const double2* src, double* dst, int mem, cudaStream_t s) {
  int st = HP_OK;
  const size_t fb = 16 * (size_t)p->n_full();
  double2* out = (double2*)dst;
  if (mem == HP_HOST) {
    out = (double2*)p->ws_get("adj.full_a", fb, &st);
    if (st) return st;
  }
  ADJ_CHECK(hp_internal_to_full(p, src, out, s));
  if (mem == HP_HOST) HP_CUDA_TRY(cudaMemcpyAsync(dst, out, fb, cudaMemcpyDeviceToHost, s));
  return HP_OK;
}

}  // namespace

extern "C" int hp_pendulum_derivative_adjoint(hp_plan* p, const double* lam, double* out, int mem) {
  if (!p || !lam || !out) { hp_set_error("null argument"); return HP_ERR_INVALID; }
  ADJ_CHECK(check_mem(mem));
  if (!p->has_model) { hp_set_error("no model: call hp_plan_set_model first"); return HP_ERR_NO_MODEL; }
  if (p->den_mR) { hp_set_error("the adjoint covers coefficient-gravity models (hp_plan_set_model)"); return HP_ERR_UNSUPPORTED; }
  if (p->so3d64) { hp_set_error("the adjoint covers the pendulum models (no attitude diffusion)"); return HP_ERR_UNSUPPORTED; }
  if (tw_init() != 0) { hp_set_error("twiddle table upload failed"); return HP_ERR_CUDA; }
  cudaStream_t s = p->stream;
  int st = HP_OK;
  const size_t ib = 16 * (size_t)p->nrows * p->nx;
  double2* li = (double2*)p->ws_get("adj.lam", ib, &st);
  if (st) return st;
  double2* lo = (double2*)p->ws_get("adj.lam2", ib, &st);
  if (st) return st;
  // no symmetrisation here: the operator is applied to the given rows
  {
    const size_t fb = 16 * (size_t)p->n_full();
    const double2* in = (const double2*)lam;
    if (mem == HP_HOST) {
      double2* a = (double2*)p->ws_get("adj.full_a", fb, &st);
      if (st) return st;
      HP_CUDA_TRY(cudaMemcpyAsync(a, lam, fb, cudaMemcpyHostToDevice, s));
      in = a;
    }
    ADJ_CHECK(hp_full_to_internal(p, in, li, s));
  }
  ADJ_CHECK(adjoint_apply(p, li, lo, 1.0, 0, s));
  ADJ_CHECK(store_full(p, lo, out, mem, s));
  HP_CUDA_TRY(cudaStreamSynchronize(s));
  return HP_OK;
}

extern "C" int hp_pendulum_adjoint(hp_plan* p, const double* F0, const double* lamT, int nsteps, double dt,
                                   int method, int checkpoint_every, double* lam0, hp_model_grad* grad, int mem) {
  if (!p || !F0 || !lamT || nsteps < 0 || checkpoint_every < 1) { hp_set_error("bad argument"); return HP_ERR_INVALID; }
  ADJ_CHECK(check_mem(mem));
  if (!p->has_model) { hp_set_error("no model: call hp_plan_set_model first"); return HP_ERR_NO_MODEL; }
  if (p->den_mR) { hp_set_error("the adjoint covers coefficient-gravity models (hp_plan_set_model)"); return HP_ERR_UNSUPPORTED; }
  if (p->so3d64) { hp_set_error("the adjoint covers the pendulum models (no attitude diffusion)"); return HP_ERR_UNSUPPORTED; }
  if (method != HP_EULER) { hp_set_error("the adjoint covers forward-Euler trajectories"); return HP_ERR_UNSUPPORTED; }
  if (!std::isfinite(dt)) { hp_set_error("dt must be finite"); return HP_ERR_INVALID; }
  if (tw_init() != 0) { hp_set_error("twiddle table upload failed"); return HP_ERR_CUDA; }
  cudaStream_t s = p->stream;
  int st = HP_OK;
  const size_t ib = 16 * (size_t)p->nrows * p->nx;
  const int ck = std::min(checkpoint_every, std::max(nsteps, 1));
  const int nseg = nsteps > 0 ? (nsteps + ck - 1) / ck : 0;
  // checkpoints [nseg] + one segment of states [ck] + the adjoint pair
  char* ckpt = (char*)p->ws_get("adj.ckpt", ib * (size_t)std::max(nseg, 1), &st);
  if (st) return st;
  char* seg = (char*)p->ws_get("adj.seg", ib * (size_t)ck, &st);
  if (st) return st;
  double2* la = (double2*)p->ws_get("adj.lam", ib, &st);
  if (st) return st;
  double2* lb = (double2*)p->ws_get("adj.lam2", ib, &st);
  if (st) return st;
  double* acc = (double*)p->ws_get("adj.acc", sizeof(double) * kSlots * kDotBlocks, &st);
  if (st) return st;
  HP_CUDA_TRY(cudaMemsetAsync(acc, 0, sizeof(double) * kSlots * kDotBlocks, s));
  auto state = [&](char* b, int i) { return reinterpret_cast<double2*>(b + ib * (size_t)i); };

  // forward sweep, keeping the state at the start of every segment
  {
    const size_t fb = 16 * (size_t)p->n_full();
    const double2* in = (const double2*)F0;
    if (mem == HP_HOST) {
      double2* a = (double2*)p->ws_get("adj.full_a", fb, &st);
      if (st) return st;
      HP_CUDA_TRY(cudaMemcpyAsync(a, F0, fb, cudaMemcpyHostToDevice, s));
      in = a;
    }
    ADJ_CHECK(hp_full_to_internal(p, in, state(ckpt, 0), s));
  }
  for (int g = 0; g + 1 < nseg; ++g) {
    double2* x = state(seg, 0);
    HP_CUDA_TRY(cudaMemcpyAsync(x, state(ckpt, g), ib, cudaMemcpyDeviceToDevice, s));
    for (int j = 0; j < ck; ++j) {
      double2* dst = (j + 1 < ck) ? state(seg, (j + 1) % ck) : state(ckpt, g + 1);
      ADJ_CHECK(hp_derivative_eval(p, state(seg, j), state(seg, j), dt, dst, nullptr, 0.0, s));
    }
  }
  // reverse sweep
  ADJ_CHECK(load_full(p, lamT, mem, la, s));
  for (int g = nseg - 1; g >= 0; --g) {
    const int len = std::min(ck, nsteps - g * ck);
    HP_CUDA_TRY(cudaMemcpyAsync(state(seg, 0), state(ckpt, g), ib, cudaMemcpyDeviceToDevice, s));
    for (int j = 1; j < len; ++j)
      ADJ_CHECK(hp_derivative_eval(p, state(seg, j - 1), state(seg, j - 1), dt, state(seg, j), nullptr, 0.0, s));
    for (int j = len - 1; j >= 0; --j) {
      ADJ_CHECK(grad_terms(p, la, state(seg, j), dt, acc, s));
      ADJ_CHECK(adjoint_apply(p, la, lb, dt, 1, s));
      std::swap(la, lb);
    }
  }
  if (lam0) ADJ_CHECK(store_full(p, la, lam0, mem, s));
  std::vector<double> h((size_t)kSlots * kDotBlocks);
  HP_CUDA_TRY(cudaMemcpyAsync(h.data(), acc, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, s));
  HP_CUDA_TRY(cudaStreamSynchronize(s));
  double tot[kSlots];
  for (int k = 0; k < kSlots; ++k) {
    double v = 0.0;
    for (int b = 0; b < kDotBlocks; ++b) v += h[(size_t)k * kDotBlocks + b];
    tot[k] = v;
  }
  if (grad) {
    for (int i = 0; i < 3; ++i) {
      grad->b[i] = tot[i];
      grad->gyro[i] = tot[3 + i];
      grad->gscale[i] = tot[6 + i];
    }
    const int pi[6] = {0, 0, 0, 1, 1, 2}, pj[6] = {0, 1, 2, 1, 2, 2};
    for (int q = 0; q < 6; ++q) {
      grad->G[pi[q] * 3 + pj[q]] = tot[9 + q];
      grad->G[pj[q] * 3 + pi[q]] = tot[9 + q];
    }
  }
  return HP_OK;
}
