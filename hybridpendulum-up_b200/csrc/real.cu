// Real-harmonic SO(3) transforms (the isreal branches of fftSO3.m:61-119 and
// ifftSO3.m:24-84), batched over independent functions on the plan's SO(3)
// grid (the omega part of the plan is not used).
//
// Real harmonics are built from Wigner-d through Psi(m, n, l, beta)
// (fftSO3.m:62-88): for n <= 0
//   m = n = 0 : d^l_00 ;  m = 0 or n = 0 : (-1)^(m-n) sqrt2 d^l_{|m||n|} ;
//   else      : (-1)^(m-n) d^l_{|m||n|} + (-1)^m sign(m) d^l_{|m|,-|n|},
// and Psi(m, n) = Psi(m, -n) for n > 0.  The coefficients F(m, n, l) are real.
//
// Forward, per function b and beta_j:
//   S[m][n] = sum_{a,c} f(a, j, c) e^{-2 pi i (a m + c n) / 2B}       (fft2, fftshift-ed)
// then per (l, m, n): F = sum_j w_j [ -1/2 (X(m,-n) -+ X(m,n)) Psi(-m,n) + 1/2 (X(m,-n) +- X(m,n)) Psi(m,n) ]
// with X = Re S for m, n of the same sign class (both >= 0 or both < 0) and
// X = -Im S (and the other sign pattern) otherwise (fftSO3.m:96-117).
// Backward, per (m, j, n): S1 = sum_l (2l+1) F Psi(m,n), F1 = sum_l (2l+1) F Psi(-m,n),
// then f(a, j, c) = sum_{m,n} F1 (-sin m alpha_a) t1(n, gamma_c) + S1 cos(m alpha_a) t2(n, gamma_c)
// with (t1, t2) = (sin, cos) for m, n of the same sign class, (cos, sin) otherwise
// (ifftSO3.m:69-83).  Both 2-D sums over (alpha, gamma) are done separably per
// (beta, function) block in shared memory; everything is FP64.
#include <cmath>
#include <vector>
#include "common.cuh"
#include "plan.hpp"

using namespace hp;

#define HP_CHECK(expr)              \
  do {                              \
    int _s = (expr);                \
    if (_s != HP_OK) return _s;     \
  } while (0)

// Psi in the layout of the Wigner-d table: (m+lmax) + D (n+lmax) + D^2 l + D^2 (lmax+1) j
__global__ void k_real_psi(int B, const double* __restrict__ d, double* __restrict__ psi) {
  const int lmax = B - 1, D = 2 * lmax + 1;
  const long long tot = (long long)D * D * (lmax + 1) * 2 * B;
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= tot) return;
  const int m = (int)(t % D) - lmax, n = (int)((t / D) % D) - lmax;
  const int l = (int)((t / ((long long)D * D)) % (lmax + 1));
  const long long j = t / ((long long)D * D * (lmax + 1));
  const long long js = (long long)D * D * (lmax + 1) * j;
  double v = 0.0;
  if (abs(m) <= l && abs(n) <= l) {
    const int am = abs(m), an = abs(n);
    const double sg = ((m - n) & 1) ? -1.0 : 1.0;   // (-1)^(m-n), and (-1)^(m+n) alike
    auto dd = [&](int a, int b) { return d[(a + lmax) + (long long)D * (b + lmax) + (long long)D * D * l + js]; };
    if (m == 0 && n == 0) v = dd(0, 0);
    else if (m == 0 || n == 0) v = sg * M_SQRT2 * dd(am, an);
    else v = sg * dd(am, an) + ((m & 1) ? -1.0 : 1.0) * (m > 0 ? 1.0 : -1.0) * dd(am, -an);
  }
  psi[t] = v;
}

// e^{-2 pi i k / N} for k in [0, N)
__device__ __forceinline__ double2 unit_root(int k, int N) {
  double s, c;
  sincospi(2.0 * (double)k / (double)N, &s, &c);
  return make_double2(c, -s);
}

// Forward, stage 1: S[b][j][m][n] for m, n in [-lmax, lmax]; one block per (j, b).
__global__ void k_real_fwd_slice(int B, const double* __restrict__ f, double2* __restrict__ S) {
  const int N = 2 * B, lmax = B - 1, D = 2 * lmax + 1;
  const int j = blockIdx.x, b = blockIdx.y;
  extern __shared__ __align__(16) unsigned char smraw[];
  double* sf = reinterpret_cast<double*>(smraw);              // [c][a]
  double2* sy = reinterpret_cast<double2*>(sf + N * N);       // [c][m] after the alpha sums
  double2* tw = sy + N * D;                                   // [N] roots
  const int tid = threadIdx.x, nth = blockDim.x;
  for (int k = tid; k < N; k += nth) tw[k] = unit_root(k, N);
  for (int e = tid; e < N * N; e += nth) {
    const int a = e % N, c = e / N;
    sf[e] = f[a + (long long)N * (j + (long long)N * (c + (long long)N * b))];
  }
  __syncthreads();
  // Y[c][m] = sum_a f(a, c) e^{-2 pi i a m / N}
  for (int e = tid; e < N * D; e += nth) {
    const int c = e / D, m = e % D - lmax;
    double2 acc = make_double2(0, 0);
    for (int a = 0; a < N; ++a) {
      const double2 w = tw[((a * m) % N + N) % N];
      acc.x += sf[c * N + a] * w.x;
      acc.y += sf[c * N + a] * w.y;
    }
    sy[e] = acc;
  }
  __syncthreads();
  // S[m][n] = sum_c Y[c][m] e^{-2 pi i c n / N}
  double2* out = S + ((long long)b * N + j) * D * D;
  for (int e = tid; e < D * D; e += nth) {
    const int mi = e / D, n = e % D - lmax;
    double2 acc = make_double2(0, 0);
    for (int c = 0; c < N; ++c) {
      const double2 y = sy[c * D + mi], w = tw[((c * n) % N + N) % N];
      acc.x += y.x * w.x - y.y * w.y;
      acc.y += y.x * w.y + y.y * w.x;
    }
    out[e] = acc;
  }
}

// Forward, stage 2: one thread per (l, m, n, b), the weighted beta sum.
__global__ void k_real_fwd_beta(int B, int nb, const double2* __restrict__ S, const double* __restrict__ psi,
                                const double* __restrict__ w, double* __restrict__ F) {
  const int N = 2 * B, lmax = B - 1, D = 2 * lmax + 1;
  const long long per = (long long)D * D * (lmax + 1);
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= per * nb) return;
  const int m = (int)(t % D) - lmax, n = (int)((t / D) % D) - lmax;
  const int l = (int)((t / ((long long)D * D)) % (lmax + 1));
  const int b = (int)(t / per);
  double acc = 0.0;
  if (abs(m) <= l && abs(n) <= l) {
    const bool same = (m >= 0) == (n >= 0);
    for (int j = 0; j < N; ++j) {
      const double2* Sj = S + ((long long)b * N + j) * D * D;
      const double2 smn = Sj[(m + lmax) * D + (n + lmax)], smn_ = Sj[(m + lmax) * D + (-n + lmax)];
      const long long js = per * j;
      const double p1 = psi[(-m + lmax) + (long long)D * (n + lmax) + (long long)D * D * l + js];
      const double p2 = psi[(m + lmax) + (long long)D * (n + lmax) + (long long)D * D * l + js];
      double v;
      if (same) v = -0.5 * (smn_.x - smn.x) * p1 + 0.5 * (smn_.x + smn.x) * p2;
      else v = -0.5 * (-smn.y - smn_.y) * p1 + 0.5 * (-smn.y + smn_.y) * p2;
      acc += w[j] * v;
    }
  }
  F[t] = acc;
}

// Backward, stage 1: S1, F1 [b][j][m][n]; one thread per (m, n, j, b).
__global__ void k_real_bwd_beta(int B, int nb, const double* __restrict__ F, const double* __restrict__ psi,
                                double2* __restrict__ SF) {
  const int N = 2 * B, lmax = B - 1, D = 2 * lmax + 1;
  const long long per = (long long)D * D * (lmax + 1);
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)D * D * N * nb) return;
  const int mi = (int)(t % D), ni = (int)((t / D) % D);
  const int j = (int)((t / ((long long)D * D)) % N), b = (int)(t / ((long long)D * D * N));
  const int m = mi - lmax, n = ni - lmax;
  const int lmin = max(abs(m), abs(n));
  double s1 = 0.0, f1 = 0.0;
  for (int l = lmin; l <= lmax; ++l) {
    const double fl = (2.0 * l + 1.0) * F[mi + (long long)D * ni + (long long)D * D * l + per * b];
    const long long o = (long long)D * ni + (long long)D * D * l + per * j;
    s1 += fl * psi[mi + o];
    f1 += fl * psi[(-m + lmax) + o];
  }
  SF[((long long)b * N + j) * D * D + (long long)mi * D + ni] = make_double2(s1, f1);
}

// Backward, stage 2: one block per (j, b): Q[m][c] = sum_n (F1 t1, S1 t2), then
// f(a, j, c) = sum_m -sin(m alpha_a) Q1[m][c] + cos(m alpha_a) Q2[m][c].
__global__ void k_real_bwd_slice(int B, const double2* __restrict__ SF, double* __restrict__ f) {
  const int N = 2 * B, lmax = B - 1, D = 2 * lmax + 1;
  const int j = blockIdx.x, b = blockIdx.y;
  extern __shared__ __align__(16) unsigned char smraw[];
  double2* ssf = reinterpret_cast<double2*>(smraw);   // [m][n] (S1, F1)
  double2* sq = ssf + D * D;                          // [m][c] (Q1, Q2)
  double2* tw = sq + D * N;                           // [N] (cos, sin) of 2 pi k / N
  const int tid = threadIdx.x, nth = blockDim.x;
  for (int k = tid; k < N; k += nth) {
    double s, c;
    sincospi(2.0 * (double)k / (double)N, &s, &c);
    tw[k] = make_double2(c, s);
  }
  const double2* src = SF + ((long long)b * N + j) * D * D;
  for (int e = tid; e < D * D; e += nth) ssf[e] = src[e];
  __syncthreads();
  for (int e = tid; e < D * N; e += nth) {
    const int mi = e / N, c = e % N, m = mi - lmax;
    double q1 = 0.0, q2 = 0.0;
    for (int ni = 0; ni < D; ++ni) {
      const int n = ni - lmax;
      const double2 cs = tw[((n * c) % N + N) % N];   // cos, sin of n gamma_c
      const double2 v = ssf[mi * D + ni];              // (S1, F1)
      const bool same = (m >= 0) == (n >= 0);
      q1 += v.y * (same ? cs.y : cs.x);
      q2 += v.x * (same ? cs.x : cs.y);
    }
    sq[e] = make_double2(q1, q2);
  }
  __syncthreads();
  for (int e = tid; e < N * N; e += nth) {
    const int a = e % N, c = e / N;
    double acc = 0.0;
    for (int mi = 0; mi < D; ++mi) {
      const int m = mi - lmax;
      const double2 cs = tw[((m * a) % N + N) % N];
      const double2 q = sq[mi * N + c];
      acc += -cs.y * q.x + cs.x * q.y;
    }
    f[a + (long long)N * (j + (long long)N * (c + (long long)N * b))] = acc;
  }
}

static const double* real_psi(hp_plan* p, int* st) {
  bool fresh = true;
  for (auto& kv : p->ws) if (kv.first == "real.psi") fresh = false;
  const long long n = (long long)p->D * p->D * (p->lmax + 1) * 2 * p->B;
  double* psi = (double*)p->ws_get("real.psi", sizeof(double) * n, st);
  if (*st) return nullptr;
  if (fresh) {
    k_real_psi<<<(unsigned)((n + 255) / 256), 256, 0, p->stream>>>(p->B, p->wfull, psi);
    if (cudaGetLastError() != cudaSuccess) { hp_set_error("psi table launch failed"); *st = HP_ERR_CUDA; return nullptr; }
  }
  return psi;
}

static int real_args(hp_plan* p, const void* a, const void* b, int nbatch, int mem) {
  if (!p || !a || !b) { hp_set_error("null argument"); return HP_ERR_INVALID; }
  if (mem != HP_DEVICE && mem != HP_HOST) { hp_set_error("mem must be HP_DEVICE or HP_HOST"); return HP_ERR_INVALID; }
  if (nbatch < 1 || nbatch > 65535) { hp_set_error("nbatch must be in 1..65535"); return HP_ERR_INVALID; }
  return HP_OK;
}

extern "C" int hp_fftSO3_real_forward(hp_plan* p, const double* f, double* F, int nbatch, int mem) {
  HP_CHECK(real_args(p, f, F, nbatch, mem));
  const int B = p->B, N = 2 * B, D = p->D;
  const size_t nf = (size_t)N * N * N * nbatch, nF = (size_t)D * D * B * nbatch;
  int st = HP_OK;
  const double* psi = real_psi(p, &st);
  if (st) return st;
  double2* S = (double2*)p->ws_get("real.S", sizeof(double2) * (size_t)D * D * N * nbatch, &st);
  if (st) return st;
  const double* fd = f;
  double* Fd = F;
  if (mem == HP_HOST) {
    double* a = (double*)p->ws_get("real.f", sizeof(double) * nf, &st);
    if (st) return st;
    Fd = (double*)p->ws_get("real.F", sizeof(double) * nF, &st);
    if (st) return st;
    HP_CUDA_TRY(cudaMemcpyAsync(a, f, sizeof(double) * nf, cudaMemcpyHostToDevice, p->stream));
    fd = a;
  }
  {
    ProfScope _ps(p, "real.fwd", p->stream);
    const size_t sm = sizeof(double) * N * N + sizeof(double2) * ((size_t)N * D + N);
    HP_CUDA_TRY(cudaFuncSetAttribute(k_real_fwd_slice, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    k_real_fwd_slice<<<dim3(N, nbatch), 256, sm, p->stream>>>(B, fd, S);
    const long long nt = (long long)nF;
    k_real_fwd_beta<<<(unsigned)((nt + 127) / 128), 128, 0, p->stream>>>(B, nbatch, S, psi, p->qw, Fd);
    HP_CUDA_TRY(cudaGetLastError());
  }
  if (mem == HP_HOST) HP_CUDA_TRY(cudaMemcpyAsync(F, Fd, sizeof(double) * nF, cudaMemcpyDeviceToHost, p->stream));
  HP_CUDA_TRY(cudaStreamSynchronize(p->stream));
  return HP_OK;
}

extern "C" int hp_fftSO3_real_backward(hp_plan* p, const double* F, double* f, int nbatch, int mem) {
  HP_CHECK(real_args(p, F, f, nbatch, mem));
  const int B = p->B, N = 2 * B, D = p->D;
  const size_t nf = (size_t)N * N * N * nbatch, nF = (size_t)D * D * B * nbatch;
  int st = HP_OK;
  const double* psi = real_psi(p, &st);
  if (st) return st;
  double2* SF = (double2*)p->ws_get("real.S", sizeof(double2) * (size_t)D * D * N * nbatch, &st);
  if (st) return st;
  const double* Fd = F;
  double* fd = f;
  if (mem == HP_HOST) {
    double* a = (double*)p->ws_get("real.F", sizeof(double) * nF, &st);
    if (st) return st;
    fd = (double*)p->ws_get("real.f", sizeof(double) * nf, &st);
    if (st) return st;
    HP_CUDA_TRY(cudaMemcpyAsync(a, F, sizeof(double) * nF, cudaMemcpyHostToDevice, p->stream));
    Fd = a;
  }
  {
    ProfScope _ps(p, "real.bwd", p->stream);
    const long long nt = (long long)D * D * N * nbatch;
    k_real_bwd_beta<<<(unsigned)((nt + 127) / 128), 128, 0, p->stream>>>(B, nbatch, Fd, psi, SF);
    const size_t sm = sizeof(double2) * ((size_t)D * D + (size_t)D * N + N);
    HP_CUDA_TRY(cudaFuncSetAttribute(k_real_bwd_slice, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    k_real_bwd_slice<<<dim3(N, nbatch), 256, sm, p->stream>>>(B, SF, fd);
    HP_CUDA_TRY(cudaGetLastError());
  }
  if (mem == HP_HOST) HP_CUDA_TRY(cudaMemcpyAsync(f, fd, sizeof(double) * nf, cudaMemcpyDeviceToHost, p->stream));
  HP_CUDA_TRY(cudaStreamSynchronize(p->stream));
  return HP_OK;
}

// ------------------------------------------------------- real product ----
// fftSO3_prod.m:97-205 (isreal) builds real Clebsch-Gordan matrices from the
// unitary T^l of lines 103-120; equivalently, with F_c^l = (T^l)^H F_r^l T^l the
// complex coefficients of the same function, FG_r^l = Re T^l FG_c^l (T^l)^H for
// the complex product FG_c (hp_fftSO3_prod).  T^l has two entries per row:
//   r < 0 : T[r][r] = i/sqrt2,       T[r][-r] = -i (-1)^r / sqrt2
//   r = 0 : T[0][0] = 1
//   r > 0 : T[r][r] = (-1)^r/sqrt2,  T[r][-r] = 1/sqrt2
__device__ __forceinline__ double2 t_entry(int r, int c) {
  const double h = M_SQRT1_2, sr = (r & 1) ? -1.0 : 1.0;
  if (r == 0) return make_double2(c == 0 ? 1.0 : 0.0, 0.0);
  if (c == r) return r < 0 ? make_double2(0.0, h) : make_double2(sr * h, 0.0);
  if (c == -r) return r < 0 ? make_double2(0.0, -sr * h) : make_double2(h, 0.0);
  return make_double2(0.0, 0.0);
}

// Fc[m][n] = sum_{p in {m,-m}, q in {n,-n}} conj(T[p][m]) Fr[p][q] T[q][n]
__global__ void k_real_to_cplx(int B, int nb, const double* __restrict__ Fr, double2* __restrict__ Fc) {
  const int lmax = B - 1, D = 2 * lmax + 1;
  const long long per = (long long)D * D * (lmax + 1);
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= per * nb) return;
  const int m = (int)(t % D) - lmax, n = (int)((t / D) % D) - lmax;
  const int l = (int)((t / ((long long)D * D)) % (lmax + 1));
  const long long base = t - ((long long)(m + lmax) + (long long)D * (n + lmax));
  double2 acc = make_double2(0.0, 0.0);
  if (abs(m) <= l && abs(n) <= l) {
    for (int ip = 0; ip < (m == 0 ? 1 : 2); ++ip) {
      const int p = ip ? -m : m;
      const double2 a = t_entry(p, m);              // T[p][m], conjugated below
      for (int iq = 0; iq < (n == 0 ? 1 : 2); ++iq) {
        const int q = iq ? -n : n;
        const double2 b = t_entry(q, n);
        const double v = Fr[base + (p + lmax) + (long long)D * (q + lmax)];
        // conj(a) * v * b
        const double2 ab = make_double2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
        acc.x += v * ab.x;
        acc.y += v * ab.y;
      }
    }
  }
  Fc[t] = acc;
}

// Xr[m][n] = Re sum_{p in {m,-m}, q in {n,-n}} T[m][p] Xc[p][q] conj(T[n][q])
__global__ void k_cplx_to_real(int B, int nb, const double2* __restrict__ Xc, double* __restrict__ Xr) {
  const int lmax = B - 1, D = 2 * lmax + 1;
  const long long per = (long long)D * D * (lmax + 1);
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= per * nb) return;
  const int m = (int)(t % D) - lmax, n = (int)((t / D) % D) - lmax;
  const int l = (int)((t / ((long long)D * D)) % (lmax + 1));
  const long long base = t - ((long long)(m + lmax) + (long long)D * (n + lmax));
  double acc = 0.0;
  if (abs(m) <= l && abs(n) <= l) {
    for (int ip = 0; ip < (m == 0 ? 1 : 2); ++ip) {
      const int p = ip ? -m : m;
      const double2 a = t_entry(m, p);
      for (int iq = 0; iq < (n == 0 ? 1 : 2); ++iq) {
        const int q = iq ? -n : n;
        const double2 b = t_entry(n, q);                 // conjugated below
        const double2 x = Xc[base + (p + lmax) + (long long)D * (q + lmax)];
        const double2 ax = make_double2(a.x * x.x - a.y * x.y, a.x * x.y + a.y * x.x);
        acc += ax.x * b.x + ax.y * b.y;                  // Re(ax * conj(b))
      }
    }
  }
  Xr[t] = acc;
}

extern "C" int hp_fftSO3_real_prod(hp_plan* p, const double* F, const double* G, double* FG, int batch, int mem) {
  HP_CHECK(real_args(p, F, G, batch, mem));
  if (!FG) { hp_set_error("null argument"); return HP_ERR_INVALID; }
  const int B = p->B, D = p->D;
  const size_t n = (size_t)D * D * B * batch;
  int st = HP_OK;
  double2* Fc = (double2*)p->ws_get("realprod.Fc", sizeof(double2) * n, &st);
  if (st) return st;
  double2* Gc = (double2*)p->ws_get("realprod.Gc", sizeof(double2) * n, &st);
  if (st) return st;
  double2* FGc = (double2*)p->ws_get("realprod.FGc", sizeof(double2) * n, &st);
  if (st) return st;
  const double *Fd = F, *Gd = G;
  double* FGd = FG;
  if (mem == HP_HOST) {
    double* a = (double*)p->ws_get("realprod.F", sizeof(double) * n, &st);
    if (st) return st;
    double* b = (double*)p->ws_get("realprod.G", sizeof(double) * n, &st);
    if (st) return st;
    FGd = (double*)p->ws_get("realprod.FG", sizeof(double) * n, &st);
    if (st) return st;
    HP_CUDA_TRY(cudaMemcpyAsync(a, F, sizeof(double) * n, cudaMemcpyHostToDevice, p->stream));
    HP_CUDA_TRY(cudaMemcpyAsync(b, G, sizeof(double) * n, cudaMemcpyHostToDevice, p->stream));
    Fd = a;
    Gd = b;
  }
  const unsigned g = (unsigned)((n + 127) / 128);
  {
    ProfScope _ps(p, "real.prod", p->stream);
    k_real_to_cplx<<<g, 128, 0, p->stream>>>(B, batch, Fd, Fc);
    k_real_to_cplx<<<g, 128, 0, p->stream>>>(B, batch, Gd, Gc);
    HP_CUDA_TRY(cudaGetLastError());
  }
  HP_CHECK(hp_prod_launch(p, Fc, Gc, FGc, batch, p->stream));
  {
    ProfScope _ps(p, "real.prod", p->stream);
    k_cplx_to_real<<<g, 128, 0, p->stream>>>(B, batch, FGc, FGd);
    HP_CUDA_TRY(cudaGetLastError());
  }
  if (mem == HP_HOST) HP_CUDA_TRY(cudaMemcpyAsync(FG, FGd, sizeof(double) * n, cudaMemcpyDeviceToHost, p->stream));
  HP_CUDA_TRY(cudaStreamSynchronize(p->stream));
  return HP_OK;
}
