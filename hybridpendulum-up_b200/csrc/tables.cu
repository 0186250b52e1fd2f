// Device tables in FP64 (Wigner-d, quadrature weights, Clebsch-Gordan,
// gravity taps) and the full <-> internal coefficient layout conversions.
#include <cmath>
#include <vector>
#include "common.cuh"
#include "plan.hpp"

using namespace hp;

int hp::tw_fill_host(double2* t64, float2* t32) {
  // exp(-2 pi i e / M) evaluated in long double, rounded to FP64 (and the
  // FP64 value to FP32)
  auto put = [&](int k, int e, int M) {
    const long double a = -2.0L * 3.14159265358979323846264338327950288L * (long double)e / M;
    const double c = (double)cosl(a), s = (double)sinl(a);
    t64[k] = make_double2(c, s);
    t32[k] = make_float2((float)c, (float)s);
  };
  for (int k = 0; k < kTw960; ++k) put(k, k, kTw960);
  for (int M = 1; M <= kTwMaxM; ++M)
    if (tw_own_section(M))
      for (int e = 0; e < M; ++e) put(tw_section(M) + e, e, M);
  return 0;
}

int hp_twiddles_init() {
  if (tw_init() != 0) { hp_set_error("twiddle table upload failed"); return HP_ERR_CUDA; }
  return HP_OK;
}

// ----------------------------------------------------------- Wigner-d ----
// One thread per (beta_j, m, n).  (m, n) is mapped to the entry of the
// fundamental region n <= 0, |m| <= -n that the reference's symmetry fill
// copies from (Wigner_d.m:50-63), and the recursion in l of Wigner_d.m:25-44 is
// run for that entry: closed form at l = -n, two-term step at l = -n+1, the
// three-term recursion above; the l = 1 entry of (0,0) is cos(beta) as in
// Wigner_d.m:17-21.
__global__ void k_wigner(int B, int lmax, const double* __restrict__ fact, double* __restrict__ wfull,
                         RowLayout L, double* __restrict__ wig64, float* __restrict__ wig32) {
  const int D = 2 * lmax + 1;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 2 * B * D * D) return;
  const int m = t % D - lmax, n = (t / D) % D - lmax, b = t / (D * D);
  const double beta = M_PI / (4.0 * B) * (2 * b + 1);
  int ms, ns;
  double sign = 1.0;
  if (n <= 0 && abs(m) <= -n) {
    ms = m; ns = n;
  } else if (m >= 1 && n >= -m + 1 && n <= m) {
    ms = -n; ns = -m;
  } else {  // m < n: d(m,n) = (-1)^(m-n) d(n,m)
    sign = ((m - n) & 1) ? -1.0 : 1.0;
    const int r = n, c = m;
    if (c <= 0 && abs(r) <= -c) { ms = r; ns = c; } else { ms = -c; ns = -r; }
  }
  const double cb = cos(beta), cb2 = cos(beta / 2), sb2 = sin(beta / 2);
  const int l0 = -ns;
  const double mm = ms, nn = ns;
  double dm1 = 0.0, dm2 = 0.0;
  const long long wstride = (long long)D * D * (lmax + 1);
  for (int l = l0; l <= lmax; ++l) {
    double v;
    if (l == l0) {
      v = sqrt(fact[2 * l] / fact[l + ms] / fact[l - ms]) * pow(cb2, (double)(l - ms)) *
          pow(-sb2, (double)(l + ms));
    } else if (l == 1) {
      v = cb;
    } else {
      const double ld = l;
      const double den = sqrt((ld * ld - mm * mm) * (ld * ld - nn * nn));
      v = ld * (2 * ld - 1) / den * (cb - mm * nn / (ld - 1) / ld) * dm1;
      if (l >= l0 + 2)
        v -= sqrt(((ld - 1) * (ld - 1) - mm * mm) * ((ld - 1) * (ld - 1) - nn * nn)) / den * ld /
             (ld - 1) * dm2;
    }
    dm2 = dm1;
    dm1 = v;
    const double out = sign * v;
    wfull[(m + lmax) + (long long)D * (n + lmax) + (long long)D * D * l + wstride * b] = out;
    if (m >= L.m_lo) {
      const int am = abs(m), an = abs(n);
      const long long row = L.seg[(m - L.m_lo) * D + n + lmax] + l - (am > an ? am : an);
      wig64[(long long)b * L.nrows + row] = out;
      wig32[(long long)b * L.nrows + row] = (float)out;
    }
  }
}

// Quadrature weights of fftSO3R.m:62-66.
__global__ void k_weights(int B, double* w) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= 2 * B) return;
  const double beta = M_PI / (4.0 * B) * (2 * j + 1);
  double s = 0.0;
  for (int k = 0; k < B; ++k) s += 1.0 / (2 * k + 1) * sin((2 * k + 1) * beta);
  w[j] = 1.0 / (4.0 * B * B * B) * sin(beta) * s;
}

#include "cg.cuh"

// l2 = 1 table used by the gravity product.
__global__ void k_cg1(int lmax, double* cg1) {
  const int nm = 2 * lmax + 3;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (lmax + 1) * 3 * nm) return;
  const int m = t % nm - (lmax + 1), dl = (t / nm) % 3 - 1, l1 = t / (3 * nm);
  const int l = l1 + dl;
  for (int m2 = -1; m2 <= 1; ++m2) cg1[cg1_index(lmax, l1, dl, m, m2)] = 0.0;
  if (l < 0 || l < abs(l1 - 1) || abs(m) > l) return;
  double C[3], dd[3], du[3], dlw[3], rb[3];
  const int nnz = cg_column(l1, 1, l, m, C, dd, du, dlw, rb);
  const int m1lo = max(-l1, m - 1);
  for (int k = 0; k < nnz; ++k) {
    const int m1 = m1lo + k, m2 = m - m1;
    cg1[cg1_index(lmax, l1, dl, m, m2)] = C[k];
  }
}

// Gravity taps: Grav_i^l_{mn} = sum_{l1, n2} W F^{l1}_{m, n-n2}, with
// W = (2l1+1)*3/(2l+1) <l1 m; 1 0|l m><l1 n-n2; 1 n2|l n> MR_i^1_{0 n2}
// (the l2 = 1, m2 = 0 terms of the CG loop of pendulum.m:474-502).  The
// weight factors into a real part per tap, stored here as
// tap_wr[row*9 + (l1-l+1)*3 + (n2+1)] (zero where the source row does not
// exist), and the model's MR_i^1_{0 n2}, applied per omega point.
template <typename T>
__global__ void k_gravity_taps(RowLayout L, const double* __restrict__ cg1, T* __restrict__ tap_wr) {
  const long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (r >= L.nrows) return;
  const int lmax = L.lmax;
  const char4 q = L.rows[r];
  const int l = q.x, m = q.y, n = q.z;
  for (int t = 0; t < 9; ++t) {
    const int l1 = l + t / 3 - 1, n2 = t % 3 - 1, n1 = n - n2;
    double w = 0.0;
    if (l1 >= 0 && l1 <= lmax && abs(m) <= l1 && abs(n1) <= l1) {
      const double cm = cg1[cg1_index(lmax, l1, l - l1, m, 0)];
      const double cn = cg1[cg1_index(lmax, l1, l - l1, n, n2)];
      w = (2.0 * l1 + 1.0) * 3.0 / (2.0 * l + 1.0) * cm * cn;
    }
    tap_wr[r * 9 + t] = (T)w;
  }
}

// ------------------------------------------------ layout conversions ----
// full (MATLAB F(m,n,l,w)) -> internal rows; tiles of 32 full indices x 32 omega.
__global__ void k_full_to_int(RowLayout L, const double2* __restrict__ Ff, double2* __restrict__ Fi) {
  __shared__ double2 tile[32][33];
  const int D = 2 * L.lmax + 1;
  const long long Dfull = (long long)D * D * (L.lmax + 1);
  const long long fi0 = (long long)blockIdx.x * 32, w0 = (long long)blockIdx.y * 32;
  const int tx = threadIdx.x, ty = threadIdx.y;
  for (int k = ty; k < 32; k += blockDim.y) {
    const long long fi = fi0 + tx, w = w0 + k;
    tile[k][tx] = (fi < Dfull && w < L.nx) ? Ff[fi + Dfull * w] : make_double2(0, 0);
  }
  __syncthreads();
  for (int k = ty; k < 32; k += blockDim.y) {
    const long long fi = fi0 + k, w = w0 + tx;
    if (fi >= Dfull || w >= L.nx) continue;
    const int m = (int)(fi % D) - L.lmax, n = (int)((fi / D) % D) - L.lmax, l = (int)(fi / (D * D));
    const int am = abs(m), an = abs(n);
    if (am > l || an > l || m < L.m_lo) continue;
    const long long row = L.seg[(m - L.m_lo) * D + n + L.lmax] + l - (am > an ? am : an);
    Fi[row * L.nx + w] = tile[tx][k];
  }
}

// full -> internal reading only the kept entries: block = omega point (grid
// stride), threads over the kept entries in full-layout order, so that adjacent
// lanes read adjacent source addresses (the m of one (l, n)) and nothing else
// of the omega slice is touched.  Ff may be page-locked host memory mapped into
// the device address space: only the kept entries (a fifth of the full layout
// for real plans) then cross the bus.  Ff carries no __restrict__ qualifier so
// that its loads stay on the ordinary global path.
__global__ void k_full_gather(const int2* __restrict__ fg, int nrows, long long Dfull, long long nx,
                              const double2* Ff, double2* __restrict__ Fi) {
  for (long long w = blockIdx.x; w < nx; w += gridDim.x) {
    const double2* src = Ff + Dfull * w;
    for (int e = threadIdx.x; e < nrows; e += blockDim.x) {
      const int2 g = fg[e];
      Fi[(long long)g.y * nx + w] = src[g.x];
    }
  }
}

__device__ __forceinline__ long long mirror_w(long long w, int N, int ndim) {
  long long r = 0, mul = 1;
  for (int a = 0; a < ndim; ++a) {
    const int k = (int)(w % N);
    w /= N;
    r += mul * ((N - k) % N);
    mul *= N;
  }
  return r;
}

// internal -> full; zero outside |m|,|n| <= l; rows with m < m_lo (HP_REAL)
// from F^l_{mn}[k] = (-1)^(m-n) conj F^l_{-m,-n}[-k].
__global__ void k_int_to_full(RowLayout L, const double2* __restrict__ Fi, double2* __restrict__ Ff) {
  __shared__ double2 tile[32][33];
  const int D = 2 * L.lmax + 1;
  const long long Dfull = (long long)D * D * (L.lmax + 1);
  const long long fi0 = (long long)blockIdx.x * 32, w0 = (long long)blockIdx.y * 32;
  const int tx = threadIdx.x, ty = threadIdx.y;
  for (int k = ty; k < 32; k += blockDim.y) {
    const long long fi = fi0 + k, w = w0 + tx;
    double2 v = make_double2(0, 0);
    if (fi < Dfull && w < L.nx) {
      int m = (int)(fi % D) - L.lmax, n = (int)((fi / D) % D) - L.lmax;
      const int l = (int)(fi / (D * D));
      const int am = abs(m), an = abs(n);
      if (am <= l && an <= l) {
        if (m >= L.m_lo) {
          const long long row = L.seg[(m - L.m_lo) * D + n + L.lmax] + l - (am > an ? am : an);
          v = Fi[row * L.nx + w];
        } else {
          const long long row = L.seg[(-m - L.m_lo) * D + (-n) + L.lmax] + l - (am > an ? am : an);
          v = Fi[row * L.nx + mirror_w(w, L.N, L.ndim)];
          v.y = -v.y;
          if ((m - n) & 1) { v.x = -v.x; v.y = -v.y; }
        }
      }
    }
    tile[k][tx] = v;
  }
  __syncthreads();
  for (int k = ty; k < 32; k += blockDim.y) {
    const long long fi = fi0 + tx, w = w0 + k;
    if (fi < Dfull && w < L.nx) Ff[fi + Dfull * w] = tile[tx][k];
  }
}

int hp_full_to_internal(hp_plan* p, const double2* Ff, double2* Fi, cudaStream_t s) {
  const int D = p->D;
  const long long Dfull = (long long)D * D * (p->lmax + 1);
  dim3 grid((unsigned)((Dfull + 31) / 32), (unsigned)((p->nx + 31) / 32));
  ProfScope _ps(p, "layout", s);
  k_full_to_int<<<grid, dim3(32, 8), 0, s>>>(p->layout(), Ff, Fi);
  HP_CUDA_TRY(cudaGetLastError());
  return HP_OK;
}

int hp_full_gather(hp_plan* p, const double2* Ff, double2* Fi, cudaStream_t s) {
  const long long Dfull = (long long)p->D * p->D * (p->lmax + 1);
  // every block resident at once (8 per SM at 256 threads), each walking
  // omega points
  const unsigned g = (unsigned)std::min<long long>(p->nx, 148LL * 8);
  ProfScope _ps(p, "layout", s);
  k_full_gather<<<g, 256, 0, s>>>(p->fgather, (int)p->nrows, Dfull, p->nx, Ff, Fi);
  HP_CUDA_TRY(cudaGetLastError());
  return HP_OK;
}

int hp_internal_to_full(hp_plan* p, const double2* Fi, double2* Ff, cudaStream_t s) {
  const int D = p->D;
  const long long Dfull = (long long)D * D * (p->lmax + 1);
  dim3 grid((unsigned)((Dfull + 31) / 32), (unsigned)((p->nx + 31) / 32));
  ProfScope _ps(p, "layout", s);
  k_int_to_full<<<grid, dim3(32, 8), 0, s>>>(p->layout(), Fi, Ff);
  HP_CUDA_TRY(cudaGetLastError());
  return HP_OK;
}

// -------------------------------------------------------------- build ----
int hp_tables_build(hp_plan* p) {
  int st = hp_twiddles_init();
  if (st) return st;
  const int B = p->B, lmax = p->lmax, D = p->D;
  // host row layout
  p->h_seg.assign((size_t)p->nm * D, 0);
  p->h_rows.clear();
  for (int m = p->m_lo; m <= lmax; ++m)
    for (int n = -lmax; n <= lmax; ++n) {
      p->h_seg[(size_t)(m - p->m_lo) * D + n + lmax] = (int)p->h_rows.size();
      const int l0 = std::max(std::abs(m), std::abs(n));
      for (int l = l0; l <= lmax; ++l) p->h_rows.push_back(make_char4((char)l, (char)m, (char)n, 0));
    }
  p->nrows = (long long)p->h_rows.size();
  HP_CUDA_TRY(hp_dev_alloc(&p->rows, sizeof(char4) * p->nrows));
  HP_CUDA_TRY(hp_dev_alloc(&p->seg, sizeof(int) * p->h_seg.size()));
  HP_CUDA_TRY(cudaMemcpy(p->rows, p->h_rows.data(), sizeof(char4) * p->nrows, cudaMemcpyHostToDevice));
  HP_CUDA_TRY(cudaMemcpy(p->seg, p->h_seg.data(), sizeof(int) * p->h_seg.size(), cudaMemcpyHostToDevice));
  // kept entries in full-layout order (m fastest, then n, then l), for the
  // gather that reads only them (k_full_gather)
  {
    std::vector<int2> fg;
    fg.reserve((size_t)p->nrows);
    for (int l = 0; l <= lmax; ++l)
      for (int n = -l; n <= l; ++n)
        for (int m = std::max(-l, p->m_lo); m <= l; ++m) {
          const int fi = (m + lmax) + D * (n + lmax) + D * D * l;
          const int row = p->h_seg[(size_t)(m - p->m_lo) * D + n + lmax] + l - std::max(std::abs(m), std::abs(n));
          fg.push_back(make_int2(fi, row));
        }
    if ((long long)fg.size() != p->nrows) { hp_set_error("internal: kept-entry table size"); return HP_ERR_INVALID; }
    HP_CUDA_TRY(hp_dev_alloc(&p->fgather, sizeof(int2) * fg.size()));
    HP_CUDA_TRY(cudaMemcpy(p->fgather, fg.data(), sizeof(int2) * fg.size(), cudaMemcpyHostToDevice));
  }

  std::vector<double> fact(2 * lmax + 2, 1.0);
  for (int k = 1; k < (int)fact.size(); ++k) fact[k] = fact[k - 1] * k;
  double* dfact = nullptr;
  HP_CUDA_TRY(hp_dev_alloc(&dfact, sizeof(double) * fact.size()));
  HP_CUDA_TRY(cudaMemcpy(dfact, fact.data(), sizeof(double) * fact.size(), cudaMemcpyHostToDevice));

  const long long nwfull = (long long)D * D * (lmax + 1) * 2 * B;
  HP_CUDA_TRY(hp_dev_alloc(&p->wfull, sizeof(double) * nwfull));
  HP_CUDA_TRY(cudaMemset(p->wfull, 0, sizeof(double) * nwfull));
  HP_CUDA_TRY(hp_dev_alloc(&p->wig64, sizeof(double) * 2 * B * p->nrows));
  HP_CUDA_TRY(hp_dev_alloc(&p->wig32, sizeof(float) * 2 * B * p->nrows));
  HP_CUDA_TRY(hp_dev_alloc(&p->qw, sizeof(double) * 2 * B));
  const int nth = 2 * B * D * D;
  k_wigner<<<(nth + 127) / 128, 128>>>(B, lmax, dfact, p->wfull, p->layout(), p->wig64, p->wig32);
  HP_CUDA_TRY(cudaGetLastError());
  k_weights<<<1, 2 * B>>>(B, p->qw);
  HP_CUDA_TRY(cudaGetLastError());
  const int ncg = (lmax + 1) * 3 * (2 * lmax + 3) * 3;
  HP_CUDA_TRY(hp_dev_alloc(&p->cg1, sizeof(double) * ncg));
  const int nt_cg = (lmax + 1) * 3 * (2 * lmax + 3);
  k_cg1<<<(nt_cg + 127) / 128, 128>>>(lmax, p->cg1);
  HP_CUDA_TRY(cudaGetLastError());
  HP_CUDA_TRY(cudaDeviceSynchronize());
  hp_dev_free(dfact);
  return HP_OK;
}

int hp_build_gravity_taps(hp_plan* p) {
  if (p->tap_wr) return HP_OK;
  HP_CUDA_TRY(hp_dev_alloc(&p->tap_wr, sizeof(double) * 9 * p->nrows));
  HP_CUDA_TRY(hp_dev_alloc(&p->tap_wr32, sizeof(float) * 9 * p->nrows));
  const unsigned g = (unsigned)((p->nrows + 127) / 128);
  k_gravity_taps<double><<<g, 128, 0, p->stream>>>(p->layout(), p->cg1, p->tap_wr);
  k_gravity_taps<float><<<g, 128, 0, p->stream>>>(p->layout(), p->cg1, p->tap_wr32);
  HP_CUDA_TRY(cudaGetLastError());
  return HP_OK;
}
