// Moments of the density for the per-step statistics get_stat
// (propagation/pendulum.m:547-594, pendulum_reduced_hybrid.m:304-351).
//
// Every moment get_stat needs integrates f against a polynomial of degree <= 2
// in the entries of R and in omega, so it is a finite combination of the
// transform coefficients: with F^l_mn[k] = sum_R w conj(D^l_mn(R)) DFT_omega f,
//   E[h(R)]     = c0 sum_lmn a^h_lmn F^l_mn[0]          (h = sum a^h conj(D^l_mn))
//   E[x_i h(R)] = c0/N sum_q sum_lmn a^h_lmn F^l_mn[q e_i] conj(xi(q))
//   E[x_i x_j]  = c0/N^2 sum_{q,r} F^0_00[q e_i + r e_j] conj(xi(q) xi(r))
// with c0 = (L/2Bx)^n, xi(q) = sum_t x(t) e^{-2 pi i q t/N}.  The right-hand
// sides are the same discrete sums as the reference's grid sums (the forward
// transform is itself a grid sum), so no pass over f is needed: a gather of a
// few hundred coefficients and host arithmetic.
#include <cmath>
#include <complex>
#include <cstring>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "common.cuh"
#include "plan.hpp"

using namespace hp;
using cd = std::complex<double>;

#define ST_CHECK(expr)          \
  do {                          \
    int _s = (expr);            \
    if (_s != HP_OK) return _s; \
  } while (0)

extern "C" int hp_plan_create(hp_plan** out, int B, int Bx, int ndim, int precision, int symmetry);
extern "C" int hp_plan_destroy(hp_plan* p);
extern "C" int hp_wigner_d(hp_plan* p, double* d, int mem);
extern "C" int hp_quad_weights(hp_plan* p, double* w, int mem);

namespace {

constexpr int kNB = 35;  // (l, m, n) with l <= 2
struct Lmn { int l, m, n; };
Lmn basis(int t) {
  int k = t;
  for (int l = 0; l <= 2; ++l) {
    const int sz = (2 * l + 1) * (2 * l + 1);
    if (k < sz) return {l, k / (2 * l + 1) - l, k % (2 * l + 1) - l};
    k -= sz;
  }
  return {0, 0, 0};
}

// a^h_{lmn} for h = R_kq (9) and R_kq R_k'q' (81): exact quadrature on the
// B = 3 grid, a = (2l+1) sum_g w_b h(g) D^l_mn(g), D^l_mn = e^{-im alpha} d e^{-in gamma},
// with the Wigner d table of a B = 3 plan (the reference's convention).
std::once_flag g_once;
int g_status = HP_OK;
std::vector<cd> g_aR, g_aRR;

void build_tables() {
  hp_plan* h = nullptr;
  g_status = hp_plan_create(&h, 3, 2, 2, HP_FP64, HP_REAL);
  if (g_status) return;
  const int B = 3, lmax = 2, D = 5, nb = 6;
  std::vector<double> d((size_t)D * D * (lmax + 1) * nb), w(nb);
  g_status = hp_wigner_d(h, d.data(), HP_HOST);
  if (!g_status) g_status = hp_quad_weights(h, w.data(), HP_HOST);
  hp_plan_destroy(h);
  if (g_status) return;
  g_aR.assign((size_t)9 * kNB, cd(0, 0));
  g_aRR.assign((size_t)81 * kNB, cd(0, 0));
  for (int a = 0; a < nb; ++a)
    for (int b = 0; b < nb; ++b)
      for (int c = 0; c < nb; ++c) {
        const double al = M_PI / B * a, be = M_PI / (4.0 * B) * (2 * b + 1), ga = M_PI / B * c;
        const double ca = std::cos(al), sa = std::sin(al), cb = std::cos(be), sb = std::sin(be);
        const double cg = std::cos(ga), sg = std::sin(ga);
        // R = Rz(alpha) Ry(beta) Rz(gamma) (fftSO3R.m:30-47)
        const double Ra[3][3] = {{ca, -sa, 0}, {sa, ca, 0}, {0, 0, 1}};
        const double Rb[3][3] = {{cb, 0, sb}, {0, 1, 0}, {-sb, 0, cb}};
        const double Rg[3][3] = {{cg, -sg, 0}, {sg, cg, 0}, {0, 0, 1}};
        double T[3][3] = {}, R[3][3] = {};
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j)
            for (int k = 0; k < 3; ++k) T[i][j] += Ra[i][k] * Rb[k][j];
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j)
            for (int k = 0; k < 3; ++k) R[i][j] += T[i][k] * Rg[k][j];
        for (int t = 0; t < kNB; ++t) {
          const Lmn q = basis(t);
          const double dv = d[(size_t)(q.m + lmax) + D * (q.n + lmax) + (size_t)D * D * q.l + (size_t)D * D * (lmax + 1) * b];
          const cd Dv = std::polar(1.0, -q.m * al) * dv * std::polar(1.0, -q.n * ga);
          const cd s = Dv * (w[b] * (2 * q.l + 1));
          for (int h1 = 0; h1 < 9; ++h1) {
            const double r1 = R[h1 / 3][h1 % 3];
            g_aR[(size_t)h1 * kNB + t] += s * r1;
            for (int h2 = 0; h2 < 9; ++h2) g_aRR[((size_t)h1 * 9 + h2) * kNB + t] += s * (r1 * R[h2 / 3][h2 % 3]);
          }
        }
      }
}

__global__ void k_gather(const double2* __restrict__ F, const long long* __restrict__ idx, double2* __restrict__ out,
                         int n) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) out[t] = F[idx[t]];
}

int moments_internal(hp_plan* p, const double2* Fi, hp_moments_t* out, double* fx) {
  std::call_once(g_once, build_tables);
  if (g_status) return g_status;
  if (p->lmax < 2) { hp_set_error("moments need B >= 3 (second moments of R use degree 2)"); return HP_ERR_UNSUPPORTED; }
  const int N = p->N, nd = p->ndim, lmax = p->lmax, D = p->D;
  long long stride[3] = {1, N, (long long)N * N};
  auto row_of = [&](int l, int m, int n) -> long long {
    const int am = std::abs(m), an = std::abs(n);
    return p->h_seg[(size_t)(m - p->m_lo) * D + n + lmax] + l - (am > an ? am : an);
  };
  // offsets of the stored coefficients to fetch
  std::vector<long long> idx;
  std::unordered_map<long long, int> pos;
  auto want = [&](int l, int m, int n, long long w) {
    if (m < p->m_lo) { m = -m; n = -n; long long r = 0, mul = 1, ww = w;
      for (int a = 0; a < nd; ++a) { const int k = (int)(ww % N); ww /= N; r += mul * ((N - k) % N); mul *= N; }
      w = r; }
    const long long off = row_of(l, m, n) * p->nx + w;
    if (!pos.count(off)) { pos[off] = (int)idx.size(); idx.push_back(off); }
  };
  for (int t = 0; t < kNB; ++t) { const Lmn q = basis(t); want(q.l, q.m, q.n, 0); }
  for (int t = 0; t < 10; ++t) {
    const Lmn q = basis(t);
    for (int i = 0; i < nd; ++i)
      for (int k = 0; k < N; ++k) want(q.l, q.m, q.n, k * stride[i]);
  }
  for (int i = 0; i < nd; ++i)
    for (int j = i + 1; j < nd; ++j)
      for (int k = 0; k < N; ++k)
        for (int r = 0; r < N; ++r) want(0, 0, 0, k * stride[i] + r * stride[j]);
  if (fx)
    for (long long w = 0; w < p->nx; ++w) want(0, 0, 0, w);
  const int n = (int)idx.size();
  int st = HP_OK;
  long long* didx = (long long*)p->ws_get("stats.idx", sizeof(long long) * n, &st);
  if (st) return st;
  double2* dval = (double2*)p->ws_get("stats.val", sizeof(double2) * n, &st);
  if (st) return st;
  cudaStream_t s = p->stream;
  HP_CUDA_TRY(cudaMemcpyAsync(didx, idx.data(), sizeof(long long) * n, cudaMemcpyHostToDevice, s));
  {
    ProfScope _ps(p, "stats.gather", s);
    k_gather<<<(n + 255) / 256, 256, 0, s>>>(Fi, didx, dval, n);
    HP_CUDA_TRY(cudaGetLastError());
  }
  std::vector<double2> val(n);
  HP_CUDA_TRY(cudaMemcpyAsync(val.data(), dval, sizeof(double2) * n, cudaMemcpyDeviceToHost, s));
  HP_CUDA_TRY(cudaStreamSynchronize(s));
  // full-storage coefficient F^l_mn[w], mirrored for rows not stored
  auto get = [&](int l, int m, int n, long long w) -> cd {
    if (m >= p->m_lo) {
      const double2 v = val[pos.at(row_of(l, m, n) * p->nx + w)];
      return cd(v.x, v.y);
    }
    long long r = 0, mul = 1, ww = w;
    for (int a = 0; a < nd; ++a) { const int k = (int)(ww % N); ww /= N; r += mul * ((N - k) % N); mul *= N; }
    const double2 v = val[pos.at(row_of(l, -m, -n) * p->nx + r)];
    const double sg = ((m - n) & 1) ? -1.0 : 1.0;
    return sg * std::conj(cd(v.x, v.y));
  };
  const double L = p->model.L;
  const double c0 = std::pow(L / N, nd);
  std::vector<cd> xi(N), xi2(N);
  for (int q = 0; q < N; ++q) {
    cd a(0, 0), b(0, 0);
    for (int t = 0; t < N; ++t) {
      const double x = -L / 2 + L * t / N;
      const cd e = std::polar(1.0, -2.0 * M_PI * q * t / N);
      a += x * e;
      b += x * x * e;
    }
    xi[q] = a;
    xi2[q] = b;
  }
  cd F0[kNB];
  for (int t = 0; t < kNB; ++t) { const Lmn q = basis(t); F0[t] = get(q.l, q.m, q.n, 0); }
  std::memset(out, 0, sizeof(*out));
  out->mass = c0 * F0[0].real();
  for (int h = 0; h < 9; ++h) {
    cd a(0, 0);
    for (int t = 0; t < kNB; ++t) a += g_aR[(size_t)h * kNB + t] * F0[t];
    out->ER[h] = c0 * a.real();
  }
  for (int h = 0; h < 81; ++h) {
    cd a(0, 0);
    for (int t = 0; t < kNB; ++t) a += g_aRR[(size_t)h * kNB + t] * F0[t];
    out->ERR[h] = c0 * a.real();
  }
  for (int i = 0; i < nd; ++i) {
    cd e1(0, 0), e2(0, 0);
    for (int q = 0; q < N; ++q) {
      const cd v = get(0, 0, 0, q * stride[i]);
      e1 += v * std::conj(xi[q]);
      e2 += v * std::conj(xi2[q]);
    }
    out->Ex[i] = c0 / N * e1.real();
    out->Exx[i * 3 + i] = c0 / N * e2.real();
    for (int j = i + 1; j < nd; ++j) {
      cd e(0, 0);
      for (int q = 0; q < N; ++q)
        for (int r = 0; r < N; ++r) e += get(0, 0, 0, q * stride[i] + r * stride[j]) * std::conj(xi[q] * xi[r]);
      out->Exx[i * 3 + j] = out->Exx[j * 3 + i] = c0 / ((double)N * N) * e.real();
    }
    // E[x_i R_kq]
    cd ax[10];
    for (int t = 0; t < 10; ++t) {
      const Lmn qb = basis(t);
      cd a(0, 0);
      for (int q = 0; q < N; ++q) a += get(qb.l, qb.m, qb.n, q * stride[i]) * std::conj(xi[q]);
      ax[t] = a;
    }
    for (int h = 0; h < 9; ++h) {
      cd a(0, 0);
      for (int t = 0; t < 10; ++t) a += g_aR[(size_t)h * kNB + t] * ax[t];
      out->ExR[i * 9 + h] = c0 / N * a.real();
    }
  }
  if (fx) {
    // fx(j) = sum_R w f(R, j) = inverse DFT of F^0_00 over omega (separable passes)
    std::vector<cd> a(p->nx), b(p->nx);
    for (long long w = 0; w < p->nx; ++w) a[w] = get(0, 0, 0, w);
    for (int ax = 0; ax < nd; ++ax) {
      for (long long w = 0; w < p->nx; ++w) {
        const int j = (int)((w / stride[ax]) % N);
        const long long base = w - (long long)j * stride[ax];
        cd acc(0, 0);
        for (int k = 0; k < N; ++k) acc += a[base + k * stride[ax]] * std::polar(1.0, 2.0 * M_PI * k * j / N);
        b[w] = acc / (double)N;
      }
      std::swap(a, b);
    }
    for (long long w = 0; w < p->nx; ++w) fx[w] = a[w].real();
  }
  return HP_OK;
}

}  // namespace

extern "C" int hp_moments(hp_plan* p, const double* F, int mem, hp_moments_t* out, double* fx) {
  if (!p || !F || !out) { hp_set_error("null argument"); return HP_ERR_INVALID; }
  if (mem != HP_DEVICE && mem != HP_HOST) { hp_set_error("mem must be HP_DEVICE or HP_HOST"); return HP_ERR_INVALID; }
  if (!p->has_model) { hp_set_error("no model: the omega period L comes from hp_plan_set_model"); return HP_ERR_NO_MODEL; }
  int st = HP_OK;
  const size_t fb = 16 * (size_t)p->n_full(), ib = 16 * (size_t)p->nrows * p->nx;
  const double2* in = (const double2*)F;
  if (mem == HP_HOST) {
    double2* a = (double2*)p->ws_get("api.Fin", fb, &st);
    if (st) return st;
    HP_CUDA_TRY(cudaMemcpyAsync(a, F, fb, cudaMemcpyHostToDevice, p->stream));
    in = a;
  }
  double2* Fi = (double2*)p->ws_get("api.S0", ib, &st);
  if (st) return st;
  ST_CHECK(hp_full_to_internal(p, in, Fi, p->stream));
  return moments_internal(p, Fi, out, fx);
}

extern "C" int hp_state_moments(hp_state* s, hp_moments_t* out, double* fx) {
  if (!s || !out) { hp_set_error("null argument"); return HP_ERR_INVALID; }
  if (!s->plan->has_model) { hp_set_error("no model: the omega period L comes from hp_plan_set_model"); return HP_ERR_NO_MODEL; }
  return moments_internal(s->plan, s->F, out, fx);
}
