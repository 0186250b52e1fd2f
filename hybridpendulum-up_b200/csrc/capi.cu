// C ABI (include/hp.h): plans, host/device staging, integrators, state API.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <complex>
#include <mutex>
#include <unordered_map>
#include <vector>
#include "common.cuh"
#include "plan.hpp"

using namespace hp;

static thread_local std::string g_err;
void hp_set_error(const char* msg) { g_err = msg ? msg : ""; }

// ------------------------------------------------ device memory budget ----
namespace {
std::mutex g_alloc_mu;
std::unordered_map<void*, size_t> g_alloc_sizes;
long long g_alloc_bytes = 0;    // bytes held by the library now
long long g_alloc_budget = 0;   // 0: no cap
}  // namespace

cudaError_t hp_dev_alloc_raw(void** p, size_t bytes) {
  *p = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_alloc_mu);
    if (g_alloc_budget > 0 && g_alloc_bytes + (long long)bytes > g_alloc_budget) return cudaErrorMemoryAllocation;
  }
  const cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaSuccess) {
    *p = nullptr;
    return e;
  }
  std::lock_guard<std::mutex> lk(g_alloc_mu);
  g_alloc_sizes[*p] = bytes;
  g_alloc_bytes += (long long)bytes;
  return cudaSuccess;
}

cudaError_t hp_dev_free(void* p) {
  if (!p) return cudaSuccess;
  {
    std::lock_guard<std::mutex> lk(g_alloc_mu);
    auto it = g_alloc_sizes.find(p);
    if (it != g_alloc_sizes.end()) {
      g_alloc_bytes -= (long long)it->second;
      g_alloc_sizes.erase(it);
    }
  }
  return cudaFree(p);
}

extern "C" int hp_set_device_budget(long long bytes) {
  if (bytes < 0) { hp_set_error("budget must be >= 0 (0: no cap)"); return HP_ERR_INVALID; }
  std::lock_guard<std::mutex> lk(g_alloc_mu);
  g_alloc_budget = bytes;
  return HP_OK;
}

extern "C" int hp_device_bytes(long long* bytes) {
  if (!bytes) { hp_set_error("null argument"); return HP_ERR_INVALID; }
  std::lock_guard<std::mutex> lk(g_alloc_mu);
  *bytes = g_alloc_bytes;
  return HP_OK;
}
extern "C" const char* hp_last_error(void) { return g_err.c_str(); }

#define HP_CHECK(expr)              \
  do {                              \
    int _s = (expr);                \
    if (_s != HP_OK) return _s;     \
  } while (0)

void hp_plan::ws_release(const char* name) {
  for (auto& kv : ws)
    if (kv.first == name && kv.second.p) {
      hp_dev_free(kv.second.p);
      kv.second = Buf{};
    }
}

void* hp_plan::ws_get(const char* name, size_t bytes, int* status) {
  for (auto& kv : ws) {
    if (kv.first == name) {
      if (kv.second.bytes >= bytes) return kv.second.p;
      hp_dev_free(kv.second.p);
      kv.second = Buf{};
      void* q = nullptr;
      if (hp_dev_alloc(&q, bytes) != cudaSuccess) {
        cudaGetLastError();
        hp_set_error("device allocation failed");
        *status = HP_ERR_ALLOC;
        return nullptr;
      }
      kv.second = Buf{q, bytes};
      return q;
    }
  }
  void* q = nullptr;
  if (hp_dev_alloc(&q, bytes) != cudaSuccess) {
    cudaGetLastError();
    hp_set_error("device allocation failed");
    *status = HP_ERR_ALLOC;
    return nullptr;
  }
  ws.push_back({name, Buf{q, bytes}});
  return q;
}

ProfScope::ProfScope(hp_plan* plan, const char* name, cudaStream_t stream) : p(plan), s(stream) {
  ++p->launches;
  if (!p->prof_on) return;
  for (size_t i = 0; i < p->prof.size(); ++i)
    if (p->prof[i].name == name) { idx = (int)i; break; }
  if (idx < 0) {
    p->prof.push_back(ProfEntry{});
    p->prof.back().name = name;
    idx = (int)p->prof.size() - 1;
  }
  if (cudaEventCreate(&a) != cudaSuccess) { cudaGetLastError(); a = nullptr; return; }
  cudaEventRecord(a, s);
}

ProfScope::~ProfScope() {
  if (!a) return;
  cudaEvent_t b = nullptr;
  if (cudaEventCreate(&b) != cudaSuccess) { cudaGetLastError(); cudaEventDestroy(a); return; }
  cudaEventRecord(b, s);
  p->prof[idx].pending.push_back({a, b});
}

static void prof_collect(hp_plan* p) {
  for (auto& e : p->prof) {
    for (auto& ab : e.pending) {
      float ms = 0.f;
      cudaEventSynchronize(ab.second);
      if (cudaEventElapsedTime(&ms, ab.first, ab.second) == cudaSuccess) { e.ms += ms; e.count += 1; }
      else cudaGetLastError();
      cudaEventDestroy(ab.first);
      cudaEventDestroy(ab.second);
    }
    e.pending.clear();
  }
}

extern "C" int hp_plan_profile(hp_plan* p, int enable) {
  if (!p) { hp_set_error("null plan"); return HP_ERR_INVALID; }
  prof_collect(p);
  p->prof.clear();
  p->prof_on = enable != 0;
  return HP_OK;
}

extern "C" int hp_plan_profile_get(hp_plan* p, int i, char* name, int name_cap, double* total_ms,
                                   long long* count) {
  if (!p || i < 0) { hp_set_error("bad argument"); return HP_ERR_INVALID; }
  prof_collect(p);
  if (i >= (int)p->prof.size()) return HP_ERR_INVALID;
  const ProfEntry& e = p->prof[i];
  if (name && name_cap > 0) {
    std::strncpy(name, e.name.c_str(), name_cap - 1);
    name[name_cap - 1] = 0;
  }
  if (total_ms) *total_ms = e.ms;
  if (count) *count = e.count;
  return HP_OK;
}

extern "C" int hp_plan_launch_count(hp_plan* p, long long* count) {
  if (!p || !count) { hp_set_error("null argument"); return HP_ERR_INVALID; }
  *count = p->launches;
  return HP_OK;
}

extern "C" int hp_plan_set_beta_engine(hp_plan* p, int engine) {
  if (!p) { hp_set_error("null plan"); return HP_ERR_INVALID; }
  if (engine != HP_BETA_AUTO && engine != HP_BETA_SIMT && engine != HP_BETA_TENSOR && engine != HP_BETA_TENSOR_BF16) {
    hp_set_error("engine must be HP_BETA_AUTO, HP_BETA_SIMT, HP_BETA_TENSOR or HP_BETA_TENSOR_BF16");
    return HP_ERR_INVALID;
  }
  p->beta_engine = engine;
  hp_tune_apply_cached(p);   // a tuned shape for this engine, if one was found earlier
  return HP_OK;
}

extern "C" int hp_plan_tc_errors(hp_plan* p, int* count) {
  if (!p || !count) { hp_set_error("null argument"); return HP_ERR_INVALID; }
  return hp::tc_beta_errors(p, count);
}

static bool valid_N(int N) { return N >= 4 && N <= 64 && N % 2 == 0; }
static bool valid_B(int B) { return B >= 2 && B <= 32; }

extern "C" int hp_plan_create(hp_plan** out, int B, int Bx, int ndim, int precision, int symmetry) {
  if (!out) { hp_set_error("plan pointer is null"); return HP_ERR_INVALID; }
  *out = nullptr;
  if (!valid_B(B)) { hp_set_error("bandlimit B must be 2..32"); return HP_ERR_INVALID; }
  if (!valid_N(2 * Bx)) { hp_set_error("Bx must be 2..32 (omega grids of 4..64 points per axis)"); return HP_ERR_INVALID; }
  if (ndim != 2 && ndim != 3) { hp_set_error("ndim must be 2 or 3"); return HP_ERR_INVALID; }
  if (precision != HP_FP64 && precision != HP_MIXED) { hp_set_error("bad precision"); return HP_ERR_INVALID; }
  if (symmetry != HP_REAL && symmetry != HP_COMPLEX) { hp_set_error("bad symmetry"); return HP_ERR_INVALID; }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    hp_set_error("no CUDA device");
    return HP_ERR_CUDA;
  }
  hp_plan* p = new hp_plan();
  p->B = B; p->lmax = B - 1; p->Bx = Bx; p->N = 2 * Bx; p->ndim = ndim;
  p->precision = precision; p->symmetry = symmetry;
  p->D = 2 * p->lmax + 1;
  p->m_lo = symmetry == HP_REAL ? 0 : -p->lmax;
  p->nm = p->lmax - p->m_lo + 1;
  p->nx = 1;
  for (int a = 0; a < ndim; ++a) p->nx *= p->N;
  int st = hp_tables_build(p);
  if (st) { hp_plan_destroy(p); return st; }
  hp_tune_apply_cached(p);
  *out = p;
  return HP_OK;
}

extern "C" int hp_plan_destroy(hp_plan* p) {
  if (!p) return HP_OK;
  hp_dev_free(p->rows); hp_dev_free(p->seg); hp_dev_free(p->fgather); hp_dev_free(p->wig64); hp_dev_free(p->wig32); hp_dev_free(p->wfull);
  hp_dev_free(p->qw); hp_dev_free(p->cg1); hp_dev_free(p->tap_wr); hp_dev_free(p->tap_wr32);
  p->prof_on = false;
  prof_collect(p);
  for (auto& kv : p->ws) hp_dev_free(kv.second.p);
  delete p;
  return HP_OK;
}

extern "C" int hp_plan_get_info(const hp_plan* p, hp_plan_info_t* info) {
  if (!p || !info) { hp_set_error("null argument"); return HP_ERR_INVALID; }
  info->B = p->B; info->lmax = p->lmax; info->Bx = p->Bx; info->N = p->N; info->ndim = p->ndim;
  info->precision = p->precision; info->symmetry = p->symmetry;
  info->nx = p->nx; info->nrows = p->nrows; info->n_full = p->n_full(); info->n_grid = p->n_grid();
  info->state_bytes = 16LL * p->nrows * p->nx;
  return HP_OK;
}

extern "C" int hp_plan_set_stream(hp_plan* p, void* s) {
  if (!p) { hp_set_error("null plan"); return HP_ERR_INVALID; }
  p->stream = (cudaStream_t)s;
  return HP_OK;
}

// ------------------------------------------------------------ staging ----
// Returns a device pointer holding `bytes` of `src` (copied when on the host).
static const void* stage_in(hp_plan* p, const char* name, const void* src, size_t bytes, int mem, int* st) {
  if (mem == HP_DEVICE) return src;
  void* d = p->ws_get(name, bytes, st);
  if (*st) return nullptr;
  if (cudaMemcpyAsync(d, src, bytes, cudaMemcpyHostToDevice, p->stream) != cudaSuccess) {
    hp_set_error("host to device copy failed");
    *st = HP_ERR_CUDA;
    return nullptr;
  }
  return d;
}
static void* stage_out(hp_plan* p, const char* name, void* dst, size_t bytes, int mem, int* st) {
  if (mem == HP_DEVICE) return dst;
  return p->ws_get(name, bytes, st);
}
static int finish_out(hp_plan* p, void* host, const void* dev, size_t bytes, int mem) {
  if (mem == HP_DEVICE) return HP_OK;
  HP_CUDA_TRY(cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, p->stream));
  HP_CUDA_TRY(cudaStreamSynchronize(p->stream));
  return HP_OK;
}
// Device address of a 16-byte aligned host buffer that is page-locked and
// mapped into the current device's address space at its first and its last
// byte, contiguously; null otherwise (pageable memory, a range that leaves the
// mapping, or an alignment the kernel's 16-byte loads cannot take).
static const void* mapped_host(const void* h, size_t bytes) {
  if (!h || bytes == 0 || (reinterpret_cast<uintptr_t>(h) & 15u)) return nullptr;
  cudaPointerAttributes a{}, b{};
  if (cudaPointerGetAttributes(&a, h) != cudaSuccess) { cudaGetLastError(); return nullptr; }
  if (a.type != cudaMemoryTypeHost || !a.devicePointer) return nullptr;
  const char* last = static_cast<const char*>(h) + (bytes - 1);
  if (cudaPointerGetAttributes(&b, last) != cudaSuccess) { cudaGetLastError(); return nullptr; }
  if (b.type != cudaMemoryTypeHost || !b.devicePointer) return nullptr;
  if (static_cast<const char*>(b.devicePointer) - static_cast<const char*>(a.devicePointer) != (ptrdiff_t)(bytes - 1))
    return nullptr;
  return a.devicePointer;
}

extern "C" int hp_host_read_in_place(const void* ptr, long long bytes, int* in_place) {
  if (!ptr || !in_place || bytes <= 0) { hp_set_error("null argument or empty range"); return HP_ERR_INVALID; }
  *in_place = mapped_host(ptr, (size_t)bytes) ? 1 : 0;
  return HP_OK;
}

// F in the full layout (host or device) -> [row][omega] rows in Fi.  A mapped
// host buffer is read in place, only its kept entries; another host buffer is
// copied whole into the workspace and converted there.
static int load_full(hp_plan* p, const double* F, int mem, double2* Fi) {
  const size_t fb = 16 * (size_t)p->n_full();
  if (mem == HP_HOST)
    if (const void* m = mapped_host(F, fb)) return hp_full_gather(p, static_cast<const double2*>(m), Fi, p->stream);
  int st = HP_OK;
  const double2* d = (const double2*)stage_in(p, "api.Fin", F, fb, mem, &st);
  if (st) return st;
  return hp_full_to_internal(p, d, Fi, p->stream);
}

static int check_mem(int mem) {
  if (mem != HP_DEVICE && mem != HP_HOST) { hp_set_error("mem must be HP_DEVICE or HP_HOST"); return HP_ERR_INVALID; }
  return HP_OK;
}

// ---------------------------------------------------------------- model ----
extern "C" int hp_plan_set_model(hp_plan* p, const hp_model* m, const double* MR, int mem) {
  if (!p || !m || !MR) { hp_set_error("null argument"); return HP_ERR_INVALID; }
  HP_CHECK(check_mem(mem));
  if (!(m->L > 0) || !std::isfinite(m->L)) { hp_set_error("L must be positive"); return HP_ERR_INVALID; }
  const int D = p->D, lmax = p->lmax;
  const size_t nMR = (size_t)D * D * (lmax + 1) * p->ndim;
  std::vector<double2> h(nMR);
  if (mem == HP_HOST) std::memcpy(h.data(), MR, sizeof(double2) * nMR);
  else HP_CUDA_TRY(cudaMemcpy(h.data(), MR, sizeof(double2) * nMR, cudaMemcpyDeviceToHost));
  // only the degree-1, m2 = 0 block may carry weight (gravity depends on R^T e3)
  double big = 0.0, stray = 0.0;
  for (int i = 0; i < p->ndim; ++i)
    for (int l = 0; l <= lmax; ++l)
      for (int n = -l; n <= l; ++n)
        for (int mm = -l; mm <= l; ++mm) {
          const double2 v = h[(mm + lmax) + (size_t)D * (n + lmax) + (size_t)D * D * l + (size_t)D * D * (lmax + 1) * i];
          const double a = std::hypot(v.x, v.y);
          if (!std::isfinite(a)) { hp_set_error("MR has non-finite entries"); return HP_ERR_NONFINITE; }
          if (l == 1 && mm == 0) big = std::max(big, a);
          else stray = std::max(stray, a);
        }
  if (stray > 1e-9 * std::max(big, 1e-300) && stray > 1e-300) {
    hp_set_error("MR has components outside the degree-1, m2=0 block (alpha-dependent multiplier)");
    return HP_ERR_UNSUPPORTED;
  }
  HP_CHECK(hp_build_gravity_taps(p));
  for (int n2 = -1; n2 <= 1; ++n2)
    for (int i = 0; i < 3; ++i)
      p->mr1[n2 + 1][i] = (i < p->ndim && lmax >= 1)
                              ? h[lmax + (size_t)D * (n2 + lmax) + (size_t)D * D * 1 + (size_t)D * D * (lmax + 1) * i]
                              : make_double2(0.0, 0.0);
  HP_CUDA_TRY(cudaStreamSynchronize(p->stream));
  p->model = *m;
  p->den_mR = nullptr;
  p->so3d64 = nullptr;
  p->so3d32 = nullptr;
  p->has_model = true;
  return HP_OK;
}

extern "C" int hp_plan_set_den_model(hp_plan* p, const hp_model* m, const double* mR, int mem) {
  if (!p || !m || !mR) { hp_set_error("null argument"); return HP_ERR_INVALID; }
  HP_CHECK(check_mem(mem));
  if (p->ndim != 2 || p->symmetry != HP_REAL) {
    hp_set_error("density gravity needs a 2-D plan with HP_REAL symmetry");
    return HP_ERR_UNSUPPORTED;
  }
  if (!(m->L > 0) || !std::isfinite(m->L)) { hp_set_error("L must be positive"); return HP_ERR_INVALID; }
  const size_t ng = (size_t)8 * p->B * p->B * p->B;
  std::vector<double> h(2 * ng), dein(2 * ng);
  if (mem == HP_HOST) std::memcpy(h.data(), mR, sizeof(double) * 2 * ng);
  else HP_CUDA_TRY(cudaMemcpy(h.data(), mR, sizeof(double) * 2 * ng, cudaMemcpyDeviceToHost));
  for (size_t e = 0; e < ng; ++e)
    for (int i = 0; i < 2; ++i) {
      const double v = h[2 * e + i];  // mR(i, a, b, c), component fastest
      if (!std::isfinite(v)) { hp_set_error("mR has non-finite entries"); return HP_ERR_NONFINITE; }
      dein[i * ng + e] = v;
    }
  int st = HP_OK;
  double* d = (double*)p->ws_get("model.denmR", sizeof(double) * 2 * ng, &st);
  if (st) return st;
  HP_CUDA_TRY(cudaMemcpy(d, dein.data(), sizeof(double) * 2 * ng, cudaMemcpyHostToDevice));
  HP_CHECK(hp_build_gravity_taps(p));
  for (int n2 = 0; n2 < 3; ++n2)
    for (int i = 0; i < 3; ++i) p->mr1[n2][i] = make_double2(0.0, 0.0);  // no coefficient-space gravity
  HP_CUDA_TRY(cudaStreamSynchronize(p->stream));
  p->model = *m;
  p->den_mR = d;
  p->so3d64 = nullptr;
  p->so3d32 = nullptr;
  p->has_model = true;
  return HP_OK;
}

// Attitude-diffusion weights of the gyro-bias model (gyro_bias.m:274-283):
//   sum_ij G1_ij F^l u_i^T u_j^T = F^l K^T,  K = sum_ij G1_ij u_j u_i,
// so output (l, m, n) takes K[n][k] F^l_{m,k} for k = n-2..n+2 (u_1, u_2 are
// bidiagonal in n and u_3 is diagonal).  u as in getu.m:132-163:
//   u_1[n-1][n] = -i/2 sqrt((l+n)(l-n+1)),  u_1[n+1][n] = -i/2 sqrt((l-n)(l+n+1)),
//   u_2[n-1][n] =  1/2 sqrt((l+n)(l-n+1)),  u_2[n+1][n] = -1/2 sqrt((l-n)(l+n+1)),
//   u_3[n][n]   = -i n.
static std::complex<double> getu_entry(int l, int a, int b, int i) {
  using cd = std::complex<double>;
  if (a < -l || a > l || b < -l || b > l) return cd(0, 0);
  if (i == 2) return a == b ? cd(0, -a) : cd(0, 0);
  if (a == b - 1) {
    const double v = 0.5 * std::sqrt((double)(l + b) * (l - b + 1));
    return i == 0 ? cd(0, -v) : cd(v, 0);
  }
  if (a == b + 1) {
    const double v = 0.5 * std::sqrt((double)(l - b) * (l + b + 1));
    return i == 0 ? cd(0, -v) : cd(-v, 0);
  }
  return cd(0, 0);
}

extern "C" int hp_plan_set_gyro_bias_model(hp_plan* p, double L, const double* G1, const double* G2) {
  if (!p || !G1 || !G2) { hp_set_error("null argument"); return HP_ERR_INVALID; }
  if (p->ndim != 3) { hp_set_error("the gyro-bias model has a 3-D bias (ndim = 3)"); return HP_ERR_UNSUPPORTED; }
  if (!(L > 0) || !std::isfinite(L)) { hp_set_error("L must be positive"); return HP_ERR_INVALID; }
  for (int e = 0; e < 9; ++e)
    if (!std::isfinite(G1[e]) || !std::isfinite(G2[e])) { hp_set_error("G1/G2 have non-finite entries"); return HP_ERR_NONFINITE; }
  using cd = std::complex<double>;
  std::vector<double2> w64((size_t)p->nrows * 5);
  std::vector<float2> w32((size_t)p->nrows * 5);
  for (long long r = 0; r < p->nrows; ++r) {
    const int l = p->h_rows[r].x, n = p->h_rows[r].z;
    for (int o = 0; o < 5; ++o) {
      const int k = n + o - 2;
      cd K(0, 0);
      if (k >= -l && k <= l)
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j) {
            if (G1[i * 3 + j] == 0.0) continue;
            cd uu(0, 0);   // (u_j u_i)[n][k]
            for (int q = std::max(-l, n - 1); q <= std::min(l, n + 1); ++q) uu += getu_entry(l, n, q, j) * getu_entry(l, q, k, i);
            K += G1[i * 3 + j] * uu;
          }
      w64[(size_t)r * 5 + o] = make_double2(K.real(), K.imag());
      w32[(size_t)r * 5 + o] = make_float2((float)K.real(), (float)K.imag());
    }
  }
  int st = HP_OK;
  double2* d64 = (double2*)p->ws_get("model.so3d64", sizeof(double2) * w64.size(), &st);
  if (st) return st;
  float2* d32 = (float2*)p->ws_get("model.so3d32", sizeof(float2) * w32.size(), &st);
  if (st) return st;
  HP_CUDA_TRY(cudaMemcpy(d64, w64.data(), sizeof(double2) * w64.size(), cudaMemcpyHostToDevice));
  HP_CUDA_TRY(cudaMemcpy(d32, w32.data(), sizeof(float2) * w32.size(), cudaMemcpyHostToDevice));
  HP_CHECK(hp_build_gravity_taps(p));
  for (int n2 = 0; n2 < 3; ++n2)
    for (int i = 0; i < 3; ++i) p->mr1[n2][i] = make_double2(0.0, 0.0);   // no gravity
  HP_CUDA_TRY(cudaStreamSynchronize(p->stream));
  hp_model m{};
  m.L = L;
  for (int e = 0; e < 9; ++e) m.G[e] = G2[e];   // bias random walk (gyro_bias.m:285-297)
  p->model = m;                                  // b = 0, no gyroscopic term
  p->den_mR = nullptr;
  p->so3d64 = d64;
  p->so3d32 = d32;
  p->has_model = true;
  return HP_OK;
}

extern "C" int hp_wigner_d(hp_plan* p, double* d, int mem) {
  if (!p || !d) { hp_set_error("null argument"); return HP_ERR_INVALID; }
  HP_CHECK(check_mem(mem));
  const size_t n = (size_t)p->D * p->D * (p->lmax + 1) * 2 * p->B;
  HP_CUDA_TRY(cudaMemcpy(d, p->wfull, sizeof(double) * n, mem == HP_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice));
  return HP_OK;
}

extern "C" int hp_quad_weights(hp_plan* p, double* w, int mem) {
  if (!p || !w) { hp_set_error("null argument"); return HP_ERR_INVALID; }
  HP_CHECK(check_mem(mem));
  HP_CUDA_TRY(cudaMemcpy(w, p->qw, sizeof(double) * 2 * p->B, mem == HP_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice));
  return HP_OK;
}

// ----------------------------------------------------- grid conversions ----
__global__ void k_d2f(const double* __restrict__ a, float* __restrict__ b, long long n) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n) b[i] = (float)a[i];
}
__global__ void k_f2d(const float* __restrict__ a, double* __restrict__ b, long long n) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n) b[i] = (double)a[i];
}

// ----------------------------------------------------------- transforms ----
extern "C" int hp_fftSO3R_forward(hp_plan* p, const double* f, double* F, int mem) {
  if (!p || !f || !F) { hp_set_error("null argument"); return HP_ERR_INVALID; }
  HP_CHECK(check_mem(mem));
  int st = HP_OK;
  const bool cplx = p->symmetry == HP_COMPLEX;
  const long long ng = p->n_grid() * (cplx ? 2 : 1);
  const double* df = (const double*)stage_in(p, "api.fin", f, sizeof(double) * ng, mem, &st);
  if (st) return st;
  const void* src = df;
  if (p->precision == HP_MIXED) {
    float* t = (float*)p->ws_get("api.f32", sizeof(float) * ng, &st);
    if (st) return st;
    ProfScope _ps(p, "convert", p->stream);
    k_d2f<<<(unsigned)((ng + 255) / 256), 256, 0, p->stream>>>(df, t, ng);
    HP_CUDA_TRY(cudaGetLastError());
    src = t;
  }
  double2* Fi = (double2*)p->ws_get("api.Fint", 16 * (size_t)p->nrows * p->nx, &st);
  if (st) return st;
  HP_CHECK(hp_forward_internal(p, src, cplx, Fi, p->stream));
  double2* dF = (double2*)stage_out(p, "api.Fout", F, 16 * (size_t)p->n_full(), mem, &st);
  if (st) return st;
  HP_CHECK(hp_internal_to_full(p, Fi, dF, p->stream));
  HP_CHECK(finish_out(p, F, dF, 16 * (size_t)p->n_full(), mem));
  HP_CUDA_TRY(cudaStreamSynchronize(p->stream));
  return HP_OK;
}

extern "C" int hp_fftSO3R_backward(hp_plan* p, const double* F, double* f, int mem) {
  if (!p || !F || !f) { hp_set_error("null argument"); return HP_ERR_INVALID; }
  HP_CHECK(check_mem(mem));
  int st = HP_OK;
  const bool cplx = p->symmetry == HP_COMPLEX;
  const long long ng = p->n_grid() * (cplx ? 2 : 1);
  double2* Fi = (double2*)p->ws_get("api.Fint", 16 * (size_t)p->nrows * p->nx, &st);
  if (st) return st;
  HP_CHECK(load_full(p, F, mem, Fi));
  double* df = (double*)stage_out(p, "api.fout", f, sizeof(double) * ng, mem, &st);
  if (st) return st;
  if (p->precision == HP_MIXED) {
    float* t = (float*)p->ws_get("api.f32", sizeof(float) * ng, &st);
    if (st) return st;
    HP_CHECK(hp_backward_internal(p, Fi, t, cplx, p->stream));
    ProfScope _ps(p, "convert", p->stream);
    k_f2d<<<(unsigned)((ng + 255) / 256), 256, 0, p->stream>>>(t, df, ng);
    HP_CUDA_TRY(cudaGetLastError());
  } else {
    HP_CHECK(hp_backward_internal(p, Fi, df, cplx, p->stream));
  }
  HP_CHECK(finish_out(p, f, df, sizeof(double) * ng, mem));
  HP_CUDA_TRY(cudaStreamSynchronize(p->stream));
  return HP_OK;
}

// ----------------------------------------------------------- integrators ----
// One step of `method` on internal-layout buffers; the result lands in *F
// (buffers are swapped, never aliased inside one derivative evaluation).
// fgrid: grid density of *F for the first stage of a density-gravity model
// (null: recomputed from *F), as pendulum_reduced_den.m:359-399 passes f to the
// first derivative only.
// fin32 (may be null): *F already in FP32, read by the first derivative
// evaluation; fout32 (may be null): receives the new F in FP32 from the last one.
static int integrate_internal(hp_plan* p, double2** F, double2** F2, double2** F3, double2* acc, double dt,
                              int method, const void* fgrid = nullptr, const void* fin32 = nullptr,
                              void* fout32 = nullptr) {
  cudaStream_t s = p->stream;
  const size_t bytes = 16 * (size_t)p->nrows * p->nx;
  switch (method) {
    case HP_EULER:
      HP_CHECK(hp_derivative_eval(p, *F, *F, dt, *F2, nullptr, 0.0, s, fgrid, fin32, fout32));
      std::swap(*F, *F2);
      return HP_OK;
    case HP_MIDPOINT:
      HP_CHECK(hp_derivative_eval(p, *F, *F, dt / 2, *F2, nullptr, 0.0, s, fgrid, fin32));
      HP_CHECK(hp_derivative_eval(p, *F2, *F, dt, *F3, nullptr, 0.0, s, nullptr, nullptr, fout32));
      std::swap(*F, *F3);
      return HP_OK;
    case HP_RK2:
      HP_CUDA_TRY(cudaMemcpyAsync(acc, *F, bytes, cudaMemcpyDeviceToDevice, s));
      HP_CHECK(hp_derivative_eval(p, *F, *F, dt, *F2, acc, dt / 2, s, fgrid, fin32));
      HP_CHECK(hp_derivative_eval(p, *F2, acc, dt / 2, *F3, nullptr, 0.0, s, nullptr, nullptr, fout32));
      std::swap(*F, *F3);
      return HP_OK;
    case HP_RK4:
      HP_CUDA_TRY(cudaMemcpyAsync(acc, *F, bytes, cudaMemcpyDeviceToDevice, s));
      HP_CHECK(hp_derivative_eval(p, *F, *F, dt / 2, *F2, acc, dt / 6, s, fgrid, fin32));
      HP_CHECK(hp_derivative_eval(p, *F2, *F, dt / 2, *F3, acc, dt / 3, s));
      HP_CHECK(hp_derivative_eval(p, *F3, *F, dt, *F2, acc, dt / 3, s));
      HP_CHECK(hp_derivative_eval(p, *F2, acc, dt / 6, *F3, nullptr, 0.0, s, nullptr, nullptr, fout32));
      std::swap(*F, *F3);
      return HP_OK;
    default:
      hp_set_error("method must be HP_EULER, HP_MIDPOINT, HP_RK2 or HP_RK4");
      return HP_ERR_INVALID;
  }
}

extern "C" int hp_pendulum_propagate(hp_plan* p, const double* Fold, double* Fnew, double dt, int method,
                                     int mem) {
  if (!p || !Fold || !Fnew) { hp_set_error("null argument"); return HP_ERR_INVALID; }
  HP_CHECK(check_mem(mem));
  if (!p->has_model) { hp_set_error("no model: call hp_plan_set_model first"); return HP_ERR_NO_MODEL; }
  if (method < HP_EULER || method > HP_RK4) { hp_set_error("bad method"); return HP_ERR_INVALID; }
  if (!std::isfinite(dt)) { hp_set_error("dt must be finite"); return HP_ERR_INVALID; }
  int st = HP_OK;
  const size_t fb = 16 * (size_t)p->n_full(), ib = 16 * (size_t)p->nrows * p->nx;
  double2* b0 = (double2*)p->ws_get("api.S0", ib, &st); if (st) return st;
  double2* b1 = (double2*)p->ws_get("api.S1", ib, &st); if (st) return st;
  double2* b2 = (method == HP_EULER) ? nullptr : (double2*)p->ws_get("api.S2", ib, &st); if (st) return st;
  double2* ac = (method == HP_RK2 || method == HP_RK4) ? (double2*)p->ws_get("api.S3", ib, &st) : nullptr;
  if (st) return st;
  HP_CHECK(load_full(p, Fold, mem, b0));
  double2 *F = b0, *F2 = b1, *F3 = b2;
  HP_CHECK(integrate_internal(p, &F, &F2, &F3, ac, dt, method));
  double2* dOut = (double2*)stage_out(p, "api.Fout", Fnew, fb, mem, &st);
  if (st) return st;
  HP_CHECK(hp_internal_to_full(p, F, dOut, p->stream));
  HP_CHECK(finish_out(p, Fnew, dOut, fb, mem));
  HP_CUDA_TRY(cudaStreamSynchronize(p->stream));
  return HP_OK;
}

extern "C" int hp_gyrobias_propagate(hp_plan* p, const double* Fold, double* Fnew, double dt, int mem) {
  if (!p) { hp_set_error("null argument"); return HP_ERR_INVALID; }
  if (!p->has_model || !p->so3d64) { hp_set_error("no gyro-bias model: call hp_plan_set_gyro_bias_model first"); return HP_ERR_NO_MODEL; }
  return hp_pendulum_propagate(p, Fold, Fnew, dt, HP_EULER, mem);
}

extern "C" int hp_pendulum_propagate_den(hp_plan* p, const double* Fold, const double* f, double* Fnew,
                                         double dt, int method, int mem) {
  if (!p || !Fold || !Fnew) { hp_set_error("null argument"); return HP_ERR_INVALID; }
  HP_CHECK(check_mem(mem));
  if (!p->has_model || !p->den_mR) { hp_set_error("no density-gravity model: call hp_plan_set_den_model first"); return HP_ERR_NO_MODEL; }
  if (method < HP_EULER || method > HP_RK4) { hp_set_error("bad method"); return HP_ERR_INVALID; }
  if (!std::isfinite(dt)) { hp_set_error("dt must be finite"); return HP_ERR_INVALID; }
  int st = HP_OK;
  const void* fg = nullptr;
  if (f) {
    const long long ng = p->n_grid();
    const double* df = (const double*)stage_in(p, "api.fin", f, sizeof(double) * ng, mem, &st);
    if (st) return st;
    fg = df;
    if (p->precision == HP_MIXED) {
      float* t = (float*)p->ws_get("api.f32", sizeof(float) * ng, &st);
      if (st) return st;
      ProfScope _ps(p, "convert", p->stream);
      k_d2f<<<(unsigned)((ng + 255) / 256), 256, 0, p->stream>>>(df, t, ng);
      HP_CUDA_TRY(cudaGetLastError());
      fg = t;
    }
  }
  const size_t fb = 16 * (size_t)p->n_full(), ib = 16 * (size_t)p->nrows * p->nx;
  double2* b0 = (double2*)p->ws_get("api.S0", ib, &st); if (st) return st;
  double2* b1 = (double2*)p->ws_get("api.S1", ib, &st); if (st) return st;
  double2* b2 = (method == HP_EULER) ? nullptr : (double2*)p->ws_get("api.S2", ib, &st); if (st) return st;
  double2* ac = (method == HP_RK2 || method == HP_RK4) ? (double2*)p->ws_get("api.S3", ib, &st) : nullptr;
  if (st) return st;
  HP_CHECK(load_full(p, Fold, mem, b0));
  double2 *F = b0, *F2 = b1, *F3 = b2;
  HP_CHECK(integrate_internal(p, &F, &F2, &F3, ac, dt, method, fg));
  double2* dOut = (double2*)stage_out(p, "api.Fout", Fnew, fb, mem, &st);
  if (st) return st;
  HP_CHECK(hp_internal_to_full(p, F, dOut, p->stream));
  HP_CHECK(finish_out(p, Fnew, dOut, fb, mem));
  HP_CUDA_TRY(cudaStreamSynchronize(p->stream));
  return HP_OK;
}

extern "C" int hp_pendulum_derivative(hp_plan* p, const double* F, double* dF, int mem) {
  if (!p || !F || !dF) { hp_set_error("null argument"); return HP_ERR_INVALID; }
  HP_CHECK(check_mem(mem));
  if (!p->has_model) { hp_set_error("no model: call hp_plan_set_model first"); return HP_ERR_NO_MODEL; }
  int st = HP_OK;
  const size_t fb = 16 * (size_t)p->n_full(), ib = 16 * (size_t)p->nrows * p->nx;
  double2* b0 = (double2*)p->ws_get("api.S0", ib, &st); if (st) return st;
  double2* b1 = (double2*)p->ws_get("api.S1", ib, &st); if (st) return st;
  HP_CHECK(load_full(p, F, mem, b0));
  HP_CHECK(hp_derivative_eval(p, b0, nullptr, 1.0, b1, nullptr, 0.0, p->stream));
  double2* dOut = (double2*)stage_out(p, "api.Fout", dF, fb, mem, &st);
  if (st) return st;
  HP_CHECK(hp_internal_to_full(p, b1, dOut, p->stream));
  HP_CHECK(finish_out(p, dF, dOut, fb, mem));
  HP_CUDA_TRY(cudaStreamSynchronize(p->stream));
  return HP_OK;
}

extern "C" int hp_fftSO3_prod(hp_plan* p, const double* F, const double* G, double* FG, int batch, int mem) {
  if (!p || !F || !G || !FG || batch < 1) { hp_set_error("bad argument"); return HP_ERR_INVALID; }
  HP_CHECK(check_mem(mem));
  int st = HP_OK;
  const size_t nb = 16 * (size_t)p->D * p->D * p->B * batch;
  const double2* dFa = (const double2*)stage_in(p, "prod.F", F, nb, mem, &st); if (st) return st;
  const double2* dGa = (const double2*)stage_in(p, "prod.G", G, nb, mem, &st); if (st) return st;
  double2* dO = (double2*)stage_out(p, "prod.FG", FG, nb, mem, &st); if (st) return st;
  HP_CHECK(hp_prod_launch(p, dFa, dGa, dO, batch, p->stream));
  HP_CHECK(finish_out(p, FG, dO, nb, mem));
  HP_CUDA_TRY(cudaStreamSynchronize(p->stream));
  return HP_OK;
}

// ---------------------------------------------------------------- state ----
extern "C" int hp_state_create(hp_plan* p, hp_state** out) {
  if (!p || !out) { hp_set_error("null argument"); return HP_ERR_INVALID; }
  *out = nullptr;
  hp_state* s = new hp_state();
  s->plan = p;
  const size_t ib = 16 * (size_t)p->nrows * p->nx;
  // F3 and acc are allocated on first use by a method that needs them
  double2** bufs[2] = {&s->F, &s->F2};
  for (auto b : bufs) {
    if (hp_dev_alloc(b, ib) != cudaSuccess) {
      cudaGetLastError();
      hp_state_destroy(s);
      hp_set_error("device allocation failed");
      return HP_ERR_ALLOC;
    }
  }
  HP_CUDA_TRY(cudaMemset(s->F, 0, ib));
  *out = s;
  return HP_OK;
}

extern "C" int hp_state_destroy(hp_state* s) {
  if (!s) return HP_OK;
  hp_dev_free(s->guard_flag);
  hp_dev_free(s->F); hp_dev_free(s->F2); hp_dev_free(s->F3); hp_dev_free(s->acc); hp_dev_free(s->fg);
  hp_dev_free(s->F32[0]); hp_dev_free(s->F32[1]);
  delete s;
  return HP_OK;
}

extern "C" int hp_state_load(hp_state* s, const double* F, int mem) {
  if (!s || !F) { hp_set_error("null argument"); return HP_ERR_INVALID; }
  HP_CHECK(check_mem(mem));
  hp_plan* p = s->plan;
  HP_CHECK(load_full(p, F, mem, s->F));
  HP_CUDA_TRY(cudaStreamSynchronize(p->stream));
  s->fg_valid = false;
  s->f32_valid = false;
  return HP_OK;
}

extern "C" int hp_state_store(hp_state* s, double* F, int mem) {
  if (!s || !F) { hp_set_error("null argument"); return HP_ERR_INVALID; }
  HP_CHECK(check_mem(mem));
  hp_plan* p = s->plan;
  int st = HP_OK;
  const size_t fb = 16 * (size_t)p->n_full();
  double2* d = (double2*)stage_out(p, "api.Fout", F, fb, mem, &st);
  if (st) return st;
  HP_CHECK(hp_internal_to_full(p, s->F, d, p->stream));
  HP_CHECK(finish_out(p, F, d, fb, mem));
  HP_CUDA_TRY(cudaStreamSynchronize(p->stream));
  return HP_OK;
}

// stage buffers of the midpoint and Runge-Kutta methods, allocated on first use
static int state_bufs(hp_state* s, int method) {
  const size_t ib = 16 * (size_t)s->plan->nrows * s->plan->nx;
  if (method != HP_EULER && !s->F3) {
    if (hp_dev_alloc(&s->F3, ib) != cudaSuccess) { cudaGetLastError(); s->F3 = nullptr; hp_set_error("device allocation failed"); return HP_ERR_ALLOC; }
  }
  if ((method == HP_RK2 || method == HP_RK4) && !s->acc) {
    if (hp_dev_alloc(&s->acc, ib) != cudaSuccess) { cudaGetLastError(); s->acc = nullptr; hp_set_error("device allocation failed"); return HP_ERR_ALLOC; }
  }
  return HP_OK;
}

extern "C" int hp_state_step(hp_state* s, double dt, int method, int nsteps) {
  if (!s || nsteps < 0) { hp_set_error("bad argument"); return HP_ERR_INVALID; }
  hp_plan* p = s->plan;
  if (!p->has_model) { hp_set_error("no model: call hp_plan_set_model first"); return HP_ERR_NO_MODEL; }
  if (method < HP_EULER || method > HP_RK4) { hp_set_error("bad method"); return HP_ERR_INVALID; }
  HP_CHECK(state_bufs(s, method));
  if (nsteps > 0) s->fg_valid = false;
  // Mixed 3-D plans carry F in FP32 from step to step: the last plane pass of
  // a step writes it, the next step's first evaluation and the density read it.
  const bool carry = p->ndim == 3 && p->precision == HP_MIXED;
  if (carry && !s->F32[0]) {
    const size_t b32 = 8 * (size_t)p->nrows * p->nx;
    if (hp_dev_alloc(&s->F32[0], b32) != cudaSuccess || hp_dev_alloc(&s->F32[1], b32) != cudaSuccess) {
      cudaGetLastError();
      hp_dev_free(s->F32[0]); hp_dev_free(s->F32[1]);
      s->F32[0] = s->F32[1] = nullptr;
      hp_set_error("device allocation failed");
      return HP_ERR_ALLOC;
    }
    s->f32_valid = false;
  }
  for (int k = 0; k < nsteps; ++k) {
    if (carry) {
      const float2* in = s->f32_valid ? s->F32[s->f32_cur] : nullptr;
      s->f32_valid = false;
      HP_CHECK(integrate_internal(p, &s->F, &s->F2, &s->F3, s->acc, dt, method, nullptr, in,
                                  s->F32[1 - s->f32_cur]));
      s->f32_cur = 1 - s->f32_cur;
      s->f32_valid = true;
    } else {
      HP_CHECK(integrate_internal(p, &s->F, &s->F2, &s->F3, s->acc, dt, method));
    }
    HP_CHECK(hp_state_guard_check(s, false));
  }
  return HP_OK;
}

// ------------------------------------------------------ health guard ----
__global__ void k_nonfinite(const double2* __restrict__ a, long long n, int* __restrict__ flag) {
  bool bad = false;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double2 v = a[i];
    bad |= !isfinite(v.x) || !isfinite(v.y);
  }
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(flag, 1);
}

extern "C" int hp_state_set_guard(hp_state* s, int check_every, double mass_rtol) {
  if (!s || check_every < 0 || !std::isfinite(mass_rtol)) { hp_set_error("bad argument"); return HP_ERR_INVALID; }
  if (check_every > 0 && !s->guard_flag) {
    if (hp_dev_alloc(&s->guard_flag, sizeof(int)) != cudaSuccess) {
      cudaGetLastError();
      s->guard_flag = nullptr;
      hp_set_error("device allocation failed");
      return HP_ERR_ALLOC;
    }
  }
  double m0 = 0.0;
  if (check_every > 0 && mass_rtol > 0) {
    HP_CHECK(hp_state_mass(s, &m0));
    if (!std::isfinite(m0) || m0 == 0.0) { hp_set_error("the state's l = 0 mass is zero or not finite"); return HP_ERR_NONFINITE; }
  }
  s->guard_every = check_every;
  s->guard_rtol = mass_rtol > 0 ? mass_rtol : 0.0;
  s->guard_mass0 = m0;
  s->guard_count = 0;
  return HP_OK;
}

int hp_state_guard_check(hp_state* s, bool force) {
  if (s->guard_every <= 0 || !s->guard_flag) return HP_OK;
  // inside a batch step whose plane passes are collected the state is not
  // final yet: the batch checks its guarded members after the step
  if (hp_plane_collecting()) return HP_OK;
  if (!force && ++s->guard_count % s->guard_every) return HP_OK;
  hp_plan* p = s->plan;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  HP_CUDA_TRY(cudaStreamIsCapturing(p->stream, &cs));
  if (cs != cudaStreamCaptureStatusNone) return HP_OK;
  const long long n = p->nrows * p->nx;
  HP_CUDA_TRY(cudaMemsetAsync(s->guard_flag, 0, sizeof(int), p->stream));
  {
    ProfScope _ps(p, "guard", p->stream);
    const long long nb = std::min<long long>((n + 255) / 256, 148LL * 8);
    k_nonfinite<<<(unsigned)nb, 256, 0, p->stream>>>(s->F, n, s->guard_flag);
  }
  HP_CUDA_TRY(cudaGetLastError());
  int flag = 0;
  const long long row = p->h_seg[(size_t)(0 - p->m_lo) * p->D + p->lmax];
  double2 m;
  HP_CUDA_TRY(cudaMemcpyAsync(&flag, s->guard_flag, sizeof(int), cudaMemcpyDeviceToHost, p->stream));
  HP_CUDA_TRY(cudaMemcpyAsync(&m, s->F + row * p->nx, sizeof(double2), cudaMemcpyDeviceToHost, p->stream));
  HP_CUDA_TRY(cudaStreamSynchronize(p->stream));
  char msg[160];
  if (flag) {
    snprintf(msg, sizeof msg, "non-finite coefficients after step %lld since the guard was set", s->guard_count);
    hp_set_error(msg);
    return HP_ERR_NONFINITE;
  }
  if (s->guard_rtol > 0) {
    const double drift = std::fabs(m.x - s->guard_mass0) / std::fabs(s->guard_mass0);
    if (!(drift <= s->guard_rtol)) {
      snprintf(msg, sizeof msg, "l = 0 mass drifted by %.3e (tolerance %.3e) after step %lld since the guard was set",
               drift, s->guard_rtol, s->guard_count);
      hp_set_error(msg);
      return HP_ERR_MASS_DRIFT;
    }
  }
  return HP_OK;
}

// Loads the state from a grid density on the device in the plan's compute
// precision (double for HP_FP64, float for HP_MIXED; complex interleaved for
// HP_COMPLEX plans): F = fftSO3R(f).
extern "C" int hp_state_load_density(hp_state* s, const void* f) {
  if (!s || !f) { hp_set_error("null argument"); return HP_ERR_INVALID; }
  hp_plan* p = s->plan;
  HP_CHECK(hp_forward_internal(p, f, p->symmetry == HP_COMPLEX, s->F, p->stream));
  s->fg_valid = false;
  s->f32_valid = false;
  HP_CUDA_TRY(cudaStreamSynchronize(p->stream));
  return HP_OK;
}

// pendulum_reduced_hybrid.m:226-234 per step: F = propagate_den(F, f);
// f = backward(F); f += dt * df(f); F = forward(f).
extern "C" int hp_state_hybrid_step(hp_state* s, hp_collision* c, double dt, int method, int nsteps) {
  if (!s || !c || nsteps < 0) { hp_set_error("bad argument"); return HP_ERR_INVALID; }
  hp_plan* p = s->plan;
  if (hp_collision_plan(c) != p) { hp_set_error("collision operator belongs to another plan"); return HP_ERR_INVALID; }
  if (!p->has_model) { hp_set_error("no model: call hp_plan_set_den_model or hp_plan_set_model first"); return HP_ERR_NO_MODEL; }
  if (method < HP_EULER || method > HP_RK4) { hp_set_error("bad method"); return HP_ERR_INVALID; }
  if (!std::isfinite(dt)) { hp_set_error("dt must be finite"); return HP_ERR_INVALID; }
  cudaStream_t st = p->stream;
  HP_CHECK(state_bufs(s, method));
  if (!s->fg) {
    const size_t eb = p->precision == HP_FP64 ? sizeof(double) : sizeof(float);
    if (hp_dev_alloc(&s->fg, eb * (size_t)p->n_grid()) != cudaSuccess) {
      cudaGetLastError();
      s->fg = nullptr;
      hp_set_error("device allocation failed");
      return HP_ERR_ALLOC;
    }
  }
  if (nsteps > 0) s->f32_valid = false;   // the forward transform below rewrites F
  if (!s->fg_valid && nsteps > 0) HP_CHECK(hp_backward_internal(p, s->F, s->fg, 0, st));
  for (int k = 0; k < nsteps; ++k) {
    s->fg_valid = false;
    HP_CHECK(integrate_internal(p, &s->F, &s->F2, &s->F3, s->acc, dt, method, s->fg));
    HP_CHECK(hp_backward_internal(p, s->F, s->fg, 0, st));
    HP_CHECK(hp_collision_apply(c, s->fg, dt, st));
    HP_CHECK(hp_forward_internal(p, s->fg, 0, s->F, st));
    s->fg_valid = true;
    HP_CHECK(hp_state_guard_check(s, false));
  }
  return HP_OK;
}

// The grid density of the state: after hybrid steps the post-collision
// density (the f of pendulum_reduced_hybrid.m:233), else backward(F).
extern "C" int hp_state_density(hp_state* s, void* f) {
  if (!s || !f) { hp_set_error("null argument"); return HP_ERR_INVALID; }
  hp_plan* p = s->plan;
  if (s->fg_valid) {
    const size_t eb = p->precision == HP_FP64 ? sizeof(double) : sizeof(float);
    HP_CUDA_TRY(cudaMemcpyAsync(f, s->fg, eb * (size_t)p->n_grid(), cudaMemcpyDeviceToDevice, p->stream));
    return HP_OK;
  }
  if (s->f32_valid)   // the FP32 copy the last step left: the values the FP32 transform converts to
    return hp_backward_internal32(p, s->F32[s->f32_cur], f, p->symmetry == HP_COMPLEX, p->stream);
  return hp_backward_internal(p, s->F, f, p->symmetry == HP_COMPLEX, p->stream);
}

__global__ void k_scale_c64(double2* __restrict__ a, long long n, double s) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n) { a[i].x *= s; a[i].y *= s; }
}

extern "C" int hp_state_normalize(hp_state* s, double mass, double* scale) {
  if (!s || !(mass > 0) || !std::isfinite(mass)) { hp_set_error("bad argument"); return HP_ERR_INVALID; }
  double m0 = 0.0;
  HP_CHECK(hp_state_mass(s, &m0));
  if (!(m0 > 0) || !std::isfinite(m0)) { hp_set_error("state mass is not positive and finite"); return HP_ERR_NONFINITE; }
  hp_plan* p = s->plan;
  const double f = mass / m0;
  const long long n = p->nrows * p->nx;
  s->fg_valid = false;
  s->f32_valid = false;
  {
    ProfScope _ps(p, "normalize", p->stream);
    k_scale_c64<<<(unsigned)((n + 255) / 256), 256, 0, p->stream>>>(s->F, n, f);
  }
  HP_CUDA_TRY(cudaGetLastError());
  if (scale) *scale = f;
  return HP_OK;
}

extern "C" int hp_state_mass(hp_state* s, double* mass) {
  if (!s || !mass) { hp_set_error("null argument"); return HP_ERR_INVALID; }
  hp_plan* p = s->plan;
  // row (l=0, m=0, n=0) at omega index 0
  const long long row = p->h_seg[(size_t)(0 - p->m_lo) * p->D + p->lmax];
  double2 v;
  HP_CUDA_TRY(cudaMemcpyAsync(&v, s->F + row * p->nx, sizeof(double2), cudaMemcpyDeviceToHost, p->stream));
  HP_CUDA_TRY(cudaStreamSynchronize(p->stream));
  *mass = v.x;
  return HP_OK;
}
