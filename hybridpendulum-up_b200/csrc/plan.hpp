// Plan: sizes, row layout, device tables and workspace of one (B, Bx, ndim,
// precision, symmetry) configuration.
#pragma once
#include <string>
#include <vector>
#include <cuda_runtime.h>
#include "../../include/hp.h"

// Device-side view of the row layout, passed by value to kernels.
//
// Internal coefficient layout ("row-major over omega"): F[row * nx + w], where
// w = k1 + N*k2 (+ N^2*k3) runs over the omega Fourier grid in FFT order and a
// row is one (l, m, n) with m in [m_lo, lmax] (m_lo = 0 for HP_REAL, -lmax for
// HP_COMPLEX), n in [-lmax, lmax] and l in [max(|m|,|n|), lmax], ordered by
// m, then n, then l.  Rows of one (m, n) segment are therefore consecutive in l.
struct RowLayout {
  int B, lmax, N, ndim, m_lo, nm;   // nm = number of stored m values
  long long nx, nrows;
  const char4* rows;                // (l, m, n, 0) per row
  const int* seg;                   // first row of segment (m, n): seg[(m-m_lo)*(2lmax+1) + n+lmax]
};

struct hp_state;

struct Buf {
  void* p = nullptr;
  size_t bytes = 0;
};

// Per-kernel-family CUDA-event timing (opt-in) and a launch counter.
struct ProfEntry {
  std::string name;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> pending;
  double ms = 0.0;
  long long count = 0;
};

struct hp_plan {
  int B = 0, lmax = 0, Bx = 0, N = 0, ndim = 0, precision = 0, symmetry = 0;
  int m_lo = 0, nm = 0, D = 0;     // D = 2lmax+1
  long long nx = 0, nrows = 0;
  cudaStream_t stream = nullptr;

  std::vector<char4> h_rows;
  std::vector<int> h_seg;

  // device tables
  char4* rows = nullptr;
  int* seg = nullptr;
  // the kept entries in full-layout order (m fastest, then n, then l):
  // (full index within one omega slice, row)
  int2* fgather = nullptr;
  double* wig64 = nullptr;   // [b][row] d^l_mn(beta_b)
  float* wig32 = nullptr;
  double* wfull = nullptr;   // d(2lmax+1,2lmax+1,lmax+1,2B) in the MATLAB layout
  double* qw = nullptr;      // quadrature weights [2B]
  double* cg1 = nullptr;     // <l1 m1; 1 m2 | l m> table, see cg1_index()

  // model
  bool has_model = false;
  hp_model model{};
  double* tap_wr = nullptr;  // [row][9] real gravity tap weights, tap (l1-l+1)*3 + (n2+1)
  float* tap_wr32 = nullptr;
  double2 mr1[3][3] = {};    // MR_i^1_{0 n2} of the model: [n2+1][i]
  double* den_mR = nullptr;  // [2][(2B)^3] density-side gravity multipliers (pendulum_reduced_den)
  // attitude diffusion sum_ij G1_ij F^l u_i^T u_j^T of the gyro-bias model:
  // [row][5] complex weights of F^l_{m, n+o-2}, o = 0..4 (null when absent)
  double2* so3d64 = nullptr;
  float2* so3d32 = nullptr;

  // engine of the forward transform's beta contraction (enum hp_beta_engine)
  int beta_engine = 0;
  // launch shapes chosen by hp_plan_autotune (defaults: the hand-picked ones)
  struct Tune {
    int synth_pt = 1;      // omega points per beta-stage item of the synthesis (1, 2, 4; FP32)
    int synth_waves = 8;   // resident waves of synthesis blocks per SM set
    int tc_waves = 16;     // waves of tensor-core CTAs of the forward beta contraction
    int tc_form = 0;       // 0: the staged tensor-core kernel, 1: the warp-specialised TMA-fed one
  } tune;

  // profiling
  bool prof_on = false;
  std::vector<ProfEntry> prof;
  long long launches = 0;

  // workspace (grow-only), keyed by name
  std::vector<std::pair<std::string, Buf>> ws;
  void* ws_get(const char* name, size_t bytes, int* status);
  void ws_release(const char* name);   // frees a workspace buffer (re-created on demand)

  RowLayout layout() const {
    RowLayout L;
    L.B = B; L.lmax = lmax; L.N = N; L.ndim = ndim; L.m_lo = m_lo; L.nm = nm;
    L.nx = nx; L.nrows = nrows; L.rows = rows; L.seg = seg;
    return L;
  }
  size_t cplx_bytes() const { return precision == HP_FP64 ? 16 : 8; }
  long long n_full() const { return (long long)D * D * (lmax + 1) * nx; }
  long long n_grid() const { return 8LL * B * B * B * nx; }
};

struct hp_state {
  hp_plan* plan = nullptr;
  double2* F = nullptr;     // current coefficients, FP64, internal layout
  double2* F2 = nullptr;    // ping-pong / stage buffers
  double2* F3 = nullptr;
  double2* acc = nullptr;
  void* fg = nullptr;       // grid density of the hybrid step (compute precision)
  bool fg_valid = false;    // fg holds the post-collision density of F
  // mixed 3-D plans: F converted to FP32 by the last plane pass of a step,
  // ping-pong pair; F32[f32_cur] is valid for the current F when f32_valid
  float2* F32[2] = {nullptr, nullptr};
  int f32_cur = 0;
  bool f32_valid = false;
  // per-step health check (hp_state_set_guard): every guard_every steps
  int guard_every = 0;
  double guard_rtol = 0.0;      // l = 0 mass drift tolerance (<= 0: not checked)
  double guard_mass0 = 0.0;     // F^0_00[0] when the guard was set
  long long guard_count = 0;    // steps since the guard was set
  int* guard_flag = nullptr;    // device flag of the non-finite scan
};
// The check of hp_state_set_guard after a step (force: whatever the count);
// returns HP_ERR_NONFINITE / HP_ERR_MASS_DRIFT when it fails.
int hp_state_guard_check(hp_state* s, bool force);

struct hp_collision;
// f += dt * df(f), in place, f in the plan's compute precision (device).
int hp_collision_apply(hp_collision* c, void* f, double dt, cudaStream_t s);
hp_plan* hp_collision_plan(const hp_collision* c);

// <l1 m1; 1 m2 | l m> with m1 = m - m2, l = l1 + dl (dl in -1..1):
// cg1[((l1 * 3 + (dl+1)) * (2*lmax+3) + (m + lmax+1)) * 3 + (m2+1)]
inline __host__ __device__ int cg1_index(int lmax, int l1, int dl, int m, int m2) {
  return ((l1 * 3 + (dl + 1)) * (2 * lmax + 3) + (m + lmax + 1)) * 3 + (m2 + 1);
}

// RAII: counts one launch on plan p and, when profiling is on, brackets it
// with CUDA events recorded on stream s under the family `name`.
struct ProfScope {
  hp_plan* p;
  int idx = -1;
  cudaEvent_t a = nullptr;
  cudaStream_t s;
  ProfScope(hp_plan* plan, const char* name, cudaStream_t stream);
  ~ProfScope();
};

// launch shapes found earlier by hp_plan_autotune for the plan's key, if any
void hp_tune_apply_cached(hp_plan* p);

// ---- launchers implemented in the .cu files (return hp_status) ----
int hp_tables_build(hp_plan* p);
int hp_twiddles_init();
int hp_build_gravity_taps(hp_plan* p);
int hp_full_to_internal(hp_plan* p, const double2* Ffull, double2* Fint, cudaStream_t s);
int hp_internal_to_full(hp_plan* p, const double2* Fint, double2* Ffull, cudaStream_t s);
// full layout -> [row][omega], reading only the kept entries of Ff, which may be
// host memory mapped into the device address space (read in place)
int hp_full_gather(hp_plan* p, const double2* Ff, double2* Fi, cudaStream_t s);
// Coefficients of the derivative terms: lie scales the Lie (u) term, gs[i]
// the gravity component i (coefficient taps, or the density-side term of a
// density-gravity model when gs[0] or gs[1] is non-zero); b, G, gyro as in hp_model.
struct DerivParams {
  double L;
  double b[3];
  double G[9];
  double gyro[3];
  double lie;
  double gs[3];
  double mr[3][3][2];  // MR_i^1_{0 n2}: [n2+1][i][re, im]
};
// Persistent batched plane pass (deriv.cu): between hp_plane_collect_begin and
// _end, the plane passes of 3-D derivative evaluations are recorded as jobs
// (per compute precision) instead of launched; hp_plane_batch_prepare numbers
// their work items, hp_plane_batch_launch runs one precision's jobs (copied
// to d_jobs by the caller) in one persistent launch.
struct PlaneTile { int m, l, n0, cnt; };   // (m, l) row, rows n0 .. n0+cnt-1 of the plane pass
struct PlaneJob {
  RowLayout L;
  const PlaneTile* tiles;
  int ntiles, N;
  const void* Fev;   // compute-precision input (the FP32 copy, or the FP64 state of FP64 plans)
  const void* P3;
  const void* G;
  const double2* F0;
  double a;
  double2* out;
  double2* acc;
  double bacc;
  void* out32;
  DerivParams prm;
  long long item0;   // first queue item of this job
};
void hp_plane_collect_begin(std::vector<PlaneJob>* f32, std::vector<PlaneJob>* f64);
void hp_plane_collect_end();
bool hp_plane_collecting();
void hp_plane_batch_prepare(std::vector<PlaneJob>& jobs);
size_t hp_plane_job_bytes();
int hp_plane_batch_launch(int precision, const std::vector<PlaneJob>& jobs, const PlaneJob* d_jobs, int* counter,
                          cudaStream_t s);

DerivParams hp_model_params(const hp_plan* p);
// fev32 (mixed 3-D plans, may be null): Feval already converted to FP32 in the
// [row][omega] layout; out32 (may be null): receives out converted to FP32.
int hp_derivative_eval_prm(hp_plan* p, const DerivParams& prm, const double2* Feval, const double2* F0,
                           double a, double2* out, double2* acc, double bacc, cudaStream_t s,
                           const void* fgrid = nullptr, const void* fev32 = nullptr, void* out32 = nullptr);
// The gravity and noise terms of the derivative alone (the pointwise-in-omega
// pass), in FP64 whatever the plan's precision: out = noise F + gravity F
// ([row][omega] layout, FP64 in and out).
int hp_gravity_noise_eval64(hp_plan* p, const DerivParams& prm, const double2* F, double2* out, cudaStream_t s);
int hp_derivative_eval(hp_plan* p, const double2* Feval, const double2* F0, double a,
                       double2* out, double2* acc, double bacc, cudaStream_t s,
                       const void* fgrid = nullptr, const void* fev32 = nullptr, void* out32 = nullptr);
// backward transform from FP32 coefficients in the [row][omega] layout (mixed plans)
int hp_backward_internal32(hp_plan* p, const float2* Fint32, void* f, int complex_out, cudaStream_t s);
// Forward transform of mult . f (mult: (2B)^3 grid samples, may be null) into
// [row][omega] coefficients in the plan's compute precision (c2<T>).
int hp_forward_internal_T(hp_plan* p, const void* f, const double* mult, void* out, cudaStream_t s);
int hp_backward_internal(hp_plan* p, const double2* Fint, void* f, int complex_out, cudaStream_t s);
namespace hp {
// Tensor-core (tcgen05, TF32-split) beta contraction of the forward transform
// (tc_beta.cu): FP32 plans with B <= 32.  Qg: stage-1 tiles of the omega chunk
// [w0, w0 + nwc), stride nwc; out: [row][nx] FP32 coefficients.
bool tc_beta_supported(const hp_plan* p);
int tc_beta_forward(hp_plan* p, const float2* Qg, const int2* pairs, int npairs, float2* out, long long w0,
                    long long nwc, cudaStream_t s);
// number of launches whose wait on the tensor cores gave up (0 when none ran)
int tc_beta_errors(hp_plan* p, int* count);
}  // namespace hp
int hp_forward_internal(hp_plan* p, const void* f, int complex_in, double2* Fint, cudaStream_t s);
int hp_forward_internal64(hp_plan* p, const double* f, double2* Fint, cudaStream_t s);
// inverse (scaled 1/nx) / forward omega FFT of every row, in the plan's compute precision
int hp_omega_ifft_rows(hp_plan* p, const double2* in, void* out, cudaStream_t s);
int hp_omega_fft_rows(hp_plan* p, void* inout, cudaStream_t s);
int hp_prod_launch(hp_plan* p, const double2* F, const double2* G, double2* FG, int batch,
                   cudaStream_t s);
