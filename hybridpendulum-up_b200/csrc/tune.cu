// Autotuner of a plan's launch shapes, with a process-wide cache keyed by
// (B, Bx, ndim, precision, symmetry, beta engine) that can be saved to and
// loaded from a text file.
//
// The knobs are the runtime launch shapes of the two transforms:
//   synth_pt    omega points per beta-stage item of the synthesis (FP32
//               plans: 1, 2 or 4; an item then holds an NB x PT output tile)
//   synth_waves resident waves of synthesis blocks (4, 8 or 16): how many
//               omega chunks each block walks through
//   tc_waves    waves of tensor-core CTAs of the forward beta contraction
//               (8, 16 or 32), i.e. omega tiles per CTA
//   tc_form     the tensor-core kernel: 1 the warp-specialised TMA-fed
//               pipeline, 0 the staged single-warpgroup form
// Each candidate is timed with CUDA events on the plan's stream, on scratch
// coefficients and densities of the plan's own sizes (zeros: the kernels have
// no value-dependent control flow), and the fastest kept.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "common.cuh"
#include "plan.hpp"

namespace {

using Key = std::tuple<int, int, int, int, int, int>;
std::mutex g_mu;
std::map<Key, hp_plan::Tune> g_cache;

Key key_of(const hp_plan* p) { return Key(p->B, p->Bx, p->ndim, p->precision, p->symmetry, p->beta_engine); }

struct Scratch {
  void* p = nullptr;
  ~Scratch() { hp_dev_free(p); }
};

// median of `reps` timed calls of fn (one untimed call first)
template <typename F>
int time_it(cudaStream_t s, int reps, F fn, float* ms) {
  cudaEvent_t a, b;
  HP_CUDA_TRY(cudaEventCreate(&a));
  HP_CUDA_TRY(cudaEventCreate(&b));
  int st = fn();
  std::vector<float> t;
  for (int r = 0; r < reps && st == HP_OK; ++r) {
    cudaEventRecord(a, s);
    st = fn();
    cudaEventRecord(b, s);
    float x = 0;
    if (st == HP_OK && cudaEventSynchronize(b) == cudaSuccess && cudaEventElapsedTime(&x, a, b) == cudaSuccess)
      t.push_back(x);
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (st) return st;
  if (t.empty()) { hp_set_error("timing failed"); return HP_ERR_CUDA; }
  std::sort(t.begin(), t.end());
  *ms = t[t.size() / 2];
  return HP_OK;
}

}  // namespace

void hp_tune_apply_cached(hp_plan* p) {
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = g_cache.find(key_of(p));
  if (it != g_cache.end()) p->tune = it->second;
}

extern "C" int hp_plan_set_tune(hp_plan* p, int synth_pt, int synth_waves, int tc_waves, int tc_form) {
  if (!p) { hp_set_error("null plan"); return HP_ERR_INVALID; }
  if ((synth_pt && synth_pt != 1 && synth_pt != 2 && synth_pt != 4) || synth_waves < 0 || synth_waves > 64 ||
      tc_waves < 0 || tc_waves > 256 || tc_form < -1 || tc_form > 1) {
    hp_set_error("synth_pt must be 1, 2 or 4; waves in 1..64 (synthesis) and 1..256 (tensor cores); tc_form 0 or 1; "
                 "0 (-1 for tc_form) keeps a knob");
    return HP_ERR_INVALID;
  }
  if (synth_pt) p->tune.synth_pt = synth_pt;
  if (synth_waves) p->tune.synth_waves = synth_waves;
  if (tc_waves) p->tune.tc_waves = tc_waves;
  if (tc_form >= 0) p->tune.tc_form = tc_form;
  return HP_OK;
}

extern "C" int hp_plan_get_tune(const hp_plan* p, int* synth_pt, int* synth_waves, int* tc_waves, int* tc_form) {
  if (!p) { hp_set_error("null plan"); return HP_ERR_INVALID; }
  if (synth_pt) *synth_pt = p->tune.synth_pt;
  if (synth_waves) *synth_waves = p->tune.synth_waves;
  if (tc_waves) *tc_waves = p->tune.tc_waves;
  if (tc_form) *tc_form = p->tune.tc_form;
  return HP_OK;
}

extern "C" int hp_plan_autotune(hp_plan* p, double* best_backward_ms, double* best_forward_ms) {
  if (!p) { hp_set_error("null plan"); return HP_ERR_INVALID; }
  if (p->prof_on) { hp_set_error("disable plan profiling before tuning"); return HP_ERR_INVALID; }
  cudaStream_t s = p->stream;
  const bool cplx = p->symmetry == HP_COMPLEX;
  const size_t fe = (p->precision == HP_FP64 ? 8 : 4) * (cplx ? 2 : 1);
  Scratch F, f;
  HP_CUDA_TRY(hp_dev_alloc(&F.p, 16 * (size_t)p->nrows * p->nx));
  HP_CUDA_TRY(hp_dev_alloc(&f.p, fe * (size_t)p->n_grid()));
  HP_CUDA_TRY(cudaMemsetAsync(F.p, 0, 16 * (size_t)p->nrows * p->nx, s));
  HP_CUDA_TRY(cudaMemsetAsync(f.p, 0, fe * (size_t)p->n_grid(), s));
  const hp_plan::Tune start = p->tune;
  hp_plan::Tune best = start;
  float best_b = 1e30f;
  const std::vector<int> pts = p->precision == HP_FP64 ? std::vector<int>{1} : std::vector<int>{1, 2, 4};
  for (int pt : pts)
    for (int waves : {4, 8, 16}) {
      p->tune.synth_pt = pt;
      p->tune.synth_waves = waves;
      float ms = 0;
      const int st = time_it(s, 3, [&] { return hp_backward_internal(p, (const double2*)F.p, f.p, cplx, s); }, &ms);
      if (st) { p->tune = start; return st; }
      if (ms < best_b) {
        best_b = ms;
        best.synth_pt = pt;
        best.synth_waves = waves;
      }
    }
  p->tune = best;
  float best_f = 0;
  const bool tc = p->precision == HP_MIXED && hp::tc_beta_supported(p) &&
                  (p->beta_engine == HP_BETA_TENSOR || p->beta_engine == HP_BETA_TENSOR_BF16 ||
                   (p->beta_engine == HP_BETA_AUTO && p->B >= 15));
  if (tc) {
    best_f = 1e30f;
    for (int form : {1, 0})
      for (int waves : form == 1 ? std::vector<int>{1, 2, 4} : std::vector<int>{8, 16, 32}) {
        p->tune.tc_form = form;
        p->tune.tc_waves = waves;
        float ms = 0;
        const int st = time_it(s, 3, [&] { return hp_forward_internal(p, f.p, cplx, (double2*)F.p, s); }, &ms);
        if (st) { p->tune = best; return st; }
        if (ms < best_f) {
          best_f = ms;
          best.tc_form = form;
          best.tc_waves = waves;
        }
      }
    p->tune = best;
  }
  HP_CUDA_TRY(cudaStreamSynchronize(s));
  {
    std::lock_guard<std::mutex> lk(g_mu);
    g_cache[key_of(p)] = best;
  }
  if (best_backward_ms) *best_backward_ms = best_b;
  if (best_forward_ms) *best_forward_ms = best_f;
  return HP_OK;
}

extern "C" int hp_tune_cache_save(const char* path) {
  if (!path) { hp_set_error("null path"); return HP_ERR_INVALID; }
  FILE* fp = std::fopen(path, "w");
  if (!fp) { hp_set_error("cannot open the tuning cache file for writing"); return HP_ERR_INVALID; }
  std::fprintf(fp, "# B Bx ndim precision symmetry beta_engine synth_pt synth_waves tc_waves tc_form\n");
  std::lock_guard<std::mutex> lk(g_mu);
  for (auto& kv : g_cache) {
    const Key& k = kv.first;
    std::fprintf(fp, "%d %d %d %d %d %d %d %d %d %d\n", std::get<0>(k), std::get<1>(k), std::get<2>(k), std::get<3>(k),
                 std::get<4>(k), std::get<5>(k), kv.second.synth_pt, kv.second.synth_waves, kv.second.tc_waves,
                 kv.second.tc_form);
  }
  std::fclose(fp);
  return HP_OK;
}

extern "C" int hp_tune_cache_load(const char* path) {
  if (!path) { hp_set_error("null path"); return HP_ERR_INVALID; }
  FILE* fp = std::fopen(path, "r");
  if (!fp) { hp_set_error("cannot open the tuning cache file"); return HP_ERR_INVALID; }
  char line[256];
  int bad = 0;
  std::lock_guard<std::mutex> lk(g_mu);
  while (std::fgets(line, sizeof line, fp)) {
    if (line[0] == '#' || line[0] == '\n') continue;
    int v[10];
    if (std::sscanf(line, "%d %d %d %d %d %d %d %d %d %d", &v[0], &v[1], &v[2], &v[3], &v[4], &v[5], &v[6], &v[7],
                    &v[8], &v[9]) != 10 ||
        (v[6] != 1 && v[6] != 2 && v[6] != 4) || v[7] < 1 || v[7] > 64 || v[8] < 1 || v[8] > 256 || v[9] < 0 ||
        v[9] > 1) {
      ++bad;
      continue;
    }
    hp_plan::Tune t;
    t.synth_pt = v[6];
    t.synth_waves = v[7];
    t.tc_waves = v[8];
    t.tc_form = v[9];
    g_cache[Key(v[0], v[1], v[2], v[3], v[4], v[5])] = t;
  }
  std::fclose(fp);
  if (bad) { hp_set_error("malformed lines in the tuning cache file were skipped"); return HP_ERR_INVALID; }
  return HP_OK;
}
