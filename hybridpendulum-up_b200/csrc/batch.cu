// Batched propagation: many independent densities (each its own resident
// state, of any bandlimit and omega grid) advance together.  Members whose
// plans differ run concurrently on their own streams; members that share a
// plan (and so its workspace) run one after the other on that plan's stream.
// After one eager warm-up step (which sizes every workspace), two steps of the
// whole batch are captured into one CUDA graph and replayed: the state
// buffers ping-pong with period two for every method, so a two-step graph
// starts and ends on the same buffers.  An odd remainder runs eagerly.
#include <algorithm>
#include <cmath>
#include <vector>

#include "common.cuh"
#include "plan.hpp"

extern "C" int hp_state_step(hp_state* s, double dt, int method, int nsteps);
extern "C" int hp_state_hybrid_step(hp_state* s, hp_collision* c, double dt, int method, int nsteps);
extern "C" int hp_plan_set_stream(hp_plan* p, void* stream);

struct hp_batch {
  bool persistent = false;                  // plane passes of plain Euler members in one launch per round
  std::vector<std::vector<int>> rounds;     // members grouped so that a round has one member per plan
  // jobs per (step parity, round, precision) and their device copies
  std::vector<std::vector<PlaneJob>> jobs;
  std::vector<void*> d_jobs;
  std::vector<size_t> d_cap;
  std::vector<bool> pending_upload;         // recorded during a capture, copied after it
  int* counter = nullptr;
  int step_parity = 0;
  std::vector<hp_state*> st;
  std::vector<hp_collision*> coll;
  std::vector<hp_plan*> plans;              // distinct plans
  std::vector<int> plan_of;                 // member -> index in plans
  std::vector<cudaStream_t> streams;        // one per distinct plan
  std::vector<cudaStream_t> saved;          // the plans' own streams
  cudaStream_t origin = nullptr;
  cudaEvent_t fork = nullptr;
  std::vector<cudaEvent_t> joins;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  double dt = 0.0;
  int method = -1;
  std::vector<double2*> capF;               // each member's F at capture
  std::vector<int> capF32;                  // and its FP32-copy state: valid * 2 + current slot
  long long graph_launches = 0;
};

namespace {

#define BT_CHECK(expr)          \
  do {                          \
    int _s = (expr);            \
    if (_s != HP_OK) return _s; \
  } while (0)
#define HP_CHECK_B(expr) BT_CHECK(expr)

// slot of (parity, round, precision) in the job arrays
size_t job_slot(const hp_batch* b, int parity, size_t round, int prec) {
  return ((size_t)parity * b->rounds.size() + round) * 2 + (size_t)prec;
}

// one step of one round of members whose plane passes are collected into
// persistent launches (plain Euler members; the others step as usual)
int round_step(hp_batch* b, size_t r, double dt, int method, bool capturing) {
  for (auto s : b->streams) HP_CUDA_TRY(cudaStreamWaitEvent(s, b->fork, 0));
  std::vector<PlaneJob>* jv[2];
  for (int prec = 0; prec < 2; ++prec) {
    jv[prec] = &b->jobs[job_slot(b, b->step_parity, r, prec)];
    jv[prec]->clear();
  }
  for (int i : b->rounds[r]) {
    const bool defer = b->coll[i] == nullptr && method == HP_EULER && b->st[i]->plan->ndim == 3;
    if (defer) hp_plane_collect_begin(jv[0], jv[1]);
    const int st = b->coll[i] ? hp_state_hybrid_step(b->st[i], b->coll[i], dt, method, 1)
                              : hp_state_step(b->st[i], dt, method, 1);
    hp_plane_collect_end();
    if (st) return st;
  }
  for (size_t k = 0; k < b->streams.size(); ++k) {
    HP_CUDA_TRY(cudaEventRecord(b->joins[k], b->streams[k]));
    HP_CUDA_TRY(cudaStreamWaitEvent(b->origin, b->joins[k], 0));
  }
  for (int prec = 0; prec < 2; ++prec) {
    std::vector<PlaneJob>& jobs = *jv[prec];
    if (jobs.empty()) continue;
    hp_plane_batch_prepare(jobs);
    const size_t slot = job_slot(b, b->step_parity, r, prec);
    const size_t bytes = jobs.size() * hp_plane_job_bytes();
    if (b->d_cap[slot] < bytes) {
      if (capturing) { hp_set_error("batched plane jobs grew during a capture"); return HP_ERR_INVALID; }
      hp_dev_free(b->d_jobs[slot]);
      b->d_jobs[slot] = nullptr;
      HP_CUDA_TRY(hp_dev_alloc(&b->d_jobs[slot], bytes));
      b->d_cap[slot] = bytes;
    }
    if (capturing) {
      b->pending_upload[slot] = true;   // the graph's launch reads the array, copied once the capture ends
    } else {
      HP_CUDA_TRY(cudaMemcpyAsync(b->d_jobs[slot], jobs.data(), bytes, cudaMemcpyHostToDevice, b->origin));
      HP_CUDA_TRY(cudaStreamSynchronize(b->origin));   // the host array is rewritten by the next step
    }
    HP_CHECK_B(hp_plane_batch_launch(prec == 0 ? HP_MIXED : HP_FP64, jobs, (const PlaneJob*)b->d_jobs[slot],
                                     b->counter, b->origin));
  }
  HP_CUDA_TRY(cudaEventRecord(b->fork, b->origin));
  return HP_OK;
}

void drop_graph(hp_batch* b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
}

int use_streams(hp_batch* b, bool on) {
  for (size_t i = 0; i < b->plans.size(); ++i)
    BT_CHECK(hp_plan_set_stream(b->plans[i], on ? (void*)b->streams[i] : (void*)b->saved[i]));
  return HP_OK;
}

int member_step(hp_batch* b, size_t i, double dt, int method) {
  return b->coll[i] ? hp_state_hybrid_step(b->st[i], b->coll[i], dt, method, 1)
                    : hp_state_step(b->st[i], dt, method, 1);
}

// one step of every member, forked from `origin` and joined back into it
int batch_step(hp_batch* b, double dt, int method, bool capturing = false) {
  if (b->persistent) {
    HP_CUDA_TRY(cudaEventRecord(b->fork, b->origin));
    for (size_t r = 0; r < b->rounds.size(); ++r) BT_CHECK(round_step(b, r, dt, method, capturing));
    b->step_parity ^= 1;
    return HP_OK;
  }
  HP_CUDA_TRY(cudaEventRecord(b->fork, b->origin));
  for (auto s : b->streams) HP_CUDA_TRY(cudaStreamWaitEvent(s, b->fork, 0));
  for (size_t i = 0; i < b->st.size(); ++i) BT_CHECK(member_step(b, i, dt, method));
  for (size_t k = 0; k < b->streams.size(); ++k) {
    HP_CUDA_TRY(cudaEventRecord(b->joins[k], b->streams[k]));
    HP_CUDA_TRY(cudaStreamWaitEvent(b->origin, b->joins[k], 0));
  }
  return HP_OK;
}

// The replayed graph reads the FP32 copy the capture saw as valid: a member
// whose copy was invalidated (or whose slot moved) since must step eagerly.
int f32_tag(const hp_state* s) { return (s->f32_valid ? 2 : 0) + s->f32_cur; }

bool at_capture_buffers(const hp_batch* b) {
  for (size_t i = 0; i < b->st.size(); ++i)
    if (b->st[i]->F != b->capF[i] || f32_tag(b->st[i]) != b->capF32[i]) return false;
  return true;
}

int capture(hp_batch* b, double dt, int method) {
  b->capF.clear();
  b->capF32.clear();
  for (auto s : b->st) {
    b->capF.push_back(s->F);
    b->capF32.push_back(f32_tag(s));
  }
  std::vector<bool> fg(b->st.size());
  for (size_t i = 0; i < b->st.size(); ++i) fg[i] = b->st[i]->fg_valid;
  const int parity0 = b->step_parity;
  HP_CUDA_TRY(cudaStreamBeginCapture(b->origin, cudaStreamCaptureModeRelaxed));
  int st = batch_step(b, dt, method, true);
  if (st == HP_OK) st = batch_step(b, dt, method, true);
  cudaGraph_t g = nullptr;
  const cudaError_t e = cudaStreamEndCapture(b->origin, &g);
  if (st != HP_OK) { if (g) cudaGraphDestroy(g); return st; }
  if (e != cudaSuccess) { hp_set_error(cudaGetErrorString(e)); return HP_ERR_CUDA; }
  b->step_parity = parity0;   // capturing enqueued nothing
  // the job arrays the captured launches read: copied now, fixed while the graph lives
  for (size_t slot = 0; slot < b->pending_upload.size(); ++slot)
    if (b->pending_upload[slot]) {
      HP_CUDA_TRY(cudaMemcpy(b->d_jobs[slot], b->jobs[slot].data(), b->jobs[slot].size() * hp_plane_job_bytes(),
                             cudaMemcpyHostToDevice));
      b->pending_upload[slot] = false;
    }
  b->graph = g;
  HP_CUDA_TRY(cudaGraphInstantiate(&b->exec, g, 0));
  // capturing enqueued nothing: the buffers are back where they started
  for (size_t i = 0; i < b->st.size(); ++i) {
    if (b->st[i]->F != b->capF[i] || f32_tag(b->st[i]) != b->capF32[i]) {
      hp_set_error("state buffers do not cycle with period two");
      return HP_ERR_UNSUPPORTED;
    }
    b->st[i]->fg_valid = fg[i];
  }
  b->dt = dt;
  b->method = method;
  return HP_OK;
}

}  // namespace

extern "C" int hp_batch_create(hp_state* const* states, hp_collision* const* colls, int n, hp_batch** out) {
  if (!states || n < 1 || !out) { hp_set_error("bad argument"); return HP_ERR_INVALID; }
  *out = nullptr;
  hp_batch* b = new hp_batch();
  for (int i = 0; i < n; ++i) {
    if (!states[i]) { delete b; hp_set_error("null state"); return HP_ERR_INVALID; }
    for (int j = 0; j < i; ++j)
      if (states[j] == states[i]) { delete b; hp_set_error("a state appears twice in the batch"); return HP_ERR_INVALID; }
    b->st.push_back(states[i]);
    b->coll.push_back(colls ? colls[i] : nullptr);
    hp_plan* p = states[i]->plan;
    auto it = std::find(b->plans.begin(), b->plans.end(), p);
    if (it == b->plans.end()) {
      b->plans.push_back(p);
      b->plan_of.push_back((int)b->plans.size() - 1);
    } else {
      b->plan_of.push_back((int)(it - b->plans.begin()));
    }
  }
  auto fail = [&](cudaError_t e) {
    hp_set_error(cudaGetErrorString(e));
    for (auto s : b->streams) cudaStreamDestroy(s);
    for (auto ev : b->joins) cudaEventDestroy(ev);
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->origin) cudaStreamDestroy(b->origin);
    delete b;
    return HP_ERR_CUDA;
  };
  cudaError_t e;
  if ((e = cudaStreamCreateWithFlags(&b->origin, cudaStreamNonBlocking)) != cudaSuccess) return fail(e);
  if ((e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming)) != cudaSuccess) return fail(e);
  for (auto p : b->plans) {
    cudaStream_t s;
    cudaEvent_t ev;
    if ((e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)) != cudaSuccess) return fail(e);
    b->streams.push_back(s);
    if ((e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming)) != cudaSuccess) return fail(e);
    b->joins.push_back(ev);
    b->saved.push_back(p->stream);
  }
  *out = b;
  return HP_OK;
}

extern "C" int hp_batch_destroy(hp_batch* b) {
  if (!b) return HP_OK;
  drop_graph(b);
  for (void* d : b->d_jobs) hp_dev_free(d);
  hp_dev_free(b->counter);
  for (auto s : b->streams) cudaStreamDestroy(s);
  for (auto ev : b->joins) cudaEventDestroy(ev);
  if (b->fork) cudaEventDestroy(b->fork);
  if (b->origin) cudaStreamDestroy(b->origin);
  delete b;
  return HP_OK;
}

extern "C" int hp_batch_step(hp_batch* b, double dt, int method, int nsteps) {
  if (!b || nsteps < 0) { hp_set_error("bad argument"); return HP_ERR_INVALID; }
  if (method < HP_EULER || method > HP_RK4) { hp_set_error("bad method"); return HP_ERR_INVALID; }
  if (!std::isfinite(dt)) { hp_set_error("dt must be finite"); return HP_ERR_INVALID; }
  for (auto p : b->plans)
    if (p->prof_on) { hp_set_error("disable plan profiling before batched steps"); return HP_ERR_INVALID; }
  if (b->exec && (dt != b->dt || method != b->method)) drop_graph(b);
  BT_CHECK(use_streams(b, true));
  int st = HP_OK;
  int done = 0;
  if (!b->exec && nsteps >= 3) {
    st = batch_step(b, dt, method);   // warm-up: every workspace and table exists afterwards
    ++done;
    if (st == HP_OK) {
      const cudaError_t e = cudaStreamSynchronize(b->origin);
      if (e != cudaSuccess) { hp_set_error(cudaGetErrorString(e)); st = HP_ERR_CUDA; }
    }
    if (st == HP_OK) st = capture(b, dt, method);
  }
  if (st == HP_OK && b->exec) {
    if (!at_capture_buffers(b) && nsteps - done >= 1) {
      st = batch_step(b, dt, method);
      ++done;
    }
    while (st == HP_OK && nsteps - done >= 2 && at_capture_buffers(b)) {
      const cudaError_t e = cudaGraphLaunch(b->exec, b->origin);
      if (e != cudaSuccess) { hp_set_error(cudaGetErrorString(e)); st = HP_ERR_CUDA; break; }
      ++b->graph_launches;
      done += 2;
    }
  }
  while (st == HP_OK && done < nsteps) {
    st = batch_step(b, dt, method);
    ++done;
  }
  // the hybrid members' resident densities are valid after any full step
  if (st == HP_OK && nsteps > 0)
    for (size_t i = 0; i < b->st.size(); ++i)
      if (b->coll[i]) b->st[i]->fg_valid = true;
  const cudaError_t e = cudaStreamSynchronize(b->origin);
  const int rs = use_streams(b, false);
  if (st != HP_OK) return st;
  if (e != cudaSuccess) { hp_set_error(cudaGetErrorString(e)); return HP_ERR_CUDA; }
  // the replayed steps ran no guard checks: check every guarded member now
  if (nsteps > 0)
    for (auto s : b->st) BT_CHECK(hp_state_guard_check(s, true));
  return rs;
}

extern "C" int hp_batch_set_persistent(hp_batch* b, int enable) {
  if (!b) { hp_set_error("null argument"); return HP_ERR_INVALID; }
  drop_graph(b);
  b->persistent = enable != 0;
  if (!b->persistent) return HP_OK;
  // round r: the r-th member of every plan (members sharing a plan share its
  // workspace, so their collected plane passes cannot share a launch)
  b->rounds.clear();
  std::vector<int> seen(b->plans.size(), 0);
  for (size_t i = 0; i < b->st.size(); ++i) {
    const int r = seen[b->plan_of[i]]++;
    if ((int)b->rounds.size() <= r) b->rounds.resize(r + 1);
    b->rounds[r].push_back((int)i);
  }
  const size_t nslots = 2 * b->rounds.size() * 2;
  for (void* d : b->d_jobs) hp_dev_free(d);
  b->jobs.assign(nslots, {});
  b->d_jobs.assign(nslots, nullptr);
  b->d_cap.assign(nslots, 0);
  b->pending_upload.assign(nslots, false);
  // every slot sized for a round's members up front (a capture cannot allocate)
  for (size_t slot = 0; slot < nslots; ++slot) {
    const size_t r = (slot / 2) % b->rounds.size();
    const size_t bytes = std::max<size_t>(1, b->rounds[r].size()) * hp_plane_job_bytes();
    HP_CUDA_TRY(hp_dev_alloc(&b->d_jobs[slot], bytes));
    b->d_cap[slot] = bytes;
  }
  if (!b->counter) HP_CUDA_TRY(hp_dev_alloc(&b->counter, sizeof(int)));
  b->step_parity = 0;
  return HP_OK;
}

extern "C" int hp_batch_info(hp_batch* b, long long* graph_launches, int* concurrent_streams) {
  if (!b) { hp_set_error("null argument"); return HP_ERR_INVALID; }
  if (graph_launches) *graph_launches = b->graph_launches;
  if (concurrent_streams) *concurrent_streams = (int)b->streams.size();
  return HP_OK;
}
