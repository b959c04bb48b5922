// Many solves on one device: the batched ensemble (one CUDA graph per batch step, one branch
// per solve) and the continuous-batching server (HBM-budget admission, per-solve step graphs
// on per-solve streams, retirement at the horizon).  Neither exists in the reference, which
// runs one solve per process; both drive the same per-solve handles as sns_step, so every
// solve computes exactly what it computes alone.
#include "sns_kernels.cuh"
#include "../../include/sns_b200.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <deque>
#include <map>
#include <utility>
#include <new>
#include <string>
#include <vector>

namespace {

constexpr double kPi = 3.141592653589793238462643383279502884;

std::string cuda_msg(const char* what, cudaError_t e) { return std::string(what) + ": " + cudaGetErrorString(e); }

// Fixed step of a solve: the given dt, or the CFL step from the initial field's vmax
// (the reference's rule, ava_taylor_green_impl.hpp:1363-1368, evaluated once).
int choose_dt(sns_handle* h, int n, double dt, double cfl, double dt_max, double* out, std::string* err) {
  if (dt > 0.0) {
    *out = dt;
    return SNS_OK;
  }
  if (!(cfl > 0.0) || !(dt_max > 0.0)) {
    *err = "a CFL step needs cfl > 0 and dt_max > 0";
    return SNS_ERR_INVALID;
  }
  double vmax = 0.0;
  const int rc = sns_max_velocity(h, &vmax);
  if (rc != SNS_OK) {
    *err = sns_last_error(h);
    return rc;
  }
  const double dx = 2.0 * kPi / (double)n;
  double d = dt_max;
  if (vmax > 1.0e-14) d = std::fmin(d, cfl * dx / vmax);
  *out = d;
  return SNS_OK;
}

}  // namespace

// ---------------------------------------------------------------------------------------
// Batched ensemble.
struct sns_batch {
  std::vector<sns_handle*> h;
  std::vector<double> dt;      // fixed step, or the first CFL step of an adaptive member
  std::vector<char> adaptive;  // the member takes a CFL step from its device clock every step
  std::vector<cudaEvent_t> join;
  cudaStream_t origin = nullptr;
  cudaEvent_t fork = nullptr, ev0 = nullptr, ev1 = nullptr;
  cudaGraphExec_t exec = nullptr;
  int device = 0;
  std::string err;
};

namespace {

void batch_release(sns_batch* b) {
  if (!b) return;
  cudaSetDevice(b->device);
  if (b->origin) cudaStreamSynchronize(b->origin);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  for (cudaEvent_t e : b->join)
    if (e) cudaEventDestroy(e);
  if (b->fork) cudaEventDestroy(b->fork);
  if (b->ev0) cudaEventDestroy(b->ev0);
  if (b->ev1) cudaEventDestroy(b->ev1);
  if (b->origin) cudaStreamDestroy(b->origin);
  for (sns_handle* h : b->h)
    if (h) sns_destroy(h);
  delete b;
}

int batch_fail(sns_batch* b, int code, const std::string& msg) {
  b->err = msg;
  return code;
}

// Capture one batch step: fork from the origin stream into every solve's stream, the
// solve's step there, join back.  The graph's branches are independent, so the executor
// runs the solves' kernels concurrently.
int batch_capture(sns_batch* b) {
  cudaError_t e = cudaStreamBeginCapture(b->origin, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return batch_fail(b, SNS_ERR_CUDA, cuda_msg("cudaStreamBeginCapture", e));
  e = cudaEventRecord(b->fork, b->origin);
  for (size_t i = 0; i < b->h.size() && e == cudaSuccess; ++i) {
    cudaStream_t st = sns::handle_stream(b->h[i]);
    e = cudaStreamWaitEvent(st, b->fork, 0);
    if (e != cudaSuccess) break;
    if (b->adaptive[i]) sns::enqueue_clock_step(b->h[i]);
    else sns::enqueue_step(b->h[i], b->dt[i]);
    e = cudaEventRecord(b->join[i], st);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(b->origin, b->join[i], 0);
  }
  cudaGraph_t graph = nullptr;
  const cudaError_t e2 = cudaStreamEndCapture(b->origin, &graph);
  if (e != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    return batch_fail(b, SNS_ERR_CUDA, cuda_msg("batch capture", e));
  }
  if (e2 != cudaSuccess) return batch_fail(b, SNS_ERR_CUDA, cuda_msg("cudaStreamEndCapture", e2));
  e = cudaGraphInstantiate(&b->exec, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) return batch_fail(b, SNS_ERR_CUDA, cuda_msg("cudaGraphInstantiate", e));
  return SNS_OK;
}

int batch_finish(sns_batch* b, const char* what) {
  cudaError_t e = cudaStreamSynchronize(b->origin);
  if (e != cudaSuccess) return batch_fail(b, SNS_ERR_CUDA, cuda_msg(what, e));
  for (sns_handle* h : b->h) {
    const int rc = sns::finish_handle(h, what);
    if (rc != SNS_OK) return batch_fail(b, rc, sns::handle_error(h));
  }
  return SNS_OK;
}

}  // namespace

// ---------------------------------------------------------------------------------------
// Continuous-batching server.
//
// Steps: every solve takes the reference's adaptive CFL step (ava_taylor_green_impl.hpp:
// 1363-1378) at every step, computed on the device from the current state's vmax by the
// handle's clock, and stops exactly at its horizon; one step is one graph replay, captured
// once per handle.  After its horizon a replay leaves the state as it is.
// Memory: a solve's handle (fields, tables, stream, graph) is not freed when the solve
// retires; it joins an idle pool keyed by N and the next request of that N takes it over
// (its state re-initialised in place), so a steady stream admits and retires without
// cudaMalloc or cudaFree, which would synchronise the whole device.  The budget counts
// resident and idle handles; an idle handle of another N is freed only when a request needs
// its room and no solve of the request's N is resident (else the request waits for that
// handle, and queued requests with an idle handle start in the meantime).
// Time: a tick never waits for GPU work.  It queues a resident solve's next batch of steps
// only when at most one earlier batch is still in flight (two batches queued per solve keep
// the device busy between ticks); each batch ends with a copy of the clock to pinned host
// memory, from which the host learns the solve's time, and the solve retires once the
// batch that reached the horizon has completed.
struct sns_server {
  struct Pending {
    int64_t id;
    sns_request req;
  };
  struct Slot {  // a handle with its step graph, events and clock copies, resident or idle
    sns_handle* h = nullptr;
    cudaGraphExec_t step = nullptr;  // one adaptive step on the handle's clock
    cudaEvent_t ev[2] = {nullptr, nullptr};
    double* snap = nullptr;          // pinned: the clock after batch 0 / 1 (kClockWords each)
    size_t bytes = 0;
    int n = 0;
  };
  struct Resident {
    Slot slot;
    int64_t id = 0;
    sns_request req{};
    double t = 0.0, dt = 0.0;  // the clock as of the last completed batch
    long long steps = 0;       // steps of the completed batches
    long long launched = 0;    // steps queued so far
    int head = 0;              // next event slot to record
    int pending = 0;           // recorded batches not yet seen complete (0..2)
  };
  size_t budget = 0, used = 0, idle_bytes = 0;
  int precision = 0;
  int device = 0;
  int64_t next_id = 1;
  long long allocations = 0;  // handles created (the pool's misses)
  std::deque<Pending> queue;
  std::vector<Resident> resident;
  std::vector<Slot> idle;
  std::deque<sns_result> done;  // finished, not yet returned
  std::string err;
};

namespace {

int server_fail(sns_server* s, int code, const std::string& msg) {
  s->err = msg;
  return code;
}

void free_slot(sns_server::Slot& sl) {
  if (sl.step) cudaGraphExecDestroy(sl.step);
  for (cudaEvent_t& e : sl.ev)
    if (e) cudaEventDestroy(e);
  if (sl.snap) cudaFreeHost(sl.snap);
  if (sl.h) sns_destroy(sl.h);
  sl = sns_server::Slot{};
}

// A retired solve's handle goes to the idle pool (no device memory is released).
void retire(sns_server* s, size_t i) {
  sns_server::Resident& r = s->resident[i];
  s->used -= r.slot.bytes;
  s->idle_bytes += r.slot.bytes;
  s->idle.push_back(r.slot);
  s->resident.erase(s->resident.begin() + (long)i);
}

// Room for `bytes` more under the budget, freeing idle handles of other sizes (largest
// first) if that makes it fit; false if it does not fit even then.
bool make_room(sns_server* s, size_t bytes) {
  if (s->used + s->idle_bytes + bytes <= s->budget) return true;
  if (s->used + bytes > s->budget) return false;
  std::sort(s->idle.begin(), s->idle.end(),
            [](const sns_server::Slot& a, const sns_server::Slot& b) { return a.bytes < b.bytes; });
  while (!s->idle.empty() && s->used + s->idle_bytes + bytes > s->budget) {
    s->idle_bytes -= s->idle.back().bytes;
    free_slot(s->idle.back());
    s->idle.pop_back();
  }
  return s->used + s->idle_bytes + bytes <= s->budget;
}

// A new handle of size n with its step graph, events and pinned clock copies.
int make_slot(sns_server* s, const sns_request& q, size_t bytes, sns_server::Slot* out, std::string* err) {
  sns_server::Slot sl;
  int rc = sns_create(q.n, q.nu, s->precision, SNS_VISCOUS_EXPLICIT, q.seed, q.pert_amp, q.pert_kmax, &sl.h);
  if (rc != SNS_OK) {
    *err = sns_last_error(nullptr);
    return rc;
  }
  sl.bytes = bytes;
  sl.n = q.n;
  cudaError_t e = cudaEventCreateWithFlags(&sl.ev[0], cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sl.ev[1], cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaHostAlloc((void**)&sl.snap, 2 * sns::kClockWords * sizeof(double), cudaHostAllocDefault);
  if (e != cudaSuccess) {
    *err = cuda_msg("server slot", e);
    free_slot(sl);
    return SNS_ERR_CUDA;
  }
  // the graph: one adaptive step on the handle's clock (its step size is read on the device)
  cudaStream_t st = sns::handle_stream(sl.h);
  cudaGraph_t graph = nullptr;
  e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    sns::enqueue_clock_step(sl.h);
    e = cudaStreamEndCapture(st, &graph);
  }
  if (e == cudaSuccess) e = cudaGraphInstantiate(&sl.step, graph, 0);
  if (graph) cudaGraphDestroy(graph);
  if (e != cudaSuccess) {
    *err = cuda_msg("server step graph", e);
    free_slot(sl);
    return SNS_ERR_CUDA;
  }
  *out = sl;
  return SNS_OK;
}

// Start request p on an idle handle of its N (re-initialised in place, no allocation) or on
// a new handle `fresh`; false with the error set if the handle cannot take it.
int start_request(sns_server* s, const sns_server::Pending& p, sns_server::Slot slot, bool fresh) {
  sns_server::Resident r;
  r.id = p.id;
  r.req = p.req;
  r.slot = slot;
  int rc = SNS_OK;
  std::string err;
  if (!fresh) {
    rc = sns::reset_handle(r.slot.h, p.req.nu, p.req.seed, p.req.pert_amp, p.req.pert_kmax);
    if (rc != SNS_OK) err = sns_last_error(r.slot.h);
  }
  if (rc == SNS_OK) {
    rc = sns_set_clock(r.slot.h, 0.0, p.req.t_end, p.req.cfl, p.req.dt_max);
    if (rc != SNS_OK) err = sns_last_error(r.slot.h);
  }
  if (rc != SNS_OK) {
    free_slot(r.slot);
    return server_fail(s, rc, "request " + std::to_string(p.id) + ": " + err);
  }
  s->used += r.slot.bytes;
  s->resident.push_back(r);
  return SNS_OK;
}

// The idle handle of size n, taken out of the pool (false if there is none).
bool take_idle(sns_server* s, int n, sns_server::Slot* out) {
  for (size_t k = 0; k < s->idle.size(); ++k)
    if (s->idle[k].n == n) {
      *out = s->idle[k];
      s->idle.erase(s->idle.begin() + (long)k);
      s->idle_bytes -= out->bytes;
      return true;
    }
  return false;
}

// Queued requests behind a waiting head that may start on an idle handle meanwhile.
constexpr size_t kLookahead = 64;

// Admit queued requests in arrival order while their device bytes fit the budget.  The head
// request takes an idle handle of its N, else unused budget, else -- when no solve of its N
// is resident -- the room of idle handles of other sizes (freed).  When a solve of its N is
// resident, the head waits for that handle instead of freeing and allocating (cudaFree and
// cudaMalloc synchronise the device), and requests behind it whose N has an idle handle
// start meanwhile, so the pool's memory keeps working.
int admit(sns_server* s) {
  while (!s->queue.empty()) {
    const sns_server::Pending p = s->queue.front();
    const size_t bytes = sns_bytes_required(p.req.n, s->precision);
    if (bytes == 0) {
      s->queue.pop_front();
      return server_fail(s, SNS_ERR_UNSUPPORTED, "request " + std::to_string(p.id) + ": unsupported grid size");
    }
    if (bytes > s->budget)
      return server_fail(s, SNS_ERR_NOMEM, "request " + std::to_string(p.id) + " needs " + std::to_string(bytes) +
                                               " bytes, more than the whole HBM budget");
    sns_server::Slot slot;
    if (take_idle(s, p.req.n, &slot)) {
      s->queue.pop_front();
      const int rc = start_request(s, p, slot, false);
      if (rc != SNS_OK) return rc;
      continue;
    }
    const bool unused_room = s->used + s->idle_bytes + bytes <= s->budget;
    bool same_n_resident = false;
    for (const sns_server::Resident& r : s->resident) same_n_resident = same_n_resident || r.req.n == p.req.n;
    if (!unused_room && same_n_resident) {
      // the head waits for a handle of its N; later requests with an idle handle start now
      for (size_t q = 1; q < s->queue.size() && q <= kLookahead && !s->idle.empty();) {
        const sns_server::Pending pq = s->queue[q];
        if (take_idle(s, pq.req.n, &slot)) {
          s->queue.erase(s->queue.begin() + (long)q);
          const int rc = start_request(s, pq, slot, false);
          if (rc != SNS_OK) return rc;
        } else {
          ++q;
        }
      }
      return SNS_OK;
    }
    if (!make_room(s, bytes)) return SNS_OK;  // waits until retirements free memory
    std::string err;
    const int rc = make_slot(s, p.req, bytes, &slot, &err);
    if (rc == SNS_ERR_NOMEM && !s->resident.empty()) return SNS_OK;  // the device itself is full: wait
    if (rc != SNS_OK) {
      s->queue.pop_front();
      return server_fail(s, rc, "request " + std::to_string(p.id) + ": " + err);
    }
    ++s->allocations;
    s->queue.pop_front();
    const int rc2 = start_request(s, p, slot, true);
    if (rc2 != SNS_OK) return rc2;
  }
  return SNS_OK;
}

// Take in the batches of the resident that have completed: `pending` drops and the host
// copy of the clock advances to the latest completed batch's.
int poll(sns_server* s, sns_server::Resident& r) {
  while (r.pending > 0) {
    const int idx = (r.head + 2 - r.pending) & 1;
    const cudaError_t e = cudaEventQuery(r.slot.ev[idx]);
    if (e == cudaErrorNotReady) return SNS_OK;
    if (e != cudaSuccess) return server_fail(s, SNS_ERR_CUDA, cuda_msg("cudaEventQuery", e));
    const double* c = r.slot.snap + idx * sns::kClockWords;
    r.t = c[sns::kClockT];
    if (c[sns::kClockDt] > 0.0) r.dt = c[sns::kClockDt];
    r.steps = (long long)c[sns::kClockSteps];
    --r.pending;
  }
  return SNS_OK;
}

bool reached(const sns_server::Resident& r) { return !(r.t < r.req.t_end - 1.0e-14); }

}  // namespace

extern "C" {

int sns_batch_create(const sns_solve_spec* specs, int count, int autotune_trials, const char* autotune_cache,
                     sns_batch** out, double* out_dt) {
  if (out == nullptr) return SNS_ERR_INVALID;
  *out = nullptr;
  if (specs == nullptr || count <= 0) {
    sns::set_handleless_error("sns_batch_create: need at least one solve spec");
    return SNS_ERR_INVALID;
  }
  sns_batch* b = new (std::nothrow) sns_batch();
  if (b == nullptr) return SNS_ERR_NOMEM;
  cudaGetDevice(&b->device);
  b->h.assign(count, nullptr);
  b->dt.assign(count, 0.0);
  b->adaptive.assign(count, 0);
  b->join.assign(count, nullptr);
  for (int i = 0; i < count; ++i) {
    const sns_solve_spec& sp = specs[i];
    int rc = sns_create(sp.n, sp.nu, sp.precision, sp.viscous_mode, sp.seed, sp.pert_amp, sp.pert_kmax, &b->h[i]);
    if (rc != SNS_OK) {
      sns::set_handleless_error(("sns_batch_create: solve " + std::to_string(i) + ": " + sns_last_error(nullptr)).c_str());
      batch_release(b);
      return rc;
    }
    std::string err;
    rc = choose_dt(b->h[i], sp.n, sp.dt, sp.cfl, sp.dt_max, &b->dt[i], &err);
    if (rc == SNS_OK && !(sp.dt > 0.0)) {
      // the reference's adaptive rule every step, on the device: no horizon
      b->adaptive[i] = 1;
      rc = sns_set_clock(b->h[i], 0.0, INFINITY, sp.cfl, sp.dt_max);
      if (rc != SNS_OK) err = sns_last_error(b->h[i]);
    }
    if (rc != SNS_OK) {
      sns::set_handleless_error(("sns_batch_create: solve " + std::to_string(i) + ": " + err).c_str());
      batch_release(b);
      return rc;
    }
    if (out_dt) out_dt[i] = b->dt[i];
  }
  if (autotune_trials > 0) {
    // one launch-shape search per distinct (N, precision), on a scratch handle so the
    // batch's own states are untouched by the trial steps; every member then runs it
    std::map<std::pair<int, int>, std::array<int, 3>> shapes;
    for (int i = 0; i < count; ++i) {
      const auto key = std::make_pair(specs[i].n, specs[i].precision);
      auto it = shapes.find(key);
      if (it == shapes.end()) {
        sns_handle* scratch = nullptr;
        int rc = sns_create(specs[i].n, specs[i].nu, specs[i].precision, specs[i].viscous_mode, 0, 0.0, 0, &scratch);
        std::array<int, 3> cfg{};
        if (rc == SNS_OK) {
          rc = sns_autotune(scratch, autotune_trials, autotune_cache, cfg.data());
          if (rc != SNS_OK) sns::set_handleless_error(sns_last_error(scratch));
          sns_destroy(scratch);
        }
        if (rc != SNS_OK) {
          batch_release(b);
          return rc;
        }
        it = shapes.emplace(key, cfg).first;
      }
      sns::set_launch_shape(b->h[i], it->second.data());
    }
  }
  cudaError_t e = cudaStreamCreateWithFlags(&b->origin, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
  for (int i = 0; i < count && e == cudaSuccess; ++i) e = cudaEventCreateWithFlags(&b->join[i], cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreate(&b->ev0);
  if (e == cudaSuccess) e = cudaEventCreate(&b->ev1);
  if (e != cudaSuccess) {
    sns::set_handleless_error(cuda_msg("sns_batch_create", e).c_str());
    batch_release(b);
    return SNS_ERR_CUDA;
  }
  const int rc = batch_capture(b);
  if (rc != SNS_OK) {
    sns::set_handleless_error(("sns_batch_create: " + b->err).c_str());
    batch_release(b);
    return rc;
  }
  *out = b;
  return SNS_OK;
}

int sns_batch_destroy(sns_batch* b) {
  if (b == nullptr) return SNS_ERR_INVALID;
  batch_release(b);
  return SNS_OK;
}

int sns_batch_step(sns_batch* b, int nsteps) {
  if (b == nullptr) return SNS_ERR_INVALID;
  if (nsteps < 0) return batch_fail(b, SNS_ERR_INVALID, "negative step count");
  cudaSetDevice(b->device);
  for (int k = 0; k < nsteps; ++k) {
    const cudaError_t e = cudaGraphLaunch(b->exec, b->origin);
    if (e != cudaSuccess) return batch_fail(b, SNS_ERR_CUDA, cuda_msg("cudaGraphLaunch", e));
  }
  return batch_finish(b, "sns_batch_step");
}

int sns_batch_time_steps(sns_batch* b, int nsteps, double* elapsed_ms) {
  if (b == nullptr) return SNS_ERR_INVALID;
  if (nsteps < 0 || elapsed_ms == nullptr) return batch_fail(b, SNS_ERR_INVALID, "invalid argument");
  cudaSetDevice(b->device);
  cudaError_t e = cudaEventRecord(b->ev0, b->origin);
  for (int k = 0; k < nsteps && e == cudaSuccess; ++k) e = cudaGraphLaunch(b->exec, b->origin);
  if (e == cudaSuccess) e = cudaEventRecord(b->ev1, b->origin);
  if (e != cudaSuccess) return batch_fail(b, SNS_ERR_CUDA, cuda_msg("sns_batch_time_steps", e));
  const int rc = batch_finish(b, "sns_batch_time_steps");
  if (rc != SNS_OK) return rc;
  float ms = 0.f;
  e = cudaEventElapsedTime(&ms, b->ev0, b->ev1);
  if (e != cudaSuccess) return batch_fail(b, SNS_ERR_CUDA, cuda_msg("cudaEventElapsedTime", e));
  *elapsed_ms = ms;
  return SNS_OK;
}

sns_handle* sns_batch_handle(sns_batch* b, int i) {
  if (b == nullptr || i < 0 || i >= (int)b->h.size()) return nullptr;
  return b->h[i];
}

int sns_batch_size(const sns_batch* b) { return b ? (int)b->h.size() : 0; }

const char* sns_batch_last_error(const sns_batch* b) { return b ? b->err.c_str() : ""; }

int sns_server_create(size_t hbm_budget_bytes, int precision, sns_server** out) {
  if (out == nullptr) return SNS_ERR_INVALID;
  *out = nullptr;
  if (hbm_budget_bytes == 0 || sns_bytes_required(64, precision) == 0) {
    sns::set_handleless_error("sns_server_create: need a positive budget and a known precision");
    return SNS_ERR_INVALID;
  }
  sns_server* s = new (std::nothrow) sns_server();
  if (s == nullptr) return SNS_ERR_NOMEM;
  s->budget = hbm_budget_bytes;
  s->precision = precision;
  cudaGetDevice(&s->device);
  *out = s;
  return SNS_OK;
}

int sns_server_destroy(sns_server* s) {
  if (s == nullptr) return SNS_ERR_INVALID;
  cudaSetDevice(s->device);
  while (!s->resident.empty()) {
    sns_server::Resident& r = s->resident.back();
    cudaStreamSynchronize(sns::handle_stream(r.slot.h));
    free_slot(r.slot);
    s->resident.pop_back();
  }
  for (sns_server::Slot& sl : s->idle) free_slot(sl);
  delete s;
  return SNS_OK;
}

int sns_server_submit(sns_server* s, const sns_request* r, int64_t* out_id) {
  if (s == nullptr) return SNS_ERR_INVALID;
  if (r == nullptr || !(r->t_end > 0.0) || !(r->nu >= 0.0) || r->n <= 0)
    return server_fail(s, SNS_ERR_INVALID, "request needs n > 0, nu >= 0 and t_end > 0");
  if (sns_bytes_required(r->n, s->precision) == 0) return server_fail(s, SNS_ERR_UNSUPPORTED, "unsupported request");
  const int64_t id = s->next_id++;
  s->queue.push_back({id, *r});
  if (out_id) *out_id = id;
  return SNS_OK;
}

int sns_server_step(sns_server* s, sns_result* done, int max_done, int* ndone, int* resident, int* queued,
                    size_t* bytes_in_use) {
  if (s == nullptr) return SNS_ERR_INVALID;
  if (ndone) *ndone = 0;
  cudaSetDevice(s->device);
  int rc = admit(s);
  if (rc != SNS_OK) return rc;
  // Every resident solve with room in its two-batch window gets its next batch of steps on
  // its own stream: the largest by one step and smaller ones by proportionally more
  // (N_max^3 / N^3 steps, at most kMaxTickSteps), so a small solve is not held to the pace
  // of the largest; no more than the steps its horizon still needs at the last known step
  // size (a step past the horizon is a no-op replay).
  constexpr double kMaxTickSteps = 64.0;
  double wmax = 0.0;
  for (const sns_server::Resident& r : s->resident) wmax = std::fmax(wmax, std::pow((double)r.req.n, 3.0));
  for (sns_server::Resident& r : s->resident) {
    rc = poll(s, r);
    if (rc != SNS_OK) return rc;
    if (r.pending >= 2 || reached(r)) continue;
    long long k = (long long)std::fmin(kMaxTickSteps, std::fmax(1.0, std::floor(wmax / std::pow((double)r.req.n, 3.0))));
    if (r.dt > 0.0) {
      const long long need = (long long)std::ceil((r.req.t_end - r.t) / r.dt) + 1;
      k = std::min(k, need - (r.launched - r.steps));
    }
    if (k <= 0) continue;
    cudaStream_t st = sns::handle_stream(r.slot.h);
    for (long long j = 0; j < k; ++j) {
      const cudaError_t e = cudaGraphLaunch(r.slot.step, st);
      if (e != cudaSuccess) return server_fail(s, SNS_ERR_CUDA, cuda_msg("cudaGraphLaunch", e));
    }
    r.launched += k;
    double* snap = r.slot.snap + r.head * sns::kClockWords;
    cudaError_t e = cudaMemcpyAsync(snap, sns::handle_clock(r.slot.h), sns::kClockWords * sizeof(double),
                                    cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaEventRecord(r.slot.ev[r.head], st);
    if (e != cudaSuccess) return server_fail(s, SNS_ERR_CUDA, cuda_msg("server batch", e));
    r.head ^= 1;
    ++r.pending;
  }
  // retire the solves whose horizon a completed batch reached
  for (size_t i = s->resident.size(); i-- > 0;) {
    sns_server::Resident& r = s->resident[i];
    rc = poll(s, r);
    if (rc != SNS_OK) return rc;
    if (!reached(r) || r.pending > 0) continue;
    rc = sns::finish_handle(r.slot.h, "sns_server_step");  // the device error word
    if (rc != SNS_OK) return server_fail(s, rc, sns::handle_error(r.slot.h));
    sns_result res{};
    res.id = r.id;
    res.n = r.req.n;
    res.steps = (int)r.steps;
    res.dt = r.steps > 0 ? r.req.t_end / (double)r.steps : 0.0;
    rc = sns_diagnostics(r.slot.h, r.req.t_end, &res.final);
    if (rc != SNS_OK) return server_fail(s, rc, sns_last_error(r.slot.h));
    s->done.push_back(res);
    retire(s, i);
  }
  int nd = 0;
  while (!s->done.empty() && nd < max_done && done != nullptr) {
    done[nd++] = s->done.front();
    s->done.pop_front();
  }
  if (ndone) *ndone = nd;
  if (resident) *resident = (int)s->resident.size();
  if (queued) *queued = (int)s->queue.size();
  if (bytes_in_use) *bytes_in_use = s->used;
  return SNS_OK;
}

int sns_server_stats(const sns_server* s, size_t* idle_bytes, long long* handles_created) {
  if (s == nullptr) return SNS_ERR_INVALID;
  if (idle_bytes) *idle_bytes = s->idle_bytes;
  if (handles_created) *handles_created = s->allocations;
  return SNS_OK;
}

const char* sns_server_last_error(const sns_server* s) { return s ? s->err.c_str() : ""; }

}  // extern "C"
