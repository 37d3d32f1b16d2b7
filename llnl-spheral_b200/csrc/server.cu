// Continuous-batching request loop: simulations arrive, are admitted by
// device-memory footprint, advance together one batched RK2 step per tick
// with their state resident on the device, and retire when done.
//
// No counterpart in the reference, which runs one problem per process.
// Admission is first-come first-served: the head of the queue is admitted
// when its footprint fits under the budget beside the running simulations
// (and the member cap); a request larger than the whole budget fails with
// SPHGPU_ERR_ADMISSION.  A running simulation's footprint is its estimate
// until its first step, then the bytes its buffers actually hold.  Every
// tick is one call of the batched step over all running simulations, so a
// simulation's results are those it gives alone.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <deque>
#include <map>
#include <new>
#include <string>
#include <vector>

#include "problem.cuh"

namespace sphgpu {
namespace {

enum RequestState { REQ_QUEUED = 0, REQ_RUNNING = 1, REQ_DONE = 2, REQ_FAILED = 3, REQ_CANCELLED = 4 };

struct Request {
  sphgpu_config cfg{};
  int64_t n = 0;
  int64_t nsteps = 0;
  int64_t stepsDone = 0;
  int64_t pairs = 0;            // pair interactions evaluated (one evaluation per step)
  int state = REQ_QUEUED;
  int64_t footprint = 0;        // device bytes charged against the budget
  bool measured = false;        // footprint measured (after the first step)
  std::vector<double> pos, vel, mass, rho, eps, H;   // initial, then final state
  double time = 0.0;
  sphgpu_problem* prob = nullptr;
  std::string error;
};

// Kernel extents of the TableKernels (BSplineKernel, WendlandC4Kernel).
double kernel_extent(int kernel) { return kernel == SPHGPU_KERNEL_BSPLINE ? 2.0 : 1.0; }

// Footprint estimate before allocation: ghosts from the periodic layers of
// width kappa*hmax, neighbors from the node density inside kappa*hmax, cells
// of side kappa*hmax over the box with its ghost layers.  The problem's first
// neighbor build is planned from these sizes (Problem::hint*), so the bytes
// it holds after that build are exactly planned_bytes of them, unless a size
// turns out larger than estimated and the build grows its buffers.
struct Estimate {
  int64_t G = 0, E = 0, cells = 0, bytes = 0;
};

Estimate estimate_sizes(const sphgpu_config& c, int64_t n, const double* pos, const double* H) {
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  double hmax = 0.0;
  for (int64_t i = 0; i < n; ++i) {
    for (int a = 0; a < 3; ++a) {
      lo[a] = std::min(lo[a], pos[3*i + a]);
      hi[a] = std::max(hi[a], pos[3*i + a]);
    }
    const double* h = &H[6*i];
    const double hmin = std::min(h[0], std::min(h[3], h[5]));
    if (hmin > 0.0) hmax = std::max(hmax, 1.0/hmin);
  }
  const double reach = kernel_extent(c.kernel)*hmax;
  // cells of half a kernel reach (the finest subdivision the neighbor walk uses)
  const double cell = reach*1.001/2.0;
  double vol = 1.0, ext = 1.0, cells = 1.0;
  for (int a = 0; a < 3; ++a) {
    const double L = c.periodic[a] ? c.xmax[a] - c.xmin[a] : std::max(hi[a] - lo[a], reach);
    vol *= L;
    ext *= c.periodic[a] ? (L + 2.0*reach)/L : 1.0;
    cells *= std::floor((c.periodic[a] ? L + 2.0*reach : L)/cell) + 1.0;   // the grid's cells per axis
  }
  Estimate e;
  e.G = (int64_t)(1.1*(double)n*(ext - 1.0)) + 64;
  const double density = (double)n/vol;
  const double nbrs = 1.3*density*(4.0/3.0)*3.14159265358979323846*reach*reach*reach + 8.0;
  e.E = (int64_t)(nbrs*(double)n);
  e.cells = (int64_t)(1.1*cells) + 64;
  e.bytes = planned_bytes(c, n, e.G, e.E, e.cells);
  return e;
}

Estimate estimate_sizes(const Request& r) { return estimate_sizes(r.cfg, r.n, r.pos.data(), r.H.data()); }

}  // namespace
}  // namespace sphgpu

using namespace sphgpu;

struct sphgpu_server {
  int64_t budget = 0;
  int32_t maxMembers = 0;
  int64_t nextId = 1;
  std::deque<int64_t> queue;
  std::map<int64_t, Request> reqs;
  std::vector<int64_t> running;       // admission order
  std::vector<int64_t> finished;      // not yet reported by sphgpu_server_finished
  Batch batch;
  bool deviceReady = false;           // stream and batch set up (first tick)
  int64_t inUse = 0, peak = 0;
  int64_t pairsTotal = 0, ticks = 0, completed = 0, steps = 0;
};

namespace {

void release(sphgpu_server& s, Request& r) {
  if (r.prob) {
    sphgpu_destroy(r.prob);
    r.prob = nullptr;
  }
  s.inUse -= r.footprint;
  r.footprint = 0;
}

// The server's stream and batch descriptors, made on the first tick: queue
// management (submit, cancel, status) needs no device.
int server_device(sphgpu_server& s) {
  if (s.deviceReady) return SPHGPU_OK;
  cudaStream_t st = nullptr;
  int rc = cuda_status(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "server stream");
  if (rc != SPHGPU_OK) return rc;
  rc = batch_init(s.batch, st);
  s.batch.ownStream = true;
  if (rc != SPHGPU_OK) {
    batch_free(s.batch);
    return rc;
  }
  s.deviceReady = true;
  return SPHGPU_OK;
}

int admit(sphgpu_server& s, int64_t id, const Estimate& est) {
  Request& r = s.reqs[id];
  int rc = sphgpu_create(&r.cfg, r.n, &r.prob);
  if (rc == SPHGPU_OK) {
    r.prob->hintG = est.G;
    r.prob->hintE = est.E;
    r.prob->hintCells = est.cells;
    rc = sphgpu_set_state(r.prob, r.pos.data(), r.vel.data(), r.mass.data(), r.rho.data(), r.eps.data(), r.H.data());
  }
  if (rc != SPHGPU_OK) {
    r.error = sphgpu_last_error();
    release(s, r);
    r.state = REQ_FAILED;
    s.finished.push_back(id);
    return rc;
  }
  r.state = REQ_RUNNING;
  s.running.push_back(id);
  return SPHGPU_OK;
}

}  // namespace

extern "C" {

int sphgpu_estimate_footprint(const sphgpu_config* cfg, int64_t n, const double* position, const double* H,
                              int64_t* bytes) {
  if (cfg == nullptr || n <= 0 || position == nullptr || H == nullptr || bytes == nullptr) {
    set_error("sphgpu_estimate_footprint: bad arguments");
    return SPHGPU_ERR_ARG;
  }
  *bytes = estimate_sizes(*cfg, n, position, H).bytes;
  return SPHGPU_OK;
}

int sphgpu_server_create(double hbm_budget_bytes, int32_t max_members, sphgpu_server** out) {
  if (out == nullptr || !(hbm_budget_bytes > 0.0) || max_members <= 0) {
    set_error("sphgpu_server_create: bad arguments");
    return SPHGPU_ERR_ARG;
  }
  *out = nullptr;
  sphgpu_server* s = new (std::nothrow) sphgpu_server();
  if (s == nullptr) { set_error("host allocation failed"); return SPHGPU_ERR_NOMEM; }
  s->budget = (int64_t)hbm_budget_bytes;
  s->maxMembers = max_members;
  *out = s;
  return SPHGPU_OK;
}

void sphgpu_server_destroy(sphgpu_server* s) {
  if (s == nullptr) return;
  for (auto& kv : s->reqs) if (kv.second.prob) sphgpu_destroy(kv.second.prob);
  if (s->deviceReady) batch_free(s->batch);
  delete s;
}

int sphgpu_server_submit(sphgpu_server* s, const sphgpu_config* cfg, int64_t n, const double* position,
                         const double* velocity, const double* mass, const double* massDensity,
                         const double* specificThermalEnergy, const double* H, int64_t nsteps, int64_t* id) {
  if (s == nullptr || cfg == nullptr || id == nullptr || n <= 0 || nsteps < 0 || position == nullptr ||
      velocity == nullptr || mass == nullptr || massDensity == nullptr || specificThermalEnergy == nullptr ||
      H == nullptr) {
    set_error("sphgpu_server_submit: bad arguments");
    return SPHGPU_ERR_ARG;
  }
  const int64_t rid = s->nextId++;
  Request& r = s->reqs[rid];
  r.cfg = *cfg;
  r.n = n;
  r.nsteps = nsteps;
  r.pos.assign(position, position + 3*n);
  r.vel.assign(velocity, velocity + 3*n);
  r.mass.assign(mass, mass + n);
  r.rho.assign(massDensity, massDensity + n);
  r.eps.assign(specificThermalEnergy, specificThermalEnergy + n);
  r.H.assign(H, H + 6*n);
  s->queue.push_back(rid);
  *id = rid;
  return SPHGPU_OK;
}

int sphgpu_server_tick(sphgpu_server* s, int32_t* running, int32_t* queued) {
  if (s == nullptr) return SPHGPU_ERR_ARG;
  SPH_TRY(server_device(*s));
  // ---- admission, first come first served
  while (!s->queue.empty() && (int32_t)s->running.size() < s->maxMembers) {
    const int64_t id = s->queue.front();
    Request& r = s->reqs[id];
    const Estimate est = estimate_sizes(r);
    const int64_t need = est.bytes;
    if (need > s->budget) {
      s->queue.pop_front();
      r.state = REQ_FAILED;
      r.error = "request footprint exceeds the server's device-memory budget";
      s->finished.push_back(id);
      continue;
    }
    if (s->inUse + need > s->budget) break;
    s->queue.pop_front();
    r.footprint = need;
    s->inUse += need;
    admit(*s, id, est);
  }
  s->peak = std::max(s->peak, s->inUse);
  // ---- one batched RK2 step of every running simulation
  if (!s->running.empty()) {
    s->batch.mem.clear();
    std::vector<int64_t> stepping;
    for (int64_t id : s->running) {
      Request& r = s->reqs[id];
      if (r.stepsDone < r.nsteps) {
        s->batch.mem.push_back(r.prob);
        stepping.push_back(id);
      }
    }
    if (!s->batch.mem.empty()) {
      const int rc = batch_step_rk2(s->batch);
      if (rc != SPHGPU_OK) return rc;
      s->ticks += 1;
    }
    for (int64_t id : stepping) {
      Request& r = s->reqs[id];
      r.stepsDone += 1;
      r.pairs += r.prob->pairs;
      s->pairsTotal += r.prob->pairs;
      s->steps += 1;
      if (!r.measured) {
        // charge what the buffers hold now instead of the estimate
        const int64_t actual = problem_bytes(*r.prob);
        s->inUse += actual - r.footprint;
        r.footprint = actual;
        r.measured = true;
      }
    }
    s->peak = std::max(s->peak, s->inUse);
    // ---- retire finished simulations: final state to the host, memory freed
    std::vector<int64_t> still;
    for (int64_t id : s->running) {
      Request& r = s->reqs[id];
      if (r.stepsDone < r.nsteps) { still.push_back(id); continue; }
      int rc = sphgpu_get_state(r.prob, r.pos.data(), r.vel.data(), r.mass.data(), r.rho.data(), r.eps.data(),
                                r.H.data());
      double lastDt = 0.0;
      if (rc == SPHGPU_OK) rc = sphgpu_time(r.prob, &r.time, &lastDt);
      r.state = rc == SPHGPU_OK ? REQ_DONE : REQ_FAILED;
      if (rc != SPHGPU_OK) r.error = sphgpu_last_error();
      release(*s, r);
      s->finished.push_back(id);
      s->completed += 1;
    }
    s->running.swap(still);
  }
  if (running) *running = (int32_t)s->running.size();
  if (queued) *queued = (int32_t)s->queue.size();
  return SPHGPU_OK;
}

int sphgpu_server_cancel(sphgpu_server* s, int64_t id) {
  if (s == nullptr) return SPHGPU_ERR_ARG;
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) { set_error("sphgpu_server_cancel: unknown request"); return SPHGPU_ERR_ARG; }
  Request& r = it->second;
  if (r.state == REQ_QUEUED) {
    s->queue.erase(std::find(s->queue.begin(), s->queue.end(), id));
  } else if (r.state == REQ_RUNNING) {
    // Between ticks no kernel of the request is in flight on the server's
    // stream once it is drained; its buffers go back to the pool.
    if (s->deviceReady) SPH_CHECK(cudaStreamSynchronize(s->batch.stream));
    release(*s, r);
    s->running.erase(std::find(s->running.begin(), s->running.end(), id));
  } else {
    set_error("sphgpu_server_cancel: request already finished");
    return SPHGPU_ERR_STATE;
  }
  r.state = REQ_CANCELLED;
  r.error = "request cancelled";
  r.pos.clear(); r.vel.clear(); r.mass.clear(); r.rho.clear(); r.eps.clear(); r.H.clear();
  s->finished.push_back(id);
  return SPHGPU_OK;
}

int sphgpu_server_finished(sphgpu_server* s, int64_t* ids, int32_t capacity, int32_t* count) {
  if (s == nullptr || count == nullptr || (capacity > 0 && ids == nullptr)) return SPHGPU_ERR_ARG;
  const int32_t k = std::min<int32_t>(capacity, (int32_t)s->finished.size());
  for (int32_t t = 0; t < k; ++t) ids[t] = s->finished[t];
  s->finished.erase(s->finished.begin(), s->finished.begin() + k);
  *count = k;
  return SPHGPU_OK;
}

int sphgpu_server_status(sphgpu_server* s, int64_t id, int32_t* state, int64_t* steps_done, int64_t* pairs) {
  if (s == nullptr) return SPHGPU_ERR_ARG;
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) { set_error("sphgpu_server_status: unknown request"); return SPHGPU_ERR_ARG; }
  if (state) *state = it->second.state;
  if (steps_done) *steps_done = it->second.stepsDone;
  if (pairs) *pairs = it->second.pairs;
  if (it->second.state == REQ_FAILED || it->second.state == REQ_CANCELLED) set_error(it->second.error);
  return SPHGPU_OK;
}

int sphgpu_server_fetch(sphgpu_server* s, int64_t id, double* position, double* velocity, double* mass,
                        double* massDensity, double* specificThermalEnergy, double* H, double* time) {
  if (s == nullptr) return SPHGPU_ERR_ARG;
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) { set_error("sphgpu_server_fetch: unknown request"); return SPHGPU_ERR_ARG; }
  Request& r = it->second;
  if (r.state == REQ_FAILED || r.state == REQ_CANCELLED) {
    set_error(r.error);
    s->reqs.erase(it);
    return SPHGPU_ERR_STATE;
  }
  if (r.state != REQ_DONE) { set_error("sphgpu_server_fetch: request not finished"); return SPHGPU_ERR_STATE; }
  const int64_t n = r.n;
  if (position) std::memcpy(position, r.pos.data(), sizeof(double)*3*n);
  if (velocity) std::memcpy(velocity, r.vel.data(), sizeof(double)*3*n);
  if (mass) std::memcpy(mass, r.mass.data(), sizeof(double)*n);
  if (massDensity) std::memcpy(massDensity, r.rho.data(), sizeof(double)*n);
  if (specificThermalEnergy) std::memcpy(specificThermalEnergy, r.eps.data(), sizeof(double)*n);
  if (H) std::memcpy(H, r.H.data(), sizeof(double)*6*n);
  if (time) *time = r.time;
  s->reqs.erase(it);
  return SPHGPU_OK;
}

int sphgpu_server_stats(sphgpu_server* s, double out[8]) {
  if (s == nullptr || out == nullptr) return SPHGPU_ERR_ARG;
  out[0] = (double)s->inUse;
  out[1] = (double)s->peak;
  out[2] = (double)s->budget;
  out[3] = (double)s->pairsTotal;
  out[4] = (double)s->ticks;
  out[5] = (double)s->completed;
  out[6] = (double)s->steps;
  out[7] = (double)s->batch.launches;
  return SPHGPU_OK;
}

}  // extern "C"
