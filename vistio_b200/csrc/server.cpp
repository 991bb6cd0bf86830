// Serving layer: continuous batching of drape requests over the C ABI
// (include/vistio_cuda.h). The reference has no counterpart (its runner,
// crates/vistio-bench/src/runner.rs, simulates one scenario at a time).
//
// Request life: submit copies the request's host data and queues it for a
// set-up thread; the thread builds (or clones from the cache) the garment's
// solver; each tick packs ready requests that share a step configuration into
// a new cohort (one vistio_batch on its own context and stream) while the
// device-memory budget allows, queues step slices of every running cohort
// (two slices in flight each, so a stream never idles on the host), and
// retires cohorts whose last slice finished: their states are read back, the
// requests marked done and the batch freed in the order of its own stream
// (no device-wide synchronisation, so other cohorts keep running).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <list>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/vistio_cuda.h"

namespace {

using Clock = std::chrono::steady_clock;

static_assert(sizeof(vistio_solver_config) % 8 == 0, "hashed as bytes: no tail padding");

struct Fnv {
  uint64_t h = 1469598103934665603ull;
  void add(const void* p, size_t n) {
    const unsigned char* b = static_cast<const unsigned char*>(p);
    for (size_t i = 0; i < n; ++i) h = (h ^ b[i]) * 1099511628211ull;
  }
  template <class T> void add_vec(const std::vector<T>& v) {
    uint64_t n = v.size();
    add(&n, sizeof(n));
    if (n) add(v.data(), n * sizeof(T));
  }
};

struct Request {
  uint64_t id = 0;
  std::vector<float> px, py, pz;
  std::vector<uint32_t> tris;
  std::vector<uint8_t> pinned;
  vistio_solver_config cfg{};
  vistio_setup_desc setup{};
  int32_t ipc = 0;
  vistio_contact_desc contact{};
  float dt = 0.f;
  uint32_t steps = 0;
  int32_t state = VISTIO_REQ_QUEUED, status = VISTIO_OK;
  vistio_solver* solver = nullptr;
  uint64_t bytes = 0;      // admission estimate
  uint64_t cohort_key = 0;
  uint32_t cohort = 0;
  int32_t cache_hit = 0;
  double t_submit = 0, t_ready = 0, t_start = 0, t_done = 0;
  std::vector<float> out;  // px, py, pz, vx, vy, vz (nv each)
  std::string error;
};

struct CacheEntry {
  std::shared_ptr<vistio_solver> proto;
  uint64_t bytes = 0;
  uint64_t last_use = 0;
};

struct Cohort {
  uint32_t id = 0;
  vistio_ctx* ctx = nullptr;
  vistio_batch* batch = nullptr;
  std::vector<Request*> reqs;
  uint32_t steps_total = 0, steps_queued = 0;
  float dt = 0.f;
  int32_t ipc = 0;
  vistio_contact_desc contact{};
  std::deque<cudaEvent_t> pending;  // one event after each queued slice
  uint64_t bytes = 0;
};

double seconds_since(Clock::time_point t0) {
  return std::chrono::duration<double>(Clock::now() - t0).count();
}

}  // namespace

struct vistio_server {
  vistio_server_config cfg{};
  Clock::time_point t0 = Clock::now();
  std::string last_error;
  // shared with the set-up threads
  std::mutex mu;
  std::condition_variable cv;
  bool stop = false;
  std::deque<Request*> setup_queue;
  std::vector<Request*> ready;  // set up, waiting for admission, in arrival order
  std::unordered_map<uint64_t, CacheEntry> cache;
  uint64_t cache_used = 0, use_clock = 0;
  uint64_t cache_hits = 0, cache_misses = 0;
  std::vector<std::thread> workers;
  std::vector<vistio_ctx*> worker_ctx;
  // owned by the thread calling the server
  std::unordered_map<uint64_t, std::unique_ptr<Request>> requests;
  std::list<Cohort> cohorts;
  uint64_t next_id = 1;
  uint32_t next_cohort = 1;
  uint64_t bytes_in_use = 0, max_bytes_in_use = 0;
  uint64_t submitted = 0, completed = 0, failed = 0, cohorts_started = 0, max_cohorts_active = 0;
  uint64_t instance_steps = 0;
  double first_submit = -1, last_done = 0;
  std::vector<double> latencies;
};

namespace {

vistio_status srv_fail(vistio_server* s, vistio_status st, const std::string& msg) {
  if (s) s->last_error = msg;
  return st;
}

// Set-up cache key: mesh, pins, material and configuration (the factor
// depends on the material and the matrix dt; the solver carries the
// configuration). 64-bit FNV-1a together with the mesh sizes.
uint64_t setup_key(const Request& r) {
  Fnv f;
  f.add_vec(r.px); f.add_vec(r.py); f.add_vec(r.pz);
  f.add_vec(r.tris); f.add_vec(r.pinned);
  f.add(&r.setup, sizeof(r.setup));
  f.add(&r.cfg, sizeof(r.cfg));
  uint32_t g[2] = {uint32_t(r.ipc == 0 && r.contact.has_ground), 0u};
  float gh = g[0] ? r.contact.ground_height : 0.f;
  f.add(g, sizeof(g)); f.add(&gh, sizeof(gh));
  return f.h;
}

// Requests of one cohort step together: same configuration, contact set-up,
// dt and step count.
uint64_t cohort_key(const Request& r) {
  Fnv f;
  f.add(&r.cfg, sizeof(r.cfg));
  f.add(&r.ipc, sizeof(r.ipc));
  if (r.ipc) f.add(&r.contact, sizeof(r.contact));
  f.add(&r.dt, sizeof(r.dt));
  f.add(&r.steps, sizeof(r.steps));
  return f.h;
}

void cache_insert(vistio_server* S, uint64_t key, std::shared_ptr<vistio_solver> proto, uint64_t bytes) {
  // caller holds S->mu
  if (S->cfg.cache_bytes == 0 || bytes > S->cfg.cache_bytes || S->cache.count(key)) return;
  while (S->cache_used + bytes > S->cfg.cache_bytes && !S->cache.empty()) {
    auto victim = S->cache.begin();
    for (auto it = S->cache.begin(); it != S->cache.end(); ++it)
      if (it->second.last_use < victim->second.last_use) victim = it;
    S->cache_used -= victim->second.bytes;
    S->cache.erase(victim);
  }
  S->cache[key] = CacheEntry{std::move(proto), bytes, ++S->use_clock};
  S->cache_used += bytes;
}

void setup_worker(vistio_server* S, vistio_ctx* ctx) {
  for (;;) {
    Request* r;
    {
      std::unique_lock<std::mutex> lock(S->mu);
      S->cv.wait(lock, [&] { return S->stop || !S->setup_queue.empty(); });
      if (S->stop) return;
      r = S->setup_queue.front();
      S->setup_queue.pop_front();
      r->state = VISTIO_REQ_SETUP;
    }
    const uint64_t key = setup_key(*r);
    std::shared_ptr<vistio_solver> proto;
    {
      std::lock_guard<std::mutex> lock(S->mu);
      auto it = S->cache.find(key);
      if (it != S->cache.end()) {
        it->second.last_use = ++S->use_clock;
        proto = it->second.proto;
      }
    }
    vistio_solver* sol = nullptr;
    vistio_status st;
    int32_t hit = proto != nullptr;
    if (proto) {
      st = vistio_solver_clone(proto.get(), ctx, &sol);
    } else {
      vistio_mesh_desc m{uint32_t(r->px.size()), uint32_t(r->tris.size() / 3), r->px.data(), r->py.data(),
                         r->pz.data(), r->tris.data()};
      vistio_solver_config cfg = r->cfg;
      if (!S->cfg.gpu_factorization) cfg.host_factorization = 1;  // in this thread, beside the GPU's work
      st = vistio_solver_init_explicit(ctx, &m, &cfg, &r->setup, r->pinned.empty() ? nullptr : r->pinned.data(),
                                       &sol);
      if (st == VISTIO_OK && r->ipc == 0 && r->contact.has_ground)
        st = vistio_solver_set_ground(sol, 1, r->contact.ground_height);
    }
    uint64_t bytes = 0;
    if (st == VISTIO_OK) st = vistio_solver_device_bytes(sol, r->ipc && r->contact.self_collision, &bytes);
    std::shared_ptr<vistio_solver> keep;
    if (st == VISTIO_OK && !proto && S->cfg.cache_bytes) {
      vistio_solver* c = nullptr;
      if (vistio_solver_clone(sol, ctx, &c) == VISTIO_OK)
        keep = std::shared_ptr<vistio_solver>(c, [](vistio_solver* x) { vistio_solver_destroy(x); });
    }
    const std::string err = st == VISTIO_OK ? std::string() : std::string(vistio_last_error(ctx));
    {
      std::lock_guard<std::mutex> lock(S->mu);
      if (keep) cache_insert(S, key, keep, 2 * bytes);  // host copy: FP64 factor, about twice the device bytes
      (hit ? S->cache_hits : S->cache_misses)++;
      r->cache_hit = hit;
      r->t_ready = seconds_since(S->t0);
      if (st != VISTIO_OK) {
        if (sol) vistio_solver_destroy(sol);
        r->state = VISTIO_REQ_FAILED;
        r->status = st;
        r->error = err;
      } else {
        r->solver = sol;
        r->bytes = bytes;
        r->state = VISTIO_REQ_READY;
        S->ready.push_back(r);
      }
    }
  }
}

void release_cohort(Cohort& c) {
  for (cudaEvent_t e : c.pending) cudaEventDestroy(e);
  c.pending.clear();
  if (c.batch) vistio_batch_destroy(c.batch);
  c.batch = nullptr;
  for (Request* r : c.reqs) {
    if (r->solver) vistio_solver_destroy(r->solver);
    r->solver = nullptr;
  }
  if (c.ctx) vistio_ctx_destroy(c.ctx);  // freed once the batch's buffers are
  c.ctx = nullptr;
}

vistio_status queue_slice(vistio_server* S, Cohort& c) {
  const uint32_t n = std::min(S->cfg.steps_per_slice, c.steps_total - c.steps_queued);
  vistio_status st = vistio_batch_step(c.batch, c.dt, n, c.ipc ? &c.contact : nullptr);
  if (st != VISTIO_OK) return srv_fail(S, st, vistio_last_error(c.ctx));
  cudaEvent_t e;
  cudaError_t ce = cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
  if (ce == cudaSuccess) ce = cudaEventRecord(e, static_cast<cudaStream_t>(vistio_batch_stream(c.batch)));
  if (ce != cudaSuccess) return srv_fail(S, VISTIO_ERR_GPU, std::string("event: ") + cudaGetErrorString(ce));
  c.pending.push_back(e);
  c.steps_queued += n;
  return VISTIO_OK;
}

void finish_request(vistio_server* S, Request* r, int32_t state, int32_t status, const std::string& err) {
  r->state = state;
  r->status = status;
  r->error = err;
  r->t_done = seconds_since(S->t0);
  if (state == VISTIO_REQ_DONE) {
    S->completed++;
    S->instance_steps += r->steps;
    S->latencies.push_back(r->t_done - r->t_submit);
    S->last_done = std::max(S->last_done, r->t_done);
  } else {
    S->failed++;
  }
}

// Advances one cohort; returns true when it is retired.
bool advance_cohort(vistio_server* S, Cohort& c) {
  while (!c.pending.empty()) {
    cudaError_t q = cudaEventQuery(c.pending.front());
    if (q == cudaErrorNotReady) break;
    cudaEventDestroy(c.pending.front());
    c.pending.pop_front();
    if (q != cudaSuccess) {
      for (Request* r : c.reqs) finish_request(S, r, VISTIO_REQ_FAILED, VISTIO_ERR_GPU, cudaGetErrorString(q));
      return true;
    }
  }
  while (c.pending.size() < 2 && c.steps_queued < c.steps_total) {
    vistio_status st = queue_slice(S, c);
    if (st != VISTIO_OK) {
      for (Request* r : c.reqs) finish_request(S, r, VISTIO_REQ_FAILED, st, S->last_error);
      return true;
    }
  }
  if (c.steps_queued < c.steps_total || !c.pending.empty()) return false;
  for (uint32_t k = 0; k < c.reqs.size(); ++k) {
    Request* r = c.reqs[k];
    const size_t n = r->px.size();
    r->out.resize(6 * n);
    float* o = r->out.data();
    vistio_status st = vistio_batch_get_state(c.batch, k, o, o + n, o + 2 * n, o + 3 * n, o + 4 * n, o + 5 * n);
    if (st == VISTIO_OK) finish_request(S, r, VISTIO_REQ_DONE, VISTIO_OK, "");
    else finish_request(S, r, VISTIO_REQ_FAILED, st, vistio_last_error(c.ctx));
  }
  return true;
}

vistio_status start_cohort(vistio_server* S, const std::vector<Request*>& take, uint64_t est) {
  Cohort c;
  c.id = S->next_cohort++;
  c.reqs = take;
  c.steps_total = take[0]->steps;
  c.dt = take[0]->dt;
  c.ipc = take[0]->ipc;
  c.contact = take[0]->contact;
  vistio_status st = vistio_ctx_create(S->cfg.device, &c.ctx);
  if (st != VISTIO_OK) return srv_fail(S, st, vistio_last_error(nullptr));
  std::vector<vistio_solver*> sv;
  for (Request* r : take) sv.push_back(r->solver);
  st = vistio_batch_create(c.ctx, sv.data(), uint32_t(sv.size()), &c.batch);
  if (st == VISTIO_OK) st = vistio_batch_set_sweep_mode(c.batch, S->cfg.sweep_mode);
  if (st != VISTIO_OK) {
    std::string err = vistio_last_error(c.ctx);
    vistio_ctx_destroy(c.ctx);
    return srv_fail(S, st, err);
  }
  uint64_t dev_bytes = 0;
  vistio_batch_info(c.batch, nullptr, nullptr, nullptr, nullptr, nullptr, &dev_bytes);
  c.bytes = std::max(est, dev_bytes);
  const double now = seconds_since(S->t0);
  for (Request* r : take) {
    r->state = VISTIO_REQ_RUNNING;
    r->cohort = c.id;
    r->t_start = now;
  }
  S->bytes_in_use += c.bytes;
  S->max_bytes_in_use = std::max(S->max_bytes_in_use, S->bytes_in_use);
  S->cohorts_started++;
  S->cohorts.push_back(std::move(c));
  S->max_cohorts_active = std::max<uint64_t>(S->max_cohorts_active, S->cohorts.size());
  return VISTIO_OK;
}

void admit(vistio_server* S) {
  std::vector<Request*> ready;
  {
    std::lock_guard<std::mutex> lock(S->mu);
    ready.swap(S->ready);
  }
  if (ready.empty()) return;
  std::vector<uint64_t> order;  // cohort keys by first arrival
  std::unordered_map<uint64_t, std::vector<Request*>> groups;
  for (Request* r : ready) {
    r->cohort_key = cohort_key(*r);
    auto& g = groups[r->cohort_key];
    if (g.empty()) order.push_back(r->cohort_key);
    g.push_back(r);
  }
  std::vector<Request*> left;
  bool full = false;
  const double now = seconds_since(S->t0);
  for (uint64_t key : order) {
    std::vector<Request*>& g = groups[key];
    size_t i = 0;
    // the admission window: while the GPU has work, let a small set wait
    // for company (bounded by admit_wait_ms from its first readiness)
    if (S->cfg.admit_wait_ms && !S->cohorts.empty() && g.size() < S->cfg.max_cohort) {
      double first = g[0]->t_ready;
      for (Request* r : g) first = std::min(first, r->t_ready);
      if (now - first < 1e-3 * double(S->cfg.admit_wait_ms)) {
        left.insert(left.end(), g.begin(), g.end());
        continue;
      }
    }
    while (i < g.size() && !full) {
      std::vector<Request*> take;
      uint64_t sum = 0;
      while (i < g.size() && take.size() < S->cfg.max_cohort &&
             S->bytes_in_use + sum + g[i]->bytes <= S->cfg.hbm_budget_bytes) {
        sum += g[i]->bytes;
        take.push_back(g[i++]);
      }
      if (take.empty()) {
        if (S->cohorts.empty() && g[i]->bytes > S->cfg.hbm_budget_bytes) {  // can never fit
          finish_request(S, g[i], VISTIO_REQ_FAILED, VISTIO_ERR_OOM, "request needs more device memory than the budget");
          vistio_solver_destroy(g[i]->solver);
          g[i]->solver = nullptr;
          ++i;
          continue;
        }
        full = true;
        break;
      }
      if (start_cohort(S, take, sum) != VISTIO_OK) {  // e.g. out of memory: retry later
        i -= take.size();
        full = true;
        break;
      }
    }
    for (; i < g.size(); ++i) left.push_back(g[i]);
  }
  if (!left.empty()) {
    std::sort(left.begin(), left.end(), [](const Request* a, const Request* b) { return a->id < b->id; });
    std::lock_guard<std::mutex> lock(S->mu);
    S->ready.insert(S->ready.begin(), left.begin(), left.end());
  }
}

}  // namespace

extern "C" {

vistio_status vistio_server_create(const vistio_server_config* cfg, vistio_server** out) {
  if (!cfg || !out) return VISTIO_ERR_INVALID_CONFIG;
  if (cfg->max_cohort == 0 || cfg->setup_threads == 0 || cfg->steps_per_slice == 0 || cfg->hbm_budget_bytes == 0 ||
      cfg->sweep_mode > 1)
    return VISTIO_ERR_INVALID_CONFIG;
  auto S = std::make_unique<vistio_server>();
  S->cfg = *cfg;
  for (uint32_t k = 0; k < cfg->setup_threads; ++k) {
    vistio_ctx* c = nullptr;
    vistio_status st = vistio_ctx_create(cfg->device, &c);
    if (st != VISTIO_OK) {
      for (vistio_ctx* x : S->worker_ctx) vistio_ctx_destroy(x);
      return st;
    }
    S->worker_ctx.push_back(c);
  }
  for (vistio_ctx* c : S->worker_ctx) S->workers.emplace_back(setup_worker, S.get(), c);
  *out = S.release();
  return VISTIO_OK;
}

vistio_status vistio_server_destroy(vistio_server* S) {
  if (!S) return VISTIO_OK;
  {
    std::lock_guard<std::mutex> lock(S->mu);
    S->stop = true;
  }
  S->cv.notify_all();
  for (auto& t : S->workers) t.join();
  for (Cohort& c : S->cohorts) release_cohort(c);
  S->cohorts.clear();
  for (auto& kv : S->requests)
    if (kv.second->solver) vistio_solver_destroy(kv.second->solver);
  S->cache.clear();  // prototypes before their contexts
  for (vistio_ctx* c : S->worker_ctx) vistio_ctx_destroy(c);
  delete S;
  return VISTIO_OK;
}

const char* vistio_server_last_error(const vistio_server* S) { return S ? S->last_error.c_str() : ""; }

vistio_status vistio_server_submit(vistio_server* S, const vistio_request* r, uint64_t* id) {
  if (!S || !r || !id) return srv_fail(S, VISTIO_ERR_INVALID_CONFIG, "null argument");
  const vistio_mesh_desc& m = r->mesh;
  if (!m.pos_x || !m.pos_y || !m.pos_z || !m.indices || m.vertex_count == 0 || m.triangle_count == 0)
    return srv_fail(S, VISTIO_ERR_INVALID_MESH, "empty mesh");
  if (!(r->dt > 0.f) || r->steps == 0) return srv_fail(S, VISTIO_ERR_INVALID_CONFIG, "dt and steps must be positive");
  auto q = std::make_unique<Request>();
  q->id = S->next_id++;
  q->px.assign(m.pos_x, m.pos_x + m.vertex_count);
  q->py.assign(m.pos_y, m.pos_y + m.vertex_count);
  q->pz.assign(m.pos_z, m.pos_z + m.vertex_count);
  q->tris.assign(m.indices, m.indices + 3ull * m.triangle_count);
  if (r->pinned) q->pinned.assign(r->pinned, r->pinned + m.vertex_count);
  q->cfg = r->config;
  q->setup = r->setup;
  q->ipc = r->has_contact != 0;
  q->contact = r->contact;
  q->dt = r->dt;
  q->steps = r->steps;
  q->t_submit = seconds_since(S->t0);
  if (S->first_submit < 0) S->first_submit = q->t_submit;
  Request* raw = q.get();
  S->requests[q->id] = std::move(q);
  S->submitted++;
  {
    std::lock_guard<std::mutex> lock(S->mu);
    S->setup_queue.push_back(raw);
  }
  S->cv.notify_one();
  *id = raw->id;
  return VISTIO_OK;
}

vistio_status vistio_server_tick(vistio_server* S, uint32_t* unfinished) {
  if (!S) return VISTIO_ERR_INVALID_CONFIG;
  cudaSetDevice(S->cfg.device);
  for (auto it = S->cohorts.begin(); it != S->cohorts.end();) {
    if (advance_cohort(S, *it)) {
      S->bytes_in_use -= it->bytes;
      release_cohort(*it);
      it = S->cohorts.erase(it);
    } else {
      ++it;
    }
  }
  admit(S);
  for (Cohort& c : S->cohorts)  // queue the first slices of new cohorts
    if (c.steps_queued == 0) advance_cohort(S, c);
  if (unfinished) {
    uint32_t n = 0;
    std::lock_guard<std::mutex> lock(S->mu);
    for (auto& kv : S->requests)
      if (kv.second->state != VISTIO_REQ_DONE && kv.second->state != VISTIO_REQ_FAILED) ++n;
    *unfinished = n;
  }
  return VISTIO_OK;
}

vistio_status vistio_server_drain(vistio_server* S, double timeout_s) {
  if (!S) return VISTIO_ERR_INVALID_CONFIG;
  const Clock::time_point t = Clock::now();
  for (;;) {
    uint32_t n = 0;
    vistio_status st = vistio_server_tick(S, &n);
    if (st != VISTIO_OK) return st;
    if (n == 0) return VISTIO_OK;
    if (std::chrono::duration<double>(Clock::now() - t).count() > timeout_s)
      return srv_fail(S, VISTIO_ERR_TIMEOUT, "requests still unfinished at the drain timeout");
    std::this_thread::sleep_for(std::chrono::microseconds(200));
  }
}

vistio_status vistio_server_query(vistio_server* S, uint64_t id, vistio_request_info* info) {
  if (!S || !info) return VISTIO_ERR_INVALID_CONFIG;
  auto it = S->requests.find(id);
  if (it == S->requests.end()) return srv_fail(S, VISTIO_ERR_INVALID_CONFIG, "unknown request");
  std::lock_guard<std::mutex> lock(S->mu);
  const Request& r = *it->second;
  info->state = r.state;
  info->status = r.status;
  info->vertex_count = uint32_t(r.px.size());
  info->cohort = r.cohort;
  info->cache_hit = r.cache_hit;
  info->submit_s = r.t_submit;
  info->ready_s = r.t_ready;
  info->start_s = r.t_start;
  info->done_s = r.t_done;
  if (r.state == VISTIO_REQ_FAILED) S->last_error = r.error;
  return VISTIO_OK;
}

vistio_status vistio_server_result(vistio_server* S, uint64_t id, float* px, float* py, float* pz, float* vx,
                                   float* vy, float* vz) {
  if (!S) return VISTIO_ERR_INVALID_CONFIG;
  auto it = S->requests.find(id);
  if (it == S->requests.end()) return srv_fail(S, VISTIO_ERR_INVALID_CONFIG, "unknown request");
  const Request& r = *it->second;
  if (r.state == VISTIO_REQ_FAILED) return srv_fail(S, vistio_status(r.status), r.error);
  if (r.state != VISTIO_REQ_DONE) return srv_fail(S, VISTIO_ERR_INVALID_CONFIG, "request not done");
  const size_t n = r.px.size();
  float* dst[6] = {px, py, pz, vx, vy, vz};
  for (int k = 0; k < 6; ++k)
    if (dst[k]) std::memcpy(dst[k], r.out.data() + k * n, n * sizeof(float));
  return VISTIO_OK;
}

vistio_status vistio_server_release(vistio_server* S, uint64_t id) {
  if (!S) return VISTIO_ERR_INVALID_CONFIG;
  auto it = S->requests.find(id);
  if (it == S->requests.end()) return srv_fail(S, VISTIO_ERR_INVALID_CONFIG, "unknown request");
  if (it->second->state != VISTIO_REQ_DONE && it->second->state != VISTIO_REQ_FAILED)
    return srv_fail(S, VISTIO_ERR_INVALID_CONFIG, "request still in progress");
  S->requests.erase(it);
  return VISTIO_OK;
}

vistio_status vistio_server_get_stats(vistio_server* S, vistio_server_stats* st) {
  if (!S || !st) return VISTIO_ERR_INVALID_CONFIG;
  std::memset(st, 0, sizeof(*st));
  st->submitted = S->submitted;
  st->completed = S->completed;
  st->failed = S->failed;
  st->cohorts_started = S->cohorts_started;
  st->cohorts_active = S->cohorts.size();
  st->max_cohorts_active = S->max_cohorts_active;
  st->bytes_in_use = S->bytes_in_use;
  st->max_bytes_in_use = S->max_bytes_in_use;
  {
    std::lock_guard<std::mutex> lock(S->mu);
    st->cache_hits = S->cache_hits;
    st->cache_misses = S->cache_misses;
  }
  st->instance_steps = S->instance_steps;
  if (!S->latencies.empty()) {
    std::vector<double> l = S->latencies;
    std::sort(l.begin(), l.end());
    auto pct = [&](double p) {  // nearest rank
      size_t k = size_t(std::ceil(p * double(l.size()))) ;
      return l[std::min(l.size() - 1, k ? k - 1 : 0)];
    };
    st->p50_latency_s = pct(0.50);
    st->p99_latency_s = pct(0.99);
    double sum = 0;
    for (double x : l) sum += x;
    st->mean_latency_s = sum / double(l.size());
  }
  const double span = S->last_done - std::max(0.0, S->first_submit);
  st->throughput = span > 0 ? double(S->instance_steps) / span : 0.0;
  return VISTIO_OK;
}

}  // extern "C"
