// Batched and served execution of independent instances (orctm_serve_*,
// orctm_batch_run).
//
// A server owns `slots` worker threads.  Requests wait in a FIFO queue; a
// worker takes the head when the head's estimated device memory fits the
// budget (or nothing is in flight), creates a handle on its own stream,
// uploads the request's fields, runs its steps, downloads the requested
// fields and destroys the handle.  Handles allocate from the library's
// stream-ordered pool, so creating and destroying instances does not
// synchronise the device and the other slots' work keeps running.  Each
// step is timed on the host (the step's launches plus a synchronisation of
// its stream) for the latency percentiles.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/orctm_gpu.h"

namespace {

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

// p-th percentile (nearest rank) of v; v is reordered
double percentile(std::vector<double>& v, double p) {
  if (v.empty()) return 0.0;
  size_t k = (size_t)(p / 100.0 * (double)v.size());
  if (k >= v.size()) k = v.size() - 1;
  std::nth_element(v.begin(), v.begin() + (long)k, v.end());
  return v[k];
}

struct Request {
  unsigned long long id = 0;
  orctm_request req{};
  orctm_desc desc{};
  unsigned long long est = 0;
  double cells = 0;
  Clock::time_point t_submit, t_admit;
  orctm_request_stats stats{};
  bool done = false;
};

}  // namespace

struct orctm_server {
  orctm_serve_opts opts{};
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Request*> queue;
  std::unordered_map<unsigned long long, Request*> recs;
  std::vector<std::thread> workers;
  unsigned long long next_id = 1;
  unsigned long long budget = 0, reserved = 0, peak_reserved = 0;
  int in_flight = 0, peak_in_flight = 0;
  bool stop = false;
  long long submitted = 0, completed = 0, failed = 0, steps = 0;
  double cell_steps = 0;
  bool started = false;
  Clock::time_point t_first, t_last;
  std::vector<double> step_ms;

  bool admissible(const Request* r) const {
    return in_flight == 0 || reserved + r->est <= budget;
  }
  void run(Request* r);
  void worker();
};

void orctm_server::run(Request* r) {
  orctm_request_stats& s = r->stats;
  std::vector<double> lat;
  orctm_handle* h = nullptr;
  int st = orctm_create(&r->desc, &h);
  if (!st) st = orctm_set_solver(h, opts.solver, opts.rtol, opts.maxit);
  for (int k = 0; !st && k < r->req.nin; ++k) {
    size_t n = 0;
    st = orctm_field_size(h, r->req.in_fields[k], &n);
    if (!st) st = orctm_upload(h, r->req.in_fields[k], r->req.in_data[k], n);
  }
  for (int k = 0; !st && k < r->req.nsteps; ++k) {
    const Clock::time_point t0 = Clock::now();
    orctm_solve_stats ss{};
    st = orctm_step_hotpath(h, &ss);
    if (!st) st = orctm_synchronize(h);
    const Clock::time_point t1 = Clock::now();
    if (st) break;
    lat.push_back(ms_between(t0, t1));
    s.steps_done++;
    s.iterations += ss.iterations;
    s.relres_max = std::max(s.relres_max, ss.relres);
  }
  for (int k = 0; !st && k < r->req.nout; ++k) {
    size_t n = 0;
    st = orctm_field_size(h, r->req.out_fields[k], &n);
    if (!st) st = orctm_download(h, r->req.out_fields[k], r->req.out_data[k], n);
  }
  if (h) {
    orctm_device_bytes(h, &s.device_bytes);
    orctm_destroy(h);
  }
  s.status = st;
  s.estimated_bytes = r->est;
  s.step_ms_max = lat.empty() ? 0.0 : *std::max_element(lat.begin(), lat.end());
  {
    std::vector<double> v = lat;
    s.step_ms_p50 = percentile(v, 50.0);
    s.step_ms_p99 = percentile(v, 99.0);
  }
  const Clock::time_point t_end = Clock::now();
  s.queued_ms = ms_between(r->t_submit, r->t_admit);
  s.run_ms = ms_between(r->t_admit, t_end);
  std::lock_guard<std::mutex> lk(mu);
  step_ms.insert(step_ms.end(), lat.begin(), lat.end());
  steps += s.steps_done;
  cell_steps += r->cells * s.steps_done;
  if (st) failed++;
  else completed++;
  t_last = t_end;
  reserved -= r->est;
  in_flight--;
  r->done = true;
  cv_done.notify_all();
  cv_work.notify_all();
}

void orctm_server::worker() {
  cudaSetDevice(opts.device);
  for (;;) {
    Request* r = nullptr;
    {
      std::unique_lock<std::mutex> lk(mu);
      cv_work.wait(lk, [&] {
        return (stop && queue.empty()) || (!queue.empty() && admissible(queue.front()));
      });
      if (queue.empty()) return;
      r = queue.front();
      queue.pop_front();
      reserved += r->est;
      peak_reserved = std::max(peak_reserved, reserved);
      in_flight++;
      peak_in_flight = std::max(peak_in_flight, in_flight);
      r->t_admit = Clock::now();
      // another worker may be able to take the next request as well
      cv_work.notify_all();
    }
    run(r);
  }
}

extern "C" {

int orctm_serve_create(const orctm_serve_opts* opts, orctm_server** out) {
  if (!opts || !out || opts->slots < 1 || opts->slots > 1024 || !(opts->memory_fraction > 0.0) ||
      opts->memory_fraction > 1.0 || opts->rtol <= 0.0 || opts->maxit < 1 ||
      (opts->solver != ORCTM_SOLVER_FP64 && opts->solver != ORCTM_SOLVER_FP32_REFINED))
    return ORCTM_E_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return ORCTM_E_NODEVICE;
  if (opts->device < 0 || opts->device >= ndev) return ORCTM_E_ARG;
  size_t free_b = 0, total_b = 0;
  if (cudaSetDevice(opts->device) != cudaSuccess ||
      cudaMemGetInfo(&free_b, &total_b) != cudaSuccess)
    return ORCTM_E_CUDA;
  orctm_server* s = new orctm_server();
  s->opts = *opts;
  s->budget = (unsigned long long)(opts->memory_fraction * (double)free_b);
  for (int k = 0; k < opts->slots; ++k) s->workers.emplace_back([s] { s->worker(); });
  *out = s;
  return ORCTM_OK;
}

int orctm_serve_submit(orctm_server* s, const orctm_request* req, unsigned long long* id) {
  if (!s || !req || !req->desc || req->nsteps < 0 || req->nin < 0 || req->nout < 0 ||
      (req->nin > 0 && (!req->in_fields || !req->in_data)) ||
      (req->nout > 0 && (!req->out_fields || !req->out_data)))
    return ORCTM_E_ARG;
  Request* r = new Request();
  r->req = *req;
  r->desc = *req->desc;
  r->desc.device = s->opts.device;
  int st = orctm_estimate_device_bytes(&r->desc, s->opts.solver, &r->est);
  if (st) {
    delete r;
    return st;
  }
  r->cells = (double)(r->desc.ie - 2) * (double)(r->desc.je - 2) * (double)r->desc.ke;
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->stop) {
    delete r;
    return ORCTM_E_ARG;
  }
  r->id = s->next_id++;
  r->t_submit = Clock::now();
  if (!s->started) {
    s->started = true;
    s->t_first = r->t_submit;
  }
  s->recs[r->id] = r;
  s->queue.push_back(r);
  s->submitted++;
  if (id) *id = r->id;
  s->cv_work.notify_all();
  return ORCTM_OK;
}

int orctm_serve_wait(orctm_server* s, unsigned long long id, orctm_request_stats* stats) {
  if (!s) return ORCTM_E_ARG;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->recs.find(id);
  if (it == s->recs.end()) return ORCTM_E_ARG;
  Request* r = it->second;
  s->cv_done.wait(lk, [&] { return r->done; });
  if (stats) *stats = r->stats;
  s->recs.erase(it);
  delete r;
  return ORCTM_OK;
}

int orctm_serve_poll(orctm_server* s, unsigned long long id, int* done,
                     orctm_request_stats* stats) {
  if (!s || !done) return ORCTM_E_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->recs.find(id);
  if (it == s->recs.end()) return ORCTM_E_ARG;
  Request* r = it->second;
  *done = r->done ? 1 : 0;
  if (r->done) {
    if (stats) *stats = r->stats;
    s->recs.erase(it);
    delete r;
  }
  return ORCTM_OK;
}

int orctm_serve_drain(orctm_server* s) {
  if (!s) return ORCTM_E_ARG;
  std::unique_lock<std::mutex> lk(s->mu);
  s->cv_done.wait(lk, [&] { return s->completed + s->failed == s->submitted; });
  return ORCTM_OK;
}

int orctm_serve_get_stats(orctm_server* s, orctm_serve_stats* out) {
  if (!s || !out) return ORCTM_E_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  orctm_serve_stats t{};
  t.submitted = s->submitted;
  t.completed = s->completed;
  t.failed = s->failed;
  t.steps = s->steps;
  t.cell_steps = s->cell_steps;
  t.elapsed_ms = s->started ? ms_between(s->t_first, s->t_last) : 0.0;
  if (t.elapsed_ms < 0) t.elapsed_ms = 0;
  std::vector<double> v = s->step_ms;
  t.step_ms_p50 = percentile(v, 50.0);
  t.step_ms_p99 = percentile(v, 99.0);
  t.peak_in_flight = s->peak_in_flight;
  t.peak_reserved_bytes = s->peak_reserved;
  t.budget_bytes = s->budget;
  *out = t;
  return ORCTM_OK;
}

int orctm_serve_destroy(orctm_server* s) {
  if (!s) return ORCTM_E_ARG;
  orctm_serve_drain(s);
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  for (auto& w : s->workers) w.join();
  for (auto& kv : s->recs) delete kv.second;
  delete s;
  return ORCTM_OK;
}

int orctm_batch_run(const orctm_serve_opts* opts, int n, const orctm_request* reqs,
                    orctm_request_stats* per_request, orctm_serve_stats* total) {
  if (n < 0 || (n > 0 && !reqs)) return ORCTM_E_ARG;
  orctm_server* s = nullptr;
  int st = orctm_serve_create(opts, &s);
  if (st) return st;
  std::vector<unsigned long long> ids((size_t)n, 0);
  for (int k = 0; k < n && !st; ++k) st = orctm_serve_submit(s, &reqs[k], &ids[(size_t)k]);
  int first_err = st;
  for (int k = 0; k < n; ++k) {
    if (!ids[(size_t)k]) continue;
    orctm_request_stats rs{};
    orctm_serve_wait(s, ids[(size_t)k], &rs);
    if (per_request) per_request[k] = rs;
    if (!first_err && rs.status) first_err = rs.status;
  }
  if (total) orctm_serve_get_stats(s, total);
  orctm_serve_destroy(s);
  return first_err;
}

}  // extern "C"
