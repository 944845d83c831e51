// serve.cu -- request loop on one GPU: continuous batching of exact and
// Monte-Carlo permanent requests of mixed sizes.
//
// No counterpart in the reference (its CLI computes one matrix per process).
// Design:
//  * `slots` worker threads, each owning a perm_ctx (its own stream, resident
//    scratch for partial sums, pinned staging).  Work of different slots runs
//    concurrently on the device.
//  * Admission: a request is admitted when a slot is idle and its device
//    memory need (operand image + per-trial buffers) fits in the remaining
//    budget; requests that arrive while others run are admitted as slots and
//    memory free up (FIFO; a request that does not fit may be passed by
//    later ones that do, at most kMaxPasses times, after which nothing passes
//    it until enough memory frees up -- so a large request cannot starve
//    behind a steady stream of small ones).
//  * Exact requests whose Gray walk exceeds `slice_steps` run as several
//    shard launches (perm_exact_dense_shard) so that one large permanent does
//    not hold the whole GPU for tens of milliseconds while small requests
//    wait; shard results are added in double-double and the sum gets the
//    context's accuracy policy (perm_exact_dense_refine), like an unsliced
//    request.  A request whose policy starts with a certified walk
//    (perm_exact_dense_plan: integer matrices, sparse or strongly cancelling
//    real ones) runs unsliced: that walk is its whole evaluation, where
//    sliced FP64-X or int32-X shards would be followed by it.
//  * Every request gets a status; a failing request (bad size, CUDA error)
//    fails alone.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

#include "../../include/perman_b200.h"
#include "matrix_io.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Job {
  uint64_t ticket = 0;
  perm_request req{};
  std::vector<double> mat;
  size_t bytes = 0;
  Clock::time_point t_submit;
  perm_response resp{};
  bool done = false;
  int passes = 0;  // times a later job was admitted ahead of this one
};

// How often a pending job that does not fit the memory budget may be passed
// by later jobs before admission stops at it.
constexpr int kMaxPasses = 8;

size_t request_bytes(const perm_request& r) {
  const size_t n = (size_t)std::max(r.n, 1);
  const size_t np = (n + 1) & ~(size_t)1;
  switch (r.kind) {
    case PERM_REQ_SCALING: return 2 * n * np * sizeof(double) + np * 8 + 4096;
    case PERM_REQ_RASMUSSEN: return np * 8 + 4096;
    default: return n * np * sizeof(double) + 4096;
  }
}

void dd_add(double& hi, double& lo, double h2, double l2) {
  const double s = hi + h2, bb = s - hi;
  const double e = (hi - (s - bb)) + (h2 - bb);
  hi = s;
  lo += e + l2;
}

}  // namespace

struct perm_server {
  int device = 0;
  int slots = 1;
  size_t budget = 0, in_use = 0;
  uint64_t slice_steps = 1ull << 31;
  Clock::time_point t0;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Job*> pending;
  std::map<uint64_t, Job*> jobs;
  uint64_t next_ticket = 1;
  uint64_t submitted = 0, completed = 0, in_flight = 0;
  bool stop = false;
  int waiters = 0;  // threads inside perm_server_wait
  std::vector<std::thread> workers;
  std::vector<perm_ctx*> ctxs;
};

namespace {

double ms_since(const perm_server* s, Clock::time_point t) {
  return std::chrono::duration<double, std::milli>(t - s->t0).count();
}

// Pick the next job this worker may run (caller holds the lock): the oldest
// pending job whose memory need fits the remaining budget; a job larger than
// the whole budget runs alone once nothing else holds memory.  Jobs that are
// passed over are counted, and one passed kMaxPasses times blocks every job
// behind it until it fits.
Job* take_admissible(perm_server* s) {
  for (auto it = s->pending.begin(); it != s->pending.end(); ++it) {
    Job* j = *it;
    if (s->in_use + j->bytes <= s->budget || s->in_use == 0) {
      for (auto p = s->pending.begin(); p != it; ++p) (*p)->passes++;
      s->pending.erase(it);
      s->in_use += j->bytes;
      s->in_flight++;
      return j;
    }
    if (j->passes >= kMaxPasses) return nullptr;
  }
  return nullptr;
}

void run_job(perm_server* s, perm_ctx* ctx, Job* j) {
  perm_response& r = j->resp;
  const perm_request& q = j->req;
  const double* a = j->mat.data();
  int rc = PERM_OK;
  switch (q.kind) {
    case PERM_REQ_EXACT_DENSE:
    case PERM_REQ_EXACT_SPARSE: {
      perm_result pr{};
      if (q.kind == PERM_REQ_EXACT_SPARSE && q.n >= 1 && q.n <= PERM_MAX_EXACT_N) {
        std::vector<double> tmp(j->mat);
        perm::Compressed c;
        perm::compress(tmp.data(), q.n, &c);
        rc = perm_exact_sparse(ctx, q.n, c.rptrs.data(), c.cols.data(), c.rvals.data(), c.cptrs.data(),
                               c.rows.data(), c.cvals.data(), &pr);
        r.hi = pr.hi;
        r.lo = pr.lo;
        r.device_ms = pr.kernel_ms;
        r.kernel = pr.kernel;
      } else {
        const double total = q.n >= 1 && q.n <= PERM_MAX_EXACT_N ? std::ldexp(1.0, q.n - 1) : 1.0;
        int plan = 0;
        if (total > (double)s->slice_steps) rc = perm_exact_dense_plan(ctx, a, q.n, PERM_F64, &plan, nullptr);
        const int shards =
            plan ? 1 : (int)std::min(4096.0, std::max(1.0, std::ceil(total / (double)s->slice_steps)));
        double hi = 0, lo = 0, dev = 0;
        for (int k = 0; k < shards && rc == PERM_OK; k++) {
          rc = perm_exact_dense_shard(ctx, a, q.n, PERM_F64, k, shards, &pr);
          if (rc == PERM_OK) {
            dd_add(hi, lo, pr.hi, pr.lo);
            dev += pr.kernel_ms;
          }
        }
        r.hi = hi + lo;
        r.lo = lo - (r.hi - hi);
        r.device_ms = dev;
        r.kernel = pr.kernel;
        if (rc == PERM_OK && shards > 1) {
          // the single-shard call applied the accuracy policy itself; a
          // sliced request gets it on the assembled value
          pr.hi = r.hi;
          pr.lo = r.lo;
          pr.kernel_ms = dev;
          rc = perm_exact_dense_refine(ctx, a, q.n, PERM_F64, &pr);
          if (rc == PERM_OK) {
            r.hi = pr.hi;
            r.lo = pr.lo;
            r.device_ms = pr.kernel_ms;
            r.kernel = pr.kernel;
          }
        }
      }
      r.value = r.hi + r.lo;
      r.std_error = 0;
      break;
    }
    case PERM_REQ_RASMUSSEN:
    case PERM_REQ_SCALING: {
      perm_estimate e{};
      rc = q.kind == PERM_REQ_SCALING
               ? perm_approx_scaling(ctx, a, q.n, PERM_F64, q.trials, q.scale_intervals, q.scale_times, q.seed,
                                     nullptr, &e)
               : perm_approx_rasmussen(ctx, a, q.n, PERM_F64, q.trials, q.seed, nullptr, &e);
      r.value = r.hi = e.mean;
      r.lo = 0;
      r.std_error = e.std_error;
      r.device_ms = e.kernel_ms;
      r.kernel = 0;
      break;
    }
    default:
      rc = PERM_EINVAL;
  }
  r.status = rc;
  if (rc != PERM_OK) snprintf(r.message, sizeof r.message, "%s", perm_ctx_last_error(ctx));
}

void worker(perm_server* s, int slot) {
  perm_ctx* ctx = s->ctxs[slot];
  for (;;) {
    Job* j = nullptr;
    {
      std::unique_lock<std::mutex> lock(s->mu);
      s->cv_work.wait(lock, [&] { return s->stop || (j = take_admissible(s)) != nullptr; });
      if (!j) return;  // stopping
      j->resp.t_admit_ms = ms_since(s, Clock::now());
    }
    run_job(s, ctx, j);
    {
      std::lock_guard<std::mutex> lock(s->mu);
      j->resp.t_done_ms = ms_since(s, Clock::now());
      j->done = true;
      s->in_use -= j->bytes;
      s->in_flight--;
      s->completed++;
    }
    s->cv_done.notify_all();
    s->cv_work.notify_all();
  }
}

}  // namespace

extern "C" int perm_server_create(int device, int slots, size_t memory_budget, uint64_t slice_steps,
                                  perm_server** out) {
  if (!out || slots < 1 || slots > 64) return PERM_EINVAL;
  *out = nullptr;
  perm_server* s = new perm_server();
  s->device = device;
  s->slots = slots;
  s->t0 = Clock::now();
  if (slice_steps) s->slice_steps = slice_steps;
  if (memory_budget == 0) {
    size_t free_b = 0, total_b = 0;
    cudaSetDevice(device);
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
      cudaGetLastError();
      delete s;
      return PERM_ECUDA;
    }
    memory_budget = free_b / 2;
  }
  s->budget = memory_budget;
  for (int i = 0; i < slots; i++) {
    perm_ctx* c = nullptr;
    int rc = perm_ctx_create(device, &c);
    if (rc != PERM_OK) {
      for (perm_ctx* p : s->ctxs) perm_ctx_destroy(p);
      delete s;
      return rc;
    }
    s->ctxs.push_back(c);
  }
  for (int i = 0; i < slots; i++) s->workers.emplace_back(worker, s, i);
  *out = s;
  return PERM_OK;
}

extern "C" int perm_server_submit(perm_server* s, const perm_request* req, uint64_t* ticket) {
  if (!s || !req || !ticket) return PERM_EINVAL;
  Job* j = new Job();
  j->req = *req;
  const int n = req->n;
  if (n >= 1 && n <= 4096 && req->mat) j->mat.assign(req->mat, req->mat + (size_t)n * n);
  j->req.mat = nullptr;
  j->bytes = request_bytes(*req);
  j->t_submit = Clock::now();
  {
    std::lock_guard<std::mutex> lock(s->mu);
    j->ticket = s->next_ticket++;
    j->resp.t_submit_ms = ms_since(s, j->t_submit);
    s->jobs[j->ticket] = j;
    s->pending.push_back(j);
    s->submitted++;
    *ticket = j->ticket;
  }
  s->cv_work.notify_one();
  return PERM_OK;
}

extern "C" int perm_server_wait(perm_server* s, uint64_t ticket, int timeout_ms, perm_response* out) {
  if (!s || !out) return PERM_EINVAL;
  std::unique_lock<std::mutex> lock(s->mu);
  auto it = s->jobs.find(ticket);
  if (it == s->jobs.end()) return PERM_EINVAL;
  Job* j = it->second;
  auto ready = [&] { return j->done; };
  s->waiters++;
  bool got = true;
  if (timeout_ms < 0)
    s->cv_done.wait(lock, ready);
  else
    got = s->cv_done.wait_for(lock, std::chrono::milliseconds(timeout_ms), ready);
  s->waiters--;
  if (s->stop) s->cv_done.notify_all();  // perm_server_destroy waits for the last waiter
  if (!got) return PERM_ETIMEOUT;
  *out = j->resp;
  s->jobs.erase(ticket);
  delete j;
  return PERM_OK;
}

extern "C" int perm_server_stats(perm_server* s, double* out5) {
  if (!s || !out5) return PERM_EINVAL;
  std::lock_guard<std::mutex> lock(s->mu);
  out5[0] = (double)s->submitted;
  out5[1] = (double)s->completed;
  out5[2] = (double)s->in_flight;
  out5[3] = (double)s->pending.size();
  out5[4] = (double)s->in_use;
  return PERM_OK;
}

extern "C" void perm_server_destroy(perm_server* s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> lock(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  for (auto& t : s->workers) t.join();
  {
    // requests that never ran end with an error, and threads blocked in
    // perm_server_wait collect their response before anything is freed
    std::unique_lock<std::mutex> lock(s->mu);
    for (Job* j : s->pending) {
      j->resp.status = PERM_EINVAL;
      snprintf(j->resp.message, sizeof j->resp.message, "server destroyed before the request ran");
      j->done = true;
    }
    s->pending.clear();
    s->cv_done.notify_all();
    s->cv_done.wait(lock, [&] { return s->waiters == 0; });
  }
  for (perm_ctx* c : s->ctxs) perm_ctx_destroy(c);
  for (auto& kv : s->jobs) delete kv.second;
  delete s;
}
