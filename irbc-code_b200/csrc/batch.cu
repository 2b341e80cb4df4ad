// batch.cu -- many independent simulations on one GPU (host code only).
//
// A batch steps its member simulations together: a pool of host threads
// issues each member's steps (irbc_step, whose 24-step stretches are single
// captured graphs), so the members' kernels overlap on the GPU through
// their own streams.  A server admits simulation requests as device memory
// frees up (footprint from irbc_footprint_bytes), keeps their state
// resident, advances all admitted simulations in rounds through the same
// machinery, and returns each one's observables (or its handle) when it
// finishes.  Nothing here changes what a simulation computes: each member
// is stepped exactly as it would be alone.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <vector>
#include <cuda_runtime.h>
#include "irbc.h"

namespace {

// a pool of host threads that each step a share of a member list
class StepPool {
 public:
  explicit StepPool(int nthreads) : n_(std::max(1, nthreads)) {
    for (int t = 0; t < n_; ++t) threads_.emplace_back([this, t] { run(t); });
  }
  ~StepPool() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    for (auto& th : threads_) th.join();
  }
  // advances members[i] by steps[i] (interleaved in chunks of `chunk`) and
  // waits for their device work; returns the first error, 0 if none
  int step(const std::vector<irbc_handle*>& members, const std::vector<int64_t>& steps, int64_t chunk) {
    std::unique_lock<std::mutex> lk(mu_);
    members_ = &members;
    steps_ = &steps;
    chunk_ = std::max<int64_t>(1, chunk);
    first_error_ = 0;
    pending_ = n_;
    ++job_;
    cv_.notify_all();
    done_.wait(lk, [this] { return pending_ == 0; });
    members_ = nullptr;
    steps_ = nullptr;
    return first_error_;
  }

 private:
  void run(int t) {
    uint64_t seen = 0;
    for (;;) {
      std::vector<irbc_handle*> mine;
      std::vector<int64_t> todo;
      int64_t chunk;
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return stop_ || job_ != seen; });
        if (stop_) return;
        seen = job_;
        chunk = chunk_;
        for (size_t i = t; i < members_->size(); i += n_) {
          mine.push_back((*members_)[i]);
          todo.push_back((*steps_)[i]);
        }
      }
      int err = 0;
      for (int64_t k = 0; !err; k += chunk) {
        bool any = false;
        for (size_t i = 0; i < mine.size() && !err; ++i) {
          const int64_t m = std::min(chunk, todo[i] - k);
          if (m <= 0) continue;
          any = true;
          err = irbc_step(mine[i], m);
        }
        if (!any) break;
      }
      for (irbc_handle* h : mine) {
        const int e = irbc_sync(h);
        if (!err) err = e;
      }
      {
        std::lock_guard<std::mutex> lk(mu_);
        if (err && !first_error_) first_error_ = err;
        if (--pending_ == 0) done_.notify_all();
      }
    }
  }

  int n_;
  std::vector<std::thread> threads_;
  std::mutex mu_;
  std::condition_variable cv_, done_;
  const std::vector<irbc_handle*>* members_ = nullptr;
  const std::vector<int64_t>* steps_ = nullptr;
  int64_t chunk_ = 24;
  uint64_t job_ = 0;
  int pending_ = 0, first_error_ = 0;
  bool stop_ = false;
};

double now_s(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace

// ---- batches --------------------------------------------------------------
struct irbc_batch {
  std::vector<irbc_handle*> members;
  StepPool pool;
  explicit irbc_batch(int nthreads) : pool(nthreads) {}
};

extern "C" int irbc_batch_create(int32_t nthreads, irbc_batch** out) {
  if (!out || nthreads < 1 || nthreads > 256) return IRBC_ERR_ARG;
  *out = new irbc_batch(nthreads);
  return 0;
}

extern "C" void irbc_batch_destroy(irbc_batch* b) { delete b; }

extern "C" int irbc_batch_add(irbc_batch* b, irbc_handle* h) {
  if (!b || !h) return IRBC_ERR_ARG;
  if (std::find(b->members.begin(), b->members.end(), h) != b->members.end()) return IRBC_ERR_ARG;
  b->members.push_back(h);
  return 0;
}

extern "C" int irbc_batch_remove(irbc_batch* b, irbc_handle* h) {
  if (!b || !h) return IRBC_ERR_ARG;
  auto it = std::find(b->members.begin(), b->members.end(), h);
  if (it == b->members.end()) return IRBC_ERR_ARG;
  b->members.erase(it);
  return 0;
}

extern "C" int32_t irbc_batch_size(const irbc_batch* b) { return b ? (int32_t)b->members.size() : 0; }

extern "C" int irbc_batch_step(irbc_batch* b, int64_t n) {
  if (!b || n < 0) return IRBC_ERR_ARG;
  std::vector<int64_t> steps(b->members.size(), n);
  return b->pool.step(b->members, steps, 24);
}

// ---- server -------------------------------------------------------------------
namespace {
struct Request {
  int64_t id = 0;
  irbc_params p{};
  std::vector<double> V;
  std::vector<int32_t> E, T;
  int32_t nknobs = 0;
  int64_t nsteps = 0;
  int32_t keep = 0;
  int64_t footprint = 0;
  double t_submit = 0;
};
struct Active {
  Request r;
  irbc_handle* h = nullptr;
  int64_t done = 0;
  double t_start = 0;
};
}  // namespace

struct irbc_server {
  int32_t device = 0;
  int64_t budget = 0, used = 0;
  int64_t round = 240;
  int32_t max_active = 256;
  StepPool pool;
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
  std::mutex mu;
  std::condition_variable cv;
  std::deque<Request> pending;
  std::vector<Active> active;
  std::deque<irbc_result> results;
  int64_t next_id = 1;
  int64_t particle_steps = 0;
  bool stop = false;
  std::thread loop;
  explicit irbc_server(int nthreads) : pool(nthreads) {}
};

namespace {
// admits what fits, steps one round, retires what finished; returns false
// when there is nothing to do
bool serve_round(irbc_server* s) {
  std::vector<Request> admit;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    while (!s->pending.empty() && (int32_t)(s->active.size() + admit.size()) < s->max_active &&
           s->used + s->pending.front().footprint <= s->budget) {
      s->used += s->pending.front().footprint;
      admit.push_back(std::move(s->pending.front()));
      s->pending.pop_front();
    }
  }
  auto finish = [s](const Request& r, irbc_handle* h, int32_t status, double t_start) {
    irbc_result res{};
    res.id = r.id;
    res.status = status;
    res.steps = r.nsteps;
    res.ns = r.p.Ns;
    res.t_submit = r.t_submit;
    res.t_start = t_start;
    res.t_end = now_s(s->t0);
    if (h && status == 0) irbc_observables(h, res.obs, 8);
    if (h && r.keep && status == 0) {
      res.handle = h;
    } else if (h) {
      irbc_destroy(h);
    }
    std::lock_guard<std::mutex> lk(s->mu);
    s->used -= r.footprint;
    s->results.push_back(res);
    s->cv.notify_all();
  };
  for (Request& r : admit) {
    const double t_start = now_s(s->t0);
    irbc_handle* h = nullptr;
    int rc = irbc_create(&r.p, &h);
    if (!rc) rc = irbc_init(h, r.V.data(), (int32_t)(r.V.size() / 3), r.E.data(), (int32_t)(r.E.size() / 2),
                            r.T.data(), (int32_t)(r.T.size() / 3), r.nknobs);
    if (rc) {
      finish(r, h, rc, t_start);
      continue;
    }
    Active a;
    a.r = std::move(r);
    a.h = h;
    a.t_start = t_start;
    s->active.push_back(std::move(a));
  }
  if (s->active.empty()) return !admit.empty();
  std::vector<irbc_handle*> hs;
  std::vector<int64_t> steps;
  for (const Active& a : s->active) {
    hs.push_back(a.h);
    steps.push_back(std::min(s->round, a.r.nsteps - a.done));
  }
  const int rc = s->pool.step(hs, steps, 24);
  std::vector<Active> still;
  for (size_t i = 0; i < s->active.size(); ++i) {
    Active& a = s->active[i];
    a.done += steps[i];
    {
      std::lock_guard<std::mutex> lk(s->mu);
      s->particle_steps += steps[i] * a.r.p.Ns;
    }
    if (rc || a.done >= a.r.nsteps) finish(a.r, a.h, rc, a.t_start);
    else still.push_back(std::move(a));
  }
  s->active = std::move(still);
  return true;
}

void serve_loop(irbc_server* s) {
  cudaSetDevice(s->device);
  for (;;) {
    {
      std::unique_lock<std::mutex> lk(s->mu);
      s->cv.wait(lk, [s] { return s->stop || !s->pending.empty() || !s->active.empty(); });
      if (s->stop) break;
    }
    serve_round(s);
  }
  for (Active& a : s->active) irbc_destroy(a.h);
  s->active.clear();
}
}  // namespace

extern "C" int irbc_server_create(int32_t device, int64_t budget_bytes, int32_t nthreads, int64_t round_steps,
                                  irbc_server** out) {
  if (!out || nthreads < 1 || nthreads > 256 || round_steps < 1) return IRBC_ERR_ARG;
  if (cudaSetDevice(device) != cudaSuccess) return IRBC_ERR_CUDA;
  if (budget_bytes <= 0) {
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) return IRBC_ERR_CUDA;
    budget_bytes = (int64_t)(0.85 * (double)fr);
  }
  irbc_server* s = new irbc_server(nthreads);
  s->device = device;
  s->budget = budget_bytes;
  s->round = round_steps;
  s->loop = std::thread(serve_loop, s);
  *out = s;
  return 0;
}

extern "C" int irbc_server_submit(irbc_server* s, const irbc_params* p, const double* V, int32_t nv,
                                  const int32_t* E, int32_t ne, const int32_t* T, int32_t nt, int32_t nknobs,
                                  int64_t nsteps, int32_t keep, int64_t* id) {
  if (!s || !p || !V || !E || !T || nv <= 0 || ne <= 0 || nt <= 0 || nsteps < 0) return IRBC_ERR_ARG;
  Request r;
  r.p = *p;
  r.p.device = s->device;
  r.V.assign(V, V + 3 * (size_t)nv);
  r.E.assign(E, E + 2 * (size_t)ne);
  r.T.assign(T, T + 3 * (size_t)nt);
  r.nknobs = nknobs;
  r.nsteps = nsteps;
  r.keep = keep;
  r.footprint = irbc_footprint_bytes(p, nv, ne, nt);
  if (r.footprint > s->budget) return IRBC_ERR_CAPACITY;  // would never be admitted
  std::lock_guard<std::mutex> lk(s->mu);
  r.id = s->next_id++;
  r.t_submit = now_s(s->t0);
  if (id) *id = r.id;
  s->pending.push_back(std::move(r));
  s->cv.notify_all();
  return 0;
}

extern "C" int32_t irbc_server_poll(irbc_server* s, irbc_result* out, int32_t max, double wait_s) {
  if (!s || !out || max <= 0) return IRBC_ERR_ARG;
  std::unique_lock<std::mutex> lk(s->mu);
  if (s->results.empty() && wait_s > 0)
    s->cv.wait_for(lk, std::chrono::duration<double>(wait_s), [s] { return !s->results.empty(); });
  int32_t n = 0;
  while (n < max && !s->results.empty()) {
    out[n++] = s->results.front();
    s->results.pop_front();
  }
  return n;
}

extern "C" int irbc_server_status(irbc_server* s, int64_t out[6]) {
  if (!s || !out) return IRBC_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  out[0] = (int64_t)s->pending.size();
  out[1] = (int64_t)s->active.size();
  out[2] = (int64_t)s->results.size();
  out[3] = s->used;
  out[4] = s->budget;
  out[5] = s->particle_steps;
  return 0;
}

extern "C" double irbc_server_clock(irbc_server* s) { return s ? now_s(s->t0) : 0.0; }

extern "C" void irbc_server_destroy(irbc_server* s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv.notify_all();
  s->loop.join();
  delete s;
}
