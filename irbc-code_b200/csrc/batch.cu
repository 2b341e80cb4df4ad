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
#include <map>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <vector>
#include <cuda_runtime.h>
#include "cohort.h"
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
  // waits for their device work.  status[i] receives member i's own result:
  // 0, or the error of its irbc_step or irbc_sync (a member that fails stops
  // stepping there; the others go on).  Returns the first error, 0 if none.
  int step(const std::vector<irbc_handle*>& members, const std::vector<int64_t>& steps, int64_t chunk,
           std::vector<int>* status = nullptr) {
    std::unique_lock<std::mutex> lk(mu_);
    members_ = &members;
    steps_ = &steps;
    status_.assign(members.size(), 0);
    chunk_ = std::max<int64_t>(1, chunk);
    pending_ = n_;
    ++job_;
    cv_.notify_all();
    done_.wait(lk, [this] { return pending_ == 0; });
    members_ = nullptr;
    steps_ = nullptr;
    int first = 0;
    for (int e : status_)
      if (e && !first) first = e;
    if (status) *status = status_;
    return first;
  }

 private:
  void run(int t) {
    uint64_t seen = 0;
    for (;;) {
      std::vector<irbc_handle*> mine;
      std::vector<int64_t> todo;
      std::vector<size_t> where;
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
          where.push_back(i);
        }
      }
      std::vector<int> err(mine.size(), 0);
      for (int64_t k = 0;; k += chunk) {
        bool any = false;
        for (size_t i = 0; i < mine.size(); ++i) {
          const int64_t m = std::min(chunk, todo[i] - k);
          if (m <= 0 || err[i]) continue;
          any = true;
          err[i] = irbc_step(mine[i], m);
        }
        if (!any) break;
      }
      for (size_t i = 0; i < mine.size(); ++i) {
        const int e = irbc_sync(mine[i]);
        if (!err[i]) err[i] = e;
      }
      {
        std::lock_guard<std::mutex> lk(mu_);
        for (size_t i = 0; i < mine.size(); ++i) status_[where[i]] = err[i];
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
  std::vector<int> status_;
  uint64_t job_ = 0;
  int pending_ = 0;
  bool stop_ = false;
};

double now_s(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// Advances members[i] by steps[i] and waits for their device work;
// status[i] receives member i's own result.  Under a fused schedule, the
// members that can share a cohort (FP32, same phase, same step count: equal
// irbc::cohort_key) go through one launch per phase, a cohort per group;
// the others through the pool of host threads, whose work overlaps the
// cohorts' on the GPU.  Returns the first error, 0 if none.
int step_members(StepPool& pool, std::vector<irbc::Cohort*>& cohorts, const std::vector<irbc_handle*>& members,
                 const std::vector<int64_t>& steps, const irbc_schedule& sched, std::vector<int>& status) {
  status.assign(members.size(), 0);
  if (!sched.fused) return pool.step(members, steps, sched.chunk, &status);
  std::map<std::pair<int64_t, int64_t>, std::vector<size_t>> groups;
  std::vector<size_t> rest;
  for (size_t i = 0; i < members.size(); ++i) {
    const int64_t k = irbc::cohort_key(members[i]);
    if (k < 0 || steps[i] <= 0) rest.push_back(i);
    else groups[{k, steps[i]}].push_back(i);
  }
  size_t g = 0;
  for (auto& kv : groups) {
    if (cohorts.size() <= g) {
      int dev = 0;
      cudaGetDevice(&dev);
      cohorts.push_back(irbc::cohort_create(dev));
    }
    std::vector<irbc_handle*> hs;
    for (size_t i : kv.second) hs.push_back(members[i]);
    std::vector<int> st;
    const int rc = irbc::cohort_step(cohorts[g], hs, kv.first.second, st);
    for (size_t j = 0; j < kv.second.size(); ++j) status[kv.second[j]] = rc ? rc : st[j];
    ++g;
  }
  if (!rest.empty()) {
    std::vector<irbc_handle*> hs;
    std::vector<int64_t> ns;
    for (size_t i : rest) { hs.push_back(members[i]); ns.push_back(steps[i]); }
    std::vector<int> st;
    pool.step(hs, ns, sched.chunk, &st);
    for (size_t j = 0; j < rest.size(); ++j) status[rest[j]] = st[j];
  }
  // the cohorts' device work (and each member's health word)
  for (auto& kv : groups)
    for (size_t i : kv.second)
      if (!status[i]) status[i] = irbc_sync(members[i]);
  for (int e : status)
    if (e) return e;
  return 0;
}

}  // namespace

// ---- batches --------------------------------------------------------------
struct irbc_batch {
  std::vector<irbc_handle*> members;
  StepPool pool;
  std::vector<irbc::Cohort*> cohorts;    // fused schedules: one per group of members
  irbc_schedule sched{2, 1, 0, 24, 1};  // the handles' defaults, the pool's chunk, fused
  bool scheduled = false;               // set explicitly: members added later get it too
  explicit irbc_batch(int nthreads) : pool(nthreads) {}
  ~irbc_batch() {
    for (irbc::Cohort* c : cohorts) irbc::cohort_destroy(c);
  }
};

namespace {
bool valid_schedule(const irbc_schedule& s) {
  return (s.streams == 1 || s.streams == 2) && (s.membrane == 1 || s.membrane == 2) &&
         (s.graphs == 0 || s.graphs == 1) && s.chunk >= 24 && s.chunk <= 2400 && s.chunk % 24 == 0 &&
         (s.fused == 0 || s.fused == 1);
}

int apply_schedule(irbc_handle* h, const irbc_schedule& s) {
  int rc = irbc_set_streams(h, s.streams);
  if (!rc) rc = irbc_set_membrane_kernels(h, s.membrane);
  if (!rc) rc = irbc_set_graphs(h, s.graphs);
  return rc;
}
}  // namespace

extern "C" int irbc_batch_create(int32_t nthreads, irbc_batch** out) {
  if (!out || nthreads < 1 || nthreads > 256) return IRBC_ERR_ARG;
  *out = new irbc_batch(nthreads);
  return 0;
}

extern "C" void irbc_batch_destroy(irbc_batch* b) { delete b; }

extern "C" int irbc_batch_add(irbc_batch* b, irbc_handle* h) {
  if (!b || !h) return IRBC_ERR_ARG;
  if (std::find(b->members.begin(), b->members.end(), h) != b->members.end()) return IRBC_ERR_ARG;
  if (b->scheduled) {
    const int rc = apply_schedule(h, b->sched);
    if (rc) return rc;
  }
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
  std::vector<int> status;
  return step_members(b->pool, b->cohorts, b->members, steps, b->sched, status);
}

// ---- launch schedules and the autotuner --------------------------------------
extern "C" int irbc_batch_set_schedule(irbc_batch* b, const irbc_schedule* s) {
  if (!b || !s || !valid_schedule(*s)) return IRBC_ERR_ARG;
  for (irbc_handle* h : b->members) {
    const int rc = apply_schedule(h, *s);
    if (rc) {
      for (irbc_handle* g : b->members) apply_schedule(g, b->sched);
      return rc;
    }
  }
  b->sched = *s;
  b->scheduled = true;
  return 0;
}

extern "C" int irbc_batch_get_schedule(const irbc_batch* b, irbc_schedule* s) {
  if (!b || !s) return IRBC_ERR_ARG;
  *s = b->sched;
  return 0;
}

extern "C" int irbc_tune_select(int32_t n, irbc_tune_measure measure, void* ctx, int32_t repeats, double margin,
                                double* medians, int32_t* best) {
  if (n < 1 || !measure || !best || repeats < 1 || repeats > 64 || !(margin >= 0.0 && margin < 1.0))
    return IRBC_ERR_ARG;
  int32_t win = -1;
  double win_t = 0.0;
  std::vector<double> t;
  for (int32_t i = 0; i < n; ++i) {
    t.clear();
    int rc = 0;
    for (int32_t r = 0; r <= repeats && !rc; ++r) {
      double sec = 0.0;
      rc = measure(i, ctx, &sec);
      if (rc) break;
      if (!(sec >= 0.0 && sec < 1e30)) return IRBC_ERR_ARG;  // not a time
      if (r > 0) t.push_back(sec);                          // run 0 warms up
    }
    if (rc && rc != IRBC_ERR_CAPACITY) return rc;
    double med = -1.0;
    if (!rc) {
      std::sort(t.begin(), t.end());
      const size_t m = t.size();
      med = (m % 2) ? t[m / 2] : 0.5 * (t[m / 2 - 1] + t[m / 2]);
      if (win < 0 || med < (1.0 - margin) * win_t) {
        win = i;
        win_t = med;
      }
    }
    if (medians) medians[i] = med;
  }
  if (win < 0) return IRBC_ERR_CAPACITY;
  *best = win;
  return 0;
}

namespace {
struct TuneRun {
  irbc_batch* b = nullptr;
  std::vector<irbc_schedule> cands;
  int64_t trial = 0, taken = 0;
};

// one timed stretch of trial steps of every member under candidate i; the
// schedule is applied first (a no-op for the one already in place, so
// captured graphs survive between the runs of one candidate)
int measure_schedule(int32_t i, void* ctx, double* seconds) {
  TuneRun* run = static_cast<TuneRun*>(ctx);
  irbc_batch* b = run->b;
  const irbc_schedule& s = run->cands[i];
  const int rc = irbc_batch_set_schedule(b, &s);
  if (rc) return rc;
  std::vector<int64_t> steps(b->members.size(), run->trial);
  std::vector<int> status;
  const auto t0 = std::chrono::steady_clock::now();
  const int e = step_members(b->pool, b->cohorts, b->members, steps, s, status);
  *seconds = now_s(t0);
  if (!e) run->taken += run->trial;
  return e;
}
}  // namespace

extern "C" int irbc_batch_autotune(irbc_batch* b, int64_t trial_steps, int32_t repeats, double margin,
                                   irbc_schedule* best, int64_t* steps_taken) {
  if (!b || trial_steps < 1 || repeats < 1 || repeats > 64 || !(margin >= 0.0 && margin < 1.0))
    return IRBC_ERR_ARG;
  if (b->members.empty()) return IRBC_ERR_STATE;
  TuneRun run;
  run.b = b;
  run.trial = trial_steps;
  irbc_schedule cur = b->sched;
  static const int32_t kChunks[] = {24, 96, 240};
  int rc = 0;
  for (int field = -1; field < 4 && !rc; ++field) {
    run.cands.assign(1, cur);
    irbc_schedule alt = cur;
    if (field == -1) {
      alt.fused = 1 - cur.fused;
      run.cands.push_back(alt);
    } else if (field == 0) {
      alt.membrane = 3 - cur.membrane;
      run.cands.push_back(alt);
    } else if (field == 1) {
      alt.streams = 3 - cur.streams;
      run.cands.push_back(alt);
    } else if (field == 2) {
      alt.graphs = 1 - cur.graphs;
      run.cands.push_back(alt);
    } else {
      for (int32_t k : kChunks)
        if (k != cur.chunk) {
          alt.chunk = k;
          run.cands.push_back(alt);
        }
    }
    int32_t w = 0;
    rc = irbc_tune_select((int32_t)run.cands.size(), measure_schedule, &run, repeats, margin, nullptr, &w);
    if (!rc) cur = run.cands[w];
  }
  if (!rc) rc = irbc_batch_set_schedule(b, &cur);
  if (!rc && best) *best = cur;
  if (steps_taken) *steps_taken = run.taken;
  return rc;
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
  // for simulations admitted from now on; the pool by default: requests
  // differ in box, mesh and list lengths, and a cohort's phases wait for
  // its slowest member where the pool's streams overlap them
  irbc_schedule sched{2, 1, 0, 24, 0};
  bool scheduled = false;                // set explicitly: applied at admission
  StepPool pool;
  std::vector<irbc::Cohort*> cohorts;    // fused schedules: one per group of simulations
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
  std::mutex mu;
  std::condition_variable cv;
  std::deque<Request> pending;  // waiting for room in the budget
  // set up (created and initialised on the device), waiting for the next
  // round; a failed set-up carries its error
  struct Ready {
    Request r;
    irbc_handle* h = nullptr;
    int rc = 0;
    double t_start = 0;
  };
  std::deque<Ready> ready;
  int32_t setting_up = 0;       // requests in the hands of the set-up threads
  std::vector<Active> active;   // owned by the stepping loop
  std::deque<irbc_result> results;
  // finished simulations handed out with keep = 1: their memory stays
  // charged to the budget until irbc_server_release
  std::vector<std::pair<irbc_handle*, int64_t>> kept;
  int64_t n_active = 0;  // active.size(), readable under mu while the loop runs
  int64_t next_id = 1;
  int64_t particle_steps = 0;
  bool stop = false;
  std::thread loop;
  std::vector<std::thread> setup;
  explicit irbc_server(int nthreads) : pool(nthreads) {}
};

namespace {
constexpr int kSetupThreads = 2;

// a result for request r (under no lock); h is destroyed unless it is
// handed out
void finish_request(irbc_server* s, const Request& r, irbc_handle* h, int32_t status, double t_start) {
  irbc_result res{};
  res.id = r.id;
  res.status = status;
  res.steps = r.nsteps;
  res.ns = r.p.Ns;
  res.t_submit = r.t_submit;
  res.t_start = t_start;
  res.t_end = now_s(s->t0);
  if (h && status == 0) irbc_observables(h, res.obs, 8);
  const bool hand_out = h && r.keep && status == 0;
  if (hand_out) {
    res.handle = h;
  } else if (h) {
    irbc_destroy(h);
  }
  std::lock_guard<std::mutex> lk(s->mu);
  if (hand_out) s->kept.push_back({h, r.footprint});
  else s->used -= r.footprint;
  s->results.push_back(res);
  s->cv.notify_all();
}

// whether the head of the queue can be admitted now (under s->mu)
bool can_admit(const irbc_server* s) {
  return !s->pending.empty() && s->used + s->pending.front().footprint <= s->budget &&
         s->n_active + (int64_t)s->ready.size() + s->setting_up < s->max_active;
}

// A set-up thread: admits the head of the queue as soon as the budget has
// room for it, creates and initialises it on the device (solvent draw,
// inside/outside ray test, lists, knobs) while the admitted simulations go
// on stepping, and hands it to the stepping loop for its next round.
void setup_loop(irbc_server* s) {
  cudaSetDevice(s->device);
  for (;;) {
    Request r;
    irbc_schedule sched;
    bool scheduled;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      s->cv.wait(lk, [s] { return s->stop || can_admit(s); });
      if (s->stop) return;
      r = std::move(s->pending.front());
      s->pending.pop_front();
      s->used += r.footprint;
      s->setting_up += 1;
      sched = s->sched;
      scheduled = s->scheduled;
    }
    irbc_server::Ready out;
    out.t_start = now_s(s->t0);
    int rc = irbc_create(&r.p, &out.h);
    if (!rc)
      rc = irbc_init(out.h, r.V.data(), (int32_t)(r.V.size() / 3), r.E.data(), (int32_t)(r.E.size() / 2),
                     r.T.data(), (int32_t)(r.T.size() / 3), r.nknobs);
    // the one-block membrane form only where the mesh fits it
    if (!rc && scheduled && apply_schedule(out.h, sched)) {
      irbc_schedule wide = sched;
      wide.membrane = 1;
      rc = apply_schedule(out.h, wide);
    }
    // its set-up work is done before it joins a round
    if (!rc) rc = irbc_sync(out.h);
    out.rc = rc;
    out.r = std::move(r);
    std::lock_guard<std::mutex> lk(s->mu);
    s->ready.push_back(std::move(out));
    s->setting_up -= 1;
    s->cv.notify_all();
  }
}

// one round of steps for the admitted simulations; the ones that finish
// (or fail) are retired
void step_active(irbc_server* s, const irbc_schedule& sched) {
  std::vector<irbc_handle*> hs;
  std::vector<int64_t> steps;
  for (const Active& a : s->active) {
    hs.push_back(a.h);
    steps.push_back(std::min(s->round, a.r.nsteps - a.done));
  }
  // each simulation's own status: one that fails (a CUDA error, or the
  // health check of irbc_sync) is retired with it, the others go on
  std::vector<int> status;
  step_members(s->pool, s->cohorts, hs, steps, sched, status);
  std::vector<Active> still;
  int64_t work = 0;
  for (size_t i = 0; i < s->active.size(); ++i) {
    Active& a = s->active[i];
    a.done += steps[i];
    work += steps[i] * a.r.p.Ns;
    if (status[i] || a.done >= a.r.nsteps) finish_request(s, a.r, a.h, status[i], a.t_start);
    else still.push_back(std::move(a));
  }
  std::lock_guard<std::mutex> lk(s->mu);
  s->particle_steps += work;
  s->active = std::move(still);
  s->n_active = (int64_t)s->active.size();
  s->cv.notify_all();  // room under max_active
}

// The stepping loop: at each round boundary the simulations set up since
// the last one join; then every admitted simulation takes the round's steps.
void serve_loop(irbc_server* s) {
  cudaSetDevice(s->device);
  for (;;) {
    std::deque<irbc_server::Ready> joined;
    irbc_schedule sched;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      s->cv.wait(lk, [s] { return s->stop || !s->active.empty() || !s->ready.empty(); });
      if (s->stop) break;
      joined.swap(s->ready);
      sched = s->sched;
    }
    for (irbc_server::Ready& q : joined) {
      if (q.rc) {
        finish_request(s, q.r, q.h, q.rc, q.t_start);
        continue;
      }
      Active a;
      a.r = std::move(q.r);
      a.h = q.h;
      a.t_start = q.t_start;
      if (a.r.nsteps == 0) {
        finish_request(s, a.r, a.h, 0, a.t_start);
        continue;
      }
      std::lock_guard<std::mutex> lk(s->mu);
      s->active.push_back(std::move(a));
      s->n_active = (int64_t)s->active.size();
    }
    if (!s->active.empty()) step_active(s, sched);
  }
  for (Active& a : s->active) irbc_destroy(a.h);
  for (irbc::Cohort* c : s->cohorts) irbc::cohort_destroy(c);
  s->cohorts.clear();
  std::lock_guard<std::mutex> lk(s->mu);
  s->active.clear();
  s->n_active = 0;
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
  for (int k = 0; k < kSetupThreads; ++k) s->setup.emplace_back(setup_loop, s);
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
  out[1] = s->n_active;
  out[2] = (int64_t)s->results.size();
  out[3] = s->used;
  out[4] = s->budget;
  out[5] = s->particle_steps;
  return 0;
}

extern "C" int irbc_server_set_schedule(irbc_server* s, const irbc_schedule* sched) {
  if (!s || !sched || !valid_schedule(*sched)) return IRBC_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  s->sched = *sched;
  s->scheduled = true;
  return 0;
}

extern "C" double irbc_server_clock(irbc_server* s) { return s ? now_s(s->t0) : 0.0; }

extern "C" int irbc_server_release(irbc_server* s, irbc_handle* h) {
  if (!s || !h) return IRBC_ERR_ARG;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = std::find_if(s->kept.begin(), s->kept.end(),
                           [h](const std::pair<irbc_handle*, int64_t>& k) { return k.first == h; });
    if (it == s->kept.end()) return IRBC_ERR_ARG;
    // a result not yet polled still names the handle: it may not go
    for (const irbc_result& r : s->results)
      if (r.handle == h) return IRBC_ERR_STATE;
    s->used -= it->second;
    s->kept.erase(it);
  }
  irbc_destroy(h);
  s->cv.notify_all();  // the memory may admit a pending request
  return 0;
}

extern "C" void irbc_server_destroy(irbc_server* s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv.notify_all();
  s->loop.join();
  for (std::thread& th : s->setup) th.join();
  // set up but never stepped
  for (irbc_server::Ready& q : s->ready)
    if (q.h) irbc_destroy(q.h);
  // handles of results never polled were never handed out
  for (irbc_result& r : s->results)
    if (r.handle) irbc_destroy(r.handle);
  delete s;
}
