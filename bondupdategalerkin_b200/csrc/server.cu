// Serving BUG time-evolution jobs on one GPU: a pool of worker threads, each with its own engine
// context (stream, caching allocator, descriptor staging), taking jobs from one FIFO queue.
//
// The reference has no serving layer; this is the caller of `cbe_bug_step!` that the batched and
// served workloads need. Design:
//   * a job is `nsteps` steps of one chain. The caller's `load` callback builds the job's state and
//     MPO on the worker's context (so every tensor of a job lives on one stream), the worker runs
//     the steps through `bug_mps_step`, and the caller's `done` callback reads the result before
//     the worker frees the job's tensors;
//   * jobs arriving while others run are admitted as soon as a worker is idle and the sum of the
//     running jobs' projected HBM footprints plus the new one fits the budget (FIFO: a job that
//     does not fit waits, and so do the jobs behind it; a job is always admitted when nothing
//     runs, so an oversized one cannot block forever);
//   * the running jobs' kernels overlap on the device (one stream per worker) and their host-side
//     sweep logic overlaps on the host cores; every job's arithmetic is the same as alone (the
//     kernels are deterministic and each job draws from its own generator), so a job's result
//     does not depend on the mix;
//   * per-step latency (host wall clock around the step, the stream drained) and per-job submit /
//     start / end times are recorded for p50 / p99 reporting.
#include "engine.h"

#include <chrono>
#include <condition_variable>
#include <deque>
#include <functional>
#include <mutex>
#include <thread>

namespace {

using Clock = std::chrono::steady_clock;

struct Job {
  bug_job_spec spec{};
  int state = BUG_JOB_QUEUED;
  int status = BUG_OK;
  bool cancel = false;
  int worker = -1;
  int steps_done = 0;
  double t_submit = 0, t_start = 0, t_end = 0;
  std::vector<double> step_s;
  std::string error;
};

}  // namespace

struct bug_server {
  int device = 0;
  int64_t budget = 0;
  int64_t admitted = 0;
  int running = 0;
  bool stop = false;
  int64_t next_id = 1;
  Clock::time_point t0 = Clock::now();
  std::mutex mu;
  std::condition_variable work_cv;  // workers wait for admissible jobs
  std::condition_variable done_cv;  // waiters wait for job completion
  std::deque<int64_t> queue;
  std::map<int64_t, std::unique_ptr<Job>> jobs;
  std::vector<std::thread> threads;
  std::vector<bug_ctx*> ctxs;
  // The workers' contexts share one stream, and their stage lists go through one combiner: the
  // lists the running jobs drain at about the same time become one launch (a cluster per job).
  bugi::Combiner combiner;
  cudaStream_t shared = nullptr;

  double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }

  // The head of the queue, if it may start now (caller holds mu).
  bool head_admissible() const {
    if (queue.empty()) return false;
    const Job& j = *jobs.at(queue.front());
    return running == 0 || admitted + j.spec.footprint_bytes <= budget;
  }

  void run_job(int w, int64_t id, Job& job);
  void worker(int w);
};

void bug_server::run_job(int w, int64_t id, Job& job) {
  (void)id;
  bug_ctx* ctx = ctxs[w];
  if (shared) combiner.job_begin();
  struct End {
    bug_server* s;
    ~End() {
      if (s->shared) s->combiner.job_end();
    }
  } end_{this};
  std::vector<bug_tensor*> psi(BUG_MAX_SITES + 1, nullptr), mpo(BUG_MAX_SITES + 1, nullptr);
  std::vector<bug_tensor*> io(BUG_MAX_SITES + 1, nullptr);
  int L = 0, center = 0;
  int rc = job.spec.load(job.spec.user, ctx, &L, psi.data(), &center, mpo.data());
  if (rc == BUG_OK && (L < 2 || L > BUG_MAX_SITES + 1)) rc = BUG_EINVAL;
  if (rc != BUG_OK) {
    std::lock_guard<std::mutex> lk(mu);
    job.status = rc;
    job.error = "the job's load callback failed";
  }
  bug_step_info info{};
  for (int s = 0; rc == BUG_OK && s < job.spec.nsteps; ++s) {
    {
      std::lock_guard<std::mutex> lk(mu);
      if (job.cancel) break;
    }
    const double t1 = now();
    for (int i = 0; i < L; ++i) io[i] = psi[i];
    int nlog = 0;
    rc = bug_mps_step(ctx, L, io.data(), &center, mpo.data(), job.spec.tau_re, job.spec.tau_im,
                      &job.spec.params, job.spec.draw, job.spec.draw_user, &info, nullptr, 0, &nlog);
    if (rc == BUG_OK) rc = bug_ctx_synchronize(ctx);
    const double t2 = now();
    if (rc != BUG_OK) {
      std::lock_guard<std::mutex> lk(mu);
      job.status = rc;
      job.error = bug_last_error();
      break;
    }
    for (int i = 0; i < L; ++i)
      if (io[i]) {  // a replaced site: the step hands back a new handle, the old one is ours
        delete psi[i];
        psi[i] = io[i];
      }
    std::lock_guard<std::mutex> lk(mu);
    job.step_s.push_back(t2 - t1);
    job.steps_done = s + 1;
  }
  if (job.spec.done)
    job.spec.done(job.spec.user, ctx, rc == BUG_OK ? BUG_OK : rc, L, psi.data(), center);
  for (int i = 0; i < L; ++i) {
    delete psi[i];
    delete mpo[i];
  }
  bug_ctx_synchronize(ctx);
}

void bug_server::worker(int w) {
  cudaSetDevice(device);
  for (;;) {
    int64_t id = 0;
    Job* job = nullptr;
    {
      std::unique_lock<std::mutex> lk(mu);
      work_cv.wait(lk, [&] { return stop || head_admissible(); });
      if (stop) return;
      id = queue.front();
      queue.pop_front();
      job = jobs.at(id).get();
      admitted += job->spec.footprint_bytes;
      ++running;
      job->state = BUG_JOB_RUNNING;
      job->worker = w;
      job->t_start = now();
    }
    run_job(w, id, *job);
    {
      std::lock_guard<std::mutex> lk(mu);
      admitted -= job->spec.footprint_bytes;
      --running;
      job->t_end = now();
      job->state = job->status != BUG_OK ? BUG_JOB_FAILED
                   : (job->cancel && job->steps_done < job->spec.nsteps) ? BUG_JOB_CANCELLED
                                                                         : BUG_JOB_DONE;
    }
    work_cv.notify_all();
    done_cv.notify_all();
  }
}

using bugi::guard;
using bugi::require;

// Puts the contexts on one new stream with one combiner (their own streams are destroyed).
static void share_stream(int device, std::vector<bug_ctx*>& ctxs, bugi::Combiner& comb,
                         cudaStream_t& shared) {
  BUG_CUDA(cudaSetDevice(device));
  BUG_CUDA(cudaStreamCreateWithFlags(&shared, cudaStreamNonBlocking));
  comb.stream = shared;
  comb.cluster = ctxs[0]->list_cluster;
  for (bug_ctx* c : ctxs) {
    BUG_CUDA(cudaStreamSynchronize(c->stream));
    BUG_CUDA(cudaStreamDestroy(c->stream));
    c->stream = shared;
    c->owns_stream = false;
    c->combiner = &comb;
    BUG_CUDA(cudaEventCreateWithFlags(&c->sync_ev, cudaEventDisableTiming));
  }
}

extern "C" int bug_server_create(int device, int workers, int64_t budget_bytes, bug_server** out) {
  return guard([&] {
    require(out != nullptr && workers >= 1 && workers <= 256 && budget_bytes > 0, "bad argument");
    auto s = std::make_unique<bug_server>();
    s->device = device;
    s->budget = budget_bytes;
    for (int w = 0; w < workers; ++w) {
      bug_ctx* c = nullptr;
      const int rc = bug_ctx_create(device, &c);
      if (rc != BUG_OK) {
        for (bug_ctx* x : s->ctxs) bug_ctx_destroy(x);
        throw bugi::BugError(rc, std::string("bug_server_create: ") + bug_last_error());
      }
      s->ctxs.push_back(c);
    }
    // BUG_SERVER_COMBINE=1 puts the workers on one stream and merges their stage lists into
    // shared launches. Off by default: measured on B200 (32 chains, 16 workers) it ran 3.67
    // chain-steps/s against 10.86 with a stream per worker, whose kernels overlap on the device.
    const char* comb = std::getenv("BUG_SERVER_COMBINE");
    const bool combine = comb && std::string(comb) == "1" && workers <= bugk::kMaxLists &&
                         s->ctxs[0]->list_cluster > 0 && s->ctxs[0]->queue_enabled;
    if (combine) share_stream(device, s->ctxs, s->combiner, s->shared);
    bug_server* raw = s.get();
    for (int w = 0; w < workers; ++w) raw->threads.emplace_back([raw, w] { raw->worker(w); });
    *out = s.release();
  });
}

extern "C" int bug_server_submit(bug_server* s, const bug_job_spec* spec, int64_t* job_id) {
  return guard([&] {
    require(s && spec && job_id && spec->load && spec->draw && spec->nsteps >= 0 &&
                spec->footprint_bytes >= 0,
            "bad argument");
    auto j = std::make_unique<Job>();
    j->spec = *spec;
    {
      std::lock_guard<std::mutex> lk(s->mu);
      require(!s->stop, "the server is shutting down");
      j->t_submit = s->now();
      const int64_t id = s->next_id++;
      s->queue.push_back(id);
      s->jobs[id] = std::move(j);
      *job_id = id;
    }
    s->work_cv.notify_all();
  });
}

extern "C" int bug_server_cancel(bug_server* s, int64_t job_id) {
  return guard([&] {
    require(s != nullptr, "null server");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->jobs.find(job_id);
    require(it != s->jobs.end(), "no such job");
    Job& j = *it->second;
    j.cancel = true;
    if (j.state == BUG_JOB_QUEUED) {  // never started: leaves the queue at once
      for (auto q = s->queue.begin(); q != s->queue.end(); ++q)
        if (*q == job_id) {
          s->queue.erase(q);
          break;
        }
      j.state = BUG_JOB_CANCELLED;
      j.t_start = j.t_end = s->now();
    }
    s->done_cv.notify_all();
    s->work_cv.notify_all();
  });
}

static bool finished_state(int st) { return st == BUG_JOB_DONE || st == BUG_JOB_FAILED || st == BUG_JOB_CANCELLED; }

extern "C" int bug_server_wait(bug_server* s, int64_t job_id, double timeout_s, int* finished) {
  return guard([&] {
    require(s && finished, "bad argument");
    std::unique_lock<std::mutex> lk(s->mu);
    auto all_done = [&] {
      if (job_id > 0) {
        auto it = s->jobs.find(job_id);
        return it == s->jobs.end() || finished_state(it->second->state);
      }
      for (auto& kv : s->jobs)
        if (!finished_state(kv.second->state)) return false;
      return true;
    };
    if (timeout_s < 0) {
      s->done_cv.wait(lk, all_done);
    } else {
      s->done_cv.wait_for(lk, std::chrono::duration<double>(timeout_s), all_done);
    }
    *finished = all_done() ? 1 : 0;
  });
}

extern "C" int bug_server_job_stats(bug_server* s, int64_t job_id, bug_job_stats* out) {
  return guard([&] {
    require(s && out, "bad argument");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->jobs.find(job_id);
    require(it != s->jobs.end(), "no such job");
    const Job& j = *it->second;
    out->state = j.state;
    out->status = j.status;
    out->worker = j.worker;
    out->steps_done = j.steps_done;
    out->t_submit = j.t_submit;
    out->t_start = j.t_start;
    out->t_end = j.t_end;
    double sum = 0.0, mx = 0.0;
    for (double x : j.step_s) {
      sum += x;
      mx = std::max(mx, x);
    }
    out->step_s_sum = sum;
    out->step_s_max = mx;
  });
}

extern "C" int bug_server_step_times(bug_server* s, int64_t job_id, double* out, int cap, int* n) {
  return guard([&] {
    require(s && n && (cap == 0 || out), "bad argument");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->jobs.find(job_id);
    require(it != s->jobs.end(), "no such job");
    const auto& v = it->second->step_s;
    *n = int(v.size());
    for (int i = 0; i < cap && i < int(v.size()); ++i) out[i] = v[size_t(i)];
  });
}

extern "C" int bug_server_destroy(bug_server* s) {
  return guard([&] {
    if (!s) return;
    {
      std::lock_guard<std::mutex> lk(s->mu);
      for (int64_t id : s->queue) {  // queued jobs never start
        Job& j = *s->jobs.at(id);
        j.state = BUG_JOB_CANCELLED;
      }
      s->queue.clear();
      for (auto& kv : s->jobs) kv.second->cancel = true;  // running jobs stop after their step
      s->stop = true;
    }
    s->work_cv.notify_all();
    s->done_cv.notify_all();
    for (auto& t : s->threads) t.join();
    for (bug_ctx* c : s->ctxs) bug_ctx_destroy(c);
    if (s->shared) cudaStreamDestroy(s->shared);
    delete s;
  });
}

extern "C" int bug_server_job_error(bug_server* s, int64_t job_id, char* buf, int cap) {
  return guard([&] {
    require(s && buf && cap > 0, "bad argument");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->jobs.find(job_id);
    require(it != s->jobs.end(), "no such job");
    const std::string& e = it->second->error;
    const size_t n = std::min(e.size(), size_t(cap - 1));
    std::memcpy(buf, e.data(), n);
    buf[n] = 0;
  });
}

extern "C" int64_t bug_server_launches(const bug_server* s) {
  if (!s) return 0;
  int64_t n = 0;
  for (const bug_ctx* c : s->ctxs) n += bug_ctx_launches(c);
  return n + const_cast<bug_server*>(s)->combiner.launches;
}

// ── batched steps ─────────────────────────────────────────────────────────────────────────────
// n chains stepped together: n contexts on one shared stream with one combiner (their stage
// lists merge into shared launches) and n persistent host threads, one per chain.

struct bug_batch {
  int device = 0;
  std::vector<bug_ctx*> ctxs;
  bugi::Combiner combiner;
  cudaStream_t shared = nullptr;
  std::vector<std::thread> threads;
  std::mutex mu;
  std::condition_variable go_cv, done_cv;
  uint64_t gen = 0;
  int nrun = 0, remaining = 0;
  bool stop = false;
  std::function<void(int)> task;

  void worker(int i) {
    cudaSetDevice(device);
    uint64_t seen = 0;
    for (;;) {
      std::function<void(int)> t;
      {
        std::unique_lock<std::mutex> lk(mu);
        go_cv.wait(lk, [&] { return stop || gen != seen; });
        if (stop) return;
        seen = gen;
        if (i >= nrun) continue;
        t = task;
      }
      if (shared) combiner.job_begin();
      t(i);
      if (shared) combiner.job_end();
      {
        std::lock_guard<std::mutex> lk(mu);
        if (--remaining == 0) done_cv.notify_all();
      }
    }
  }
};

extern "C" int bug_batch_create(int device, int n, int combine, bug_batch** out) {
  return guard([&] {
    require(out != nullptr && n >= 1 && n <= bugk::kMaxLists, "bug_batch_create: bad argument");
    auto b = std::make_unique<bug_batch>();
    b->device = device;
    for (int i = 0; i < n; ++i) {
      bug_ctx* c = nullptr;
      const int rc = bug_ctx_create(device, &c);
      if (rc != BUG_OK) {
        for (bug_ctx* x : b->ctxs) bug_ctx_destroy(x);
        throw bugi::BugError(rc, std::string("bug_batch_create: ") + bug_last_error());
      }
      b->ctxs.push_back(c);
    }
    if (combine && b->ctxs[0]->list_cluster > 0 && b->ctxs[0]->queue_enabled)
      share_stream(device, b->ctxs, b->combiner, b->shared);
    bug_batch* raw = b.get();
    for (int i = 0; i < n; ++i) raw->threads.emplace_back([raw, i] { raw->worker(i); });
    *out = b.release();
  });
}

extern "C" int bug_batch_context(bug_batch* b, int i, bug_ctx** out) {
  return guard([&] {
    require(b && out && i >= 0 && i < int(b->ctxs.size()), "bug_batch_context: bad argument");
    *out = b->ctxs[size_t(i)];
  });
}

extern "C" int bug_step_batch(bug_batch* b, int n, const int* L, bug_tensor** const* psi_io,
                              int* center_io, const bug_tensor* const* const* mpo,
                              const double* tau_re, const double* tau_im,
                              const bug_step_params* params, bug_normal_fn draw,
                              void* const* draw_user, bug_step_info* info, int* status) {
  int first_rc = BUG_OK;
  std::string first_err;
  const int rc0 = guard([&] {
    require(b && n >= 1 && n <= int(b->ctxs.size()) && L && psi_io && center_io && mpo && tau_re &&
                tau_im && params && draw && draw_user && info && status,
            "bug_step_batch: bad argument");
    std::vector<std::string> chain_err(static_cast<size_t>(n));
    std::unique_lock<std::mutex> lk(b->mu);
    b->task = [&](int i) {
      int nlog = 0;
      status[i] = bug_mps_step(b->ctxs[size_t(i)], L[i], psi_io[i], &center_io[i], mpo[i], tau_re[i],
                               tau_im[i], &params[i], draw, draw_user[i], &info[i], nullptr, 0, &nlog);
      if (status[i] != BUG_OK) chain_err[static_cast<size_t>(i)] = bug_last_error();
    };
    b->nrun = n;
    b->remaining = n;
    ++b->gen;
    b->go_cv.notify_all();
    b->done_cv.wait(lk, [&] { return b->remaining == 0; });
    b->task = nullptr;
    for (int i = 0; i < n; ++i)
      if (status[i] != BUG_OK && first_rc == BUG_OK) {
        first_rc = status[i];
        first_err = "chain " + std::to_string(i) + ": " + chain_err[static_cast<size_t>(i)];
      }
  });
  if (rc0 != BUG_OK) return rc0;
  if (first_rc != BUG_OK) bugi::g_err = first_err;
  return first_rc;
}

extern "C" int64_t bug_batch_launches(const bug_batch* b) {
  if (!b) return 0;
  int64_t n = 0;
  for (const bug_ctx* c : b->ctxs) n += bug_ctx_launches(c);
  return n + const_cast<bug_batch*>(b)->combiner.launches;
}

extern "C" int bug_batch_destroy(bug_batch* b) {
  return guard([&] {
    if (!b) return;
    {
      std::lock_guard<std::mutex> lk(b->mu);
      b->stop = true;
    }
    b->go_cv.notify_all();
    for (auto& t : b->threads) t.join();
    for (bug_ctx* c : b->ctxs) bug_ctx_destroy(c);
    if (b->shared) cudaStreamDestroy(b->shared);
    delete b;
  });
}

extern "C" int64_t bug_projected_footprint(int L, int d, int maxdim, int mpo_dim) {
  if (L < 1 || d < 1 || maxdim < 1 || mpo_dim < 1) return 0;
  const int64_t D2 = int64_t(maxdim) * maxdim, c = 16;  // complex FP64
  const int64_t state = int64_t(L) * d * D2;
  const int64_t envs = 2 * int64_t(L) * mpo_dim * D2;
  const int64_t krylov = int64_t(64 + 16) * d * D2;   // Krylov basis + probes of one bond
  const int64_t twosite = 4 * int64_t(d) * d * D2;     // two-site work tensors
  return 2 * c * (state + envs + krylov + twosite);    // x2: temporaries and copies
}
