// server.cpp -- the job engine of include/eplace.h: many placement jobs on
// one GPU, continuously batched.  No reference counterpart.
//
// One scheduler thread owns the device.  Each turn it admits queued jobs
// (while fewer than max_jobs run and the estimated device footprint of the
// running jobs plus the next one fits the budget), then advances every
// running job without blocking (job_pump: launch the next interval graph,
// read finished intervals, fold finished legalisations) and completes the
// finished ones.  A job runs on a context of its own; contexts are kept
// after their job and re-loaded for the next one (their device buffers only
// grow, a context whose bin grid matches is preferred so the DCT matrices,
// tensor maps and interval graph stay, and twice max_jobs contexts are made
// at start so that each grid of a mixed stream finds one), so a steady
// stream of jobs allocates and frees nothing.  All jobs
// share one host legaliser pool.  Every job's arithmetic is its own (its
// own buffers, streams and deterministic reductions), so its result equals
// a single eplace_run of it.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

#include "eplace_internal.h"
#include "job.h"

using namespace eplace;

namespace {

using Clock = std::chrono::steady_clock;

double secs(Clock::time_point a, Clock::time_point b) { return std::chrono::duration<double>(b - a).count(); }

struct JobRec {
  uint64_t id = 0;
  HostProblem hp;  // validated copy of the inputs (moved into a context at admission)
  eplace_cfg cfg{};
  uint64_t footprint = 0;
  uint32_t n = 0;
  // result buffers
  std::vector<int32_t> bel_tile, bel_index;
  std::vector<float> x, y;
  std::vector<eplace_traj_entry> traj;
  eplace_result res{};
  eplace_status st = EPLACE_OK;
  std::string err;
  Clock::time_point t_submit, t_admit, t_done;
  bool admitted = false;
  bool done = false;
};

struct Running {
  JobRec *rec;
  eplace_ctx *ctx;
  JobState *job;
};

// A job a loader thread has loaded and started (or failed to).
struct Ready {
  JobRec *rec;
  eplace_ctx *ctx;
  JobState *job;  // nullptr when the load failed
  eplace_status st;
};

}  // namespace

struct eplace_server {
  eplace_server_cfg cfg{};
  uint64_t budget = 0;
  std::unique_ptr<Pool> pool;     // host legaliser, shared by all jobs
  std::unique_ptr<Pool> loaders;  // admission work: context load + job start
  std::vector<Ready> ready;       // loaded jobs waiting for the scheduler (under m)
  int loading = 0;                // jobs handed to the loaders (scheduler thread)
  std::thread sched;
  std::mutex m;
  std::condition_variable cv_work, cv_done;
  bool stop = false;
  uint64_t next_id = 1;
  std::deque<JobRec *> queue;
  std::unordered_map<uint64_t, std::unique_ptr<JobRec>> jobs;
  uint64_t submitted = 0, finished = 0, running_n = 0, contexts = 0;
  uint64_t device_bytes = 0;  // held by all contexts, refreshed after each job
  double t_admit = 0.0, t_pump = 0.0, t_idle = 0.0;  // scheduler time split (under m)
  // scheduler-thread state
  std::vector<Running> running;
  std::vector<eplace_ctx *> idle;
  uint64_t used = 0;

  ~eplace_server() {
    for (auto *c : idle) eplace_ctx_destroy(c);
  }

  void loop() {
    cudaSetDevice(cfg.device);
    for (;;) {
      {
        std::unique_lock<std::mutex> g(m);
        if (stop && running.empty() && loading == 0) break;
        if (running.empty() && queue.empty() && loading == 0) {
          cv_work.wait(g, [&] { return stop || !queue.empty(); });
          continue;
        }
      }
      const auto a0 = Clock::now();
      take_ready();
      admit();
      const auto a1 = Clock::now();
      bool progressed = false;
      for (size_t k = 0; k < running.size();) {
        Running &r = running[k];
        progressed |= job_pump(r.job, false);
        if (job_done(r.job)) {
          complete(r);
          running.erase(running.begin() + k);
          progressed = true;
        } else {
          ++k;
        }
      }
      const auto a2 = Clock::now();
      if (!progressed) std::this_thread::sleep_for(std::chrono::microseconds(20));
      const auto a3 = Clock::now();
      std::lock_guard<std::mutex> g(m);
      t_admit += secs(a0, a1);
      t_pump += secs(a1, a2);
      t_idle += secs(a2, a3);
    }
  }

  // Context for a job: an idle one with the same bin grid (its DCT matrices
  // stay), else any idle one, else a new one.
  eplace_ctx *take_context(const JobRec &r, eplace_status *st) {
    *st = EPLACE_OK;
    // An idle context with this bin grid keeps its DCT matrices, tensor
    // maps and interval graph; else one never loaded (the server creates
    // twice max_jobs of them at start, so a mixed stream's grids each find
    // one) while the memory the contexts hold leaves room; else any.
    size_t pick = idle.size(), fresh = idle.size();
    for (size_t k = 0; k < idle.size(); ++k) {
      if (ctx_bins_x(idle[k]) == r.hp.BX && ctx_bins_y(idle[k]) == r.hp.BY) {
        pick = k;
        break;
      }
      if (ctx_bins_x(idle[k]) <= 0 && fresh == idle.size()) fresh = k;
    }
    uint64_t held;
    {
      std::lock_guard<std::mutex> g(m);
      held = device_bytes;
    }
    if (pick == idle.size() && fresh < idle.size() && held + r.footprint <= budget) pick = fresh;
    if (pick == idle.size() && !idle.empty()) pick = idle.size() - 1;
    if (pick < idle.size()) {
      eplace_ctx *c = idle[pick];
      idle.erase(idle.begin() + pick);
      return c;
    }
    eplace_ctx *c = ctx_new(cfg.device, st);
    if (c) {
      std::lock_guard<std::mutex> g(m);
      ++contexts;
    }
    return c;
  }

  void admit() {
    for (;;) {
      JobRec *r = nullptr;
      {
        std::lock_guard<std::mutex> g(m);
        if (stop || queue.empty() || (int)running.size() + loading >= cfg.max_jobs) return;
        JobRec *front = queue.front();
        if ((!running.empty() || loading > 0) && used + front->footprint > budget) return;
        queue.pop_front();
        r = front;
        ++running_n;
      }
      r->t_admit = Clock::now();
      r->admitted = true;
      used += r->footprint;
      // The tensor-core transform needs bins_y % 128 == 0 and bins_x % 64 == 0;
      // smaller grids of a mixed stream run the FP32 transform.
      eplace_opts jo = cfg.opts;
      if (jo.dct_mode == EPLACE_DCT_BF16X3_TC && !problem_tc_supported(r->hp)) jo.dct_mode = EPLACE_DCT_FP32_FFT;
      eplace_status st = EPLACE_OK;
      eplace_ctx *c = take_context(*r, &st);
      if (!c) {
        fail(r, st);
        continue;
      }
      // The host work of admission (CSR copies, initial placement, uploads)
      // runs on a loader thread while this thread keeps the others going.
      ++loading;
      const bool shared = cfg.max_jobs > 1;
      Pool *lp = pool.get();
      loaders->submit([this, r, c, jo, shared, lp](int) {
        Ready rd{r, c, nullptr, EPLACE_OK};
        rd.st = ctx_load_problem(c, std::move(r->hp));
        if (rd.st != EPLACE_OK) {
          char buf[512];
          eplace_last_error(c, buf, sizeof buf);
          r->err = buf;
        } else {
          ctx_set_shared(c, shared);
          r->bel_tile.assign(r->n, 0);
          r->bel_index.assign(r->n, 0);
          r->x.assign(r->n, 0.f);
          r->y.assign(r->n, 0.f);
          r->traj.assign(r->cfg.max_iters / std::max<uint64_t>(1, r->cfg.legalize_interval) + 2,
                         eplace_traj_entry{});
          r->res = eplace_result{};
          r->res.bel_tile = r->bel_tile.data();
          r->res.bel_index = r->bel_index.data();
          r->res.x = r->x.data();
          r->res.y = r->y.data();
          r->res.traj = r->traj.data();
          r->res.traj_capacity = (uint32_t)r->traj.size();
          rd.job = job_create(c, r->cfg, jo, &r->res, lp);
          const eplace_status st2 = job_start(rd.job);
          if (st2 != EPLACE_OK) r->st = st2;  // the job is done(); complete() records it
        }
        {
          std::lock_guard<std::mutex> g(m);
          ready.push_back(rd);
        }
        cv_work.notify_one();
      });
    }
  }

  // Moves the loaders' finished admissions into the running set.
  void take_ready() {
    std::vector<Ready> got;
    {
      std::lock_guard<std::mutex> g(m);
      got.swap(ready);
    }
    for (const Ready &rd : got) {
      --loading;
      if (!rd.job) {
        idle.push_back(rd.ctx);
        fail(rd.rec, rd.st);
      } else {
        running.push_back({rd.rec, rd.ctx, rd.job});
      }
    }
  }

  void complete(Running &run) {
    JobRec *r = run.rec;
    eplace_status st = job_finish(run.job);
    if (r->st != EPLACE_OK) st = r->st;
    if (st != EPLACE_OK) {
      char buf[512];
      eplace_last_error(run.ctx, buf, sizeof buf);
      r->err = buf;
    }
    job_destroy(run.job);
    idle.push_back(run.ctx);
    used -= r->footprint;
    uint64_t held = 0;
    for (auto *c : idle) held += ctx_device_bytes(c);
    for (auto &o : running)
      if (o.ctx != run.ctx) held += ctx_device_bytes(o.ctx);
    std::lock_guard<std::mutex> g(m);
    device_bytes = held;
    r->st = st;
    r->t_done = Clock::now();
    r->done = true;
    --running_n;
    ++finished;
    cv_done.notify_all();
  }

  void fail(JobRec *r, eplace_status st) {
    used -= r->footprint;
    std::lock_guard<std::mutex> g(m);
    r->st = st;
    if (r->err.empty()) r->err = "job could not be admitted";
    r->t_done = Clock::now();
    r->done = true;
    --running_n;
    ++finished;
    cv_done.notify_all();
  }
};

extern "C" {

void eplace_server_cfg_default(eplace_server_cfg *cfg) {
  if (!cfg) return;
  std::memset(cfg, 0, sizeof *cfg);
  cfg->device = 0;
  cfg->max_jobs = 16;
  cfg->hbm_budget = 0;
  cfg->legal_threads = 0;
  eplace_opts_default(&cfg->opts);
}

eplace_status eplace_server_create(const eplace_server_cfg *cfg, eplace_server **out) {
  if (!out) return EPLACE_ERR_INVALID;
  *out = nullptr;
  std::unique_ptr<eplace_server> s(new eplace_server());
  if (cfg) s->cfg = *cfg;
  else eplace_server_cfg_default(&s->cfg);
  if (s->cfg.max_jobs <= 0) s->cfg.max_jobs = 16;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    set_thread_error("no CUDA device");
    return EPLACE_ERR_NO_DEVICE;
  }
  if (s->cfg.device < 0 || s->cfg.device >= ndev) {
    set_thread_error("device index out of range");
    return EPLACE_ERR_INVALID;
  }
  if (cudaSetDevice(s->cfg.device) != cudaSuccess) {
    set_thread_error("cudaSetDevice failed");
    return EPLACE_ERR_CUDA;
  }
  s->budget = s->cfg.hbm_budget;
  if (s->budget == 0) {
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
      set_thread_error("cudaMemGetInfo failed");
      return EPLACE_ERR_CUDA;
    }
    s->budget = fr / 2;
  }
  const int nt = s->cfg.legal_threads > 0 ? s->cfg.legal_threads : (int)std::max(1u, std::thread::hardware_concurrency());
  s->pool.reset(new Pool(std::min(nt, 64), 5));
  s->loaders.reset(new Pool(4));
  // Contexts made up front (streams, events, a few scalars each): made
  // while jobs run, their set-up would stall the other jobs' streams.
  for (int k = 0; k < 2 * s->cfg.max_jobs; ++k) {
    eplace_status st = EPLACE_OK;
    eplace_ctx *c = ctx_new(s->cfg.device, &st);
    if (!c) return st;
    s->idle.push_back(c);
    ++s->contexts;
  }
  eplace_server *raw = s.get();
  s->sched = std::thread([raw] { raw->loop(); });
  *out = s.release();
  return EPLACE_OK;
}

void eplace_server_destroy(eplace_server *s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> g(s->m);
    s->stop = true;
    for (JobRec *r : s->queue) {
      r->st = EPLACE_ERR_INVALID;
      r->err = "engine shut down before the job ran";
      r->done = true;
    }
    s->queue.clear();
  }
  s->cv_work.notify_all();
  if (s->sched.joinable()) s->sched.join();
  s->cv_done.notify_all();
  delete s;
}

eplace_status eplace_server_submit(eplace_server *s, const eplace_netlist *nl, const eplace_chip *chip,
                                   const eplace_cfg *cfg, uint64_t *job_id) {
  if (!s || !job_id) return EPLACE_ERR_INVALID;
  std::unique_ptr<JobRec> r(new JobRec());
  std::string msg;
  eplace_status st = load_problem(nl, chip, r->hp, msg);
  if (st != EPLACE_OK) {
    set_thread_error(msg);
    return st;
  }
  if (cfg) r->cfg = *cfg;
  else eplace_cfg_default(&r->cfg);
  r->footprint = problem_device_bytes(r->hp);
  r->n = r->hp.N;
  r->t_submit = Clock::now();
  {
    std::lock_guard<std::mutex> g(s->m);
    if (s->stop) {
      set_thread_error("engine is shutting down");
      return EPLACE_ERR_INVALID;
    }
    r->id = s->next_id++;
    *job_id = r->id;
    s->queue.push_back(r.get());
    s->jobs.emplace(r->id, std::move(r));
    ++s->submitted;
  }
  s->cv_work.notify_one();
  return EPLACE_OK;
}

eplace_status eplace_server_wait(eplace_server *s, uint64_t job_id, int32_t timeout_ms, eplace_result *res,
                                 eplace_job_info *info) {
  if (!s) return EPLACE_ERR_INVALID;
  std::unique_ptr<JobRec> r;
  {
    std::unique_lock<std::mutex> g(s->m);
    auto it = s->jobs.find(job_id);
    if (it == s->jobs.end()) {
      set_thread_error("unknown job id");
      return EPLACE_ERR_INVALID;
    }
    JobRec *p = it->second.get();
    auto ready = [p] { return p->done; };
    if (timeout_ms < 0) s->cv_done.wait(g, ready);
    else if (timeout_ms > 0) s->cv_done.wait_for(g, std::chrono::milliseconds(timeout_ms), ready);
    if (!p->done) return EPLACE_PENDING;
    r = std::move(it->second);
    s->jobs.erase(it);
  }
  if (info) {
    info->queued_seconds = r->admitted ? secs(r->t_submit, r->t_admit) : 0.0;
    info->run_seconds = r->admitted ? secs(r->t_admit, r->t_done) : 0.0;
    info->latency_seconds = secs(r->t_submit, r->t_done);
    info->footprint_bytes = r->footprint;
  }
  if (r->st != EPLACE_OK) {
    set_thread_error(r->err);
    return r->st;
  }
  if (res) {
    const eplace_result &o = r->res;
    if (res->bel_tile && r->n) std::memcpy(res->bel_tile, r->bel_tile.data(), sizeof(int32_t) * r->n);
    if (res->bel_index && r->n) std::memcpy(res->bel_index, r->bel_index.data(), sizeof(int32_t) * r->n);
    if (res->x && r->n) std::memcpy(res->x, r->x.data(), sizeof(float) * r->n);
    if (res->y && r->n) std::memcpy(res->y, r->y.data(), sizeof(float) * r->n);
    const uint32_t nt = res->traj ? std::min(res->traj_capacity, o.traj_len) : 0;
    if (nt) std::memcpy(res->traj, r->traj.data(), sizeof(eplace_traj_entry) * nt);
    res->traj_len = nt;
    res->hpwl = o.hpwl;
    res->overlap = o.overlap;
    res->iters = o.iters;
    res->best_iter = o.best_iter;
    res->converged = o.converged;
    res->gpu_seconds = o.gpu_seconds;
    res->total_seconds = o.total_seconds;
    res->gpu_launches = o.gpu_launches;
    res->h2d_bytes = o.h2d_bytes;
    res->d2h_bytes = o.d2h_bytes;
  }
  return EPLACE_OK;
}

eplace_status eplace_server_stats_get(eplace_server *s, eplace_server_stats *out) {
  if (!s || !out) return EPLACE_ERR_INVALID;
  std::lock_guard<std::mutex> g(s->m);
  out->submitted = s->submitted;
  out->finished = s->finished;
  out->running = s->running_n;
  out->queued = s->queue.size();
  out->contexts = s->contexts;
  out->device_bytes = s->device_bytes;
  out->admit_seconds = s->t_admit;
  out->pump_seconds = s->t_pump;
  out->idle_seconds = s->t_idle;
  return EPLACE_OK;
}

uint64_t eplace_footprint(const eplace_netlist *nl, const eplace_chip *chip) {
  HostProblem hp;
  std::string msg;
  if (load_problem(nl, chip, hp, msg) != EPLACE_OK) return 0;
  return problem_device_bytes(hp);
}

}  // extern "C"
