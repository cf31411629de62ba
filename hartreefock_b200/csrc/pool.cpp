// Serving pool: RHF/UHF jobs submitted at any time, run by a fixed number of
// worker threads (slots) whose SCFs share the device, admitted in arrival
// order against a device-memory budget.  The C ABI is declared in
// include/hfgpu_driver.h (hfg_pool_create ... hfg_pool_destroy).
//
// The reference runs one algorithm object per std::thread with no shared
// state (HartreeFockDoc.cpp:372-405) and stops it through its terminate flag
// (HartreeFockAlgorithm.h:57, polled between iterations at
// HartreeFockAlgorithm.cpp:142,159,187).  A slot here is that thread; a
// cancelled or timed-out job sets the running algorithm's terminate flag, so
// it stops between two SCF iterations, never inside a kernel.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/hfgpu_driver.h"
#include "driver_internal.h"

namespace {

using Clock = std::chrono::steady_clock;

struct JobRec {
  int64_t id = 0;
  std::string basis;
  std::vector<int32_t> Z;
  std::vector<double> xyz;
  hfd_scf_opts opts{};
  double timeout_s = 0;
  int64_t bytes = 0;
  int32_t state = HFG_JOB_QUEUED;
  hfg_status status = HFG_OK;
  hfd_scf_result result{};
  std::string error;
  Clock::time_point t_submit, t_start, t_end;
  std::atomic_bool *term = nullptr;  // the running algorithm's terminate flag
  bool cancel = false, timed_out = false;
};

bool terminal(int32_t s) { return s >= HFG_JOB_DONE; }

double seconds(Clock::time_point a, Clock::time_point b) { return std::chrono::duration<double>(b - a).count(); }

thread_local std::string g_pool_error;

hfg_status pool_fail(hfg_status st, const std::string &msg) {
  g_pool_error = msg;
  return st;
}

}  // namespace

struct hfg_pool {
  int slots = 1;
  int64_t budget = 0, used = 0;
  int running = 0;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<std::shared_ptr<JobRec>> queue;
  std::unordered_map<int64_t, std::shared_ptr<JobRec>> jobs;
  std::vector<std::thread> workers;
  std::thread monitor;
  bool stop = false;
  int64_t next_id = 1;

  // the head of the queue fits what is left of the budget (arrival order:
  // a job never overtakes an earlier one)
  bool head_fits() const { return !queue.empty() && used + queue.front()->bytes <= budget; }

  void finish(const std::shared_ptr<JobRec> &j, int32_t state, hfg_status st) {
    j->state = state;
    j->status = st;
    j->t_end = Clock::now();
    cv_done.notify_all();
  }

  void work() {
    for (;;) {
      std::shared_ptr<JobRec> j;
      {
        std::unique_lock<std::mutex> lk(mu);
        cv_work.wait(lk, [&] { return stop || head_fits(); });
        if (stop) break;
        j = queue.front();
        queue.pop_front();
        used += j->bytes;
        ++running;
        j->state = HFG_JOB_RUNNING;
        j->t_start = Clock::now();
      }
      hfd_scf_result r{};
      std::string err;
      const hfg_status st = hfgpu::run_scf(
          j->basis.c_str(), (int32_t)j->Z.size(), j->Z.data(), j->xyz.data(), &j->opts, &r, nullptr, 0,
          [&](std::atomic_bool *flag) {
            std::lock_guard<std::mutex> lk(mu);
            j->term = flag;
            if (flag && (j->cancel || j->timed_out)) flag->store(true);
          },
          &err);
      {
        std::lock_guard<std::mutex> lk(mu);
        used -= j->bytes;
        --running;
        j->result = r;
        j->error = err;
        if (j->cancel) finish(j, HFG_JOB_CANCELLED, HFG_CANCELLED);
        else if (j->timed_out) finish(j, HFG_JOB_TIMEOUT, HFG_TIMEOUT);
        else if (st == HFG_OK) finish(j, HFG_JOB_DONE, HFG_OK);
        else finish(j, HFG_JOB_FAILED, st);
        cv_work.notify_all();  // budget freed: the next head may fit
      }
    }
    hfgpu::release_driver_thread();
  }

  // timeouts: every job's bound runs from its submission; queued jobs past it
  // leave the queue, running ones get their terminate flag set
  void watch() {
    std::unique_lock<std::mutex> lk(mu);
    while (!stop) {
      cv_done.wait_for(lk, std::chrono::milliseconds(20));
      const auto now = Clock::now();
      for (auto it = queue.begin(); it != queue.end();) {
        const auto &j = *it;
        if (j->timeout_s > 0 && seconds(j->t_submit, now) > j->timeout_s) {
          j->timed_out = true;
          finish(j, HFG_JOB_TIMEOUT, HFG_TIMEOUT);
          it = queue.erase(it);
        } else {
          ++it;
        }
      }
      for (auto &kv : jobs) {
        auto &j = kv.second;
        if (j->state == HFG_JOB_RUNNING && j->timeout_s > 0 && !j->timed_out &&
            seconds(j->t_submit, now) > j->timeout_s) {
          j->timed_out = true;
          if (j->term) j->term->store(true);
        }
      }
      cv_work.notify_all();
    }
  }
};

namespace {

void fill_info(const JobRec &j, hfg_job_info *info) {
  std::memset(info, 0, sizeof *info);
  info->state = j.state;
  info->status = j.status;
  info->footprint_bytes = j.bytes;
  const auto now = Clock::now();
  if (j.state == HFG_JOB_QUEUED) {
    info->queue_s = seconds(j.t_submit, now);
  } else {
    const bool started = j.t_start != Clock::time_point{};
    info->queue_s = started ? seconds(j.t_submit, j.t_start) : seconds(j.t_submit, terminal(j.state) ? j.t_end : now);
    info->run_s = started ? seconds(j.t_start, terminal(j.state) ? j.t_end : now) : 0.0;
    info->latency_s = terminal(j.state) ? seconds(j.t_submit, j.t_end) : seconds(j.t_submit, now);
  }
  if (terminal(j.state)) info->result = j.result;
}

}  // namespace

extern "C" {

const char *hfg_pool_last_error(void) { return g_pool_error.c_str(); }

hfg_status hfg_pool_create(int32_t slots, int64_t hbm_budget_bytes, hfg_pool **out) {
  if (!out || slots < 1 || hbm_budget_bytes <= 0) return pool_fail(HFG_INVALID_ARG, "hfg_pool_create: arguments");
  auto p = std::make_unique<hfg_pool>();
  p->slots = slots;
  p->budget = hbm_budget_bytes;
  for (int i = 0; i < slots; ++i) p->workers.emplace_back([q = p.get()] { q->work(); });
  p->monitor = std::thread([q = p.get()] { q->watch(); });
  *out = p.release();
  return HFG_OK;
}

hfg_status hfg_job_submit(hfg_pool *p, const hfg_job_spec *spec, int64_t *job_id) {
  if (!p || !spec || !job_id || !spec->basis_path || spec->natoms <= 0 || !spec->Z || !spec->xyz)
    return pool_fail(HFG_INVALID_ARG, "hfg_job_submit: arguments");
  auto j = std::make_shared<JobRec>();
  j->basis = spec->basis_path;
  j->Z.assign(spec->Z, spec->Z + spec->natoms);
  j->xyz.assign(spec->xyz, spec->xyz + 3 * spec->natoms);
  j->opts = spec->opts;
  j->timeout_s = spec->timeout_s;
  try {
    j->bytes = hfgpu::job_footprint_bytes(spec->basis_path, spec->natoms, spec->Z, spec->xyz,
                                          spec->opts.unrestricted != 0);
  } catch (const std::exception &ex) {
    return pool_fail(HFG_INVALID_ARG, std::string("hfg_job_submit: ") + ex.what());
  }
  std::lock_guard<std::mutex> lk(p->mu);
  if (j->bytes > p->budget)
    return pool_fail(HFG_OOM_BUDGET, "hfg_job_submit: the job's estimated " + std::to_string(j->bytes) +
                                         " device bytes exceed the pool's whole budget");
  j->id = p->next_id++;
  j->t_submit = Clock::now();
  p->jobs[j->id] = j;
  p->queue.push_back(j);
  *job_id = j->id;
  p->cv_work.notify_all();
  return HFG_OK;
}

hfg_status hfg_job_poll(hfg_pool *p, int64_t job_id, hfg_job_info *info) {
  if (!p || !info) return pool_fail(HFG_INVALID_ARG, "hfg_job_poll: arguments");
  std::lock_guard<std::mutex> lk(p->mu);
  auto it = p->jobs.find(job_id);
  if (it == p->jobs.end()) return pool_fail(HFG_INVALID_ARG, "hfg_job_poll: unknown job");
  fill_info(*it->second, info);
  return HFG_OK;
}

hfg_status hfg_job_wait(hfg_pool *p, int64_t job_id, double timeout_s, hfg_job_info *info) {
  if (!p || !info) return pool_fail(HFG_INVALID_ARG, "hfg_job_wait: arguments");
  std::unique_lock<std::mutex> lk(p->mu);
  auto it = p->jobs.find(job_id);
  if (it == p->jobs.end()) return pool_fail(HFG_INVALID_ARG, "hfg_job_wait: unknown job");
  auto j = it->second;
  auto done = [&] { return terminal(j->state); };
  if (timeout_s > 0) p->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), done);
  else p->cv_done.wait(lk, done);
  fill_info(*j, info);
  return terminal(j->state) ? HFG_OK : HFG_TIMEOUT;
}

hfg_status hfg_job_cancel(hfg_pool *p, int64_t job_id) {
  if (!p) return pool_fail(HFG_INVALID_ARG, "hfg_job_cancel: arguments");
  std::lock_guard<std::mutex> lk(p->mu);
  auto it = p->jobs.find(job_id);
  if (it == p->jobs.end()) return pool_fail(HFG_INVALID_ARG, "hfg_job_cancel: unknown job");
  auto &j = it->second;
  if (j->state == HFG_JOB_QUEUED) {
    p->queue.erase(std::remove(p->queue.begin(), p->queue.end(), j), p->queue.end());
    j->cancel = true;
    p->finish(j, HFG_JOB_CANCELLED, HFG_CANCELLED);
    p->cv_work.notify_all();
  } else if (j->state == HFG_JOB_RUNNING) {
    j->cancel = true;
    if (j->term) j->term->store(true);
  }
  return HFG_OK;
}

hfg_status hfg_pool_stats(hfg_pool *p, int32_t *running, int32_t *queued, int64_t *used_bytes) {
  if (!p) return pool_fail(HFG_INVALID_ARG, "hfg_pool_stats: arguments");
  std::lock_guard<std::mutex> lk(p->mu);
  if (running) *running = p->running;
  if (queued) *queued = (int32_t)p->queue.size();
  if (used_bytes) *used_bytes = p->used;
  return HFG_OK;
}

void hfg_pool_destroy(hfg_pool *p) {
  if (!p) return;
  {
    std::lock_guard<std::mutex> lk(p->mu);
    for (auto &j : p->queue) {
      j->cancel = true;
      p->finish(j, HFG_JOB_CANCELLED, HFG_CANCELLED);
    }
    p->queue.clear();
    for (auto &kv : p->jobs)
      if (kv.second->state == HFG_JOB_RUNNING) {
        kv.second->cancel = true;
        if (kv.second->term) kv.second->term->store(true);
      }
    p->stop = true;
  }
  p->cv_work.notify_all();
  p->cv_done.notify_all();
  for (auto &t : p->workers) t.join();
  if (p->monitor.joinable()) p->monitor.join();
  delete p;
}

}  // extern "C"
