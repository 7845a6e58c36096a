// Serving loop: model-construction jobs admitted by HBM budget and run
// concurrently on one GPU.
//
// A job is one GALIC run (main.c:69-107) from the point where the grids and
// the initial particles exist: upload them into a fresh context (they stay
// resident on the device for the whole job), calc_all_response_fields, then
// MaximumNumberOfSteps iterations of IndepenentOptimizationsPerStep
// repetitions, each optimising the next n_per_cpu particles of the
// permutation (main.c:120-146), optionally ending early once Sall (main.c:1270)
// improves by less than a given fraction over an iteration.
//
// Worker threads take queued jobs first-fit in arrival order as soon as a
// worker is free and the job's device footprint fits the remaining budget;
// each job runs on its context's own non-blocking stream, so the kernels of
// concurrent jobs overlap on the device.  A job's result does not depend on
// what else runs: its kernels and its random streams (seed, particle,
// repetition) are its own.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "galic_gpu.h"

namespace galic_internal {
// galic_ctx_create with a stream priority (api.cu)
int ctx_create(const galic_params_t *prm, int priority, galic_ctx **out);
}

namespace {

struct Job {
  int id = 0;
  galic_job_t desc{};
  size_t bytes = 0;
  int state = 0;  // 0 queued, 1 running, 2 done
  galic_job_result_t res{};
};

double sall(const double *fit)
{
  // main.c:1270, summed over the particle types present
  double s = 0;
  for(int t = 1; t <= 3; t++) {
    const double *f = fit + 7 * t;
    const double cnt = f[6] != 0 ? f[6] : 1.0;
    s += f[0] + (f[1] + f[2] + f[3] + f[4]) / cnt;
  }
  return s;
}

// particles optimised per repetition (main.c:128 with NTask = 1)
size_t job_count(const galic_job_t &d)
{
  return std::min((size_t) d.n, (size_t) (1 + d.fraction_per_rep * d.n));
}

// device bytes of the per-orbit grids of one window of repetitions: the
// whole iteration, capped at 8 GiB (at least one repetition); a job holds
// two windows at once (galic_optimize_reps)
size_t job_window_bytes(const galic_job_t &d)
{
  const size_t G = (size_t) 1 << (2 * d.prm->DG_MaxLevel);
  const size_t per_rep = job_count(d) * 2 * (5 * G * 8 + 128);
  const size_t iter = per_rep * (size_t) std::max(d.reps_per_iteration, 1);
  return std::max(per_rep, std::min(iter, (size_t) 8 << 30));
}

int run_job(const galic_job_t &d, galic_job_result_t &r, double *t_first, const std::function<double()> &now,
            int priority)
{
  galic_ctx *ctx = nullptr;
  int st = galic_internal::ctx_create(d.prm, priority, &ctx);
  if(st) return st;
  auto done = [&](int status) {
    galic_ctx_destroy(ctx);
    return status;
  };
  if((st = galic_set_force_grid(ctx, d.fg_pot, d.fg_dpotdr, d.fg_dpotdz))) return done(st);
  for(int t = 1; t <= 3; t++)
    if(d.vstream[t] && (st = galic_set_vstream(ctx, t, d.vstream[t]))) return done(st);
  if((st = galic_set_density_geometry(ctx, d.cellsize, d.dgs_distance))) return done(st);
  for(int t = 1; t <= 3; t++)
    if(d.prm->NType[t] > 0) {
      const double *const *g = d.targets[t];
      if((st = galic_set_targets(ctx, t, g[0], g[1], g[2], g[3], g[4], g[5]))) return done(st);
    }
  if((st = galic_set_particles(ctx, d.n, d.pos, d.vel, d.mass, d.tint, d.vesc, d.type, d.ptargets)))
    return done(st);
  if((st = galic_calc_all_response_fields(ctx, d.form))) return done(st);
  r.orbit_steps += galic_last_orbit_steps(ctx);
  double fit[28];
  galic_get_fit(ctx, fit);
  r.sall_first = r.sall_last = sall(fit);
  *t_first = now();
  // optimize_some_particles (main.c:120-146): n_per_cpu from the fraction,
  // a cursor through the permutation that persists across repetitions
  const int n_per = std::min(d.n, (int) (1 + d.fraction_per_rep * d.n));
  // one iteration's repetitions in one call: their orbits run in windows of
  // repetitions (galic_optimize_reps), the repetitions commit in order
  std::vector<int> idx((size_t) n_per * std::max(d.reps_per_iteration, 0));
  const size_t window = job_window_bytes(d);
  int cursor = 0;
  uint32_t rep_serial = 0;
  for(int it = 0; it < d.max_iterations; it++) {
    const double before = r.sall_last;
    for(size_t i = 0; i < idx.size(); i++, cursor++) {
      if(cursor >= d.n) cursor = 0;
      idx[i] = d.permutation ? d.permutation[cursor] : cursor;
    }
    if(d.reps_per_iteration > 0) {
      if((st = galic_optimize_reps(ctx, idx.data(), n_per, d.reps_per_iteration, d.seed, rep_serial, d.form,
                                   window, nullptr)))
        return done(st);
      r.orbit_steps += galic_last_orbit_steps(ctx);
      rep_serial += (uint32_t) d.reps_per_iteration;
      r.reps += d.reps_per_iteration;
    }
    galic_get_fit(ctx, fit);
    r.sall_last = sall(fit);
    r.iterations = it + 1;
    if(d.converge_rel > 0 && before > 0 && (before - r.sall_last) < d.converge_rel * before) break;
  }
  std::memcpy(r.fit, fit, sizeof(fit));
  if(d.vel_out) galic_get_particles(ctx, d.vel_out, nullptr, nullptr);
  return done(GALIC_OK);
}

}  // namespace

struct galic_server {
  int device = 0;
  size_t budget = 0, used = 0, peak_used = 0;
  int running = 0, peak_running = 0;
  std::vector<std::thread> workers;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Job *> queue;
  std::map<int, std::unique_ptr<Job>> jobs;
  int next_id = 1;
  bool stopping = false;
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();

  double now() const { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); }

  // first queued job that fits the budget (arrival order), or null
  Job *pick()
  {
    for(auto it = queue.begin(); it != queue.end(); ++it)
      if(used + (*it)->bytes <= budget) {
        Job *j = *it;
        queue.erase(it);
        return j;
      }
    return nullptr;
  }

  int prio_least = 0, prio_greatest = 0;  // cudaDeviceGetStreamPriorityRange

  void worker()
  {
    cudaSetDevice(device);
    for(;;) {
      Job *j = nullptr;
      int prio = 0;
      {
        std::unique_lock<std::mutex> lk(mu);
        cv_work.wait(lk, [&] { return (j = pick()) != nullptr || (stopping && queue.empty()); });
        if(!j) return;
        used += j->bytes;
        peak_used = std::max(peak_used, used);
        running++;
        peak_running = std::max(peak_running, running);
        j->state = 1;
        j->res.t_admit = now();
        // a job admitted while k others run gets the k-th highest stream
        // priority: earlier jobs run first where they compete (approximates
        // first-come first-served, which lowers the median time to
        // convergence; every job keeps progressing)
        prio = std::min(prio_least, prio_greatest + (running - 1));
      }
      double t_first = -1;
      const int st = run_job(j->desc, j->res, &t_first, [&] { return now(); }, prio);
      {
        std::lock_guard<std::mutex> lk(mu);
        j->res.status = st;
        j->res.t_first_response = t_first;
        j->res.t_done = now();
        j->state = 2;
        used -= j->bytes;
        running--;
      }
      cv_done.notify_all();
      cv_work.notify_all();
    }
  }
};

extern "C" size_t galic_job_device_bytes(const galic_job_t *job)
{
  if(!job || !job->prm || job->n <= 0) return 0;
  const galic_params_t &p = *job->prm;
  const size_t n = (size_t) job->n;
  const size_t NF = (size_t) p.FG_Nbin * p.FG_Nbin;
  const size_t G = (size_t) 1 << (2 * p.DG_MaxLevel);
  const size_t Ns = (((size_t) 1 << (2 + 2 * p.DG_MaxLevel)) - 1) / 3;
  size_t b = n * 160;                       // particle state (allvars.h:844-868) and processing order
  b += NF * (16 + 8 + 3 * 8 + 3 * 64);      // FP64 force tables, streaming velocities, FP32 quad tables
  b += G * (8 + 4 + 320 + 640) + Ns * 520;  // geometry, committed grids, fixed point, stacks, targets
  b += 2 * job_window_bytes(*job) + job_count(*job) * 64;  // per-orbit grids of two windows of repetitions
  b += (size_t) 16 << 20;                   // fit scratch, allocator granularity
  return b;
}

extern "C" int galic_server_create(size_t hbm_budget_bytes, int workers, galic_server **out)
{
  if(!out || workers < 1 || workers > 64 || hbm_budget_bytes == 0) return GALIC_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  int dev = 0;
  if(cudaGetDevice(&dev) != cudaSuccess) return GALIC_ERR_NO_DEVICE;
  int count = 0;
  if(cudaGetDeviceCount(&count) != cudaSuccess || count < 1) return GALIC_ERR_NO_DEVICE;
  galic_server *s = new galic_server();
  s->device = dev;
  if(cudaDeviceGetStreamPriorityRange(&s->prio_least, &s->prio_greatest) != cudaSuccess) {
    cudaGetLastError();
    s->prio_least = s->prio_greatest = 0;
  }
  s->budget = hbm_budget_bytes;
  for(int w = 0; w < workers; w++) s->workers.emplace_back([s] { s->worker(); });
  *out = s;
  return GALIC_OK;
}

extern "C" int galic_server_submit(galic_server *s, const galic_job_t *job, int *job_id)
{
  if(!s || !job || !job_id || !job->prm || job->n <= 0 || !job->pos || !job->vel || !job->mass || !job->tint ||
     !job->vesc || !job->type || !job->ptargets || !job->fg_pot || !job->fg_dpotdr || !job->fg_dpotdz ||
     !job->cellsize || !job->dgs_distance || job->max_iterations < 0 || job->reps_per_iteration < 0 ||
     !(job->fraction_per_rep >= 0) || (job->form != GALIC_FORM_FP64 && job->form != GALIC_FORM_FP32))
    return GALIC_ERR_INVALID_ARGUMENT;
  for(int t = 1; t <= 3; t++)
    if(job->prm->NType[t] > 0)
      for(int k = 0; k < 6; k++)
        if(!job->targets[t][k]) return GALIC_ERR_INVALID_ARGUMENT;
  auto j = std::make_unique<Job>();
  j->desc = *job;
  j->bytes = galic_job_device_bytes(job);
  std::lock_guard<std::mutex> lk(s->mu);
  if(s->stopping) return GALIC_ERR_STATE;
  j->id = s->next_id++;
  j->res.t_submit = s->now();
  j->res.t_admit = j->res.t_first_response = j->res.t_done = -1;
  *job_id = j->id;
  if(j->bytes > s->budget) {  // can never be admitted
    j->state = 2;
    j->res.status = GALIC_ERR_BUDGET;
    j->res.t_done = j->res.t_submit;
    s->jobs[j->id] = std::move(j);
    s->cv_done.notify_all();
    return GALIC_OK;
  }
  s->queue.push_back(j.get());
  s->jobs[j->id] = std::move(j);
  s->cv_work.notify_all();
  return GALIC_OK;
}

extern "C" int galic_server_wait(galic_server *s, int job_id, double timeout_s, galic_job_result_t *res)
{
  if(!s || !res) return GALIC_ERR_INVALID_ARGUMENT;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->jobs.find(job_id);
  if(it == s->jobs.end()) return GALIC_ERR_INVALID_ARGUMENT;
  Job *j = it->second.get();
  const auto until = std::chrono::steady_clock::now() + std::chrono::duration<double>(timeout_s);
  if(!s->cv_done.wait_until(lk, until, [&] { return j->state == 2; })) return GALIC_ERR_STATE;  // not done yet
  *res = j->res;
  return GALIC_OK;
}

extern "C" int galic_server_stats(galic_server *s, size_t *peak_bytes, int *peak_running, int *queued, int *running)
{
  if(!s) return GALIC_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(s->mu);
  if(peak_bytes) *peak_bytes = s->peak_used;
  if(peak_running) *peak_running = s->peak_running;
  if(queued) *queued = (int) s->queue.size();
  if(running) *running = s->running;
  return GALIC_OK;
}

extern "C" void galic_server_destroy(galic_server *s)
{
  if(!s) return;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stopping = true;
  }
  s->cv_work.notify_all();
  for(auto &w : s->workers) w.join();
  delete s;
}
