// SCF serving on one GPU: independent ChebySCF jobs (each a directory with
// an INPUT and its pseudopotential files, the reference program's own
// inputs, main.cpp:20-50) run to convergence with continuous batching.
//
// The reference runs one job per process.  Here a server owns `slots`
// worker threads on one device.  A job is admitted when a worker is free
// and the sum of the admitted jobs' estimated device footprints stays within
// the HBM budget (a job larger than the whole budget runs alone); jobs that
// arrive while others run are admitted as slots and memory free up, in
// arrival order.  Each admitted job builds its own system (cell, SCF handle)
// with its own streams and runs pspw_system_cheby_scf_with, so the kernels
// of concurrent jobs overlap on the device; its wavefunction block,
// densities and mixing history stay on the device for the whole run and are
// released when it finishes.  Jobs share nothing but the device, so each
// job's arithmetic is the same alone and in the mix.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "engine.h"
#include "pspw_gpu.h"

namespace {

using clk = std::chrono::steady_clock;

struct Job {
  int id = 0;
  std::string dir;
  pspw_job_result res{};
  std::vector<double> eig;
  bool done = false;
};

}  // namespace

struct pspw_server {
  int device = 0;
  pspw_server_config cfg{};
  double budget = 0.0, used = 0.0;
  int running = 0;
  clk::time_point t0;
  std::mutex mu;
  std::condition_variable cv_queue, cv_budget, cv_done;
  std::deque<Job *> queue;
  std::vector<std::unique_ptr<Job>> jobs;
  bool stop = false;
  std::vector<std::thread> workers;
  double now() const { return std::chrono::duration<double>(clk::now() - t0).count(); }
};

namespace {

struct JobSizes {
  int ngw = 0, ngwx = 0, nnr = 0, ng = 0, nx = 0, nsp = 0, n3 = 0, nat = 0, nproj = 0,
      nsticks = 0, mixdim = 0;
};

// Device bytes a job holds while it runs: the system's set-up arrays, the
// cell (projector data in both precisions, the stored FP64 projectors, the
// stick-order copies of the filter, the FFT maps and potentials), the SCF
// handle and mixing history, the SCF loop's blocks and the workspaces of
// H*psi, the filter and the dense steps, plus a fixed allowance for the
// library handles and streams.
double footprint_bytes(const JobSizes &v) {
  const double ngw = v.ngw, ngwx = v.ngwx, nnr = v.nnr, ng = v.ng, nx2 = v.nx + 2.0;
  const double nat = v.nat, nproj = v.nproj, nsp = v.nsp, mixdim = std::max(2, v.mixdim);
  double b = 0.0;
  b += ngwx * nat * 16 + nsp * ng * 32 + 4.0 * ngwx * nsp * 8 + nnr * 8;  // set-up arrays
  b += 2.0 * (ngw * nat * 24 + 4.0 * nsp * ngw * 12 + ngw * 48);          // cell (+ stick order)
  b += 2.0 * ngw * nproj * 16;                                             // FP64 projectors
  b += nnr * 40;                                                           // potentials, maps
  b += ng * 48 + nnr * 16 + (2.0 * mixdim + 6.0) * nnr * 8;                // SCF handle
  b += ngw * nx2 * (16 * 2 + 8) + nnr * 24;                                // SCF loop blocks
  b += 3.0 * ngw * nx2 * 16;                                               // filter blocks
  b += 2.0 * std::min(96.0 * (1 << 20), nx2 * v.n3 * v.nsticks * 16.0);   // stick buffers
  b += nx2 * nx2 * 16 * 40.0 + nx2 * nproj * 16 * 40.0;                    // split-K slices
  return 1.25 * b + 64.0 * (1 << 20);
}

int job_sizes(const std::string &dir, JobSizes *v) {
  pspw_system *S = nullptr;
  int rc = pspw_system_load(dir.c_str(), -1, &S);  // host part only: no GPU touched
  if (rc) return rc;
  int d[16];
  double sc[16];
  pspw_scf_params p;
  if ((rc = pspw_system_info(S, d, sc)) || (rc = pspw_system_species(S, &v->nat, &v->nproj)) ||
      (rc = pspw_system_params(S, &p))) {
    pspw_system_destroy(S);
    return rc;
  }
  v->nnr = d[3];
  v->ngw = d[4];
  v->ngwx = d[5];
  v->ng = d[6];
  v->nx = d[8];
  v->nsp = d[11];
  v->n3 = d[2];
  v->nsticks = (int)(0.8 * d[0] * d[1]);  // the sphere's (i1, i2) columns, a bound
  v->mixdim = p.mixdim;
  pspw_system_destroy(S);
  return PSPW_OK;
}

void run_job(pspw_server *s, Job *job) {
  pspw_job_result &r = job->res;
  JobSizes v;
  int rc = job_sizes(job->dir, &v);
  const double foot = rc ? 0.0 : footprint_bytes(v);
  bool admitted = false;
  {
    std::unique_lock<std::mutex> lk(s->mu);
    r.footprint_bytes = foot;
    if (!rc) {
      // admit when it fits, or when nothing else runs (a job larger than the
      // whole budget runs alone)
      s->cv_budget.wait(lk, [&] { return s->running == 0 || s->used + foot <= s->budget; });
      s->used += foot;
      s->running++;
      admitted = true;
    }
    r.t_admit = s->now();
  }
  if (admitted) {
    cudaSetDevice(s->device);
    pspw_system *S = nullptr;
    rc = pspw_system_load(job->dir.c_str(), s->device, &S);
    if (!rc) {
      pspw_scf_params p;
      pspw_system_params(S, &p);
      p.filter_prec = s->cfg.filter_prec;
      if (s->cfg.conv_per_atom > 0.0) p.conv = s->cfg.conv_per_atom * v.nat;
      if (s->cfg.max_scf_iter > 0) p.max_scf_iter = s->cfg.max_scf_iter;
      if (s->cfg.pulay_beta > 0.0) p.pulay_beta = s->cfg.pulay_beta;
      if (s->cfg.mixdim > 0) p.mixdim = s->cfg.mixdim;
      r.natoms = v.nat;
      r.nbands = p.nx + 2;
      r.ngw = v.ngw;
      r.nnr = v.nnr;
      r.t_scf = s->now();
      job->eig.assign(p.nx, 0.0);
      double e6[6] = {0, 0, 0, 0, 0, 0};
      int its = 0, conv = 0;
      rc = pspw_system_cheby_scf_with(S, &p, nullptr, job->eig.data(), e6, &its, &conv, nullptr);
      r.etot = e6[0];
      r.iterations = its;
      r.converged = conv;
      pspw_system_destroy(S);
    }
  }
  if (rc) {
    const char *m = pspw_last_error();  // this worker thread's last message
    std::strncpy(r.error, m ? m : "", sizeof r.error - 1);
    r.error[sizeof r.error - 1] = '\0';
  }
  std::lock_guard<std::mutex> lk(s->mu);
  r.status = rc;
  r.t_done = s->now();
  if (admitted) {
    s->used -= foot;
    s->running--;
  }
  job->done = true;
  s->cv_budget.notify_all();
  s->cv_done.notify_all();
}

void worker(pspw_server *s) {
  cudaSetDevice(s->device);
  for (;;) {
    Job *job = nullptr;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      s->cv_queue.wait(lk, [&] { return s->stop || !s->queue.empty(); });
      if (s->queue.empty()) return;  // stopping
      job = s->queue.front();
      s->queue.pop_front();
    }
    run_job(s, job);
  }
}

Job *find(pspw_server *s, int id) {
  return id >= 0 && id < (int)s->jobs.size() ? s->jobs[id].get() : nullptr;
}

}  // namespace

using namespace pspw;

extern "C" {

int pspw_server_create(int device, const pspw_server_config *cfg, pspw_server **out) {
  if (!cfg || !out) return fail(PSPW_ERR_ARG, "server_create: null argument");
  if (cfg->slots < 1 || cfg->slots > 256) return fail(PSPW_ERR_ARG, "server_create: slots 1..256");
  if (cfg->filter_prec != PSPW_PREC_F64 && cfg->filter_prec != PSPW_PREC_F32)
    return fail(PSPW_ERR_ARG, "server_create: unknown filter precision");
  PSPW_CUDA(cudaSetDevice(device));
  size_t fr = 0, tot = 0;
  PSPW_CUDA(cudaMemGetInfo(&fr, &tot));
  auto *s = new pspw_server;
  s->device = device;
  s->cfg = *cfg;
  s->budget = cfg->hbm_budget_bytes > 0.0 ? cfg->hbm_budget_bytes : 0.8 * (double)fr;
  s->t0 = clk::now();
  for (int i = 0; i < cfg->slots; i++) s->workers.emplace_back(worker, s);
  *out = s;
  return PSPW_OK;
}

int pspw_server_submit(pspw_server *s, const char *dir, int *job_id) {
  if (!s || !dir || !job_id) return fail(PSPW_ERR_ARG, "server_submit: null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->stop) return fail(PSPW_ERR_ARG, "server_submit: the server is stopping");
  auto job = std::make_unique<Job>();
  job->id = (int)s->jobs.size();
  job->dir = dir;
  job->res.id = job->id;
  job->res.t_submit = s->now();
  *job_id = job->id;
  s->queue.push_back(job.get());
  s->jobs.push_back(std::move(job));
  s->cv_queue.notify_one();
  return PSPW_OK;
}

int pspw_server_wait(pspw_server *s, int job_id, pspw_job_result *res, double *eig, int neig) {
  if (!s || !res) return fail(PSPW_ERR_ARG, "server_wait: null argument");
  std::unique_lock<std::mutex> lk(s->mu);
  Job *job = find(s, job_id);
  if (!job) return fail(PSPW_ERR_ARG, "server_wait: no such job");
  s->cv_done.wait(lk, [&] { return job->done; });
  *res = job->res;
  if (eig && neig > 0)
    for (int i = 0; i < neig; i++) eig[i] = i < (int)job->eig.size() ? job->eig[i] : 0.0;
  return PSPW_OK;
}

int pspw_server_now(pspw_server *s, double *seconds) {
  if (!s || !seconds) return fail(PSPW_ERR_ARG, "server_now: null argument");
  *seconds = s->now();
  return PSPW_OK;
}

int pspw_server_destroy(pspw_server *s) {
  if (!s) return PSPW_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_queue.notify_all();
  s->cv_budget.notify_all();
  for (auto &t : s->workers) t.join();
  delete s;
  return PSPW_OK;
}

}  // extern "C"
