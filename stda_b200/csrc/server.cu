// Served form of the sTDA / sTD-DFT path: a request loop with continuous
// batching over a pool of engine contexts.
//
// The reference is a single-shot program (one molecule per process, main.f);
// serving many molecules is this engine's own layer on top of the C ABI.
// Design:
//   * `slots` contexts (std2g_create), each with its own CUDA stream, cuBLAS /
//     cuSOLVER handles and grow-only device work buffers that stay resident
//     between requests (charges, gamma products, PT buffers, Davidson subspace);
//   * one worker thread per slot; a request is admitted when a slot is free
//     and its estimated device footprint fits the HBM budget beside the
//     requests already in flight (or nothing else is in flight), in FIFO
//     order, so requests that arrive while others run start as soon as slots
//     and memory free up and their kernels overlap on the device;
//   * a request's persistent tensor-core kernels use an equal share of the
//     SMs among the requests in flight when it starts (std2g_set_sm_limit):
//     the whole device when it runs alone, a 1/k share when k run at once, so
//     a large request does not hold every SM while small ones wait;
//   * inputs are copied at submit, results are kept until std2g_server_wait;
//   * a slot that ran a large request (estimate above budget / slots) or
//     ran out of memory gets a fresh context; a request that ran out of
//     memory is retried once with the device to itself.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <string>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/std2g.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Job {
  int64_t ticket = 0;
  int ncent = 0, nmo = 0, nao = 0;
  std::vector<double> xyz, C, eps, occ, S, muL, muV, muM, omega;
  std::vector<int> iaoat;
  // primitive list: AO integrals formed on the device (std2g_load_prims)
  std::vector<int> ipty, ipao, ipat;
  std::vector<double> exip, cxip;
  std2g_params par{};
  int64_t footprint = 0;
  bool exclusive = false;   // admitted only when nothing else is in flight
  Clock::time_point t_submit, t_start, t_end;
  // results
  bool done = false;
  int status = STD2G_OK;
  std2g_result res{};
  std::vector<double> om, fL, fV, RL, RV, resid, alpha, alpha_resid, err, domc;
  std::vector<int> domi, doma;
  // trace: phase times (ms) of the solve and of alpha(omega), load time
  std::vector<double> ph_solve, ph_alpha;
  double load_ms = 0;
};

struct Server {
  std2g_server_opts opts{};
  int64_t budget = 0;
  std::vector<void *> ctxs;
  std::vector<std::thread> workers;
  std::mutex mu;
  std::condition_variable cv_queue, cv_done;
  std::deque<std::shared_ptr<Job>> queue;
  std::unordered_map<int64_t, std::shared_ptr<Job>> jobs;
  int64_t next_ticket = 1;
  int64_t inflight_bytes = 0;
  int inflight = 0;
  int alive_workers = 0;     // workers that still hold a context
  int dead_status = STD2G_OK;  // why the last worker stopped (0 while any is alive)
  bool stop = false;
  int64_t submitted = 0, completed = 0, peak_bytes = 0;
  int peak_inflight = 0;
  int dev_sms = 148;
  void *batch = nullptr;   // shared batched eigensolver (STD2G_FLAG_BATCH_EIGEN)
};

// Estimated device bytes of one request from the input sizes alone (the CSF
// count is not known before the screen): charge and gamma-product tensors
// over the largest possible window (all occupied x all virtual MOs), AO-basis
// work arrays, the PT coupling buffers up to their chunk budget, and either
// the dense CSF matrices or the matrix-free solvers' subspaces, chosen by the
// engine's own rules (std2g_solve: dense eigensolve for all roots, solver 1 or
// up to 320 CSFs; std2g_polarizability: matrix-free for solver 2, when the
// dense form needs more than 24 GB, and in the mixed form (precision 1) with
// solver 0 above 4096 CSFs).
int64_t footprint_estimate(const Job &j, int precision, bool batched) {
  int64_t nocc = 0;
  for (double o : j.occ)
    if (o > 1e-8) ++nocc;
  const int64_t nvir = j.nmo - nocc, N = j.ncent, nao = j.nao;
  const int64_t pairs = nocc * nvir;
  int64_t b = 8 * (3 * N * pairs + 2 * N * nocc * nocc + 2 * N * nvir * nvir);
  b += 8 * (16 * nao * nao + 12 * (int64_t)j.nmo * nao);
  b += std::min<int64_t>(6000000000LL, 8 * pairs * std::min<int64_t>(pairs, 4096));
  const int64_t nci = std::min<int64_t>(pairs, 30000);
  bool dense = j.par.nroots <= 0 || j.par.solver == 1 || nci <= 320;
  if (!j.omega.empty()) {
    const bool resp_mf = j.par.solver == 2 || (double)nci * nci * 8.0 * 10.0 > 24e9 ||
                         (precision == 1 && j.par.solver == 0 && nci > 4096);
    dense |= !resp_mf;
  }
  // the (ij|ab) / (ib|ja) box of a dense build (at most 1.5e8 doubles)
  const int64_t box = 8 * std::min<int64_t>(150000000LL, pairs * pairs);
  if (dense) {
    b += 12 * 8 * nci * nci + box;   // dense K, J, Kx, A+B, A-B, work copies, box
  } else {
    b += 4 * 8 * nci * 512;    // Davidson subspace and products, CG vectors
    // a batched eigensolve (up to 6144 CSFs) builds the dense K, J, Kx, A and B
    if (batched && j.omega.empty() && j.par.rpa == 0)
      b += 5 * 8 * std::min<int64_t>(nci, 6144) * std::min<int64_t>(nci, 6144) + box;
  }
  return b;
}

// result arrays of a job for cap roots, bound into its std2g_result
void room(Job &j, int cap) {
  for (auto *v : {&j.om, &j.fL, &j.fV, &j.RL, &j.RV, &j.resid, &j.err}) v->assign(cap, 0.0);
  j.domc.assign(3 * (size_t)cap, 0.0);
  j.domi.assign(3 * (size_t)cap, 0);
  j.doma.assign(3 * (size_t)cap, 0);
  j.res = std2g_result{};
  j.res.cap = cap;
  j.res.omega = j.om.data();
  j.res.fL = j.fL.data();
  j.res.fV = j.fV.data();
  j.res.RL = j.RL.data();
  j.res.RV = j.RV.data();
  j.res.resid = j.resid.data();
  j.res.err_est = j.err.data();
  j.res.dom_coef = j.domc.data();
  j.res.dom_i = j.domi.data();
  j.res.dom_a = j.doma.data();
}

std::vector<double> phases_of(void *ctx) {
  std::vector<double> ph(32, 0.0);
  ph.resize(std::min(32, std2g_phase_times(ctx, ph.data(), 32)));
  return ph;
}

void run_job(void *ctx, Job &j, bool trace) {
  j.t_start = Clock::now();
  int st = j.ipty.empty()
               ? std2g_load(ctx, j.ncent, j.nmo, j.nao, j.xyz.data(), j.C.data(), j.eps.data(),
                            j.occ.data(), j.iaoat.data(), j.S.data(), j.muL.data(),
                            j.muV.data(), j.muM.data())
               : std2g_load_prims(ctx, j.ncent, j.nmo, j.nao, j.xyz.data(), j.C.data(),
                                  j.eps.data(), j.occ.data(), (int)j.ipty.size(), j.ipty.data(),
                                  j.ipao.data(), j.ipat.data(), j.exip.data(), j.cxip.data());
  if (trace)
    j.load_ms = std::chrono::duration<double, std::milli>(Clock::now() - j.t_start).count();
  if (st == STD2G_OK) {
    const int cap = j.par.nroots > 0 ? j.par.nroots : 20000;
    room(j, cap);
    st = std2g_solve(ctx, &j.par, &j.res);
    if (st == STD2G_ECAP && j.res.nroot > cap) {
      // every root of the window was asked for and there are more than cap:
      // the solve reported the count; run it once more with that much room
      room(j, j.res.nroot);
      st = std2g_solve(ctx, &j.par, &j.res);
    }
    if (trace) j.ph_solve = phases_of(ctx);
  }
  if (st == STD2G_OK && !j.omega.empty()) {
    j.alpha.assign(9 * j.omega.size(), 0.0);
    j.alpha_resid.assign(j.omega.size(), 0.0);
    st = std2g_polarizability(ctx, &j.par, j.omega.data(), (int)j.omega.size(), j.alpha.data(),
                              j.alpha_resid.data());
    if (trace) j.ph_alpha = phases_of(ctx);
  }
  j.status = st;
  j.t_end = Clock::now();
}

void print_trace(const Job &j, int slot, int inflight, int share, bool renewed) {
  using ms = std::chrono::duration<double, std::milli>;
  std::string line = "std2g server: ticket " + std::to_string(j.ticket) + " slot " +
                     std::to_string(slot) + " atoms " + std::to_string(j.ncent) + " status " +
                     std::to_string(j.status) + " inflight " + std::to_string(inflight) +
                     " sms " + std::to_string(share) + (renewed ? " renewed" : "");
  char buf[96];
  std::snprintf(buf, sizeof buf, " queued %.1f run %.1f load %.1f ms",
                ms(j.t_start - j.t_submit).count(), ms(j.t_end - j.t_start).count(), j.load_ms);
  line += buf;
  for (int pass = 0; pass < 2; ++pass) {
    const auto &ph = pass ? j.ph_alpha : j.ph_solve;
    if (ph.empty()) continue;
    line += pass ? " | alpha" : " | solve";
    for (size_t q = 0; q < ph.size(); ++q)
      if (ph[q] >= 0.5) {
        std::snprintf(buf, sizeof buf, " %s %.1f", std2g_phase_name((int)q), ph[q]);
        line += buf;
      }
  }
  std::fprintf(stderr, "%s\n", line.c_str());
}

bool can_admit(const Server &s) {
  if (s.queue.empty()) return false;
  if (s.inflight == 0) return true;
  const Job &j = *s.queue.front();
  return !j.exclusive && s.inflight_bytes + j.footprint <= s.budget;
}

// SMs for the persistent tensor-core kernels of a request that starts with
// `inflight` requests running (itself included): all of them when it runs
// alone (0 = no cap), else an equal share.
int sm_share(const Server &s, int inflight) {
  return inflight <= 1 ? 0 : std::max(1, s.dev_sms / inflight);
}

// Fresh context for a slot: releases every device buffer the old one held.
int renew_context(Server *s, int slot) {
  std2g_destroy(s->ctxs[slot]);
  s->ctxs[slot] = nullptr;
  std2g_opts eo{};
  eo.device = s->opts.device;
  eo.precision = s->opts.precision;
  eo.flags = s->opts.flags;
  void *ctx = nullptr;
  const int st = std2g_create(&ctx, &eo);
  if (st != STD2G_OK) return st;
  s->ctxs[slot] = ctx;
  if (s->batch) std2g_attach_batch(ctx, s->batch);
  return STD2G_OK;
}

void worker(Server *s, int slot) {
  for (;;) {
    std::shared_ptr<Job> job;
    int share = 0, inflight_at_start = 1;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      s->cv_queue.wait(lk, [&] { return s->stop || can_admit(*s); });
      if (s->stop) return;
      job = s->queue.front();
      s->queue.pop_front();
      s->inflight_bytes += job->footprint;
      ++s->inflight;
      s->peak_inflight = std::max(s->peak_inflight, s->inflight);
      s->peak_bytes = std::max(s->peak_bytes, s->inflight_bytes);
      share = sm_share(*s, s->inflight);
      inflight_at_start = s->inflight;
    }
    std2g_set_sm_limit(s->ctxs[slot], share);
    run_job(s->ctxs[slot], *job, s->opts.trace > 0);
    // Context buffers only grow; after a large request (or a failed one) the
    // slot starts again from a fresh context so that idle slots do not hold
    // memory the admission rule no longer counts.
    const bool out_of_memory = job->status == STD2G_ENOMEM;
    const bool large = job->footprint > s->budget / (int64_t)s->ctxs.size();
    int renew = STD2G_OK;
    if (out_of_memory || large) renew = renew_context(s, slot);
    if (s->opts.trace > 0) print_trace(*job, slot, inflight_at_start, share, out_of_memory || large);
    const bool alive = renew == STD2G_OK;
    bool retry = out_of_memory && !job->exclusive && alive;
    {
      std::lock_guard<std::mutex> lk(s->mu);
      s->inflight_bytes -= job->footprint;
      --s->inflight;
      if (retry) {   // once more, with the device to itself
        job->exclusive = true;
        job->status = STD2G_OK;
        s->queue.push_front(job);
      } else {
        ++s->completed;
        job->done = true;
      }
    }
    if (!alive) {
      // this slot could not get a new context; when it was the last one,
      // nothing can run what is queued, so those requests fail with the
      // reason (and later submits are refused) instead of waiting forever
      std::lock_guard<std::mutex> lk(s->mu);
      if (--s->alive_workers == 0) {
        s->dead_status = renew;
        for (auto &q : s->queue) {
          q->status = renew;
          q->done = true;
          ++s->completed;
        }
        s->queue.clear();
      }
    }
    s->cv_done.notify_all();
    s->cv_queue.notify_all();
    if (!alive) return;
  }
}

template <typename T>
std::vector<T> copy_of(const T *p, size_t n) {
  return std::vector<T>(p, p + n);
}

}  // namespace

extern "C" {

int std2g_server_create(void **srv, const std2g_server_opts *o) {
  if (!srv || !o || o->slots < 1 || o->slots > 64) return STD2G_EINVAL;
  auto s = std::make_unique<Server>();
  s->opts = *o;
  if (cudaSetDevice(o->device) != cudaSuccess) return STD2G_ENODEV;
  size_t free_b = 0, total_b = 0;
  if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) return STD2G_ECUDA;
  s->budget = o->hbm_budget > 0 ? o->hbm_budget : (int64_t)(0.8 * (double)free_b);
  cudaDeviceGetAttribute(&s->dev_sms, cudaDevAttrMultiProcessorCount, o->device);
  for (int k = 0; k < o->slots; ++k) {
    std2g_opts eo{};
    eo.device = o->device;
    eo.precision = o->precision;
    eo.flags = o->flags;
    eo.verbose = 0;
    void *ctx = nullptr;
    int st = std2g_create(&ctx, &eo);
    if (st != STD2G_OK) {
      for (void *c : s->ctxs) std2g_destroy(c);
      return st;
    }
    s->ctxs.push_back(ctx);
  }
  if (o->flags & STD2G_FLAG_BATCH_EIGEN) {
    int st = std2g_batch_create(o->device, &s->batch);
    for (void *c : s->ctxs)
      if (st == STD2G_OK) st = std2g_attach_batch(c, s->batch);
    if (st != STD2G_OK) {
      for (void *c : s->ctxs) std2g_destroy(c);
      std2g_batch_destroy(s->batch);
      return st;
    }
  }
  s->alive_workers = o->slots;
  for (int k = 0; k < o->slots; ++k) s->workers.emplace_back(worker, s.get(), k);
  *srv = s.release();
  return STD2G_OK;
}

int std2g_server_submit(void *srv, const std2g_request *rq, int64_t *ticket) {
  if (!srv || !rq || !ticket || rq->ncent <= 0 || rq->nmo <= 0 || rq->nao <= 0 || !rq->xyz ||
      !rq->C || !rq->eps || !rq->occ || rq->nomega < 0 || (rq->nomega > 0 && !rq->omega) ||
      rq->nprims < 0)
    return STD2G_EINVAL;
  const bool prims = rq->nprims > 0;
  if (prims ? (!rq->ipty || !rq->ipao || !rq->ipat || !rq->exip || !rq->cxip)
            : (!rq->iaoat || !rq->S || !rq->mu_L || !rq->mu_V || !rq->mu_M))
    return STD2G_EINVAL;
  auto *s = (Server *)srv;
  auto j = std::make_shared<Job>();
  const size_t npk = (size_t)rq->nao * (rq->nao + 1) / 2;
  j->ncent = rq->ncent;
  j->nmo = rq->nmo;
  j->nao = rq->nao;
  j->xyz = copy_of(rq->xyz, 4 * (size_t)rq->ncent);
  j->C = copy_of(rq->C, (size_t)rq->nao * rq->nmo);
  j->eps = copy_of(rq->eps, (size_t)rq->nmo);
  j->occ = copy_of(rq->occ, (size_t)rq->nmo);
  if (prims) {
    const size_t np = (size_t)rq->nprims;
    j->ipty = copy_of(rq->ipty, np);
    j->ipao = copy_of(rq->ipao, np);
    j->ipat = copy_of(rq->ipat, np);
    j->exip = copy_of(rq->exip, np);
    j->cxip = copy_of(rq->cxip, np);
  } else {
    j->iaoat = copy_of(rq->iaoat, (size_t)rq->nao);
    j->S = copy_of(rq->S, npk);
    j->muL = copy_of(rq->mu_L, 3 * npk);
    j->muV = copy_of(rq->mu_V, 3 * npk);
    j->muM = copy_of(rq->mu_M, 3 * npk);
  }
  if (rq->nomega > 0) j->omega = copy_of(rq->omega, (size_t)rq->nomega);
  j->par = rq->params;
  j->footprint = footprint_estimate(*j, s->opts.precision,
                                    (s->opts.flags & STD2G_FLAG_BATCH_EIGEN) != 0);
  j->t_submit = Clock::now();
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->alive_workers == 0) return s->dead_status;   // no slot left to run it
    j->ticket = s->next_ticket++;
    s->jobs[j->ticket] = j;
    s->queue.push_back(j);
    ++s->submitted;
  }
  s->cv_queue.notify_all();
  *ticket = j->ticket;
  return STD2G_OK;
}

int std2g_server_poll(void *srv, int64_t ticket, int *done) {
  if (!srv || !done) return STD2G_EINVAL;
  auto *s = (Server *)srv;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->jobs.find(ticket);
  if (it == s->jobs.end()) return STD2G_EINVAL;
  *done = it->second->done ? 1 : 0;
  return STD2G_OK;
}

int std2g_server_wait(void *srv, int64_t ticket, std2g_result *res, double *alpha,
                      double *alpha_resid, double *timing_ms) {
  if (!srv) return STD2G_EINVAL;
  auto *s = (Server *)srv;
  std::shared_ptr<Job> j;
  {
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->jobs.find(ticket);
    if (it == s->jobs.end()) return STD2G_EINVAL;
    j = it->second;
    s->cv_done.wait(lk, [&] { return j->done; });
    if (res && j->status == STD2G_OK && res->cap < j->res.nroot) {
      // keep the ticket so that the caller can wait again with more room
      res->nroot = j->res.nroot;
      return STD2G_ECAP;
    }
    s->jobs.erase(ticket);
  }
  if (timing_ms) {
    auto ms = [](Clock::time_point a, Clock::time_point b) {
      return std::chrono::duration<double, std::milli>(b - a).count();
    };
    timing_ms[0] = ms(j->t_submit, j->t_start);   // queued
    timing_ms[1] = ms(j->t_start, j->t_end);      // running
    timing_ms[2] = ms(j->t_submit, j->t_end);     // latency
  }
  if (j->status != STD2G_OK) return j->status;
  if (res) {
    const int n = j->res.nroot;
    double *dst[8] = {res->omega, res->fL, res->fV, res->RL,
                      res->RV,    res->resid, res->err_est, res->dom_coef};
    const std::vector<double> *src[8] = {&j->om, &j->fL,    &j->fV,  &j->RL,
                                         &j->RV, &j->resid, &j->err, &j->domc};
    for (int q = 0; q < 8; ++q)
      if (dst[q]) std::copy(src[q]->begin(), src[q]->begin() + (q == 7 ? 3 * n : n), dst[q]);
    if (res->dom_i) std::copy(j->domi.begin(), j->domi.begin() + 3 * n, res->dom_i);
    if (res->dom_a) std::copy(j->doma.begin(), j->doma.begin() + 3 * n, res->dom_a);
    const int cap = res->cap;
    std2g_result keep = *res;
    *res = j->res;
    res->cap = cap;
    res->omega = keep.omega;
    res->fL = keep.fL;
    res->fV = keep.fV;
    res->RL = keep.RL;
    res->RV = keep.RV;
    res->resid = keep.resid;
    res->err_est = keep.err_est;
    res->dom_coef = keep.dom_coef;
    res->dom_i = keep.dom_i;
    res->dom_a = keep.dom_a;
  }
  if (alpha && !j->alpha.empty()) std::copy(j->alpha.begin(), j->alpha.end(), alpha);
  if (alpha_resid && !j->alpha_resid.empty())
    std::copy(j->alpha_resid.begin(), j->alpha_resid.end(), alpha_resid);
  return STD2G_OK;
}

int std2g_server_stats(void *srv, int64_t *stats) {
  if (!srv || !stats) return STD2G_EINVAL;
  auto *s = (Server *)srv;
  std::lock_guard<std::mutex> lk(s->mu);
  stats[0] = s->submitted;
  stats[1] = s->completed;
  stats[2] = s->inflight;
  stats[3] = s->peak_inflight;
  stats[4] = s->inflight_bytes;
  stats[5] = s->peak_bytes;
  stats[6] = s->budget;
  return STD2G_OK;
}

void std2g_server_destroy(void *srv) {
  if (!srv) return;
  auto *s = (Server *)srv;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_queue.notify_all();
  for (auto &t : s->workers) t.join();
  for (void *c : s->ctxs)
    if (c) std2g_destroy(c);
  std2g_batch_destroy(s->batch);
  delete s;
}

int std2g_server_batch_stats(void *srv, int64_t *problems, int64_t *iterations,
                             int64_t *members, double *ms) {
  if (!srv || !problems || !iterations || !members) return STD2G_EINVAL;
  auto *s = (Server *)srv;
  if (!s->batch) {
    *problems = *iterations = *members = 0;
    if (ms) ms[0] = ms[1] = 0.0;
    return STD2G_OK;
  }
  return std2g_batch_stats(s->batch, problems, iterations, members, ms);
}

}  // extern "C"
