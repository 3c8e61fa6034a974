// Batched Davidson: the TDA eigensolves of many molecules in lockstep.
//
// A small molecule's blocked Davidson (davidson.cuh) does microseconds of
// arithmetic per iteration but takes ~0.7 ms per iteration on the device,
// nearly all of it kernel-launch and host-synchronisation latency (about 60
// launches and three host synchronisations per iteration, the Rayleigh-Ritz
// solve alone 0.3-0.6 ms of serial cluster steps).  Here one coordinator
// thread with one stream runs the iterations of every molecule that has
// reached its eigensolve together: each step of an iteration is one launch for
// all of them (grouped FP64 products over a per-launch table of members,
// k_dgemm_grouped; batched Rayleigh-Ritz solves, symeig_small_batched; batched
// residual, preconditioner and Cholesky-QR kernels below), and the three host
// synchronisations of an iteration are shared by the whole batch.
//
// Continuous batching at the iteration level: a molecule's solve thread hands
// its problem over (dense FP64 A, its diagonal, the root request) and waits; a
// problem joins the batch at the next iteration boundary and leaves it when its
// wanted roots have converged, so molecules of different sizes and iteration
// counts flow through the same launches.  The algorithm of every member is
// davidson()'s (same buffer roots, subspace limit, preconditioner, BCGS2
// orthogonalisation with Cholesky QR, restarts, convergence test), with the
// product A V taken from the dense matrix; the reference diagonalises the
// same A with ssyevr (stda.f:1133-1150).
#pragma once

#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "common.cuh"
#include "davidson.cuh"
#include "dgemm.cuh"
#include "symeig_small.cuh"

namespace std2g {

// One member of a batched small-kernel launch (blockIdx.y or .z selects it).
struct BdJob {
  double *V, *W, *H, *Hs, *theta, *X, *R, *T, *tmp, *G, *Li, *lam, *Tb;
  const double *diag;
  const int *cols;
  int *einfo;
  int n, m, nb, k, nc, mmax;
  int off;   // offset of the member's entries in the gathered output arrays
};

// H[c + ld r] = H[r + ld c] for r < m, c in [m, m + nb) (the new rows of the
// projected matrix from the symmetry of A)
__global__ void k_bd_mirror(const BdJob *__restrict__ jobs) {
  const BdJob j = jobs[blockIdx.y];
  const int64_t total = (int64_t)j.m * j.nb;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int c = j.m + (int)(t / j.m), r = (int)(t % j.m);
    j.H[c + (int64_t)j.mmax * r] = j.H[r + (int64_t)j.mmax * c];
  }
}

// R[:, c] -= theta[c] X[:, c] for c < k; part[(b * kcap + c) * kColSplit + x]
// = partial |R[:, c]|^2 over the x-th slice of rows (grid kColSplit x kcap x b)
__global__ void k_bd_resid(const BdJob *__restrict__ jobs, int kcap, double *__restrict__ part) {
  const BdJob j = jobs[blockIdx.z];
  const int c = blockIdx.y;
  double s = 0.0;
  if (c < j.k) {
    const double th = j.theta[c];
    const int64_t chunk = (j.n + gridDim.x - 1) / gridDim.x;
    const int64_t i0 = chunk * blockIdx.x, i1 = min((int64_t)j.n, i0 + chunk);
    for (int64_t i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
      const int64_t o = i + (int64_t)j.n * c;
      const double r = j.R[o] - th * j.X[o];
      j.R[o] = r;
      s += r * r;
    }
  }
  __shared__ double red[256];
  s = block_sum256(s, red);
  if (threadIdx.x == 0)
    part[((int64_t)blockIdx.z * kcap + c) * gridDim.x + blockIdx.x] = s;
}

// gathered outputs of the residual step: out[off + c] = |R[:, c]| (in order
// of the slices), out[tot + off + c] = theta[c], info[b] = the Rayleigh-Ritz
// status of member b
__global__ void k_bd_resid_finish(const BdJob *__restrict__ jobs, int njobs, int kcap,
                                  const double *__restrict__ part, int nsplit, int tot,
                                  double *__restrict__ out, int *__restrict__ info) {
  const int b = blockIdx.x;
  if (b >= njobs) return;
  const BdJob j = jobs[b];
  for (int c = threadIdx.x; c < j.k; c += blockDim.x) {
    double s = 0.0;
    for (int x = 0; x < nsplit; ++x) s += part[((int64_t)b * kcap + c) * nsplit + x];
    out[j.off + c] = sqrt(s);
    out[tot + j.off + c] = j.theta[c];
  }
  if (threadIdx.x == 0) info[b] = *j.einfo;
}

// T[:, q] = R[:, cols[q]] / (theta[cols[q]] - diag), guarded away from zero,
// for q < nc (the preconditioner of davidson())
__global__ void k_bd_precond(const BdJob *__restrict__ jobs) {
  const BdJob j = jobs[blockIdx.y];
  const int64_t total = (int64_t)j.n * j.nc;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int q = (int)(t / j.n), i = (int)(t - (int64_t)q * j.n);
    const int c = j.cols[q];
    double d = j.theta[c] - j.diag[i];
    if (fabs(d) < 1e-4) d = d < 0 ? -1e-4 : 1e-4;
    j.T[t] = j.R[i + (int64_t)j.n * c] / d;
  }
}

// restart to the Ritz vectors: V[:, :k] = X, W[:, :k] = tmp (= W Y_k),
// H[:k, :k] = diag(theta) (ld mmax)
__global__ void k_bd_restart(const BdJob *__restrict__ jobs) {
  const BdJob j = jobs[blockIdx.y];
  const int64_t nk = (int64_t)j.n * j.k, kk = (int64_t)j.k * j.k;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nk + kk;
       t += (int64_t)gridDim.x * blockDim.x) {
    if (t < nk) {
      j.V[t] = j.X[t];
      j.W[t] = j.tmp[t];
    } else {
      const int q = (int)(t - nk), c = q / j.k, r = q - c * j.k;
      j.H[r + (int64_t)j.mmax * c] = r == c ? j.theta[r] : 0.0;
    }
  }
}

// part[(b * kcap + c) * kColSplit + x] = partial |Tb[:, c]|^2, c < nc
__global__ void k_bd_colnorm(const BdJob *__restrict__ jobs, int kcap, double *__restrict__ part) {
  const BdJob j = jobs[blockIdx.z];
  const int c = blockIdx.y;
  double s = 0.0;
  if (c < j.nc) {
    const int64_t chunk = (j.n + gridDim.x - 1) / gridDim.x;
    const int64_t i0 = chunk * blockIdx.x, i1 = min((int64_t)j.n, i0 + chunk);
    const double *t = j.Tb + (int64_t)j.n * c;
    for (int64_t i = i0 + threadIdx.x; i < i1; i += blockDim.x) s += t[i] * t[i];
  }
  __shared__ double red[256];
  s = block_sum256(s, red);
  if (threadIdx.x == 0)
    part[((int64_t)blockIdx.z * kcap + c) * gridDim.x + blockIdx.x] = s;
}

// lam[c] = |Tb[:, c]| from the partial sums (in order), c < nc
__global__ void k_bd_colnorm_finish(const BdJob *__restrict__ jobs, int njobs, int kcap,
                                    const double *__restrict__ part, int nsplit) {
  const int b = blockIdx.x;
  if (b >= njobs) return;
  const BdJob j = jobs[b];
  for (int c = threadIdx.x; c < j.nc; c += blockDim.x) {
    double s = 0.0;
    for (int x = 0; x < nsplit; ++x) s += part[((int64_t)b * kcap + c) * nsplit + x];
    j.lam[c] = sqrt(s);
  }
}

// Tb[:, c] *= 1 / lam[c] (0 for a zero column), c < nc
__global__ void k_bd_scale(const BdJob *__restrict__ jobs) {
  const BdJob j = jobs[blockIdx.y];
  const int64_t total = (int64_t)j.n * j.nc;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const double v = j.lam[t / j.n];
    j.Tb[t] *= v > 0 ? 1.0 / v : 0.0;
  }
}

// Cholesky factor and inverse of every member's Gram matrix G (nc x nc, one
// CTA each, chol_inv_body); stat[2 b], stat[2 b + 1] as k_chol_inv's
__global__ void __launch_bounds__(256)
k_bd_chol_inv(const BdJob *__restrict__ jobs, double tol, double *__restrict__ stat) {
  const BdJob j = jobs[blockIdx.x];
  chol_inv_body(j.G, j.nc, tol, j.Li, stat + 2 * blockIdx.x);
}

// Tb[:, :nc] = tmp[:, :nc] (the orthonormalised block written through tmp)
__global__ void k_bd_copy_block(const BdJob *__restrict__ jobs) {
  const BdJob j = jobs[blockIdx.y];
  const int64_t total = (int64_t)j.n * j.nc;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x)
    j.Tb[t] = j.tmp[t];
}

// k unit vectors on the given rows: V[:, q] = e_{idx[q]}
__global__ void k_bd_unit(double *__restrict__ V, int n, const int *__restrict__ idx, int k) {
  const int64_t total = (int64_t)n * k;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int q = (int)(t / n), i = (int)(t - (int64_t)q * n);
    V[t] = i == idx[q] ? 1.0 : 0.0;
  }
}

// A molecule's eigenproblem handed to the batch.  The solve thread fills the
// inputs, sizes the work buffers of its own DavidsonWork (bd_prepare), records
// `ready` on its stream and calls BatchDavidson::solve, which returns when the
// problem has left the batch; `done` (recorded on the batch's stream) orders
// the solve thread's later work after the results.
struct BatchProblem {
  // inputs
  DavidsonWork *dw = nullptr;
  cublasHandle_t blas = nullptr;
  cusolverDnHandle_t sol = nullptr;
  const double *A = nullptr, *diag = nullptr;   // dense A (n x n), diag(A)
  int n = 0, kwant = 0, max_iter = 300;
  double tol = 1e-6;
  double *omega_out = nullptr, *X_out = nullptr;   // kwant values, n x kwant
  std::vector<int> init_idx;                        // k rows of the lowest diagonal entries
  cudaEvent_t ready = nullptr, done = nullptr;
  // results
  int status = STD2G_OK;
  std::string msg;
  int nconv = 0, iters = 0;
  int64_t matvecs = 0;
  double max_resid = 0;
  std::vector<double> final_resid, final_theta;
  bool finished = false;
  // batch state
  int k = 0, mmax = 0, m = 0, nb = 0, nc = 0, ncur = 0;
  bool restart = false, ortho_open = false;
  double *Tb = nullptr;
  std::vector<int> unc;
};

// davidson()'s block sizes for kwant wanted roots of an n-dimensional problem
inline void bd_sizes(int n, int kwant, int *k, int *mmax) {
  const int kk = std::min(n, kwant + std::max(4, kwant / 4));
  *k = kk;
  *mmax = std::min(n, std::max(kk + 32, std::min(kSymEigMaxN, 6 * kk)));
}

// whether a problem fits the batched solver (its Rayleigh-Ritz and Cholesky
// QR stay within the single-CTA / cluster kernels)
inline bool bd_fits(int n, int kwant) {
  if (kwant < 1 || n < 2) return false;
  int k = 0, mmax = 0;
  bd_sizes(n, kwant, &k, &mmax);
  return k <= kCholMax && mmax <= kSymEigMaxN && k < n;
}

// Work buffers of a problem, in the solve thread's DavidsonWork (grow-only;
// allocated on the solve thread, never by the batch).
inline void bd_prepare(BatchProblem &p) {
  DavidsonWork &dw = *p.dw;
  bd_sizes(p.n, p.kwant, &p.k, &p.mmax);
  const size_t n = p.n, k = p.k, mmax = p.mmax;
  dw.V.ensure(n * mmax);
  dw.W.ensure(n * mmax);
  dw.H.ensure(mmax * mmax);
  dw.Hs.ensure(mmax * mmax);
  dw.theta.ensure(mmax);
  dw.X.ensure(n * k);
  dw.R.ensure(n * k);
  dw.T.ensure(n * k);
  dw.tmp.ensure(n * k);
  dw.proj.ensure(mmax * k + 4);
  dw.G.ensure(k * k);
  dw.Gc.ensure(k * k);
  dw.lam.ensure(k);
  dw.eigwork.ensure(symeig_work_doubles((int)mmax, (int)k));
  dw.idx.ensure(k);
  dw.einfo.ensure(1);
}

class BatchDavidson {
 public:
  // creates the batch's stream on `device` (the calling thread's current
  // device is left as it was) and starts the coordinator thread
  explicit BatchDavidson(int device) : device_(device) {
    int prev = -1;
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    S2G_CUDA(cudaSetDevice(device));
    // the highest stream priority: the batch's small launches are the
    // critical path of every attached solve, so their blocks go first when
    // the solves' own (large-grid) kernels occupy the device
    int least = 0, greatest = 0;
    cudaError_t e = cudaDeviceGetStreamPriorityRange(&least, &greatest);
    if (e == cudaSuccess)
      e = cudaStreamCreateWithPriority(&cs_, cudaStreamNonBlocking, greatest);
    if (prev >= 0) cudaSetDevice(prev);
    S2G_CUDA(e);
    th_ = std::thread([this] { loop(); });
  }
  int device() const { return device_; }
  ~BatchDavidson() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    if (th_.joinable()) th_.join();
    if (cs_) cudaStreamDestroy(cs_);
  }

  BatchDavidson(const BatchDavidson &) = delete;
  BatchDavidson &operator=(const BatchDavidson &) = delete;

  // Hands p to the batch and waits until it has left it (thread-safe).
  void solve(BatchProblem &p) {
    {
      std::unique_lock<std::mutex> lk(mu_);
      if (stop_) throw Error{STD2G_ESTATE, "batched eigensolver stopped"};
      p.finished = false;
      pending_.push_back(&p);
    }
    cv_.notify_all();
    std::unique_lock<std::mutex> lk(mu_);
    cv_done_.wait(lk, [&] { return p.finished; });
  }

  // problems solved, batched iterations run, the sum over iterations of the
  // members in flight (mean batch = members / iterations), and in ms[0..1]
  // the wall time of the iterations, total and up to their first host
  // synchronisation (products, Rayleigh-Ritz, residuals)
  void stats(int64_t *problems, int64_t *iterations, int64_t *members, double *ms) {
    std::lock_guard<std::mutex> lk(mu_);
    *problems = n_problems_;
    *iterations = n_iters_;
    *members = n_members_;
    if (ms) {
      ms[0] = t_iter_;
      ms[1] = t_first_;
    }
  }

 private:
  int device_;
  cudaStream_t cs_ = nullptr;
  std::thread th_;
  std::mutex mu_;
  std::condition_variable cv_, cv_done_;
  std::deque<BatchProblem *> pending_;
  bool stop_ = false;
  int64_t n_problems_ = 0, n_iters_ = 0, n_members_ = 0;
  double t_iter_ = 0, t_first_ = 0;   // wall ms of the iterations, up to their first sync
  double t_first_sync_ = 0;
  Dgemm dg_;
  DBuf<SymEigJob> dsj_;
  DBuf<BdJob> djob_;
  DBuf<double> part_, gout_, gstat_;
  DBuf<int> ginfo_, gcols_;
  // page-locked staging of the launch descriptors (reset after each host
  // synchronisation) and of the values read back
  PinnedArena stage_, back_;

  void loop();
  void admit(BatchProblem &p);
  void iterate(std::vector<BatchProblem *> &act);
  const BdJob *upload(const std::vector<BdJob> &jobs);
  void finish(BatchProblem &p);
};

// ---------------------------------------------------------------- host side
inline int bd_blocks(int64_t work) {
  return (int)std::max<int64_t>(1, std::min<int64_t>(div_up(work, 256), 1024));
}

inline const BdJob *BatchDavidson::upload(const std::vector<BdJob> &jobs) {
  BdJob *d = djob_.ensure(jobs.size());
  const void *h = stage_.put(jobs.data(), sizeof(BdJob) * jobs.size());
  S2G_CUDA(cudaMemcpyAsync(d, h, sizeof(BdJob) * jobs.size(), cudaMemcpyHostToDevice, cs_));
  return d;
}

inline BdJob bd_job(const BatchProblem &p) {
  const DavidsonWork &dw = *p.dw;
  BdJob j{};
  j.V = dw.V.get();
  j.W = dw.W.get();
  j.H = dw.H.get();
  j.Hs = dw.Hs.get();
  j.theta = dw.theta.get();
  j.X = dw.X.get();
  j.R = dw.R.get();
  j.T = dw.T.get();
  j.tmp = dw.tmp.get();
  j.G = dw.G.get();
  j.Li = dw.Gc.get();
  j.lam = dw.lam.get();
  j.Tb = p.Tb;
  j.diag = p.diag;
  j.einfo = dw.einfo.get();
  j.n = p.n;
  j.m = p.m;
  j.nb = p.nb;
  j.k = p.k;
  j.nc = p.nc;
  j.mmax = p.mmax;
  return j;
}

inline void BatchDavidson::admit(BatchProblem &p) {
  DavidsonWork &dw = *p.dw;
  if ((int)p.init_idx.size() < p.k) throw Error{STD2G_EINVAL, "batched Davidson: initial rows"};
  S2G_CUDA(cudaStreamWaitEvent(cs_, p.ready, 0));
  p.m = 0;
  p.nb = p.k;
  p.iters = 0;
  p.matvecs = 0;
  p.nconv = 0;
  S2G_CUDA(cudaMemcpyAsync(dw.idx.get(), stage_.put(p.init_idx.data(), sizeof(int) * p.k),
                           sizeof(int) * p.k, cudaMemcpyHostToDevice, cs_));
  S2G_LAUNCH(k_bd_unit, bd_blocks((int64_t)p.n * p.k), 256, 0, cs_, dw.V.get(), p.n, dw.idx.get(),
             p.k);
  S2G_CUDA(cudaMemsetAsync(dw.einfo.get(), 0, sizeof(int), cs_));
}

// results of a problem that leaves the batch (final_resid / final_theta set
// from its last residual step): the wanted Ritz pairs to the caller's arrays
// (on the batch's stream, then `done`).  Never throws: a failed copy becomes
// the problem's status.  The caller has already taken p out of the active set
// (once finished, its owner may return and p no longer exists).
inline void BatchDavidson::finish(BatchProblem &p) {
  DavidsonWork &dw = *p.dw;
  if (!p.final_resid.empty())
    p.max_resid = *std::max_element(p.final_resid.begin(),
                                    p.final_resid.begin() + std::min<size_t>(p.kwant,
                                                                             p.final_resid.size()));
  try {
    S2G_CUDA(cudaMemcpyAsync(p.omega_out, dw.theta.get(), sizeof(double) * p.kwant,
                             cudaMemcpyDeviceToDevice, cs_));
    S2G_CUDA(cudaMemcpyAsync(p.X_out, dw.X.get(), sizeof(double) * p.n * p.kwant,
                             cudaMemcpyDeviceToDevice, cs_));
    S2G_CUDA(cudaEventRecord(p.done, cs_));
  } catch (const Error &e) {
    if (p.status == STD2G_OK) {
      p.status = e.code;
      p.msg = e.msg;
    }
    cudaEventRecord(p.done, cs_);
  }
  {
    std::lock_guard<std::mutex> lk(mu_);
    p.finished = true;
    ++n_problems_;
  }
  cv_done_.notify_all();
}

inline void BatchDavidson::loop() {
  cudaSetDevice(device_);
  std::vector<BatchProblem *> act;
  auto fail = [&](BatchProblem *p, const Error &e) {
    p->status = e.code;
    p->msg = e.msg;
    cudaEventRecord(p->done, cs_);
    {
      std::lock_guard<std::mutex> lk(mu_);
      p->finished = true;
    }
    cv_done_.notify_all();
  };
  for (;;) {
    std::vector<BatchProblem *> add;
    {
      std::unique_lock<std::mutex> lk(mu_);
      cv_.wait(lk, [&] { return stop_ || !pending_.empty() || !act.empty(); });
      if (stop_ && pending_.empty() && act.empty()) return;
      while (!pending_.empty()) {
        add.push_back(pending_.front());
        pending_.pop_front();
      }
    }
    for (BatchProblem *p : add) {
      try {
        admit(*p);
        act.push_back(p);
      } catch (const Error &e) {
        fail(p, e);
      } catch (const std::exception &e) {
        fail(p, Error{STD2G_ECUDA, e.what()});
      }
    }
    if (act.empty()) continue;
    const int64_t members = (int64_t)act.size();
    const auto t0 = std::chrono::steady_clock::now();
    try {
      iterate(act);
    } catch (const Error &e) {
      for (BatchProblem *p : act) fail(p, e);
      act.clear();
    } catch (const std::exception &e) {
      for (BatchProblem *p : act) fail(p, Error{STD2G_ECUDA, e.what()});
      act.clear();
    }
    std::lock_guard<std::mutex> lk(mu_);
    ++n_iters_;
    n_members_ += members;
    t_iter_ += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0)
                   .count();
    t_first_ += t_first_sync_;
  }
}

// One Davidson iteration of every member of `act` (davidson()'s steps, each a
// single launch for all members); members that converge, reach their
// iteration limit or run out of new directions leave `act`.
inline void BatchDavidson::iterate(std::vector<BatchProblem *> &act) {
  const int P = (int)act.size();
  const auto t_start = std::chrono::steady_clock::now();
  // ---- sigma = A V_new and the new columns of H = V^T W (rows by symmetry)
  {
    std::vector<DgProblem> gs, gh;
    std::vector<BdJob> mj;
    for (BatchProblem *p : act) {
      DavidsonWork &dw = *p->dw;
      const int64_t n = p->n;
      double *Vn = dw.V.get() + n * p->m, *Wn = dw.W.get() + n * p->m;
      gs.push_back(DgProblem{p->n, p->nb, p->n, 1.0, 0.0, p->A, Vn, Wn, n, n, n});
      gh.push_back(DgProblem{p->m + p->nb, p->nb, p->n, 1.0, 0.0, dw.V.get(), Wn,
                             dw.H.get() + (int64_t)p->mmax * p->m, n, n, p->mmax});
      if (p->m > 0) mj.push_back(bd_job(*p));
    }
    dg_.grouped(cs_, false, false, gs, &stage_);
    dg_.grouped(cs_, true, false, gh, &stage_);
    if (!mj.empty()) {
      int64_t mx = 0;
      for (const BdJob &j : mj) mx = std::max<int64_t>(mx, (int64_t)j.m * j.nb);
      const BdJob *d = upload(mj);
      S2G_LAUNCH(k_bd_mirror, dim3(bd_blocks(mx), (unsigned)mj.size()), 256, 0, cs_, d);
    }
    for (BatchProblem *p : act) {
      p->matvecs += p->nb;
      p->m += p->nb;
      ++p->iters;
    }
  }
  // ---- Rayleigh-Ritz: lowest k pairs of every member's H (ld mmax)
  {
    std::vector<SymEigJob> sj;
    for (BatchProblem *p : act) {
      DavidsonWork &dw = *p->dw;
      sj.push_back(SymEigJob{dw.H.get(), p->mmax, p->m, std::min(p->k, p->m), dw.theta.get(),
                             dw.Hs.get(), p->m, dw.eigwork.get(), dw.einfo.get()});
    }
    symeig_small_batched(cs_, sj, dsj_, &stage_);
  }
  // ---- Ritz vectors X = V Y, residuals R = W Y - X theta and their norms
  std::vector<double> h_out;
  std::vector<int> h_info(P);
  int tot = 0, kcap = 0;
  {
    std::vector<DgProblem> gx;
    std::vector<BdJob> rj;
    for (BatchProblem *p : act) {
      DavidsonWork &dw = *p->dw;
      const int64_t n = p->n;
      gx.push_back(DgProblem{p->n, p->k, p->m, 1.0, 0.0, dw.V.get(), dw.Hs.get(), dw.X.get(), n,
                             p->m, n});
      gx.push_back(DgProblem{p->n, p->k, p->m, 1.0, 0.0, dw.W.get(), dw.Hs.get(), dw.R.get(), n,
                             p->m, n});
      BdJob j = bd_job(*p);
      j.off = tot;
      tot += p->k;
      kcap = std::max(kcap, p->k);
      rj.push_back(j);
    }
    dg_.grouped(cs_, false, false, gx, &stage_);
    const BdJob *d = upload(rj);
    double *part = part_.ensure((size_t)P * kcap * kColSplit);
    double *out = gout_.ensure(2 * (size_t)tot);
    int *info = ginfo_.ensure(P);
    S2G_LAUNCH(k_bd_resid, dim3(kColSplit, (unsigned)kcap, (unsigned)P), 256, 0, cs_, d, kcap,
               part);
    S2G_LAUNCH(k_bd_resid_finish, P, 128, 0, cs_, d, P, kcap, part, kColSplit, tot, out, info);
    back_.reset();
    double *b_out = (double *)back_.take(sizeof(double) * 2 * tot);
    int *b_info = (int *)back_.take(sizeof(int) * P);
    S2G_CUDA(cudaMemcpyAsync(b_out, out, sizeof(double) * 2 * tot, cudaMemcpyDeviceToHost, cs_));
    S2G_CUDA(cudaMemcpyAsync(b_info, info, sizeof(int) * P, cudaMemcpyDeviceToHost, cs_));
    S2G_CUDA(cudaStreamSynchronize(cs_));
    stage_.reset();
    h_out.assign(b_out, b_out + 2 * (size_t)tot);
    std::copy(b_info, b_info + P, h_info.begin());
    t_first_sync_ = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() -
                                                              t_start)
                        .count();
  }
  // ---- convergence (davidson()'s test); members that stay get their
  // unconverged columns
  std::vector<BatchProblem *> stay, leaving;
  {
    int off = 0;
    for (int b = 0; b < P; ++b) {
      BatchProblem *p = act[b];
      const double *rn = h_out.data() + off, *th = h_out.data() + tot + off;
      off += p->k;
      p->final_resid.assign(rn, rn + p->k);
      p->final_theta.assign(th, th + p->k);
      if (h_info[b] != 0) {
        p->status = STD2G_ENOCONV;
        p->msg = "Davidson: Rayleigh-Ritz eigensolve failed (" + std::to_string(h_info[b]) + ")";
        leaving.push_back(p);
        continue;
      }
      p->unc.clear();
      int nunc_wanted = 0;
      for (int j = 0; j < p->k; ++j)
        if (!(rn[j] < p->tol)) {
          p->unc.push_back(j);
          if (j < p->kwant) ++nunc_wanted;
        }
      p->nconv = p->kwant - nunc_wanted;
      if (nunc_wanted == 0 || p->iters >= p->max_iter) {
        leaving.push_back(p);
        continue;
      }
      p->nc = (int)p->unc.size();
      p->restart = p->m + p->nc > p->mmax;
      stay.push_back(p);
    }
  }
  act.swap(stay);
  for (BatchProblem *p : leaving) finish(*p);
  if (act.empty()) return;
  const int Q = (int)act.size();
  // ---- preconditioned corrections T; restarts to the Ritz vectors
  {
    std::vector<int> h_cols;
    std::vector<size_t> coff;
    for (BatchProblem *p : act) {
      coff.push_back(h_cols.size());
      h_cols.insert(h_cols.end(), p->unc.begin(), p->unc.end());
    }
    int *dcols = gcols_.ensure(h_cols.size());
    S2G_CUDA(cudaMemcpyAsync(dcols, stage_.put(h_cols.data(), sizeof(int) * h_cols.size()),
                             sizeof(int) * h_cols.size(), cudaMemcpyHostToDevice, cs_));
    std::vector<BdJob> pj, rs;
    std::vector<DgProblem> gw;
    int64_t mx = 0, mr = 0;
    for (int b = 0; b < Q; ++b) {
      BatchProblem *p = act[b];
      BdJob j = bd_job(*p);
      j.cols = dcols + coff[b];
      pj.push_back(j);
      mx = std::max<int64_t>(mx, (int64_t)p->n * p->nc);
      if (p->restart) {
        DavidsonWork &dw = *p->dw;
        gw.push_back(DgProblem{p->n, p->k, p->m, 1.0, 0.0, dw.W.get(), dw.Hs.get(), dw.tmp.get(),
                               (int64_t)p->n, p->m, (int64_t)p->n});
        rs.push_back(j);
        mr = std::max<int64_t>(mr, (int64_t)p->n * p->k + (int64_t)p->k * p->k);
      }
    }
    const BdJob *d = upload(pj);
    S2G_LAUNCH(k_bd_precond, dim3(bd_blocks(mx), (unsigned)Q), 256, 0, cs_, d);
    if (!rs.empty()) {
      dg_.grouped(cs_, false, false, gw, &stage_);
      const BdJob *dr = upload(rs);
      S2G_LAUNCH(k_bd_restart, dim3(bd_blocks(mr), (unsigned)rs.size()), 256, 0, cs_, dr);
      for (BatchProblem *p : act)
        if (p->restart) p->m = p->k;
    }
  }
  // ---- BCGS2: normalise, then two rounds of projection against V and
  // Cholesky QR, appended to V after column m
  {
    std::vector<BdJob> nj;
    int ncap = 0;
    int64_t mx = 0;
    for (BatchProblem *p : act) {
      p->Tb = p->dw->T.get();
      p->ncur = p->nc;
      p->ortho_open = true;
      nj.push_back(bd_job(*p));
      ncap = std::max(ncap, p->nc);
      mx = std::max<int64_t>(mx, (int64_t)p->n * p->nc);
    }
    const BdJob *d = upload(nj);
    double *part = part_.ensure((size_t)Q * ncap * kColSplit);
    S2G_LAUNCH(k_bd_colnorm, dim3(kColSplit, (unsigned)ncap, (unsigned)Q), 256, 0, cs_, d, ncap,
               part);
    S2G_LAUNCH(k_bd_colnorm_finish, Q, 128, 0, cs_, d, Q, ncap, part, kColSplit);
    S2G_LAUNCH(k_bd_scale, dim3(bd_blocks(mx), (unsigned)Q), 256, 0, cs_, d);
  }
  S2G_CUDA(cudaFuncSetAttribute(k_bd_chol_inv, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)(2 * sizeof(double) * kCholMax * kCholMax)));
  for (int round = 0; round < 2; ++round) {
    std::vector<BatchProblem *> o;
    for (BatchProblem *p : act)
      if (p->ortho_open && p->ncur > 0) o.push_back(p);
    if (o.empty()) break;
    std::vector<DgProblem> gp, gt, gg;
    std::vector<BdJob> cj;
    int ncmax = 0;
    for (BatchProblem *p : o) {
      DavidsonWork &dw = *p->dw;
      const int64_t n = p->n;
      gp.push_back(DgProblem{p->m, p->ncur, p->n, 1.0, 0.0, dw.V.get(), p->Tb, dw.proj.get(), n,
                             n, p->m});
      gt.push_back(DgProblem{p->n, p->ncur, p->m, -1.0, 1.0, dw.V.get(), dw.proj.get(), p->Tb, n,
                             p->m, n});
      gg.push_back(DgProblem{p->ncur, p->ncur, p->n, 1.0, 0.0, p->Tb, p->Tb, dw.G.get(), n, n,
                             p->ncur});
      BdJob j = bd_job(*p);
      j.nc = p->ncur;
      cj.push_back(j);
      ncmax = std::max(ncmax, p->ncur);
    }
    dg_.grouped(cs_, true, false, gp, &stage_);
    dg_.grouped(cs_, false, false, gt, &stage_);
    dg_.grouped(cs_, true, false, gg, &stage_);
    const BdJob *d = upload(cj);
    double *st = gstat_.ensure(2 * o.size());
    S2G_LAUNCH(k_bd_chol_inv, (int)o.size(), 256, 2 * sizeof(double) * ncmax * ncmax, cs_, d,
               1e-8, st);
    back_.reset();
    double *b_st = (double *)back_.take(sizeof(double) * 2 * o.size());
    S2G_CUDA(cudaMemcpyAsync(b_st, st, sizeof(double) * 2 * o.size(), cudaMemcpyDeviceToHost,
                             cs_));
    S2G_CUDA(cudaStreamSynchronize(cs_));
    stage_.reset();
    const std::vector<double> h_st(b_st, b_st + 2 * o.size());
    std::vector<DgProblem> gq;
    std::vector<BdJob> copies;
    int64_t mx = 0;
    for (size_t b = 0; b < o.size(); ++b) {
      BatchProblem *p = o[b];
      DavidsonWork &dw = *p->dw;
      double *dst = dw.V.get() + (int64_t)p->n * p->m;
      if (h_st[2 * b] == 0.0) {
        // dst <- Tb L^-T (through tmp when Tb already is dst)
        double *outp = p->Tb == dst ? dw.tmp.get() : dst;
        gq.push_back(DgProblem{p->n, p->ncur, p->ncur, 1.0, 0.0, p->Tb, dw.Gc.get(), outp,
                               (int64_t)p->n, p->ncur, (int64_t)p->n});
        if (outp != dst) {
          BdJob j = bd_job(*p);
          j.Tb = dst;
          j.nc = p->ncur;
          copies.push_back(j);
          mx = std::max<int64_t>(mx, (int64_t)p->n * p->ncur);
        }
        p->Tb = dst;
      } else {
        // dependent directions: davidson()'s Gram eigen-decomposition path
        // for this member alone (rare)
        p->ncur = dav_orthonormalize(dw, p->blas, p->sol, cs_, dw.V.get(), p->n, p->m, p->Tb,
                                     p->ncur, p->k);
        p->ortho_open = false;
      }
    }
    dg_.grouped(cs_, false, false, gq, &stage_);
    if (!copies.empty()) {
      const BdJob *dc = upload(copies);
      S2G_LAUNCH(k_bd_copy_block, dim3(bd_blocks(mx), (unsigned)copies.size()), 256, 0, cs_, dc);
    }
  }
  // ---- next block sizes; members without new directions leave
  std::vector<BatchProblem *> next, done;
  for (BatchProblem *p : act) {
    p->nb = p->ncur;
    (p->nb == 0 ? done : next).push_back(p);
  }
  act.swap(next);
  for (BatchProblem *p : done) finish(*p);
}

}  // namespace std2g
