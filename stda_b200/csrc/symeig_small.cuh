// Lowest k eigenpairs of a small dense symmetric matrix (n <= kSymEigMaxN),
// for the Rayleigh-Ritz step of the Davidson solver, in four kernels with no
// host synchronisation:
//   1. k_symeig_tridiag: Householder reduction to tridiagonal form
//      T = Q^T A Q (LAPACK dsytd2, lower, restated) by a cluster of 4 or 8
//      CTAs with one cluster barrier per reflector (the scheme is described
//      at the kernel); d, e, tau and the reflectors go to a global workspace;
//   2. k_symeig_values (one warp per eigenvalue, any number of CTAs): bisection
//      on Sturm counts (LAPACK dstebz's principle), each lane evaluating the
//      count at one of 32 points of the current interval per round;
//   3. k_symeig_vectors (one warp per cluster of close eigenvalues, its work
//      arrays in shared memory): inverse iteration with a pivoted tridiagonal
//      LU (LAPACK dstein's scheme: shifts of equal eigenvalues nudged apart,
//      modified Gram-Schmidt against the earlier members of the cluster, two
//      iterations from a fixed start vector (bisection leaves the eigenvalue
//      within a few ulps of ||T||, so the first solve already grows the wanted
//      component by ~1/eps); the cluster threshold is
//      1e-5 ||T||, tighter than dstein's 1e-3, so that the dense Rayleigh-Ritz
//      spectra do not collapse into one serial cluster), vectors in T's basis;
//   4. k_symeig_backtransform (one warp per eigenvector, held in registers):
//      z = Q y with the reflectors staged through shared memory in blocks
//      that all warps of the CTA apply.
// cuSOLVER's syevd takes 1-3 ms at n = 75-300, most of it launch and host
// synchronisation latency.
// Eigenvalues ascending in w[0..k), eigenvectors in the columns of Z (ld ldz).
// The *_b kernels run the same four phases for many problems per launch
// (blockIdx.y selects the problem; symeig_small_batched).
#pragma once

#include <cooperative_groups.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "common.cuh"

namespace std2g {

constexpr int kTridiagThreads = 512;
constexpr int kSymEigMaxN = 320;       // full columns of n/8 per CTA, 119 KB

// global workspace (doubles): packed reflectors, d, e, tau, 8 spare, and per
// eigenvector its final y in T's basis (n)
__host__ __device__ inline size_t symeig_work_doubles(int n, int k) {
  return (size_t)n * (n + 1) / 2 + 3 * (size_t)n + 8 + (size_t)k * n;
}

// packed lower column-major index of (i, j), i >= j
__device__ __forceinline__ int pk_idx(int i, int j, int n) {
  return j * (2 * n - j + 1) / 2 + (i - j);
}

__device__ double symeig_block_sum(double v, double *red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double t = 0.0;
  const int nw = blockDim.x >> 5;
  for (int q = 0; q < nw; ++q) t += red[q];   // every thread, same order
  return t;
}

// number of eigenvalues of T (d, e2 = e^2) below x (Sturm sequence)
__device__ __forceinline__ int sturm_count(const double *d, const double *e2, int n, double x,
                                           double pivmin) {
  double q = d[0] - x;
  if (fabs(q) < pivmin) q = -pivmin;
  int cnt = q < 0.0;
  for (int i = 1; i < n; ++i) {
    q = d[i] - x - e2[i - 1] / q;
    if (fabs(q) < pivmin) q = -pivmin;
    cnt += q < 0.0;
  }
  return cnt;
}

// Gershgorin interval [lo, hi] and ||T|| (max row sum) of T, widened by
// 2 eps ||T||; the same arithmetic in every caller
__device__ void tri_bounds(const double *d, const double *e, int n, double *lo, double *hi,
                           double *nrm, double *pivmin) {
  double l = 1e300, h = -1e300, t = 0.0, emax2 = 0.0;
  for (int i = 0; i < n; ++i) {
    const double ei = i + 1 < n ? fabs(e[i]) : 0.0, em = i > 0 ? fabs(e[i - 1]) : 0.0;
    l = fmin(l, d[i] - ei - em);
    h = fmax(h, d[i] + ei + em);
    t = fmax(t, fabs(d[i]) + ei + em);
    if (i + 1 < n) emax2 = fmax(emax2, e[i] * e[i]);
  }
  const double eps = 2.220446049250313e-16;
  *lo = l - (2.0 * eps * t + 1e-300);
  *hi = h + (2.0 * eps * t + 1e-300);
  *nrm = t;
  *pivmin = fmax(1e-300, 1e-290 * fmax(1.0, emax2));
}

struct SymEigWork {
  double *ap, *d, *e, *tau, *spare, *vec;
  __host__ __device__ SymEigWork(double *work, int n) {
    ap = work;
    d = ap + (size_t)n * (n + 1) / 2;
    e = d + n;
    tau = e + n;
    spare = tau + n;
    vec = spare + 8;
  }
};

// One problem of a batched launch (k_symeig_*_b: blockIdx.y selects the
// problem; every kernel of the batch covers the largest member, the blocks
// past a member's own size return early or stay idle as in a single launch).
struct SymEigJob {
  const double *A;
  int lda, n, k;
  double *w, *Z;
  int ldz;
  double *work;
  int *info;
};

// ---- 1. tridiagonal reduction (Q^T A Q = T, Q = H_0 ... H_{n-3}) ----------
// A cluster of C CTAs; CTA r holds the full columns j = r (mod C) in shared
// memory, and every CTA also keeps the current column c (cur) and forms the
// reflector of step c from it itself, with the same arithmetic in every CTA,
// so that a step takes one cluster barrier:
//   phase 1: each CTA forms p_j = tau (A v)_j for its own columns j > c as the
//            dot product of column j with v (A is symmetric), and the owner of
//            column c+1 publishes that column;
//   barrier;
//   phase 2: each CTA gathers p and column c+1 from the owners (distributed
//            shared memory), forms w = p - (tau p^T v / 2) v, applies the
//            rank-2 update A -= v w^T + w v^T to its own columns and to its copy
//            of column c+1, and forms the next reflector from that copy.
// The published p pieces and columns alternate between two buffers: a CTA
// that writes buffer (c+1) % 2 has passed the barrier of step c, so every CTA
// has finished reading that buffer at step c-1.  Every CTA takes the same
// barriers (all decisions depend on data the CTAs hold identically).
__host__ __device__ inline int symeig_cluster_ctas(int n) { return n <= 96 ? 4 : 8; }

__host__ __device__ inline size_t symeig_smem_bytes(int n, int C) {
  const size_t ncol = (size_t)(n + C - 1) / C;
  // own columns, v, p, w, cur, published p pieces [2][ncol], published column
  // [2][n], reduction scratch
  return sizeof(double) * (ncol * n + 4 * (size_t)n + 2 * ncol + 2 * (size_t)n + 64);
}

// reflector H_c = I - tau v v^T of the current column c (cur, rows c+1..n-1;
// LAPACK dlarfg's convention: v[c+1] = 1, beta = -sign(alpha) ||x||);
// the writer CTA stores v, tau, beta = e[c] and d[c] = cur[c]
__device__ double symeig_reflector(const double *cur, int c, int n, double *v, double *red,
                                   const SymEigWork &g, bool writer) {
  const int r0 = c + 1, tid = threadIdx.x, nt = blockDim.x;
  const double alpha = cur[r0];
  double s = 0.0;
  for (int i = r0 + 1 + tid; i < n; i += nt) s += cur[i] * cur[i];
  const double xn2 = symeig_block_sum(s, red);
  double tc = 0.0, beta = alpha, scal = 0.0;
  if (xn2 != 0.0) {
    beta = -copysign(sqrt(alpha * alpha + xn2), alpha);
    tc = (beta - alpha) / beta;
    scal = 1.0 / (alpha - beta);
  }
  for (int i = r0 + tid; i < n; i += nt) {
    const double vi = i == r0 ? 1.0 : cur[i] * scal;
    v[i] = vi;
    if (writer && i > r0) g.ap[pk_idx(i, c, n)] = vi;   // kept for the back-transformation
  }
  if (writer && tid == 0) {
    g.tau[c] = tc;
    g.e[c] = beta;
    g.d[c] = cur[c];
  }
  __syncthreads();
  return tc;
}

template <int C>
__device__ __forceinline__ void
symeig_tridiag_body(const double *__restrict__ A, int lda, int n, double *__restrict__ work) {
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();
  const int rank = (int)cl.block_rank();
  extern __shared__ double sm[];
  const int ncol = (n + C - 1) / C;   // local columns j = rank + C * lj
  double *Aloc = sm;                  // [lj * n + i]
  double *v = Aloc + (size_t)ncol * n, *p = v + n, *w = p + n, *cur = w + n;
  double *pubp = cur + n;             // [2][ncol]
  double *pubc = pubp + 2 * ncol;     // [2][n]
  double *red = pubc + 2 * n;         // [64]
  const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5;
  const int nw = nt >> 5;
  const bool writer = rank == 0;
  SymEigWork g(work, n);
  for (int lj = 0; lj < ncol; ++lj) {
    const int j = rank + C * lj;
    if (j >= n) break;
    for (int i = tid; i < n; i += nt)
      Aloc[(size_t)lj * n + i] = i >= j ? A[i + (size_t)lda * j] : A[j + (size_t)lda * i];
  }
  for (int i = tid; i < n; i += nt) cur[i] = A[i];   // column 0
  __syncthreads();
  double tc = n >= 3 ? symeig_reflector(cur, 0, n, v, red, g, writer) : 0.0;
  for (int c = 0; c + 2 < n; ++c) {
    const int r0 = c + 1, nxt = c + 1, own_nxt = nxt % C, buf = c & 1;
    // first local column with j >= r0
    const int lj0 = r0 > rank ? (r0 - rank + C - 1) / C : 0;
    // ---- phase 1
    if (tc != 0.0) {
      for (int lj = lj0 + warp; lj < ncol; lj += nw) {
        const int j = rank + C * lj;
        if (j >= n) break;
        const double *col = Aloc + (size_t)lj * n;
        double sdot = 0.0;
        for (int i = r0 + lane; i < n; i += 32) sdot += col[i] * v[i];
        for (int o = 16; o > 0; o >>= 1) sdot += __shfl_xor_sync(0xffffffffu, sdot, o);
        if (lane == 0) pubp[buf * ncol + lj] = tc * sdot;
      }
    }
    if (rank == own_nxt) {
      const double *col = Aloc + (size_t)(nxt / C) * n;
      for (int i = r0 + tid; i < n; i += nt) pubc[buf * n + i] = col[i];
    }
    cl.sync();
    // ---- phase 2
    const double *rc = cl.map_shared_rank(pubc + buf * n, own_nxt);
    double pv = 0.0;
    for (int i = r0 + tid; i < n; i += nt) {
      cur[i] = rc[i];
      if (tc != 0.0) {
        const double *rp = cl.map_shared_rank(pubp + buf * ncol, i % C);
        const double pi = rp[i / C];
        p[i] = pi;
        pv += pi * v[i];
      }
    }
    if (tc != 0.0) {
      const double K = 0.5 * tc * symeig_block_sum(pv, red);   // same value in every CTA
      for (int i = r0 + tid; i < n; i += nt) w[i] = p[i] - K * v[i];
      __syncthreads();
      const double vn = v[nxt], wn = w[nxt];
      for (int i = r0 + tid; i < n; i += nt) cur[i] -= v[i] * wn + w[i] * vn;
      for (int lj = lj0 + warp; lj < ncol; lj += nw) {
        const int j = rank + C * lj;
        if (j >= n) break;
        const double vj = v[j], wj = w[j];
        double *col = Aloc + (size_t)lj * n;
        for (int i = r0 + lane; i < n; i += 32) col[i] -= v[i] * wj + w[i] * vj;
      }
    }
    __syncthreads();
    if (c + 3 < n) tc = symeig_reflector(cur, nxt, n, v, red, g, writer);
  }
  // the trailing 2 x 2 block: cur holds column n-2, column n-1 is on its owner
  if (writer && tid == 0) {
    if (n >= 2) {
      g.d[n - 2] = cur[n - 2];
      g.e[n - 2] = cur[n - 1];
      g.tau[n - 2] = 0.0;
    }
  }
  if (rank == (n - 1) % C && tid == 0) {
    g.d[n - 1] = Aloc[(size_t)((n - 1) / C) * n + (n - 1)];
    g.e[n - 1] = 0.0;
    g.tau[n - 1] = 0.0;
  }
  cl.sync();   // no CTA leaves while others may still read its shared memory
}

template <int C>
__global__ void __cluster_dims__(C, 1, 1) __launch_bounds__(kTridiagThreads, 1)
k_symeig_tridiag(const double *__restrict__ A, int lda, int n, double *__restrict__ work) {
  symeig_tridiag_body<C>(A, lda, n, work);
}

// batched form: cluster blockIdx.y solves jobs[blockIdx.y]
template <int C>
__global__ void __cluster_dims__(C, 1, 1) __launch_bounds__(kTridiagThreads, 1)
k_symeig_tridiag_b(const SymEigJob *__restrict__ jobs) {
  const SymEigJob j = jobs[blockIdx.y];
  symeig_tridiag_body<C>(j.A, j.lda, j.n, j.work);
}

// ---- 2. eigenvalues: multisection on Sturm counts, one warp per eigenvalue --
constexpr int kSymEigWarps = 8;   // warps per CTA of phases 2 and 3
__device__ __forceinline__ void
symeig_values_body(int n, int k, const double *__restrict__ work, double *__restrict__ w) {
  extern __shared__ double sm[];
  double *d = sm, *e = sm + n, *e2 = sm + 2 * n;
  const SymEigWork g(const_cast<double *>(work), n);
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    d[i] = g.d[i];
    e[i] = g.e[i];
    e2[i] = i + 1 < n ? g.e[i] * g.e[i] : 0.0;
  }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int j = blockIdx.x * kSymEigWarps + (threadIdx.x >> 5);
  if (j >= k) return;
  const double eps = 2.220446049250313e-16;
  double a, b, nrm, pivmin;
  tri_bounds(d, e, n, &a, &b, &nrm, &pivmin);
  for (int round = 0; round < 64; ++round) {
    if (b - a <= 2.0 * eps * fmax(fabs(a), fabs(b)) + 1e-300) break;
    const double x = a + (b - a) * (double)(lane + 1) / 33.0;
    const int cnt = sturm_count(d, e2, n, x, pivmin);
    // the first point with more than j eigenvalues below it bounds eigenvalue j
    const unsigned above = __ballot_sync(0xffffffffu, cnt > j);
    const int l = above ? __ffs(above) - 1 : 32;
    const double na = l == 0 ? a : a + (b - a) * (double)l / 33.0;
    const double nb = l == 32 ? b : a + (b - a) * (double)(l + 1) / 33.0;
    a = na;
    b = nb;
  }
  if (lane == 0) w[j] = 0.5 * (a + b);
}

__global__ void __launch_bounds__(kSymEigWarps * 32)
k_symeig_values(int n, int k, const double *__restrict__ work, double *__restrict__ w) {
  symeig_values_body(n, k, work, w);
}

__global__ void __launch_bounds__(kSymEigWarps * 32)
k_symeig_values_b(const SymEigJob *__restrict__ jobs) {
  const SymEigJob j = jobs[blockIdx.y];
  symeig_values_body(j.n, j.k, j.work, j.w);
}

// ---- 3. eigenvectors of T, one warp per cluster of close eigenvalues --------
// Cluster threshold: eigenvalues closer than 1e-5 ||T|| are orthogonalised
// against each other; further apart, inverse iteration alone gives vectors
// orthogonal to ~eps ||T|| / gap <= 2e-11.  Shared memory: d, e, then per
// warp y and the rows of U (ua holds 1 / pivot), multipliers, pivot flags.
__host__ __device__ inline size_t symeig_vec_smem_bytes(int n) {
  return sizeof(double) * (2 * (size_t)n + (size_t)kSymEigWarps * 6 * n);
}

__device__ __forceinline__ void
symeig_vectors_body(int n, int k, double *__restrict__ work, const double *__restrict__ w) {
  extern __shared__ double sm[];
  double *d = sm, *e = sm + n;
  const SymEigWork g(work, n);
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    d[i] = g.d[i];
    e[i] = g.e[i];
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, wl = threadIdx.x >> 5;
  const int j0 = blockIdx.x * kSymEigWarps + wl;
  if (j0 >= k) return;
  const double eps = 2.220446049250313e-16;
  double lo_, hi_, nrm, pivmin_;
  tri_bounds(d, e, n, &lo_, &hi_, &nrm, &pivmin_);
  const double ortol = 1e-5 * nrm, pertol = 10.0 * eps * nrm, tiny = eps * nrm + 1e-300;
  if (j0 > 0 && (w[j0] - w[j0 - 1]) <= ortol) return;   // not the first of its cluster
  int j1 = j0 + 1;
  while (j1 < k && (w[j1] - w[j1 - 1]) <= ortol) ++j1;
  double *y = sm + 2 * n + (size_t)wl * 6 * n;
  double *ua = y + n, *ub = ua + n, *uc = ub + n, *mu = uc + n, *fl = mu + n;
  double lam_prev = 0.0;
  for (int m = j0; m < j1; ++m) {
    double lam = w[m];
    if (m > j0 && lam - lam_prev < pertol) lam = lam_prev + pertol;
    lam_prev = lam;
    if (lane == 0) {   // T - lam I = P L U, rows of U: (ua, ub, uc)
      double a0 = d[0] - lam, b0 = n > 1 ? e[0] : 0.0;
      for (int i = 0; i + 1 < n; ++i) {
        const double sub = e[i], dn = d[i + 1] - lam, en = i + 2 < n ? e[i + 1] : 0.0;
        double piv;
        if (fabs(a0) >= fabs(sub)) {
          const double ml = a0 != 0.0 ? sub / a0 : 0.0;
          piv = a0;
          ub[i] = b0;
          uc[i] = 0.0;
          mu[i] = ml;
          fl[i] = 0.0;
          a0 = dn - ml * b0;
          b0 = en;
        } else {   // swap rows i and i+1
          const double ml = a0 / sub;
          piv = sub;
          ub[i] = dn;
          uc[i] = en;
          mu[i] = ml;
          fl[i] = 1.0;
          a0 = b0 - ml * dn;
          b0 = -ml * en;
        }
        if (fabs(piv) < tiny) piv = piv < 0.0 ? -tiny : tiny;
        ua[i] = 1.0 / piv;
      }
      double piv = a0;
      if (fabs(piv) < tiny) piv = piv < 0.0 ? -tiny : tiny;
      ua[n - 1] = 1.0 / piv;
    }
    for (int i = lane; i < n; i += 32) y[i] = 1.0 + 0.5 * sin(0.7 * (i + 1) + 0.3 * (m + 1));
    __syncwarp();
    for (int it = 0; it < 2; ++it) {
      if (lane == 0) {
        for (int i = 0; i + 1 < n; ++i) {   // y <- L^-1 P y
          if (fl[i] != 0.0) {
            const double t = y[i];
            y[i] = y[i + 1];
            y[i + 1] = t - mu[i] * y[i];
          } else {
            y[i + 1] -= mu[i] * y[i];
          }
        }
        for (int i = n - 1; i >= 0; --i) {   // U x = y
          double s2 = y[i];
          if (i + 1 < n) s2 -= ub[i] * y[i + 1];
          if (i + 2 < n) s2 -= uc[i] * y[i + 2];
          y[i] = s2 * ua[i];
        }
      }
      __syncwarp();
      for (int q = j0; q < m; ++q) {   // MGS against earlier cluster members (in T's basis)
        const double *zq = g.vec + (size_t)q * n;
        double dot = 0.0;
        for (int i = lane; i < n; i += 32) dot += zq[i] * y[i];
        for (int o = 16; o > 0; o >>= 1) dot += __shfl_xor_sync(0xffffffffu, dot, o);
        for (int i = lane; i < n; i += 32) y[i] -= dot * zq[i];
        __syncwarp();
      }
      double nn = 0.0;
      for (int i = lane; i < n; i += 32) nn += y[i] * y[i];
      for (int o = 16; o > 0; o >>= 1) nn += __shfl_xor_sync(0xffffffffu, nn, o);
      const double inv = nn > 0.0 ? 1.0 / sqrt(nn) : 0.0;
      for (int i = lane; i < n; i += 32) y[i] *= inv;
      __syncwarp();
    }
    // the member's vector in T's basis, for the MGS of the later members
    for (int i = lane; i < n; i += 32) g.vec[(size_t)m * n + i] = y[i];
    __syncwarp();
  }
}

__global__ void __launch_bounds__(kSymEigWarps * 32)
k_symeig_vectors(int n, int k, double *__restrict__ work, const double *__restrict__ w) {
  symeig_vectors_body(n, k, work, w);
}

__global__ void __launch_bounds__(kSymEigWarps * 32)
k_symeig_vectors_b(const SymEigJob *__restrict__ jobs) {
  const SymEigJob j = jobs[blockIdx.y];
  symeig_vectors_body(j.n, j.k, j.work, j.w);
}

// ---- 4. back-transformation z = H_0 ... H_{n-3} y ----------------------------
constexpr int kBtBlock = 16;                        // reflectors staged per round
constexpr int kBtPerLane = (kSymEigMaxN + 31) / 32;  // vector elements per lane

__host__ __device__ inline size_t symeig_bt_smem_bytes(int n) {
  return sizeof(double) * ((size_t)kBtBlock * n + kBtBlock);
}

__device__ __forceinline__ void
symeig_backtransform_body(int n, int k, const double *__restrict__ work,
                       const double *__restrict__ w, double *__restrict__ Z, int ldz,
                       int *info) {
  extern __shared__ double sm[];
  double *R = sm;                      // [kBtBlock][n]: v of H_c, zero above row c+1
  double *tt = sm + (size_t)kBtBlock * n;
  const SymEigWork g(const_cast<double *>(work), n);
  const int lane = threadIdx.x & 31, wl = threadIdx.x >> 5;
  const int m = blockIdx.x * kSymEigWarps + wl;
  const bool live = m < k;
  double y[kBtPerLane];
#pragma unroll
  for (int t = 0; t < kBtPerLane; ++t) {
    const int i = lane + 32 * t;
    y[t] = live && i < n ? g.vec[(size_t)m * n + i] : 0.0;
  }
  // H_{n-3} first, H_0 last
  for (int c1 = n - 3; c1 >= 0; c1 -= kBtBlock) {
    const int nr = min(kBtBlock, c1 + 1);   // reflectors c1, c1-1, ..., c1-nr+1
    __syncthreads();
    for (int e = threadIdx.x; e < nr * n; e += blockDim.x) {
      const int r = e / n, i = e - r * n, c = c1 - r;
      R[e] = i <= c ? 0.0 : (i == c + 1 ? 1.0 : g.ap[pk_idx(i, c, n)]);
    }
    for (int r = threadIdx.x; r < nr; r += blockDim.x) tt[r] = g.tau[c1 - r];
    __syncthreads();
    if (!live) continue;
    for (int r = 0; r < nr; ++r) {
      const double tc = tt[r];
      if (tc == 0.0) continue;
      const double *vr = R + (size_t)r * n;
      double dot = 0.0;
#pragma unroll
      for (int t = 0; t < kBtPerLane; ++t) {
        const int i = lane + 32 * t;
        if (i < n) dot += vr[i] * y[t];
      }
      for (int o = 16; o > 0; o >>= 1) dot += __shfl_xor_sync(0xffffffffu, dot, o);
      const double f = tc * dot;
#pragma unroll
      for (int t = 0; t < kBtPerLane; ++t) {
        const int i = lane + 32 * t;
        if (i < n) y[t] -= f * vr[i];
      }
    }
  }
  if (!live) return;
  bool bad = false;
#pragma unroll
  for (int t = 0; t < kBtPerLane; ++t) {
    const int i = lane + 32 * t;
    if (i < n) {
      bad |= !isfinite(y[t]);
      Z[i + (size_t)ldz * m] = y[t];
    }
  }
  if (lane == 0) bad |= !isfinite(w[m]);
  if (__any_sync(0xffffffffu, bad) && lane == 0) atomicExch(info, 1);
}

__global__ void __launch_bounds__(kSymEigWarps * 32)
k_symeig_backtransform(int n, int k, const double *__restrict__ work,
                       const double *__restrict__ w, double *__restrict__ Z, int ldz,
                       int *info) {
  symeig_backtransform_body(n, k, work, w, Z, ldz, info);
}

__global__ void __launch_bounds__(kSymEigWarps * 32)
k_symeig_backtransform_b(const SymEigJob *__restrict__ jobs) {
  const SymEigJob j = jobs[blockIdx.y];
  symeig_backtransform_body(j.n, j.k, j.work, j.w, j.Z, j.ldz, j.info);
}

// host launcher: n <= kSymEigMaxN, k <= n; work: symeig_work_doubles(n, k)
inline void symeig_small(cudaStream_t s, const double *A, int lda, int n, int k, double *w,
                         double *Z, int ldz, double *work, int *info) {
  if (n < 1 || n > kSymEigMaxN || k < 1 || k > n)
    throw Error{STD2G_EINVAL, "symeig_small: size out of range"};
  const int C = symeig_cluster_ctas(n);
  // the attribute is the same for every call (contexts on other host threads
  // launch the same kernel concurrently), the launch takes what n needs
  const int tsm = (int)symeig_smem_bytes(n, C);
  if (C == 4) {
    S2G_CUDA(cudaFuncSetAttribute(k_symeig_tridiag<4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)symeig_smem_bytes(kSymEigMaxN, 4)));
    S2G_LAUNCH(k_symeig_tridiag<4>, 4, kTridiagThreads, tsm, s, A, lda, n, work);
  } else {
    S2G_CUDA(cudaFuncSetAttribute(k_symeig_tridiag<8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)symeig_smem_bytes(kSymEigMaxN, 8)));
    S2G_LAUNCH(k_symeig_tridiag<8>, 8, kTridiagThreads, tsm, s, A, lda, n, work);
  }
  S2G_CUDA(cudaFuncSetAttribute(k_symeig_vectors, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)symeig_vec_smem_bytes(kSymEigMaxN)));
  const int nb = (k + kSymEigWarps - 1) / kSymEigWarps;
  S2G_LAUNCH(k_symeig_values, nb, kSymEigWarps * 32, 3 * n * sizeof(double), s, n, k, work, w);
  S2G_LAUNCH(k_symeig_vectors, nb, kSymEigWarps * 32, symeig_vec_smem_bytes(n), s, n, k, work, w);
  S2G_LAUNCH(k_symeig_backtransform, nb, kSymEigWarps * 32, symeig_bt_smem_bytes(n), s, n, k,
             work, w, Z, ldz, info);
}

// Batched launcher: the problems of `jobs` (each n <= kSymEigMaxN, 1 <= k <= n)
// in four launches for all of them, plus one tridiagonalisation launch per
// cluster size.  The job table goes to `dj` (same stream: a later upload
// waits for these kernels), from `stage` when given.
inline void symeig_small_batched(cudaStream_t s, const std::vector<SymEigJob> &jobs,
                                 DBuf<SymEigJob> &dj, PinnedArena *stage = nullptr) {
  if (jobs.empty()) return;
  std::vector<SymEigJob> ord;
  int n4 = 0, nmax = 0, kmax = 0;
  size_t sm4 = 0, sm8 = 0;
  for (int pass = 0; pass < 2; ++pass)
    for (const SymEigJob &j : jobs) {
      if (j.n < 1 || j.n > kSymEigMaxN || j.k < 1 || j.k > j.n)
        throw Error{STD2G_EINVAL, "symeig_small_batched: size out of range"};
      const int C = symeig_cluster_ctas(j.n);
      if ((pass == 0) != (C == 4)) continue;
      ord.push_back(j);
      if (C == 4) {
        ++n4;
        sm4 = std::max(sm4, symeig_smem_bytes(j.n, 4));
      } else {
        sm8 = std::max(sm8, symeig_smem_bytes(j.n, 8));
      }
      nmax = std::max(nmax, j.n);
      kmax = std::max(kmax, j.k);
    }
  const int nj = (int)ord.size();
  SymEigJob *d = dj.ensure(ord.size());
  const void *h = stage ? stage->put(ord.data(), sizeof(SymEigJob) * ord.size()) : ord.data();
  S2G_CUDA(cudaMemcpyAsync(d, h, sizeof(SymEigJob) * ord.size(), cudaMemcpyHostToDevice, s));
  if (n4 > 0) {
    S2G_CUDA(cudaFuncSetAttribute(k_symeig_tridiag_b<4>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)symeig_smem_bytes(kSymEigMaxN, 4)));
    S2G_LAUNCH(k_symeig_tridiag_b<4>, dim3(4, n4), kTridiagThreads, sm4, s, d);
  }
  if (nj > n4) {
    S2G_CUDA(cudaFuncSetAttribute(k_symeig_tridiag_b<8>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)symeig_smem_bytes(kSymEigMaxN, 8)));
    S2G_LAUNCH(k_symeig_tridiag_b<8>, dim3(8, nj - n4), kTridiagThreads, sm8, s, d + n4);
  }
  S2G_CUDA(cudaFuncSetAttribute(k_symeig_vectors_b, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)symeig_vec_smem_bytes(kSymEigMaxN)));
  const dim3 g((kmax + kSymEigWarps - 1) / kSymEigWarps, nj);
  S2G_LAUNCH(k_symeig_values_b, g, kSymEigWarps * 32, 3 * nmax * sizeof(double), s, d);
  S2G_LAUNCH(k_symeig_vectors_b, g, kSymEigWarps * 32, symeig_vec_smem_bytes(nmax), s, d);
  S2G_LAUNCH(k_symeig_backtransform_b, g, kSymEigWarps * 32, symeig_bt_smem_bytes(nmax), s, d);
}

}  // namespace std2g
