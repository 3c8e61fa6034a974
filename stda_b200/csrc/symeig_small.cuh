// Lowest k eigenpairs of a small dense symmetric matrix (n <= kSymEigMaxN),
// for the Rayleigh-Ritz step of the Davidson solver, in three kernels with no
// host synchronisation:
//   1. k_symeig_tridiag: Householder reduction to tridiagonal form
//      T = Q^T A Q (LAPACK dsytd2, lower, restated) by a cluster of
//      kClusterCtas CTAs.  CTA r holds the full columns j = r (mod
//      kClusterCtas) in its shared memory; per reflector the owner of the
//      column broadcasts v through distributed shared memory, every CTA forms
//      its partial A v over its columns, the partials are summed in a fixed
//      order by every CTA (so all hold the same p, w), and each CTA applies the
//      rank-2 update to its own columns.  d, e, tau and the reflectors go to a
//      global workspace;
//   2. k_symeig_values (one warp per eigenvalue, any number of CTAs): bisection
//      on Sturm counts (LAPACK dstebz's principle), each lane evaluating the
//      count at one of 32 points of the current interval per round;
//   3. k_symeig_vectors (one warp per cluster of close eigenvalues, its work
//      arrays in shared memory): inverse iteration with a pivoted tridiagonal
//      LU (LAPACK dstein's scheme: shifts of equal eigenvalues nudged apart,
//      modified Gram-Schmidt against the earlier members of the cluster, three
//      iterations from a fixed start vector; the cluster threshold is
//      1e-5 ||T||, tighter than dstein's 1e-3, so that the dense Rayleigh-Ritz
//      spectra do not collapse into one serial cluster), then the
//      back-transformation z = Q y by the stored reflectors.
// cuSOLVER's syevd takes 1-3 ms at n = 75-300, most of it launch and host
// synchronisation latency.
// Eigenvalues ascending in w[0..k), eigenvectors in the columns of Z (ld ldz).
#pragma once

#include <cooperative_groups.h>

#include <cmath>

#include "common.cuh"

namespace std2g {

constexpr int kClusterCtas = 4;        // CTAs of the tridiagonal reduction
constexpr int kTridiagThreads = 512;
constexpr int kSymEigMaxN = 320;       // full columns of n/4 per CTA within 227 KB

// shared memory of one CTA of k_symeig_tridiag: its columns, v, partial p,
// p / w, reduction scratch
__host__ __device__ inline size_t symeig_smem_bytes(int n) {
  const size_t ncol = (size_t)(n + kClusterCtas - 1) / kClusterCtas;
  return sizeof(double) * (ncol * n + 3 * (size_t)n + 64);
}

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

// ---- 1. tridiagonal reduction (Q^T A Q = T, Q = H_0 ... H_{n-3}) ----------
// A: lower triangle read (lda).  Every CTA of the cluster takes the same
// number of cluster barriers (the decisions depend on data all CTAs share).
__global__ void __cluster_dims__(kClusterCtas, 1, 1) __launch_bounds__(kTridiagThreads, 1)
k_symeig_tridiag(const double *__restrict__ A, int lda, int n, double *__restrict__ work) {
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();
  const int rank = (int)cl.block_rank();
  extern __shared__ double sm[];
  const int ncol = (n + kClusterCtas - 1) / kClusterCtas;   // local columns j = rank + CL*lj
  double *Aloc = sm;                                        // [lj * n + i]
  double *v = Aloc + (size_t)ncol * n;                      // reflector, rows r0..n-1
  double *pp = v + n;                                       // this CTA's partial A v
  double *pw = pp + n;                                      // p, then w
  double *red = pw + n;                                     // [0..31] sums, [32..] scalars
  const int tid = threadIdx.x, nt = blockDim.x;
  SymEigWork g(work, n);
  for (int lj = 0; lj < ncol; ++lj) {
    const int j = rank + kClusterCtas * lj;
    if (j >= n) break;
    for (int i = tid; i < n; i += nt)
      Aloc[(size_t)lj * n + i] = i >= j ? A[i + (size_t)lda * j] : A[j + (size_t)lda * i];
  }
  __syncthreads();
  for (int c = 0; c + 2 < n; ++c) {
    const int r0 = c + 1, owner = c % kClusterCtas;
    if (rank == owner) {
      const double *col = Aloc + (size_t)(c / kClusterCtas) * n;
      const double alpha = col[r0];
      double s = 0.0;
      for (int i = r0 + 1 + tid; i < n; i += nt) s += col[i] * col[i];
      const double xn2 = symeig_block_sum(s, red);
      double tc = 0.0, beta = alpha, scal = 0.0;
      if (xn2 != 0.0) {
        beta = -copysign(sqrt(alpha * alpha + xn2), alpha);
        tc = (beta - alpha) / beta;
        scal = 1.0 / (alpha - beta);
      }
      for (int i = r0 + tid; i < n; i += nt) {
        const double vi = i == r0 ? 1.0 : col[i] * scal;
        v[i] = vi;
        if (i > r0) g.ap[pk_idx(i, c, n)] = vi;   // kept for the back-transformation
      }
      if (tid == 0) {
        red[32] = tc;
        g.tau[c] = tc;
        g.e[c] = beta;
        g.d[c] = col[c];
      }
    }
    cl.sync();   // the owner's v and tau are ready
    if (rank != owner) {
      const double *rv = cl.map_shared_rank(v, owner);
      const double *rr = cl.map_shared_rank(red, owner);
      for (int i = r0 + tid; i < n; i += nt) v[i] = rv[i];
      if (tid == 0) red[32] = rr[32];
    }
    __syncthreads();
    const double tc = red[32];
    if (tc != 0.0) {
      // partial p over this CTA's columns j >= r0, rows i >= r0
      for (int i = r0 + tid; i < n; i += nt) {
        double acc = 0.0;
        for (int lj = 0; lj < ncol; ++lj) {
          const int j = rank + kClusterCtas * lj;
          if (j >= r0 && j < n) acc += Aloc[(size_t)lj * n + i] * v[j];
        }
        pp[i] = acc;
      }
    }
    cl.sync();   // every partial is ready
    if (tc != 0.0) {
      const double *rp[kClusterCtas];
#pragma unroll
      for (int r = 0; r < kClusterCtas; ++r) rp[r] = cl.map_shared_rank(pp, r);
      double pv = 0.0;
      for (int i = r0 + tid; i < n; i += nt) {
        double s = 0.0;
#pragma unroll
        for (int r = 0; r < kClusterCtas; ++r) s += rp[r][i];   // fixed order in every CTA
        const double p = tc * s;
        pw[i] = p;
        pv += p * v[i];
      }
      const double K = 0.5 * tc * symeig_block_sum(pv, red);
      for (int i = r0 + tid; i < n; i += nt) pw[i] -= K * v[i];   // w
      __syncthreads();
      // A22 -= v w^T + w v^T on this CTA's columns (full columns, rows >= r0)
      for (int lj = 0; lj < ncol; ++lj) {
        const int j = rank + kClusterCtas * lj;
        if (j < r0 || j >= n) continue;
        const double vj = v[j], wj = pw[j];
        double *col = Aloc + (size_t)lj * n;
        for (int i = r0 + tid; i < n; i += nt) col[i] -= v[i] * wj + pw[i] * vj;
      }
    }
    __syncthreads();
  }
  // last two diagonal elements and the last off-diagonal one
  for (int c = (n >= 2 ? n - 2 : 0); c < n; ++c) {
    if (c % kClusterCtas != rank || tid != 0) continue;
    const double *col = Aloc + (size_t)(c / kClusterCtas) * n;
    g.d[c] = col[c];
    g.tau[c] = 0.0;
    if (c + 1 < n) g.e[c] = col[c + 1];
    else g.e[c] = 0.0;
  }
  cl.sync();   // no CTA leaves while others may still read its shared memory
}

// ---- 2. eigenvalues: multisection on Sturm counts, one warp per eigenvalue --
constexpr int kSymEigWarps = 8;   // warps per CTA of phases 2 and 3
__global__ void __launch_bounds__(kSymEigWarps * 32)
k_symeig_values(int n, int k, const double *__restrict__ work, double *__restrict__ w) {
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

// ---- 3. eigenvectors of T and back-transformation, one warp per cluster ----
// Cluster threshold: eigenvalues closer than 1e-5 ||T|| are orthogonalised
// against each other; further apart, inverse iteration alone gives vectors
// orthogonal to ~eps ||T|| / gap <= 2e-11.  Shared memory: d, e, then per
// warp y and the rows of U (ua holds 1 / pivot), multipliers, pivot flags.
__host__ __device__ inline size_t symeig_vec_smem_bytes(int n) {
  return sizeof(double) * (2 * (size_t)n + (size_t)kSymEigWarps * 6 * n);
}

__global__ void __launch_bounds__(kSymEigWarps * 32)
k_symeig_vectors(int n, int k, double *__restrict__ work, const double *__restrict__ w,
                 double *__restrict__ Z, int ldz, int *info) {
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
    for (int it = 0; it < 3; ++it) {
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
  // back-transformation z = H_0 ... H_{n-3} y of every member, written to Z
  for (int m = j0; m < j1; ++m) {
    double *z = y;
    for (int i = lane; i < n; i += 32) z[i] = g.vec[(size_t)m * n + i];
    __syncwarp();
    for (int c = n - 3; c >= 0; --c) {
      const double tc = g.tau[c];
      if (tc == 0.0) continue;
      const double *vc = g.ap + pk_idx(c + 1, c, n);   // v[c+1..n-1], v[c+1] = 1 implied
      double dot = 0.0;
      for (int i = c + 1 + lane; i < n; i += 32) dot += (i == c + 1 ? 1.0 : vc[i - c - 1]) * z[i];
      for (int o = 16; o > 0; o >>= 1) dot += __shfl_xor_sync(0xffffffffu, dot, o);
      const double f = tc * dot;
      for (int i = c + 1 + lane; i < n; i += 32) z[i] -= f * (i == c + 1 ? 1.0 : vc[i - c - 1]);
      __syncwarp();
    }
    bool bad = false;
    for (int i = lane; i < n; i += 32) {
      const double zi = z[i];
      bad |= !isfinite(zi);
      Z[i + (size_t)ldz * m] = zi;
    }
    if (lane == 0) bad |= !isfinite(w[m]);
    if (__any_sync(0xffffffffu, bad) && lane == 0) atomicExch(info, 1);
    __syncwarp();
  }
}

// host launcher: n <= kSymEigMaxN, k <= n; work: symeig_work_doubles(n, k)
inline void symeig_small(cudaStream_t s, const double *A, int lda, int n, int k, double *w,
                         double *Z, int ldz, double *work, int *info) {
  if (n < 1 || n > kSymEigMaxN || k < 1 || k > n)
    throw Error{STD2G_EINVAL, "symeig_small: size out of range"};
  S2G_CUDA(cudaFuncSetAttribute(k_symeig_tridiag, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)symeig_smem_bytes(kSymEigMaxN)));
  S2G_CUDA(cudaFuncSetAttribute(k_symeig_vectors, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)symeig_vec_smem_bytes(kSymEigMaxN)));
  S2G_LAUNCH(k_symeig_tridiag, kClusterCtas, kTridiagThreads, symeig_smem_bytes(n), s, A, lda, n,
             work);
  const int nb = (k + kSymEigWarps - 1) / kSymEigWarps;
  S2G_LAUNCH(k_symeig_values, nb, kSymEigWarps * 32, 3 * n * sizeof(double), s, n, k, work, w);
  S2G_LAUNCH(k_symeig_vectors, nb, kSymEigWarps * 32, symeig_vec_smem_bytes(n), s, n, k, work, w,
             Z, ldz, info);
}

}  // namespace std2g
