// Lowest k eigenpairs of a small dense symmetric matrix (n <= kSymEigMaxN) in
// one thread block, for the Rayleigh-Ritz step of the Davidson solver.
//
// cuSOLVER's syevd takes 1.2-3 ms at n = 75-300, most of it launch and host
// synchronisation latency; this kernel keeps the whole problem in one CTA.
// Its per-eigenpair phases (Sturm multisection, serial inverse iteration) grow
// with k, so it wins for few wanted pairs (k <= 40 at n <= 128) and the
// Davidson uses syevd otherwise.  Phases:
//   1. Householder reduction to tridiagonal form T = Q^T A Q on the packed
//      lower triangle held in shared memory (LAPACK dsytd2, lower, restated);
//   2. eigenvalues of T by bisection on Sturm counts (LAPACK dstebz's
//      principle), one warp per eigenvalue, each lane evaluating the count at
//      one of 32 points of the current interval per round;
//   3. eigenvectors of T by inverse iteration with a pivoted tridiagonal LU
//      (LAPACK dstein's scheme: shifts of equal eigenvalues nudged apart,
//      modified Gram-Schmidt against the earlier members of a cluster of close
//      eigenvalues, three iterations from a fixed start vector; the cluster
//      threshold is 1e-5 ||T||, tighter than dstein's 1e-3, so that the dense
//      Rayleigh-Ritz spectra do not collapse into one serial cluster);
//   4. back-transformation Z = Q Y by the stored reflectors, one warp per vector.
// Eigenvalues ascending in w[0..k), eigenvectors in the columns of Z (ld ldz).
#pragma once

#include <cmath>

#include "common.cuh"

namespace std2g {

constexpr int kSymEigMaxN = 224;
constexpr int kSymEigThreads = 1024;

__host__ __device__ inline size_t symeig_smem_bytes(int n) {
  // packed lower A, d, e, tau, v, p/w, scratch for reductions
  return sizeof(double) * ((size_t)n * (n + 1) / 2 + 5 * (size_t)n + 64);
}

// packed lower column-major index of (i, j), i >= j
__device__ __forceinline__ int pk_idx(int i, int j, int n) {
  return j * (2 * n - j + 1) / 2 + (i - j);
}
__device__ __forceinline__ int pk_sym(int i, int j, int n) {
  return i >= j ? pk_idx(i, j, n) : pk_idx(j, i, n);
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

// A: n x n column-major (lower triangle read), lda; work: >= k * 6 * n doubles.
// info: set to 1 when a result is not finite.
__global__ void __launch_bounds__(kSymEigThreads, 1)
k_symeig_small(const double *__restrict__ A, int lda, int n, int k, double *__restrict__ w,
               double *__restrict__ Z, int ldz, double *__restrict__ work, int *info) {
  extern __shared__ double sm[];
  double *ap = sm;                                   // packed lower, n(n+1)/2
  double *d = ap + (size_t)n * (n + 1) / 2;          // diagonal of T
  double *e = d + n;                                 // off-diagonal of T
  double *tau = e + n;                               // reflector scalars
  double *v = tau + n;                               // current reflector
  double *pw = v + n;                                // p, then w; later e^2
  double *red = pw + n;                              // 64 doubles
  const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5,
            nwarp = nt >> 5;
  for (int j = warp; j < n; j += nwarp)
    for (int i = j + lane; i < n; i += 32) ap[pk_idx(i, j, n)] = A[i + (size_t)lda * j];
  __syncthreads();
  // ---- 1. tridiagonal reduction (Q^T A Q = T, Q = H_0 ... H_{n-3}) ----
  for (int c = 0; c + 2 < n; ++c) {
    const int r0 = c + 1;   // trailing block rows / columns r0..n-1
    const double alpha = ap[pk_idx(r0, c, n)];
    double s = 0.0;
    for (int i = r0 + 1 + tid; i < n; i += nt) {
      const double x = ap[pk_idx(i, c, n)];
      s += x * x;
    }
    const double xn2 = symeig_block_sum(s, red);
    if (xn2 == 0.0) {   // column already reduced: H_c = I
      if (tid == 0) {
        tau[c] = 0.0;
        e[c] = alpha;
      }
      __syncthreads();
      continue;
    }
    const double beta = -copysign(sqrt(alpha * alpha + xn2), alpha);
    const double tc = (beta - alpha) / beta;
    const double scal = 1.0 / (alpha - beta);
    for (int i = r0 + tid; i < n; i += nt) {
      const double vi = i == r0 ? 1.0 : ap[pk_idx(i, c, n)] * scal;
      v[i] = vi;
      if (i > r0) ap[pk_idx(i, c, n)] = vi;   // kept for the back-transformation
    }
    if (tid == 0) {
      tau[c] = tc;
      e[c] = beta;
    }
    __syncthreads();
    // p = tau A22 v, one warp per row
    for (int i = r0 + warp; i < n; i += nwarp) {
      double acc = 0.0;
      for (int j = r0 + lane; j < n; j += 32) acc += ap[pk_sym(i, j, n)] * v[j];
      for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
      if (lane == 0) pw[i] = tc * acc;
    }
    __syncthreads();
    double pv = 0.0;
    for (int i = r0 + tid; i < n; i += nt) pv += pw[i] * v[i];
    const double K = 0.5 * tc * symeig_block_sum(pv, red);
    for (int i = r0 + tid; i < n; i += nt) pw[i] -= K * v[i];   // w
    __syncthreads();
    // A22 -= v w^T + w v^T on the lower triangle, one warp per column
    for (int j = r0 + warp; j < n; j += nwarp) {
      const double vj = v[j], wj = pw[j];
      for (int i = j + lane; i < n; i += 32) ap[pk_idx(i, j, n)] -= v[i] * wj + pw[i] * vj;
    }
    __syncthreads();
  }
  for (int i = tid; i < n; i += nt) {
    d[i] = ap[pk_idx(i, i, n)];
    if (i >= n - 2) tau[i] = 0.0;
  }
  if (tid == 0) {
    if (n >= 2) e[n - 2] = ap[pk_idx(n - 1, n - 2, n)];
    e[n - 1] = 0.0;
  }
  __syncthreads();
  // ---- 2. eigenvalues: multisection on Sturm counts, one warp per eigenvalue ----
  double lo = 1e300, hi = -1e300, nrm = 0.0, emax2 = 0.0;
  for (int i = 0; i < n; ++i) {   // every thread, identical
    const double ei = i + 1 < n ? fabs(e[i]) : 0.0, em = i > 0 ? fabs(e[i - 1]) : 0.0;
    lo = fmin(lo, d[i] - ei - em);
    hi = fmax(hi, d[i] + ei + em);
    nrm = fmax(nrm, fabs(d[i]) + ei + em);
    if (i + 1 < n) emax2 = fmax(emax2, e[i] * e[i]);
  }
  const double eps = 2.220446049250313e-16;
  const double pivmin = fmax(1e-300, 1e-290 * fmax(1.0, emax2));
  lo -= 2.0 * eps * nrm + 1e-300;
  hi += 2.0 * eps * nrm + 1e-300;
  double *e2 = pw;
  for (int i = tid; i + 1 < n; i += nt) e2[i] = e[i] * e[i];
  __syncthreads();
  for (int j = warp; j < k; j += nwarp) {
    double a = lo, b = hi;
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
  __syncthreads();
  // ---- 3. eigenvectors of T: inverse iteration, clusters handled by one warp ----
  // per eigenvector m: y, ua, ub, uc (rows of U), mu (multipliers), fl (pivots)
  // cluster threshold: eigenvalues closer than 1e-5 ||T|| are orthogonalised
  // against each other; further apart, inverse iteration alone gives vectors
  // orthogonal to ~eps ||T|| / gap <= 2e-11
  const double ortol = 1e-5 * nrm, pertol = 10.0 * eps * nrm, tiny = eps * nrm + 1e-300;
  int cstart = 0, cid = 0;
  for (int j = 1; j <= k; ++j) {   // every warp walks the cluster list identically
    if (j < k && (w[j] - w[j - 1]) <= ortol) continue;
    if (cid % nwarp == warp) {
      double lam_prev = 0.0;
      for (int m = cstart; m < j; ++m) {
        double lam = w[m];
        if (m > cstart && lam - lam_prev < pertol) lam = lam_prev + pertol;
        lam_prev = lam;
        double *y = work + (size_t)m * 6 * n;
        double *ua = y + n, *ub = ua + n, *uc = ub + n, *mu = uc + n, *fl = mu + n;
        if (lane == 0) {   // T - lam I = P L U, rows of U: (ua, ub, uc)
          double a0 = d[0] - lam, b0 = n > 1 ? e[0] : 0.0;
          for (int i = 0; i + 1 < n; ++i) {
            const double sub = e[i], dn = d[i + 1] - lam, en = i + 2 < n ? e[i + 1] : 0.0;
            if (fabs(a0) >= fabs(sub)) {
              const double ml = a0 != 0.0 ? sub / a0 : 0.0;
              ua[i] = a0;
              ub[i] = b0;
              uc[i] = 0.0;
              mu[i] = ml;
              fl[i] = 0.0;
              a0 = dn - ml * b0;
              b0 = en;
            } else {   // swap rows i and i+1
              const double ml = a0 / sub;
              ua[i] = sub;
              ub[i] = dn;
              uc[i] = en;
              mu[i] = ml;
              fl[i] = 1.0;
              a0 = b0 - ml * dn;
              b0 = -ml * en;
            }
          }
          ua[n - 1] = a0;
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
              double piv = ua[i];
              if (fabs(piv) < tiny) piv = piv < 0.0 ? -tiny : tiny;
              y[i] = s2 / piv;
            }
          }
          __syncwarp();
          for (int q = cstart; q < m; ++q) {   // MGS against earlier cluster members
            const double *zq = work + (size_t)q * 6 * n;
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
      }
    }
    cstart = j;
    ++cid;
  }
  __syncthreads();
  // ---- 4. back-transformation z = H_0 ... H_{n-3} y, one warp per vector ----
  for (int m = warp; m < k; m += nwarp) {
    double *y = work + (size_t)m * 6 * n;
    for (int c = n - 3; c >= 0; --c) {
      const double tc = tau[c];
      if (tc == 0.0) continue;
      double dot = 0.0;
      for (int i = c + 1 + lane; i < n; i += 32)
        dot += (i == c + 1 ? 1.0 : ap[pk_idx(i, c, n)]) * y[i];
      for (int o = 16; o > 0; o >>= 1) dot += __shfl_xor_sync(0xffffffffu, dot, o);
      const double f = tc * dot;
      for (int i = c + 1 + lane; i < n; i += 32)
        y[i] -= f * (i == c + 1 ? 1.0 : ap[pk_idx(i, c, n)]);
      __syncwarp();
    }
    bool bad = false;
    for (int i = lane; i < n; i += 32) {
      const double z = y[i];
      bad |= !isfinite(z);
      Z[i + (size_t)ldz * m] = z;
    }
    if (lane == 0) bad |= !isfinite(w[m]);
    if (__any_sync(0xffffffffu, bad) && lane == 0) atomicExch(info, 1);
  }
}

// host launcher: n <= kSymEigMaxN, k <= n; work: k*6*n doubles
inline void symeig_small(cudaStream_t s, const double *A, int lda, int n, int k, double *w,
                         double *Z, int ldz, double *work, int *info) {
  if (n < 1 || n > kSymEigMaxN || k < 1 || k > n)
    throw Error{STD2G_EINVAL, "symeig_small: size out of range"};
  S2G_CUDA(cudaFuncSetAttribute(k_symeig_small, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)symeig_smem_bytes(kSymEigMaxN)));
  S2G_LAUNCH(k_symeig_small, 1, kSymEigThreads, symeig_smem_bytes(n), s, A, lda, n, k, w, Z,
             ldz, work, info);
}

}  // namespace std2g
