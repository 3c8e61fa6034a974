// Lowest k eigenpairs of a small dense symmetric matrix (n <= kSymEigMaxN),
// for the Rayleigh-Ritz step of the Davidson solver, in three kernels with no
// host synchronisation:
//   1. k_symeig_tridiag (one CTA): Householder reduction to tridiagonal form
//      T = Q^T A Q on the packed lower triangle held in shared memory (LAPACK
//      dsytd2, lower, restated); d, e, the reflectors and ||T|| go to a global
//      workspace;
//   2. k_symeig_values (one warp per eigenvalue, any number of CTAs): bisection
//      on Sturm counts (LAPACK dstebz's principle), each lane evaluating the
//      count at one of 32 points of the current interval per round;
//   3. k_symeig_vectors (one warp per cluster of close eigenvalues): inverse
//      iteration with a pivoted tridiagonal LU (LAPACK dstein's scheme: shifts
//      of equal eigenvalues nudged apart, modified Gram-Schmidt against the
//      earlier members of the cluster, three iterations from a fixed start
//      vector; the cluster threshold is 1e-5 ||T||, tighter than dstein's
//      1e-3, so that the dense Rayleigh-Ritz spectra do not collapse into one
//      serial cluster), then the back-transformation z = Q y by the stored
//      reflectors.
// cuSOLVER's syevd takes 1-3 ms at n = 75-300, most of it launch and host
// synchronisation latency; phases 2 and 3 here spread over k warps on many SMs.
// Eigenvalues ascending in w[0..k), eigenvectors in the columns of Z (ld ldz).
#pragma once

#include <cmath>

#include "common.cuh"

namespace std2g {

constexpr int kSymEigMaxN = 235;   // packed lower triangle + 5 vectors within 227 KB
constexpr int kSymEigThreads = 1024;

__host__ __device__ inline size_t symeig_smem_bytes(int n) {
  // packed lower A, d, e, tau, v, p/w, scratch for reductions
  return sizeof(double) * ((size_t)n * (n + 1) / 2 + 5 * (size_t)n + 64);
}

// global workspace (doubles): packed reflectors, d, e, tau, 4 scalars, and
// per eigenvector y, U rows (ua, ub, uc), multipliers, pivots (6 n)
__host__ __device__ inline size_t symeig_work_doubles(int n, int k) {
  return (size_t)n * (n + 1) / 2 + 3 * (size_t)n + 8 + (size_t)k * 6 * n;
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

struct SymEigWork {
  double *ap, *d, *e, *tau, *scal, *vec;   // scal: lo, hi, nrm, pivmin
  __host__ __device__ SymEigWork(double *work, int n) {
    ap = work;
    d = ap + (size_t)n * (n + 1) / 2;
    e = d + n;
    tau = e + n;
    scal = tau + n;
    vec = scal + 8;
  }
};

// ---- 1. tridiagonal reduction (Q^T A Q = T, Q = H_0 ... H_{n-3}) ----------
__global__ void __launch_bounds__(kSymEigThreads, 1)
k_symeig_tridiag(const double *__restrict__ A, int lda, int n, double *__restrict__ work) {
  extern __shared__ double sm[];
  double *ap = sm;                                   // packed lower, n(n+1)/2
  double *d = ap + (size_t)n * (n + 1) / 2;          // diagonal of T
  double *e = d + n;                                 // off-diagonal of T
  double *tau = e + n;                               // reflector scalars
  double *v = tau + n;                               // current reflector
  double *pw = v + n;                                // p, then w
  double *red = pw + n;                              // 64 doubles
  const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5,
            nwarp = nt >> 5;
  for (int j = warp; j < n; j += nwarp)
    for (int i = j + lane; i < n; i += 32) ap[pk_idx(i, j, n)] = A[i + (size_t)lda * j];
  __syncthreads();
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
  SymEigWork g(work, n);
  for (int i = tid; i < n; i += nt) {
    d[i] = ap[pk_idx(i, i, n)];
    if (i >= n - 2) tau[i] = 0.0;
  }
  if (tid == 0) {
    if (n >= 2) e[n - 2] = ap[pk_idx(n - 1, n - 2, n)];
    e[n - 1] = 0.0;
  }
  __syncthreads();
  for (size_t q = tid; q < (size_t)n * (n + 1) / 2; q += nt) g.ap[q] = ap[q];
  for (int i = tid; i < n; i += nt) {
    g.d[i] = d[i];
    g.e[i] = e[i];
    g.tau[i] = tau[i];
  }
  if (tid == 0) {
    double lo = 1e300, hi = -1e300, nrm = 0.0, emax2 = 0.0;
    for (int i = 0; i < n; ++i) {
      const double ei = i + 1 < n ? fabs(e[i]) : 0.0, em = i > 0 ? fabs(e[i - 1]) : 0.0;
      lo = fmin(lo, d[i] - ei - em);
      hi = fmax(hi, d[i] + ei + em);
      nrm = fmax(nrm, fabs(d[i]) + ei + em);
      if (i + 1 < n) emax2 = fmax(emax2, e[i] * e[i]);
    }
    const double eps = 2.220446049250313e-16;
    g.scal[0] = lo - (2.0 * eps * nrm + 1e-300);
    g.scal[1] = hi + (2.0 * eps * nrm + 1e-300);
    g.scal[2] = nrm;
    g.scal[3] = fmax(1e-300, 1e-290 * fmax(1.0, emax2));
  }
}

// ---- 2. eigenvalues: multisection on Sturm counts, one warp per eigenvalue --
constexpr int kSymEigWarps = 8;   // warps per CTA of phases 2 and 3
__global__ void __launch_bounds__(kSymEigWarps * 32)
k_symeig_values(int n, int k, double *__restrict__ work, double *__restrict__ w) {
  extern __shared__ double sm[];
  double *d = sm, *e2 = sm + n;
  const SymEigWork g(work, n);
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    d[i] = g.d[i];
    e2[i] = i + 1 < n ? g.e[i] * g.e[i] : 0.0;
  }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int j = blockIdx.x * kSymEigWarps + (threadIdx.x >> 5);
  if (j >= k) return;
  const double eps = 2.220446049250313e-16;
  const double pivmin = g.scal[3];
  double a = g.scal[0], b = g.scal[1];
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
// orthogonal to ~eps ||T|| / gap <= 2e-11.
__global__ void __launch_bounds__(kSymEigWarps * 32)
k_symeig_vectors(int n, int k, double *__restrict__ work, const double *__restrict__ w,
                 double *__restrict__ Z, int ldz, int *info) {
  const SymEigWork g(work, n);
  const int lane = threadIdx.x & 31;
  const int j0 = blockIdx.x * kSymEigWarps + (threadIdx.x >> 5);
  if (j0 >= k) return;
  const double eps = 2.220446049250313e-16;
  const double nrm = g.scal[2];
  const double ortol = 1e-5 * nrm, pertol = 10.0 * eps * nrm, tiny = eps * nrm + 1e-300;
  if (j0 > 0 && (w[j0] - w[j0 - 1]) <= ortol) return;   // not the first of its cluster
  int j1 = j0 + 1;
  while (j1 < k && (w[j1] - w[j1 - 1]) <= ortol) ++j1;
  const double *d = g.d, *e = g.e;
  double lam_prev = 0.0;
  for (int m = j0; m < j1; ++m) {
    double lam = w[m];
    if (m > j0 && lam - lam_prev < pertol) lam = lam_prev + pertol;
    lam_prev = lam;
    double *y = g.vec + (size_t)m * 6 * n;
    double *ua = y + n, *ub = ua + n, *uc = ub + n, *mu = uc + n, *fl = mu + n;
    if (lane == 0) {   // T - lam I = P L U, rows of U: (ua, ub, uc); ua holds 1 / pivot
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
        const double *zq = g.vec + (size_t)q * 6 * n;
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
  // back-transformation z = H_0 ... H_{n-3} y of every member, written to Z;
  // the members' y stay in T's basis until all of them are done (MGS above)
  for (int m = j0; m < j1; ++m) {
    const double *y = g.vec + (size_t)m * 6 * n;
    double *z = g.vec + (size_t)m * 6 * n + n;   // ua is no longer needed
    for (int i = lane; i < n; i += 32) z[i] = y[i];
    __syncwarp();
    for (int c = n - 3; c >= 0; --c) {
      const double tc = g.tau[c];
      if (tc == 0.0) continue;
      double dot = 0.0;
      for (int i = c + 1 + lane; i < n; i += 32)
        dot += (i == c + 1 ? 1.0 : g.ap[pk_idx(i, c, n)]) * z[i];
      for (int o = 16; o > 0; o >>= 1) dot += __shfl_xor_sync(0xffffffffu, dot, o);
      const double f = tc * dot;
      for (int i = c + 1 + lane; i < n; i += 32)
        z[i] -= f * (i == c + 1 ? 1.0 : g.ap[pk_idx(i, c, n)]);
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
  }
}

// host launcher: n <= kSymEigMaxN, k <= n; work: symeig_work_doubles(n, k)
inline void symeig_small(cudaStream_t s, const double *A, int lda, int n, int k, double *w,
                         double *Z, int ldz, double *work, int *info) {
  if (n < 1 || n > kSymEigMaxN || k < 1 || k > n)
    throw Error{STD2G_EINVAL, "symeig_small: size out of range"};
  S2G_CUDA(cudaFuncSetAttribute(k_symeig_tridiag, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)symeig_smem_bytes(kSymEigMaxN)));
  S2G_LAUNCH(k_symeig_tridiag, 1, kSymEigThreads, symeig_smem_bytes(n), s, A, lda, n, work);
  const int nb = (k + kSymEigWarps - 1) / kSymEigWarps;
  S2G_LAUNCH(k_symeig_values, nb, kSymEigWarps * 32, 2 * n * sizeof(double), s, n, k, work, w);
  S2G_LAUNCH(k_symeig_vectors, nb, kSymEigWarps * 32, 0, s, n, k, work, w, Z, ldz, info);
}

}  // namespace std2g
