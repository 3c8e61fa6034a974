// Blocked Davidson eigensolver for the lowest k roots of the sTDA matrix A.
//
// The reference diagonalises A completely with LAPACK ssyevr and keeps the
// roots in (0, E_thr] (stda.f:1133-1150).  For large CSF spaces this engine
// finds the requested lowest roots iteratively: sigma = A V products through a
// caller-supplied operator (matrix-free, matfree.cuh), and an FP64
// Rayleigh-Ritz projection, FP64 orthogonalisation (classical Gram-Schmidt,
// applied twice) and FP64 residuals.  The preconditioner is the diagonal
// (Davidson) one, (theta - A_ii)^-1.  A few buffer roots beyond the wanted
// ones are carried along so that near-degeneracies at the edge of the wanted
// set do not stall convergence.
#pragma once

#include <algorithm>
#include <chrono>
#include <functional>
#include <numeric>
#include <vector>

#include "common.cuh"
#include "dgemm.cuh"
#include "symeig_small.cuh"

namespace std2g {

// T[:, j] = R[:, cols[j]] / (theta - diag), guarded away from zero
__global__ void k_dav_precond(double *__restrict__ T, const double *__restrict__ R,
                              const double *__restrict__ diag, const double *__restrict__ theta,
                              const int *__restrict__ cols, int n, int nc) {
  int64_t total = (int64_t)n * nc;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    int j = (int)(t / n), i = (int)(t - (int64_t)j * n);
    int c = cols[j];
    double d = theta[c] - diag[i];
    if (fabs(d) < 1e-4) d = d < 0 ? -1e-4 : 1e-4;
    T[t] = R[i + (int64_t)n * c] / d;
  }
}

// R[:, j] -= theta_j X[:, j]; rnorm[j] = ||R[:, j]||  (one block per column)
// Column norms are reduced in two fixed-order stages so that a block of
// columns spreads over the whole GPU: grid (kColSplit, ncol) writes partial
// sums of squares, k_colnorm_finish adds them in order and takes the root.
constexpr int kColSplit = 16;

__device__ __forceinline__ double block_sum256(double s, double *red) {
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  return red[0];
}

// R[:, j] -= theta[j] X[:, j]; part[j*gridDim.x + b] = partial |R[:, j]|^2
__global__ void k_dav_resid(double *__restrict__ R, const double *__restrict__ X,
                            const double *__restrict__ theta, int n, double *__restrict__ part) {
  const int j = blockIdx.y;
  const double th = theta[j];
  const int64_t chunk = (n + gridDim.x - 1) / gridDim.x;
  const int64_t i0 = chunk * blockIdx.x, i1 = min((int64_t)n, i0 + chunk);
  double s = 0.0;
  for (int64_t i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
    int64_t o = i + (int64_t)n * j;
    double r = R[o] - th * X[o];
    R[o] = r;
    s += r * r;
  }
  __shared__ double red[256];
  s = block_sum256(s, red);
  if (threadIdx.x == 0) part[(int64_t)j * gridDim.x + blockIdx.x] = s;
}

// part[j*gridDim.x + b] = partial |T[:, j]|^2
__global__ void k_colnorm_part(const double *__restrict__ T, int n, double *__restrict__ part) {
  const int j = blockIdx.y;
  const int64_t chunk = (n + gridDim.x - 1) / gridDim.x;
  const int64_t i0 = chunk * blockIdx.x, i1 = min((int64_t)n, i0 + chunk);
  const double *t = T + (int64_t)n * j;
  double s = 0.0;
  for (int64_t i = i0 + threadIdx.x; i < i1; i += blockDim.x) s += t[i] * t[i];
  __shared__ double red[256];
  s = block_sum256(s, red);
  if (threadIdx.x == 0) part[(int64_t)j * gridDim.x + blockIdx.x] = s;
}

// out[j] = sqrt(sum_b part[j*nsplit + b]), in order
__global__ void k_colnorm_finish(const double *__restrict__ part, int nsplit, int ncol,
                                 double *__restrict__ out) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= ncol) return;
  double s = 0.0;
  for (int b = 0; b < nsplit; ++b) s += part[(int64_t)j * nsplit + b];
  out[j] = sqrt(s);
}

__global__ void k_unit_vectors(double *__restrict__ V, int n, const int *__restrict__ idx, int k) {
  int64_t total = (int64_t)n * k;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    int j = (int)(t / n), i = (int)(t - (int64_t)j * n);
    V[t] = (i == idx[j]) ? 1.0 : 0.0;
  }
}

// column norms of T (one block per column)
// T[:, j] *= f(s[j]) with mode 0: 1/s, mode 1: 1/sqrt(s)
__global__ void k_scale_by(double *__restrict__ T, int n, int ncol, const double *__restrict__ sv,
                           int mode) {
  int64_t total = (int64_t)n * ncol;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    double v = sv[t / n];
    T[t] *= mode == 0 ? (v > 0 ? 1.0 / v : 0.0) : (v > 0 ? 1.0 / sqrt(v) : 0.0);
  }
}

// H[c + ld*r] = H[r + ld*c] for rows r < m of the new columns c in [m, m+nb)
__global__ void k_mirror_cols(double *__restrict__ H, int ld, int m, int nb) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= (int64_t)m * nb) return;
  int c = m + (int)(t / m), r = (int)(t % m);
  H[c + (int64_t)ld * r] = H[r + (int64_t)ld * c];
}

// H[0:k, 0:k] = diag(theta)
__global__ void k_diag_matrix(double *__restrict__ H, int ld, int k, const double *__restrict__ th) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= (int64_t)k * k) return;
  int c = (int)(t / k), r = (int)(t % k);
  H[r + (int64_t)ld * c] = r == c ? th[r] : 0.0;
}

// Cholesky QR factor of a small Gram matrix, in one CTA: G = L L^T (nc x nc,
// lower triangle read, nc <= kCholMax), then out = L^-T (upper triangular,
// column-major nc x nc, zero below the diagonal) so that T L^-T has
// orthonormal columns.  stat[0] = 1 when a pivot is not positive or its
// square root falls below sqrt(tol) (the block is numerically dependent),
// else 0; stat[1] = the smallest pivot (the diagonal of L).  Right-looking
// factorisation, then one forward substitution per column of L^-1 (thread j
// solves L x = e_j); deterministic.
constexpr int kCholMax = 112;   // 2 nc^2 doubles of shared memory
__device__ __forceinline__ void chol_inv_body(const double *__restrict__ G, int nc, double tol,
                                              double *__restrict__ out,
                                              double *__restrict__ stat) {
  extern __shared__ double sm[];
  double *L = sm;               // column-major nc x nc
  double *X = sm + nc * nc;     // X[j*nc + i] = (L^-1)[i][j]
  __shared__ int fail;
  __shared__ double dmin;
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int q = tid; q < nc * nc; q += nt) {
    const int i = q % nc, j = q / nc;
    L[q] = i >= j ? G[q] : 0.0;
  }
  if (tid == 0) {
    fail = 0;
    dmin = 1e300;
  }
  __syncthreads();
  for (int j = 0; j < nc; ++j) {
    if (tid == 0) {
      const double d = L[j + nc * j];
      if (!(d > 0.0) || !(d * d > 0.0) || !isfinite(d)) {
        fail = 1;
      } else {
        const double r = sqrt(d);
        L[j + nc * j] = r;
        dmin = fmin(dmin, r);
        if (!(r * r > tol)) fail = 1;
      }
    }
    __syncthreads();
    if (fail) break;
    const double r = L[j + nc * j];
    for (int i = j + 1 + tid; i < nc; i += nt) L[i + nc * j] /= r;
    __syncthreads();
    // trailing update of the lower triangle: columns l > j, rows i >= l
    const int m = nc - j - 1;
    for (int q = tid; q < m * m; q += nt) {
      const int l = j + 1 + q / m, i = j + 1 + q % m;
      if (i >= l) L[i + nc * l] -= L[i + nc * j] * L[l + nc * j];
    }
    __syncthreads();
  }
  if (fail) {
    if (tid == 0) {
      stat[0] = 1.0;
      stat[1] = dmin;
    }
    return;
  }
  for (int j = tid; j < nc; j += nt) {
    double *x = X + (size_t)j * nc;
    for (int i = 0; i < j; ++i) x[i] = 0.0;
    x[j] = 1.0 / L[j + nc * j];
    for (int i = j + 1; i < nc; ++i) {
      double acc = 0.0;
      for (int k = j; k < i; ++k) acc += L[i + nc * k] * x[k];
      x[i] = -acc / L[i + nc * i];
    }
  }
  __syncthreads();
  // out[r + nc*c] = (L^-1)[c][r] = X[r*nc + c]  (upper: r <= c)
  for (int q = tid; q < nc * nc; q += nt) {
    const int r = q % nc, c = q / nc;
    out[q] = r <= c ? X[(size_t)r * nc + c] : 0.0;
  }
  if (tid == 0) {
    stat[0] = 0.0;
    stat[1] = dmin;
  }
}

__global__ void __launch_bounds__(256)
k_chol_inv(const double *__restrict__ G, int nc, double tol, double *__restrict__ out,
           double *__restrict__ stat) {
  chol_inv_body(G, nc, tol, out, stat);
}


struct DavidsonWork {
  DBuf<double> V, W, H, Hs, theta, X, R, T, tmp, rn, proj, G, Gc, Gz, lam, work2, part, eigwork,
      stat;
  DBuf<int> cols, idx, info, einfo;
  DBuf<double> work;
  int iters = 0;
  int64_t matvecs = 0;
  double max_resid = 0;
  // optional section timing (synchronises at every section boundary):
  // [0] sigma products, [1] projected matrix, [2] its eigen-decomposition,
  // [3] Ritz vectors + residuals, [4] orthogonalisation
  bool profile = false;
  double sec_ms[5] = {0, 0, 0, 0, 0};
  Dgemm *dg = nullptr;   // the context's FP64 products (dgemm.cuh)
  // residual norms and Ritz values of the last Rayleigh-Ritz step (every
  // tracked pair, the buffer roots above the wanted ones included)
  std::vector<double> final_resid, final_theta;
};

// host wall-clock section timer used when DavidsonWork::profile is set
struct SectionClock {
  DavidsonWork &dw;
  cudaStream_t s;
  std::chrono::steady_clock::time_point t0;
  SectionClock(DavidsonWork &w, cudaStream_t st) : dw(w), s(st) {
    if (dw.profile) {
      S2G_CUDA(cudaStreamSynchronize(s));
      t0 = std::chrono::steady_clock::now();
    }
  }
  void tick(int slot) {
    if (!dw.profile) return;
    S2G_CUDA(cudaStreamSynchronize(s));
    auto t1 = std::chrono::steady_clock::now();
    dw.sec_ms[slot] += std::chrono::duration<double, std::milli>(t1 - t0).count();
    t0 = t1;
  }
};

using MatVec = std::function<void(const double *V, int nb, double *W)>;

// Rayleigh-Ritz problems up to this size go to the engine's own eigensolver
// (symeig_small.cuh: 0.31 / 0.58 / 1.96 ms of kernel time at m = 64 / 120 /
// 300 against 1.1 / 2.3 / 3.2 ms for syevd); larger ones to cuSOLVER syevd.
constexpr int kRRSmallMax = kSymEigMaxN;

// Orthonormalises the nc columns of T (n x nc) against the m orthonormal
// columns of V and among themselves, and appends the result to V after column
// m (BCGS2: normalise, then two rounds of one block classical Gram-Schmidt
// projection against V followed by Cholesky QR of the block, or, when its Gram
// matrix is not safely positive definite, orthonormalisation through the Gram
// matrix's eigen-decomposition that drops dependent directions).  Returns the
// number of columns appended.  kcap: capacity of the k x k work arrays.
inline int dav_orthonormalize(DavidsonWork &dw, cublasHandle_t blas, cusolverDnHandle_t sol,
                              cudaStream_t s, double *V, int n, int m, double *T, int nc,
                              int kcap) {
  const int k = kcap;
  const int grid = 148 * 4;
  const double one = 1.0, zero = 0.0, mone = -1.0;
  double *tmp = dw.tmp.ensure((size_t)n * k);
  double *proj = dw.proj.ensure((size_t)(m + k) * k + 4);
  int *info = dw.info.ensure(1);
  int nb = 0;
  {
    double *G = dw.G.ensure((size_t)k * k), *lam = dw.lam.ensure(k);
    double *part = dw.part.ensure((size_t)k * kColSplit);
    S2G_LAUNCH(k_colnorm_part, dim3(kColSplit, (unsigned)nc), 256, 0, s, T, n, part);
    S2G_LAUNCH(k_colnorm_finish, (int)div_up(nc, 128), 128, 0, s, part, kColSplit, nc, lam);
    S2G_LAUNCH(k_scale_by, grid, 256, 0, s, T, n, nc, lam, 0);
    double *Tb = T;
    int ncur = nc;
    for (int round = 0; round < 2 && ncur > 0; ++round) {
      (dw.dg->gemm(s, CUBLAS_OP_T, CUBLAS_OP_N, m, ncur, n, &one, V, n, Tb, n,
                             &zero, proj, m));
      (dw.dg->gemm(s, CUBLAS_OP_N, CUBLAS_OP_N, n, ncur, m, &mone, V, n, proj, m,
                             &one, Tb, n));
      // G = Tb^T Tb; Cholesky QR when G is safely positive definite
      (dw.dg->gemm(s, CUBLAS_OP_T, CUBLAS_OP_N, ncur, ncur, n, &one, Tb, n, Tb, n,
                             &zero, G, ncur));
      if (ncur <= kCholMax) {
        // Cholesky QR: L^-T from the engine's small factorisation kernel
        double *Li = dw.Gc.ensure((size_t)k * k), *st = dw.stat.ensure(2);
        S2G_CUDA(cudaFuncSetAttribute(k_chol_inv, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)(2 * sizeof(double) * kCholMax * kCholMax)));
        S2G_LAUNCH(k_chol_inv, 1, 256, 2 * sizeof(double) * ncur * ncur, s, G, ncur, 1e-8, Li,
                   st);
        double h_st[2];
        S2G_CUDA(cudaMemcpyAsync(h_st, st, sizeof(h_st), cudaMemcpyDeviceToHost, s));
        S2G_CUDA(cudaStreamSynchronize(s));
        if (h_st[0] == 0.0) {
          // dst <- Tb L^-T (through tmp when Tb already is dst)
          double *dst = V + (size_t)n * m;
          double *o = Tb == dst ? tmp : dst;
          (dw.dg->gemm(s, CUBLAS_OP_N, CUBLAS_OP_N, n, ncur, ncur, &one, Tb, n, Li,
                                 ncur, &zero, o, n));
          if (o != dst)
            S2G_CUDA(cudaMemcpyAsync(dst, o, sizeof(double) * n * ncur,
                                     cudaMemcpyDeviceToDevice, s));
          Tb = dst;
          continue;
        }
      }
      // eigenpairs of G ascending: drop dependent directions
      if (ncur <= kRRSmallMax) {
        double *Z = dw.Gz.ensure((size_t)k * k);
        S2G_CUDA(cudaMemsetAsync(info, 0, sizeof(int), s));
        symeig_small(s, G, ncur, ncur, ncur, lam, Z, ncur,
                     dw.eigwork.ensure(symeig_work_doubles(ncur, ncur)), info);
        S2G_CUDA(cudaMemcpyAsync(G, Z, sizeof(double) * ncur * ncur, cudaMemcpyDeviceToDevice,
                                 s));
      } else {
        int lw2 = 0;
        S2G_CUSOLVER(cusolverDnDsyevd_bufferSize(sol, CUSOLVER_EIG_MODE_VECTOR,
                                                 CUBLAS_FILL_MODE_LOWER, ncur, G, ncur, lam,
                                                 &lw2));
        double *work2 = dw.work2.ensure((size_t)lw2 + 1);
        S2G_CUSOLVER(cusolverDnDsyevd(sol, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER,
                                      ncur, G, ncur, lam, work2, lw2, info));
      }
      std::vector<double> h_lam(ncur);
      S2G_CUDA(cudaMemcpyAsync(h_lam.data(), lam, sizeof(double) * ncur, cudaMemcpyDeviceToHost,
                               s));
      S2G_CUDA(cudaStreamSynchronize(s));
      int first = 0;   // keep eigenvalues above the dependence threshold
      const double cut = round == 0 ? 1e-10 : 1e-14;
      while (first < ncur && !(h_lam[first] > cut)) ++first;
      int nkeep = ncur - first;
      if (nkeep == 0) {
        ncur = 0;
        break;
      }
      // new block = Tb U_keep diag(lam_keep)^-1/2, written into V after column m
      double *dst = V + (size_t)n * m;
      (dw.dg->gemm(s, CUBLAS_OP_N, CUBLAS_OP_N, n, nkeep, ncur, &one, Tb, n,
                             G + (size_t)ncur * first, ncur, &zero, tmp, n));
      S2G_LAUNCH(k_scale_by, grid, 256, 0, s, tmp, n, nkeep, lam + first, 1);
      S2G_CUDA(cudaMemcpyAsync(dst, tmp, sizeof(double) * n * nkeep, cudaMemcpyDeviceToDevice,
                               s));
      Tb = dst;   // second round re-orthogonalises the appended block in place
      ncur = nkeep;
    }
    nb = ncur;
  }
  return nb;
}

// Returns the number of converged wanted roots (== k on success).  `mv` forms
// W = A V for nb column vectors (n x nb, column-major); `diag` is diag(A).
// With `warm`, the first block is the k Ritz vectors left in dw.X by a
// previous call on the same problem (orthonormal), instead of unit vectors.
inline int davidson(DavidsonWork &dw, cublasHandle_t blas, cusolverDnHandle_t sol,
                    cudaStream_t s, const MatVec &mv, const double *diag, int n, int k,
                    double tol, int max_iter, double *omega_out, double *X_out,
                    bool warm = false, bool buffer_roots = true) {
  if (k > n) k = n;
  const int kwant = k;
  // buffer roots (a quarter of the wanted ones, at least 4) and a subspace of
  // up to six blocks, kept within the engine's own Rayleigh-Ritz solver when the
  // block allows: measured against k/2 buffer roots and four blocks, 124 vs
  // 135 ms for the 50 roots of the C384H48 flake, 666 vs 841 ms for 48
  // molecules of 20-150 atoms with 20 roots each
  if (buffer_roots) k = std::min(n, k + std::max(4, k / 4));
  const int mmax = std::min(n, std::max(k + 32, std::min(kSymEigMaxN, 6 * k)));
  const int grid = 148 * 4;
  if (warm && dw.X.n < (size_t)n * k) warm = false;
  double *V = dw.V.ensure((size_t)n * mmax), *W = dw.W.ensure((size_t)n * mmax);
  double *Hs = dw.Hs.ensure((size_t)mmax * mmax);
  double *H = dw.H.ensure((size_t)mmax * mmax);   // V^T W, kept across iterations (ld mmax)
  double *theta = dw.theta.ensure(mmax), *X = dw.X.ensure((size_t)n * k);
  double *R = dw.R.ensure((size_t)n * k), *T = dw.T.ensure((size_t)n * k);
  double *tmp = dw.tmp.ensure((size_t)n * k), *rn = dw.rn.ensure(k + 2);
  double *proj = dw.proj.ensure((size_t)mmax * k + 4);
  int *cols = dw.cols.ensure(k), *info = dw.info.ensure(1);
  int *einfo = dw.einfo.ensure(1);   // status of the Rayleigh-Ritz eigensolves
  S2G_CUDA(cudaMemsetAsync(einfo, 0, sizeof(int), s));
  const double one = 1.0, zero = 0.0, mone = -1.0;

  // initial guess: unit vectors on the k lowest diagonal elements
  std::vector<double> h_diag(n);
  S2G_CUDA(cudaMemcpyAsync(h_diag.data(), diag, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
  S2G_CUDA(cudaStreamSynchronize(s));
  std::vector<int> order(n);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return h_diag[a] < h_diag[b]; });
  int *idx = dw.idx.ensure(k);
  if (warm) {
    S2G_CUDA(cudaMemcpyAsync(V, X, sizeof(double) * n * k, cudaMemcpyDeviceToDevice, s));
  } else {
    S2G_CUDA(cudaMemcpyAsync(idx, order.data(), sizeof(int) * k, cudaMemcpyHostToDevice, s));
    S2G_LAUNCH(k_unit_vectors, grid, 256, 0, s, V, n, idx, k);
  }
  int m = 0, nb = k;
  int lwork = 0;
  S2G_CUSOLVER(cusolverDnDsyevd_bufferSize(sol, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER,
                                           mmax, Hs, mmax, theta, &lwork));
  double *work = dw.work.ensure((size_t)lwork + 1);
  std::vector<double> h_rn(k);
  int nconv = 0;
  dw.iters = 0;
  dw.matvecs = 0;
  SectionClock clk(dw, s);
  for (int it = 0; it < max_iter; ++it) {
    dw.iters = it + 1;
    mv(V + (size_t)n * m, nb, W + (size_t)n * m);
    dw.matvecs += nb;
    clk.tick(0);
    // H = V^T W (ld mmax): only the new columns are formed; the new rows
    // follow from the symmetry of A
    (dw.dg->gemm(s, CUBLAS_OP_T, CUBLAS_OP_N, m + nb, nb, n, &one, V, n,
                           W + (size_t)n * m, n, &zero, H + (size_t)mmax * m, mmax));
    if (m > 0)
      S2G_LAUNCH(k_mirror_cols, (int)div_up((int64_t)m * nb, 256), 256, 0, s, H, mmax, m, nb);
    m += nb;
    clk.tick(1);
    if (m <= kRRSmallMax) {
      // lowest k eigenpairs, eigenvectors into Hs (ld m), no host synchronisation
      symeig_small(s, H, mmax, m, std::min(k, m), theta, Hs, m,
                   dw.eigwork.ensure(symeig_work_doubles(m, std::min(k, m))), einfo);
    } else {
      S2G_CUDA(cudaMemcpy2DAsync(Hs, sizeof(double) * m, H, sizeof(double) * mmax,
                                 sizeof(double) * m, m, cudaMemcpyDeviceToDevice, s));
      S2G_CUSOLVER(cusolverDnDsyevd(sol, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, m, Hs,
                                    m, theta, work, lwork, einfo));
    }
    clk.tick(2);
    // Ritz vectors X = V Y_k, residuals R = W Y_k - X theta
    (dw.dg->gemm(s, CUBLAS_OP_N, CUBLAS_OP_N, n, k, m, &one, V, n, Hs, m, &zero, X, n));
    (dw.dg->gemm(s, CUBLAS_OP_N, CUBLAS_OP_N, n, k, m, &one, W, n, Hs, m, &zero, R, n));
    {
      double *part = dw.part.ensure((size_t)k * kColSplit);
      S2G_LAUNCH(k_dav_resid, dim3(kColSplit, (unsigned)k), 256, 0, s, R, X, theta, n, part);
      S2G_LAUNCH(k_colnorm_finish, (int)div_up(k, 128), 128, 0, s, part, kColSplit, k, rn);
    }
    S2G_CUDA(cudaMemcpyAsync(h_rn.data(), rn, sizeof(double) * k, cudaMemcpyDeviceToHost, s));
    int h_einfo = 0;
    S2G_CUDA(cudaMemcpyAsync(&h_einfo, einfo, sizeof(int), cudaMemcpyDeviceToHost, s));
    S2G_CUDA(cudaStreamSynchronize(s));
    if (h_einfo != 0)
      throw Error{STD2G_ENOCONV, "Davidson: Rayleigh-Ritz eigensolve failed (" +
                                     std::to_string(h_einfo) + ")"};
    std::vector<int> unc;
    int nunc_wanted = 0;
    for (int j = 0; j < k; ++j)
      if (!(h_rn[j] < tol)) {
        unc.push_back(j);
        if (j < kwant) ++nunc_wanted;
      }
    nconv = kwant - nunc_wanted;
    dw.max_resid = *std::max_element(h_rn.begin(), h_rn.begin() + kwant);
    if (dw.profile)
      std::fprintf(stderr, "  davidson iter %d: m %d, unconverged %d of %d, max residual %.3e\n",
                   it + 1, m, nunc_wanted, kwant, dw.max_resid);
    clk.tick(3);
    if (nunc_wanted == 0) break;
    int nc = (int)unc.size();
    S2G_CUDA(cudaMemcpyAsync(cols, unc.data(), sizeof(int) * nc, cudaMemcpyHostToDevice, s));
    S2G_LAUNCH(k_dav_precond, grid, 256, 0, s, T, R, diag, theta, cols, n, nc);
    if (m + nc > mmax) {
      // restart with the current Ritz vectors: V <- X, W <- W Y_k
      (dw.dg->gemm(s, CUBLAS_OP_N, CUBLAS_OP_N, n, k, m, &one, W, n, Hs, m, &zero,
                             tmp, n));
      S2G_CUDA(cudaMemcpyAsync(W, tmp, sizeof(double) * n * k, cudaMemcpyDeviceToDevice, s));
      S2G_CUDA(cudaMemcpyAsync(V, X, sizeof(double) * n * k, cudaMemcpyDeviceToDevice, s));
      m = k;
      // H restricted to the Ritz vectors is diag(theta)
      S2G_LAUNCH(k_diag_matrix, (int)div_up((int64_t)k * k, 256), 256, 0, s, H, mmax, k, theta);
    }
    // block orthogonalisation of the corrections, appended to V after column m
    nb = dav_orthonormalize(dw, blas, sol, s, V, n, m, T, nc, k);
    clk.tick(4);
    if (nb == 0) break;
  }
  S2G_CUDA(cudaMemcpyAsync(omega_out, theta, sizeof(double) * kwant, cudaMemcpyDeviceToDevice, s));
  S2G_CUDA(cudaMemcpyAsync(X_out, X, sizeof(double) * n * kwant, cudaMemcpyDeviceToDevice, s));
  dw.final_theta.assign(k, 0.0);
  S2G_CUDA(cudaMemcpyAsync(dw.final_theta.data(), theta, sizeof(double) * k,
                           cudaMemcpyDeviceToHost, s));
  S2G_CUDA(cudaStreamSynchronize(s));
  dw.final_resid = h_rn;
  return nconv;
}

}  // namespace std2g
