// Iterative sTD-DFT roots: the lowest k solutions of
//   (A-B)(A+B) |X+Y> = w^2 |X+Y>,   A-B positive definite,
// by the Davidson scheme of Stratmann, Scuseria and Frisch (J. Chem. Phys. 109,
// 8218 (1998)).  The reference diagonalises the dense problem (srpapack,
// srpapack.f:32-197: (A-B)^1/2 by sspevd, M = (A-B)^1/2 (A+B) (A-B)^1/2 by
// ssyevr); here the same reduction is applied to a subspace:
//   b (n x m, orthonormal), P = (A+B) b, Q = (A-B) b (caller-supplied products),
//   Ap = b^T P, Am = b^T Q,  S = Am^1/2,  S Ap S z = w^2 z,
//   (X+Y)_r = S z / sqrt(w),  (X-Y)_r = Ap (X+Y)_r / w,
// so that (X+Y)^T (X-Y) = 1 as srpapack normalises.  Residuals
//   R+ = (A+B)(X+Y) - w (X-Y),   R- = (A-B)(X-Y) - w (X+Y)
// are formed in FP64; the corrections solve the 2 x 2 diagonal blocks
// [[d+, -w], [-w, d-]] (d+-: the diagonals of A+-B) and both join the
// subspace (block orthonormalisation of davidson.cuh).  On restart the basis
// becomes the span of the current X+Y and X-Y (dependent directions dropped),
// with the products transformed, not recomputed.
#pragma once

#include <cmath>
#include <vector>

#include "common.cuh"
#include "davidson.cuh"
#include "kernels_fp64.cuh"
#include "symeig_small.cuh"

namespace std2g {

// U[:, j] *= sqrt(lam[j]) for an m x m matrix (ld m); lam below 0 counts as 0
__global__ void k_cols_times_sqrt(double *__restrict__ U, const double *__restrict__ lam, int m) {
  const int64_t total = (int64_t)m * m;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const double e = lam[t / m];
    U[t] *= sqrt(e > 0.0 ? e : 0.0);
  }
}

// C[:, j] *= f(w[j]): mode 0 1/sqrt(w), mode 1 1/w (ld ld, rows m, k columns)
__global__ void k_cols_scale_w(double *__restrict__ C, int ld, int m, int k,
                               const double *__restrict__ w, int mode) {
  const int64_t total = (int64_t)m * k;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int j = (int)(t / m), i = (int)(t - (int64_t)j * m);
    const double x = w[j];
    C[i + (int64_t)ld * j] *= mode == 0 ? 1.0 / sqrt(x) : 1.0 / x;
  }
}

// R+ -= w XmY, R- -= w XpY; part[j*gridDim.x + b] = partial |R+_j|^2 + |R-_j|^2
__global__ void k_rpa_resid(double *__restrict__ Rp, double *__restrict__ Rm,
                            const double *__restrict__ XpY, const double *__restrict__ XmY,
                            const double *__restrict__ w, int n, double *__restrict__ part) {
  const int j = blockIdx.y;
  const double om = w[j];
  const int64_t chunk = (n + gridDim.x - 1) / gridDim.x;
  const int64_t i0 = chunk * blockIdx.x, i1 = min((int64_t)n, i0 + chunk);
  double sacc = 0.0;
  for (int64_t i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
    const int64_t o = i + (int64_t)n * j;
    const double rp = Rp[o] - om * XmY[o], rm = Rm[o] - om * XpY[o];
    Rp[o] = rp;
    Rm[o] = rm;
    sacc += rp * rp + rm * rm;
  }
  __shared__ double red[256];
  sacc = block_sum256(sacc, red);
  if (threadIdx.x == 0) part[(int64_t)j * gridDim.x + blockIdx.x] = sacc;
}

// corrections of the unconverged roots cols[0..nc): from the diagonal 2 x 2
// blocks, T[:, j] = (d- R+ + w R-) / det, T[:, nc + j] = (w R+ + d+ R-) / det,
// det = d+ d- - w^2 (kept away from zero)
__global__ void k_rpa_precond(double *__restrict__ T, const double *__restrict__ Rp,
                              const double *__restrict__ Rm, const double *__restrict__ dp,
                              const double *__restrict__ dm, const double *__restrict__ w,
                              const int *__restrict__ cols, int n, int nc) {
  const int64_t total = (int64_t)n * nc;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int j = (int)(t / n), i = (int)(t - (int64_t)j * n);
    const int c = cols[j];
    const double om = w[c], a = dp[i], b = dm[i];
    double det = a * b - om * om;
    if (fabs(det) < 1e-8) det = det < 0 ? -1e-8 : 1e-8;
    const double rp = Rp[i + (int64_t)n * c], rm = Rm[i + (int64_t)n * c];
    T[t] = (b * rp + om * rm) / det;
    T[t + (int64_t)n * nc] = (om * rp + a * rm) / det;
  }
}

struct DavidsonRpaWork {
  DBuf<double> Q, Am, Amc, Ap2, S, T1, Mr, lam, ev, Z, Xp, Xm, Rp, Rm, C, Qc, tmpn, rn, part, om,
      wf, XpY, XmY;
  DBuf<int> cols, einfo;
  int iters = 0;
  int64_t matvecs = 0;
  // residual norms and roots of the last subspace step (all tracked pairs)
  std::vector<double> final_resid, final_omega;
};

// Symmetric eigen-decomposition of the m x m matrix A (ld lda, lower read):
// the lowest k pairs into w, Z (ld m); the engine's solver up to its size limit
// (no host synchronisation), cuSOLVER syevd beyond it
inline void rpa_small_eig(DavidsonWork &dw, DavidsonRpaWork &rw, cusolverDnHandle_t sol,
                          cudaStream_t s, const double *A, int lda, int m, int k, double *w,
                          double *Z, double *Zfull, int *einfo) {
  if (m <= kSymEigMaxN) {
    symeig_small(s, A, lda, m, k, w, Z, m, dw.eigwork.ensure(symeig_work_doubles(m, k)), einfo);
    return;
  }
  // full decomposition on a copy, the lowest k pairs are its leading columns
  S2G_CUDA(cudaMemcpy2DAsync(Zfull, sizeof(double) * m, A, sizeof(double) * lda,
                             sizeof(double) * m, m, cudaMemcpyDeviceToDevice, s));
  double *wf = rw.wf.ensure(m);
  int lwork = 0;
  S2G_CUSOLVER(cusolverDnDsyevd_bufferSize(sol, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER,
                                           m, Zfull, m, wf, &lwork));
  double *work = dw.work.ensure((size_t)lwork + 1);
  S2G_CUSOLVER(cusolverDnDsyevd(sol, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, m, Zfull,
                                m, wf, work, lwork, einfo));
  S2G_CUDA(cudaMemcpyAsync(w, wf, sizeof(double) * k, cudaMemcpyDeviceToDevice, s));
  if (Z != Zfull)
    S2G_CUDA(cudaMemcpyAsync(Z, Zfull, sizeof(double) * m * k, cudaMemcpyDeviceToDevice, s));
}

// Returns the number of converged wanted roots (== k on success).  mv_p /
// mv_m form (A+B) V and (A-B) V for nb columns; dp, dm are diag(A+B),
// diag(A-B).  On return omega_out [k], XpY_out, XmY_out (n x k).
inline int davidson_rpa(DavidsonWork &dw, DavidsonRpaWork &rw, cublasHandle_t blas,
                        cusolverDnHandle_t sol, cudaStream_t s, const MatVec &mv_p,
                        const MatVec &mv_m, const double *dp, const double *dm, int n, int k,
                        double tol, int max_iter, double *omega_out, double *XpY_out,
                        double *XmY_out) {
  if (k > n) k = n;
  const int kwant = k;
  k = std::min(n, k + std::max(4, k / 2));
  const int mmax = std::min(n, std::max(4 * k, 2 * k + 32));
  const int grid = 148 * 4;
  const double one = 1.0, zero = 0.0;
  double *B = dw.V.ensure((size_t)n * mmax), *P = dw.W.ensure((size_t)n * mmax);
  double *Q = rw.Q.ensure((size_t)n * mmax);
  double *Ap = dw.H.ensure((size_t)mmax * mmax), *Am = rw.Am.ensure((size_t)mmax * mmax);
  double *lam = rw.lam.ensure(mmax), *U = rw.Amc.ensure((size_t)mmax * mmax);
  double *S = rw.S.ensure((size_t)mmax * mmax), *T1 = rw.T1.ensure((size_t)mmax * mmax);
  double *Mr = rw.Mr.ensure((size_t)mmax * mmax), *ev = rw.ev.ensure(k);
  double *Z = rw.Z.ensure((size_t)mmax * k), *Zf = rw.Ap2.ensure((size_t)mmax * mmax);
  double *Xp = rw.Xp.ensure((size_t)mmax * k), *Xm = rw.Xm.ensure((size_t)mmax * k);
  double *XpY = rw.XpY.ensure((size_t)n * k), *XmY = rw.XmY.ensure((size_t)n * k);
  double *Rp = rw.Rp.ensure((size_t)n * k), *Rm = rw.Rm.ensure((size_t)n * k);
  double *T = dw.T.ensure((size_t)n * 2 * k), *om = rw.om.ensure(k);
  double *rn = rw.rn.ensure(k), *part = rw.part.ensure((size_t)k * kColSplit);
  int *cols = rw.cols.ensure(k), *einfo = rw.einfo.ensure(1);
  S2G_CUDA(cudaMemsetAsync(einfo, 0, sizeof(int), s));
  // initial block: unit vectors on the k lowest diagonal elements of A
  std::vector<double> h_dp(n), h_dm(n);
  S2G_CUDA(cudaMemcpyAsync(h_dp.data(), dp, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
  S2G_CUDA(cudaMemcpyAsync(h_dm.data(), dm, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
  S2G_CUDA(cudaStreamSynchronize(s));
  std::vector<int> order(n);
  for (int i = 0; i < n; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(),
                   [&](int a, int b) { return h_dp[a] + h_dm[a] < h_dp[b] + h_dm[b]; });
  int *idx = dw.idx.ensure(k);
  S2G_CUDA(cudaMemcpyAsync(idx, order.data(), sizeof(int) * k, cudaMemcpyHostToDevice, s));
  S2G_LAUNCH(k_unit_vectors, grid, 256, 0, s, B, n, idx, k);
  int m = 0, nb = k, nconv = 0, last_kk = 0;
  std::vector<double> h_rn(k), h_lam(1);
  rw.iters = 0;
  rw.matvecs = 0;
  auto add_columns = [&](double *H, const double *W, int mnew, int nbn) {
    (dw.dg->gemm(s, CUBLAS_OP_T, CUBLAS_OP_N, mnew + nbn, nbn, n, &one, B, n,
                           W + (size_t)n * mnew, n, &zero, H + (size_t)mmax * mnew, mmax));
    if (mnew > 0)
      S2G_LAUNCH(k_mirror_cols, (int)div_up((int64_t)mnew * nbn, 256), 256, 0, s, H, mmax, mnew,
                 nbn);
  };
  for (int it = 0; it < max_iter; ++it) {
    rw.iters = it + 1;
    mv_p(B + (size_t)n * m, nb, P + (size_t)n * m);
    mv_m(B + (size_t)n * m, nb, Q + (size_t)n * m);
    rw.matvecs += nb;
    add_columns(Ap, P, m, nb);
    add_columns(Am, Q, m, nb);
    m += nb;
    // S = Am^1/2
    rpa_small_eig(dw, rw, sol, s, Am, mmax, m, m, lam, U, Zf, einfo);
    S2G_CUDA(cudaMemcpyAsync(h_lam.data(), lam, sizeof(double), cudaMemcpyDeviceToHost, s));
    S2G_CUDA(cudaMemcpyAsync(T1, U, sizeof(double) * m * m, cudaMemcpyDeviceToDevice, s));
    S2G_LAUNCH(k_cols_times_sqrt, grid, 256, 0, s, T1, lam, m);
    (dw.dg->gemm(s, CUBLAS_OP_N, CUBLAS_OP_T, m, m, m, &one, T1, m, U, m, &zero, S,
                           m));
    // M_r = S Ap S, its lowest k pairs
    (dw.dg->gemm(s, CUBLAS_OP_N, CUBLAS_OP_N, m, m, m, &one, Ap, mmax, S, m, &zero,
                           T1, m));
    (dw.dg->gemm(s, CUBLAS_OP_N, CUBLAS_OP_N, m, m, m, &one, S, m, T1, m, &zero, Mr,
                           m));
    const int kk = std::min(k, m);
    last_kk = kk;
    rpa_small_eig(dw, rw, sol, s, Mr, m, m, kk, ev, Z, Zf, einfo);
    S2G_LAUNCH(k_sqrt_inplace, (int)div_up(kk, 128), 128, 0, s, ev, kk);
    S2G_CUDA(cudaMemcpyAsync(om, ev, sizeof(double) * kk, cudaMemcpyDeviceToDevice, s));
    // (X+Y)_r = S z / sqrt(w), (X-Y)_r = Ap (X+Y)_r / w
    (dw.dg->gemm(s, CUBLAS_OP_N, CUBLAS_OP_N, m, kk, m, &one, S, m, Z, m, &zero, Xp,
                           m));
    S2G_LAUNCH(k_cols_scale_w, grid, 256, 0, s, Xp, m, m, kk, om, 0);
    (dw.dg->gemm(s, CUBLAS_OP_N, CUBLAS_OP_N, m, kk, m, &one, Ap, mmax, Xp, m, &zero,
                           Xm, m));
    S2G_LAUNCH(k_cols_scale_w, grid, 256, 0, s, Xm, m, m, kk, om, 1);
    // full-space vectors and residuals
    (dw.dg->gemm(s, CUBLAS_OP_N, CUBLAS_OP_N, n, kk, m, &one, B, n, Xp, m, &zero,
                           XpY, n));
    (dw.dg->gemm(s, CUBLAS_OP_N, CUBLAS_OP_N, n, kk, m, &one, B, n, Xm, m, &zero,
                           XmY, n));
    (dw.dg->gemm(s, CUBLAS_OP_N, CUBLAS_OP_N, n, kk, m, &one, P, n, Xp, m, &zero, Rp,
                           n));
    (dw.dg->gemm(s, CUBLAS_OP_N, CUBLAS_OP_N, n, kk, m, &one, Q, n, Xm, m, &zero, Rm,
                           n));
    S2G_LAUNCH(k_rpa_resid, dim3(kColSplit, (unsigned)kk), 256, 0, s, Rp, Rm, XpY, XmY, om, n,
               part);
    S2G_LAUNCH(k_colnorm_finish, (int)div_up(kk, 128), 128, 0, s, part, kColSplit, kk, rn);
    S2G_CUDA(cudaMemcpyAsync(h_rn.data(), rn, sizeof(double) * kk, cudaMemcpyDeviceToHost, s));
    int h_einfo = 0;
    S2G_CUDA(cudaMemcpyAsync(&h_einfo, einfo, sizeof(int), cudaMemcpyDeviceToHost, s));
    S2G_CUDA(cudaStreamSynchronize(s));
    if (h_einfo != 0) throw Error{STD2G_ENOCONV, "sTD-DFT Davidson: subspace eigensolve failed"};
    if (!(h_lam[0] > 0.0))
      throw Error{STD2G_EAMB_NOT_PD, "matrix power impossible (A-B not positive definite)"};
    std::vector<int> unc;
    int nunc_wanted = 0;
    for (int j = 0; j < kk; ++j)
      if (!(h_rn[j] < tol)) {
        unc.push_back(j);
        if (j < kwant) ++nunc_wanted;
      }
    nconv = std::min(kwant, kk) - nunc_wanted;
    if (nunc_wanted == 0 && kk >= kwant) break;
    const int nc = (int)unc.size();
    S2G_CUDA(cudaMemcpyAsync(cols, unc.data(), sizeof(int) * nc, cudaMemcpyHostToDevice, s));
    S2G_LAUNCH(k_rpa_precond, grid, 256, 0, s, T, Rp, Rm, dp, dm, om, cols, n, nc);
    if (m + 2 * nc > mmax) {
      // restart on span{X+Y, X-Y} of the kk roots: C = [Xp Xm] (m x 2kk),
      // orthonormalised through its Gram matrix (dependent directions dropped;
      // in the Tamm-Dancoff limit X-Y is parallel to X+Y)
      const int nc2 = 2 * kk;
      double *C = rw.C.ensure((size_t)mmax * 2 * k);
      S2G_CUDA(cudaMemcpyAsync(C, Xp, sizeof(double) * m * kk, cudaMemcpyDeviceToDevice, s));
      S2G_CUDA(cudaMemcpyAsync(C + (size_t)m * kk, Xm, sizeof(double) * m * kk,
                               cudaMemcpyDeviceToDevice, s));
      double *G = dw.G.ensure((size_t)4 * k * k), *gl = dw.lam.ensure(2 * k);
      (dw.dg->gemm(s, CUBLAS_OP_T, CUBLAS_OP_N, nc2, nc2, m, &one, C, m, C, m, &zero,
                             G, nc2));
      double *Gz = dw.Gz.ensure((size_t)4 * k * k);
      rpa_small_eig(dw, rw, sol, s, G, nc2, nc2, nc2, gl, Gz, Zf, einfo);
      std::vector<double> h_gl(nc2);
      S2G_CUDA(cudaMemcpyAsync(h_gl.data(), gl, sizeof(double) * nc2, cudaMemcpyDeviceToHost, s));
      S2G_CUDA(cudaStreamSynchronize(s));
      int first = 0;
      while (first < nc2 && !(h_gl[first] > 1e-10 * h_gl[nc2 - 1])) ++first;
      const int nkeep = nc2 - first;
      double *Qc = rw.Qc.ensure((size_t)mmax * 2 * k);
      (dw.dg->gemm(s, CUBLAS_OP_N, CUBLAS_OP_N, m, nkeep, nc2, &one, C, m,
                             Gz + (size_t)nc2 * first, nc2, &zero, Qc, m));
      S2G_LAUNCH(k_scale_by, grid, 256, 0, s, Qc, m, nkeep, gl + first, 1);
      // b <- b Qc, P <- P Qc, Q <- Q Qc; Ap, Am <- Qc^T (.) Qc
      double *tn = rw.tmpn.ensure((size_t)n * 2 * k);
      for (double *X : {B, P, Q}) {
        (dw.dg->gemm(s, CUBLAS_OP_N, CUBLAS_OP_N, n, nkeep, m, &one, X, n, Qc, m,
                               &zero, tn, n));
        S2G_CUDA(cudaMemcpyAsync(X, tn, sizeof(double) * n * nkeep, cudaMemcpyDeviceToDevice, s));
      }
      for (double *H : {Ap, Am}) {
        (dw.dg->gemm(s, CUBLAS_OP_N, CUBLAS_OP_N, m, nkeep, m, &one, H, mmax, Qc, m,
                               &zero, T1, m));
        (dw.dg->gemm(s, CUBLAS_OP_T, CUBLAS_OP_N, nkeep, nkeep, m, &one, Qc, m, T1, m,
                               &zero, H, mmax));
      }
      m = nkeep;
    }
    nb = dav_orthonormalize(dw, blas, sol, s, B, n, m, T, 2 * nc, 2 * k);
    if (nb == 0) break;
  }
  S2G_CUDA(cudaMemcpyAsync(omega_out, om, sizeof(double) * kwant, cudaMemcpyDeviceToDevice, s));
  S2G_CUDA(cudaMemcpyAsync(XpY_out, XpY, sizeof(double) * n * kwant, cudaMemcpyDeviceToDevice, s));
  S2G_CUDA(cudaMemcpyAsync(XmY_out, XmY, sizeof(double) * n * kwant, cudaMemcpyDeviceToDevice, s));
  rw.final_omega.assign(last_kk, 0.0);
  S2G_CUDA(cudaMemcpyAsync(rw.final_omega.data(), om, sizeof(double) * last_kk,
                           cudaMemcpyDeviceToHost, s));
  S2G_CUDA(cudaStreamSynchronize(s));
  rw.final_resid.assign(h_rn.begin(), h_rn.begin() + last_kk);
  return nconv;
}

}  // namespace std2g
