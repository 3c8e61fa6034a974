// Matrix-free products with the sTDA / sTD-DFT matrices.
//
// The reference builds A (rtdamat, stda.f:2010-2056), A+B / A-B (rrpamat,
// stda.f:1870-2004) and 0.5 B (rtdacorr, apbtrafo.f:580-643) element by
// element, each element being a gathered dot product over atoms:
//   (ia|jb) = p_ia . q_jb    (gamma^K)
//   (ij|ab) = p_ij . q_ab    (gamma^J)
//   (ib|ja) = p_ib . q_ja    (gamma^K)
// Here only products M X with blocks of vectors X are formed, never M itself.
// With the Loewdin MOs C (q_pq^A = sum_{k in A} C_kp C_kq) the three couplings
// factor into dense GEMMs:
//   K X   : g = sum_v q_v X_v (N x m), then p_u . g               -- 2 GEMMs
//   J X   : Z = C_v X^T  ->  T_A = P^A_oo Z_A  ->  C_v^T T      -- 3 GEMMs
//   Kx X  : Z = C_o X    ->  U_A = P^A_ov Z_A  ->  C_v^T U      -- 3 GEMMs
// where A runs over atoms, Z_A / T_A / U_A hold the rows of the AOs on atom A
// (padded to `maxa` slots per atom) and P^A are gamma-contracted charges in
// atom-major layout.  Every term of the element-wise definition is included
// (the diagonal ones too), so A X only needs the correction
// ed - (ak K_uu - J_uu) on the diagonal.
#pragma once

#include "common.cuh"

namespace std2g {

// box[o] = X[u + nci*r] at the CSF's (j,b); layout 0: o = j + no*b + nov*r,
// layout 1: o = b + nv*j + nov*r.  The caller zeroes the box first.
__global__ void k_mf_scatter(double *__restrict__ box, const double *__restrict__ X,
                             const int *__restrict__ ci, const int *__restrict__ ca, int nci, int no,
                             int64_t nov, int m, int layout) {
  int64_t total = (int64_t)nci * m;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    int r = (int)(t / nci), u = (int)(t - (int64_t)r * nci);
    int64_t o;
    if (layout == 0)
      o = ci[u] + (int64_t)no * ca[u] + nov * r;
    else
      o = ca[u] + (nov / no) * (int64_t)ci[u] + nov * r;
    box[o] = X[t];
  }
}

// out[u + nci*r] += box[a_u + nv*(i_u + no*r)]
__global__ void k_mf_gather(double *__restrict__ out, const double *__restrict__ box,
                            const int *__restrict__ ci, const int *__restrict__ ca, int nci, int no,
                            int nv, int m) {
  int64_t total = (int64_t)nci * m;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    int r = (int)(t / nci), u = (int)(t - (int64_t)r * nci);
    out[t] += box[ca[u] + (int64_t)nv * (ci[u] + (int64_t)no * r)];
  }
}

// Z is (maxa*N x ncol*m) with row (A*maxa+s), column (c + ncol*r);
// Zt[A][c + ncol*(s + maxa*r)]
__global__ void k_mf_to_atom_major(double *__restrict__ Zt, const double *__restrict__ Z, int N,
                                   int maxa, int ncol, int m) {
  int64_t rows = (int64_t)N * maxa;
  int64_t total = rows * ncol * m;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    int64_t col = t / rows;
    int64_t row = t - col * rows;
    int r = (int)(col / ncol), c = (int)(col - (int64_t)r * ncol);
    int A = (int)(row / maxa), s = (int)(row - (int64_t)A * maxa);
    Zt[(int64_t)A * ncol * maxa * m + c + (int64_t)ncol * (s + (int64_t)maxa * r)] = Z[t];
  }
}

// inverse of k_mf_to_atom_major, scaled by f, optionally accumulating
__global__ void k_mf_from_atom_major(double *__restrict__ Z, const double *__restrict__ T, int N,
                                     int maxa, int ncol, int m, double f, int accumulate) {
  int64_t rows = (int64_t)N * maxa;
  int64_t total = rows * ncol * m;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    int64_t col = t / rows;
    int64_t row = t - col * rows;
    int r = (int)(col / ncol), c = (int)(col - (int64_t)r * ncol);
    int A = (int)(row / maxa), s = (int)(row - (int64_t)A * maxa);
    double v = f * T[(int64_t)A * ncol * maxa * m + c + (int64_t)ncol * (s + (int64_t)maxa * r)];
    Z[t] = accumulate ? Z[t] + v : v;
  }
}

// dst[A*n1*n2 + i + n1*b] = src[A + N*(i*n2 + b)]: [pair (i,b)][atom] -> per atom an
// n1 x n2 column-major matrix
__global__ void k_pair_to_atom_major(double *__restrict__ dst, const double *__restrict__ src,
                                     int N, int n1, int n2) {
  int64_t np = (int64_t)n1 * n2;
  int64_t total = (int64_t)N * np;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    int64_t A = t / np, q = t - A * np;
    int64_t b = q / n1, i = q - b * n1;
    dst[t] = src[A + (int64_t)N * (i * n2 + b)];
  }
}

// out[t] += d[t % n] * X[t]
__global__ void k_add_diag(double *__restrict__ out, const double *__restrict__ X,
                           const double *__restrict__ d, int n, int m) {
  int64_t total = (int64_t)n * m;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x)
    out[t] += d[t % n] * X[t];
}

// padded AO rows: out[(A*maxa+s) + rows*c] = C[slot_ao[A*maxa+s] + nao*(c0+c)] or 0
__global__ void k_mf_pad_rows(double *__restrict__ out, const double *__restrict__ C, int nao,
                              const int *__restrict__ slot_ao, int rows, int c0, int ncol) {
  int64_t total = (int64_t)rows * ncol;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    int c = (int)(t / rows), r = (int)(t - (int64_t)c * rows);
    int k = slot_ao[r];
    out[t] = k >= 0 ? C[k + (int64_t)nao * (c0 + c)] : 0.0;
  }
}

// diagonal correction for A: dA[u] = ed[u] - (ak*ek[u] - (ii|aa))
__global__ void k_mf_diag(double *__restrict__ dA, const double *__restrict__ ed,
                          const double *__restrict__ ekd, const double *__restrict__ uci,
                          const int *__restrict__ ci, const int *__restrict__ ca, int nci, int nv,
                          double ak) {
  int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= nci) return;
  double jd = uci[ca[u] + (int64_t)nv * ci[u]];
  dA[u] = ed[u] - (ak * ekd[u] - jd);
}

struct MatFree {
  int N = 0, maxa = 0, no = 0, nv = 0, nci = 0, nao = 0;
  DBuf<double> CvP, CoP, PooA, PovA, dA;
  DBuf<double> box, Z, Zt, T, Tacc, G;
  const double *Qs = nullptr, *Ps = nullptr;
  const int *ci = nullptr, *ca = nullptr;
};

inline void mf_dgemm(cublasHandle_t h, cublasOperation_t ta, cublasOperation_t tb, int m, int n,
                     int k, double alpha, const double *A, int lda, const double *B, int ldb,
                     double beta, double *C, int ldc) {
  if (m == 0 || n == 0) return;
  S2G_CUBLAS(cublasDgemm(h, ta, tb, m, n, k, &alpha, A, lda, B, ldb, &beta, C, ldc));
}

// out (nci x m) = cK (K X) + cJ (J X) + cX (Kx X) + diag o X   (diag may be NULL)
inline void mf_apply(MatFree &mf, cublasHandle_t h, cudaStream_t s, const double *X, int m,
                     double *out, double cK, double cJ, double cX, const double *diag) {
  const int N = mf.N, maxa = mf.maxa, no = mf.no, nv = mf.nv, nci = mf.nci;
  const int rows = N * maxa;
  const int64_t nov = (int64_t)no * nv;
  const int grid = 148 * 8;
  S2G_CUDA(cudaMemsetAsync(out, 0, sizeof(double) * nci * m, s));
  if (cK != 0.0) {
    double *G = mf.G.ensure((size_t)N * m);
    mf_dgemm(h, CUBLAS_OP_N, CUBLAS_OP_N, N, m, nci, 1.0, mf.Qs, N, X, nci, 0.0, G, N);
    mf_dgemm(h, CUBLAS_OP_T, CUBLAS_OP_N, nci, m, N, cK, mf.Ps, N, G, N, 1.0, out, nci);
  }
  if (cJ != 0.0 || cX != 0.0) {
    double *box = mf.box.ensure((size_t)nov * m);
    double *Z = mf.Z.ensure((size_t)rows * std::max(no, nv) * m);
    double *Zt = mf.Zt.ensure((size_t)rows * std::max(no, nv) * m);
    double *T = mf.T.ensure((size_t)rows * no * m);
    double *Tacc = mf.Tacc.ensure((size_t)rows * no * m);
    const double one = 1.0, zero = 0.0;
    bool have = false;
    if (cJ != 0.0) {
      S2G_CUDA(cudaMemsetAsync(box, 0, sizeof(double) * nov * m, s));
      S2G_LAUNCH(k_mf_scatter, grid, 256, 0, s, box, X, mf.ci, mf.ca, nci, no, nov, m, 1);
      // Z = CvP (rows x nv) * XbT (nv x no*m)
      mf_dgemm(h, CUBLAS_OP_N, CUBLAS_OP_N, rows, no * m, nv, 1.0, mf.CvP.get(), rows, box, nv,
               0.0, Z, rows);
      S2G_LAUNCH(k_mf_to_atom_major, grid, 256, 0, s, Zt, Z, N, maxa, no, m);
      // T_A = P^A_oo (no x no) * Zt_A (no x maxa*m), batched over atoms
      S2G_CUBLAS(cublasDgemmStridedBatched(h, CUBLAS_OP_N, CUBLAS_OP_N, no, maxa * m, no, &one,
                                           mf.PooA.get(), no, (long long)no * no, Zt, no,
                                           (long long)no * maxa * m, &zero, T, no,
                                           (long long)no * maxa * m, N));
      S2G_LAUNCH(k_mf_from_atom_major, grid, 256, 0, s, Tacc, T, N, maxa, no, m, cJ, 0);
      have = true;
    }
    if (cX != 0.0) {
      S2G_CUDA(cudaMemsetAsync(box, 0, sizeof(double) * nov * m, s));
      S2G_LAUNCH(k_mf_scatter, grid, 256, 0, s, box, X, mf.ci, mf.ca, nci, no, nov, m, 0);
      // Z2 = CoP (rows x no) * Xb (no x nv*m)
      mf_dgemm(h, CUBLAS_OP_N, CUBLAS_OP_N, rows, nv * m, no, 1.0, mf.CoP.get(), rows, box, no,
               0.0, Z, rows);
      S2G_LAUNCH(k_mf_to_atom_major, grid, 256, 0, s, Zt, Z, N, maxa, nv, m);
      // U_A = P^A_ov (no x nv) * Z2t_A (nv x maxa*m)
      S2G_CUBLAS(cublasDgemmStridedBatched(h, CUBLAS_OP_N, CUBLAS_OP_N, no, maxa * m, nv, &one,
                                           mf.PovA.get(), no, (long long)no * nv, Zt, nv,
                                           (long long)nv * maxa * m, &zero, T, no,
                                           (long long)no * maxa * m, N));
      S2G_LAUNCH(k_mf_from_atom_major, grid, 256, 0, s, Tacc, T, N, maxa, no, m, cX,
                 have ? 1 : 0);
    }
    // box[a + nv*(i + no*r)] = CvP^T (nv x rows) * Tacc (rows x no*m)
    mf_dgemm(h, CUBLAS_OP_T, CUBLAS_OP_N, nv, no * m, rows, 1.0, mf.CvP.get(), rows, Tacc, rows,
             0.0, box, nv);
    S2G_LAUNCH(k_mf_gather, grid, 256, 0, s, out, box, mf.ci, mf.ca, nci, no, nv, m);
  }
  if (diag) S2G_LAUNCH(k_add_diag, grid, 256, 0, s, out, X, diag, nci, m);
}

}  // namespace std2g
