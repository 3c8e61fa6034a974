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
#include "dgemm.cuh"

namespace std2g {

// Leading dimensions are padded to multiples of 8 elements so that every GEMM
// operand is 16-byte aligned (required for the tensor-core GEMM paths).
inline int ld8(int64_t x) { return (int)((x + 7) / 8 * 8); }

// box[o] = X[u + nci*r] at the CSF's (j,b); layout 0: o = j + ldo*b + vs*r
// (ldo >= no), layout 1: o = b + ldv*j + vs*r (ldv >= nv).  The caller zeroes
// the box first.
template <typename T>
__global__ void k_mf_scatter(T *__restrict__ box, const double *__restrict__ X,
                             const int *__restrict__ ci, const int *__restrict__ ca, int nci,
                             int ld, int64_t vs, int m, int layout) {
  int64_t total = (int64_t)nci * m;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    int r = (int)(t / nci), u = (int)(t - (int64_t)r * nci);
    int64_t o = layout == 0 ? ci[u] + (int64_t)ld * ca[u] : ca[u] + (int64_t)ld * ci[u];
    box[o + vs * r] = (T)X[t];
  }
}

// out[u + nci*r] += box[a_u + ldv*(i_u + no*r)]
template <typename T>
__global__ void k_mf_gather(double *__restrict__ out, const T *__restrict__ box,
                            const int *__restrict__ ci, const int *__restrict__ ca, int nci, int no,
                            int ldv, int m) {
  int64_t total = (int64_t)nci * m;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    int r = (int)(t / nci), u = (int)(t - (int64_t)r * nci);
    out[t] += (double)box[ca[u] + (int64_t)ldv * (ci[u] + (int64_t)no * r)];
  }
}

// Z is rows x (ncol*m) with leading dimension ldz, row R = A*maxa+s and column
// c + ncol*r; Zt[A*ldt*maxa*m + c + ldt*(s + maxa*r)].  32x32 tiles through
// shared memory (reads and writes coalesced); grid (rows/32, ncol/32, m),
// block 32x8.
template <typename T>
__global__ void k_mf_to_atom_major(T *__restrict__ Zt, const T *__restrict__ Z, int N, int maxa,
                                   int ncol, int m, int ldz, int ldt) {
  __shared__ T tile[32][33];
  const int rows = N * maxa;
  const int R0 = blockIdx.x * 32, c0 = blockIdx.y * 32, r = blockIdx.z;
  const int tx = threadIdx.x;
  for (int ty = threadIdx.y; ty < 32; ty += 8) {
    int R = R0 + tx, c = c0 + ty;
    if (R < rows && c < ncol) tile[ty][tx] = Z[R + (int64_t)ldz * (c + (int64_t)ncol * r)];
  }
  __syncthreads();
  for (int ty = threadIdx.y; ty < 32; ty += 8) {
    int R = R0 + ty, c = c0 + tx;
    if (R < rows && c < ncol) {
      int A = R / maxa, s = R - A * maxa;
      Zt[(int64_t)A * ldt * maxa * m + c + (int64_t)ldt * (s + (int64_t)maxa * r)] = tile[tx][ty];
    }
  }
}

// inverse of k_mf_to_atom_major, scaled by f, optionally accumulating
template <typename TT>
__global__ void k_mf_from_atom_major(TT *__restrict__ Z, const TT *__restrict__ T, int N,
                                     int maxa, int ncol, int m, int ldz, int ldt, double f,
                                     int accumulate) {
  __shared__ TT tile[32][33];
  const int rows = N * maxa;
  const int R0 = blockIdx.x * 32, c0 = blockIdx.y * 32, r = blockIdx.z;
  const int tx = threadIdx.x;
  for (int ty = threadIdx.y; ty < 32; ty += 8) {
    int R = R0 + ty, c = c0 + tx;
    if (R < rows && c < ncol) {
      int A = R / maxa, s = R - A * maxa;
      tile[ty][tx] = T[(int64_t)A * ldt * maxa * m + c + (int64_t)ldt * (s + (int64_t)maxa * r)];
    }
  }
  __syncthreads();
  for (int ty = threadIdx.y; ty < 32; ty += 8) {
    int R = R0 + tx, c = c0 + ty;
    if (R < rows && c < ncol) {
      int64_t o = R + (int64_t)ldz * (c + (int64_t)ncol * r);
      TT v = (TT)(f * (double)tile[tx][ty]);
      Z[o] = accumulate ? (TT)(Z[o] + v) : v;
    }
  }
}

// dst[A*ld1*n2 + i + ld1*b] = src[A + N*(i*n2 + b)]: [pair (i,b)][atom] -> per atom
// an n1 x n2 column-major matrix with leading dimension ld1.  Tiled; grid
// (N/32, <=65535), block 32x8.
template <typename T>
__global__ void k_pair_to_atom_major(T *__restrict__ dst, const double *__restrict__ src, int N,
                                     int n1, int n2, int ld1) {
  __shared__ double tile[32][33];
  const int64_t np = (int64_t)n1 * n2;
  const int A0 = blockIdx.x * 32;
  const int tx = threadIdx.x;
  for (int64_t p0 = (int64_t)blockIdx.y * 32; p0 < np; p0 += (int64_t)gridDim.y * 32) {
    // p0: pair index i + n1*b of the tile's first column
    for (int ty = threadIdx.y; ty < 32; ty += 8) {
      int64_t pp = p0 + ty;
      int A = A0 + tx;
      if (A < N && pp < np) {
        int64_t b = pp / n1, i = pp - b * n1;
        tile[ty][tx] = src[A + (int64_t)N * (i * n2 + b)];
      }
    }
    __syncthreads();
    for (int ty = threadIdx.y; ty < 32; ty += 8) {
      int A = A0 + ty;
      int64_t pp = p0 + tx;
      if (A < N && pp < np) {
        int64_t b = pp / n1, i = pp - b * n1;
        dst[(int64_t)A * ld1 * n2 + i + (int64_t)ld1 * b] = (T)tile[tx][ty];
      }
    }
    __syncthreads();
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

// padded AO rows: out[(A*maxa+s) + ldr*c] = C[slot_ao[A*maxa+s] + nao*(c0+c)] or 0
// for rows < ldr (rows beyond N*maxa are zero)
template <typename T>
__global__ void k_mf_pad_rows(T *__restrict__ out, const double *__restrict__ C, int nao,
                              const int *__restrict__ slot_ao, int rows, int ldr, int c0,
                              int ncol) {
  int64_t total = (int64_t)ldr * ncol;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    int c = (int)(t / ldr), r = (int)(t - (int64_t)c * ldr);
    int k = r < rows ? slot_ao[r] : -1;
    out[t] = k >= 0 ? (T)C[k + (int64_t)nao * (c0 + c)] : (T)0;
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

// y[u + ldy*r] = (T)x[u + n*r]
template <typename T>
__global__ void k_mf_convert_ld(T *__restrict__ y, int ldy, const double *__restrict__ x, int n,
                                int m) {
  int64_t total = (int64_t)n * m;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    int r = (int)(t / n), u = (int)(t - (int64_t)r * n);
    y[u + (int64_t)ldy * r] = (T)x[t];
  }
}

// out[u + n*r] += (double)y[u + ldy*r]
template <typename T>
__global__ void k_mf_accum_ld(double *__restrict__ out, const T *__restrict__ y, int ldy, int n,
                              int m) {
  int64_t total = (int64_t)n * m;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    int r = (int)(t / n), u = (int)(t - (int64_t)r * n);
    out[t] += (double)y[u + (int64_t)ldy * r];
  }
}

// y = (T)x
template <typename T>
__global__ void k_mf_convert(T *__restrict__ y, const double *__restrict__ x, int64_t n) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
       t += (int64_t)gridDim.x * blockDim.x)
    y[t] = (T)x[t];
}

// Operands and work arrays of one storage type: double (FP64 form) or float
// (mixed form: FP32 GEMMs executed on the tensor cores as split-BF16 products,
// cuBLAS's BF16x9 FP32 emulation, FP32 accumulation).
template <typename T>
struct MatFreeOps {
  DBuf<T> CvP, CoP, PooA, PovA, Qs, Ps;
  DBuf<T> box, Z, Zt, Tm, Tacc, G, Xc, Yc;
};

struct MatFree {
  int N = 0, maxa = 0, no = 0, nv = 0, nci = 0, nao = 0;
  bool f32 = false;
  Dgemm *dg = nullptr;   // FP64 products (dgemm.cuh); FP32 ones go to cuBLAS
  DBuf<double> dA;
  const int *ci = nullptr, *ca = nullptr;
  MatFreeOps<double> d;
  MatFreeOps<float> f;
};

inline void mf_gemm(MatFree &mf, cublasHandle_t, cudaStream_t s, cublasOperation_t ta,
                    cublasOperation_t tb, int m, int n, int k, double alpha, const double *A,
                    int lda, const double *B, int ldb, double beta, double *C, int ldc) {
  if (m == 0 || n == 0) return;
  mf.dg->run(s, ta != CUBLAS_OP_N, tb != CUBLAS_OP_N, m, n, k, alpha, A, lda, 0, B, ldb, 0, beta,
             C, ldc, 0);
}

inline void mf_gemm(MatFree &, cublasHandle_t h, cudaStream_t, cublasOperation_t ta,
                    cublasOperation_t tb, int m, int n, int k, double alpha, const float *A,
                    int lda, const float *B, int ldb, double beta, float *C, int ldc) {
  if (m == 0 || n == 0) return;
  float a = (float)alpha, b = (float)beta;
  S2G_CUBLAS(cublasGemmEx(h, ta, tb, m, n, k, &a, A, CUDA_R_32F, lda, B, CUDA_R_32F, ldb, &b, C,
                          CUDA_R_32F, ldc, CUBLAS_COMPUTE_32F_EMULATED_16BFX9,
                          CUBLAS_GEMM_DEFAULT));
}

inline void mf_gemm_batched(MatFree &mf, cublasHandle_t, cudaStream_t s, int m, int n, int k,
                            const double *A, int lda, long long sa, const double *B, int ldb,
                            long long sb, double *C, int ldc, long long sc, int batch) {
  mf.dg->run(s, false, false, m, n, k, 1.0, A, lda, sa, B, ldb, sb, 0.0, C, ldc, sc, batch);
}

inline void mf_gemm_batched(MatFree &, cublasHandle_t h, cudaStream_t, int m, int n, int k,
                            const float *A, int lda, long long sa, const float *B, int ldb,
                            long long sb, float *C, int ldc, long long sc, int batch) {
  const float one = 1.f, zero = 0.f;
  S2G_CUBLAS(cublasGemmStridedBatchedEx(h, CUBLAS_OP_N, CUBLAS_OP_N, m, n, k, &one, A, CUDA_R_32F,
                                        lda, sa, B, CUDA_R_32F, ldb, sb, &zero, C, CUDA_R_32F, ldc,
                                        sc, batch, CUBLAS_COMPUTE_32F_EMULATED_16BFX9,
                                        CUBLAS_GEMM_DEFAULT));
}

// Set up the operands from the FP64 arrays of the solve (once per solve).
template <typename T>
inline void mf_setup_ops(MatFree &mf, MatFreeOps<T> &o, cudaStream_t s, const double *Clow,
                         const int *slot_ao, const double *Poo, const double *Pia,
                         const double *Qs, const double *Ps, bool need_ov) {
  const int N = mf.N, rows = N * mf.maxa, no = mf.no, nv = mf.nv, nao = mf.nao, nci = mf.nci;
  const int lr = ld8(rows), lo = ld8(no);
  const int grid = 148 * 16;
  S2G_LAUNCH(k_mf_pad_rows<T>, grid, 256, 0, s, o.CvP.ensure((size_t)lr * nv), Clow, nao, slot_ao,
             rows, lr, no, nv);
  S2G_LAUNCH(k_mf_pad_rows<T>, grid, 256, 0, s, o.CoP.ensure((size_t)lr * no), Clow, nao, slot_ao,
             rows, lr, 0, no);
  const dim3 tb(32, 8);
  S2G_LAUNCH(k_pair_to_atom_major<T>,
             dim3((unsigned)div_up(N, 32), (unsigned)std::min<int64_t>(div_up((int64_t)no * no, 32), 65535)),
             tb, 0, s, o.PooA.ensure((size_t)N * lo * no), Poo, N, no, no, lo);
  if (need_ov)
    S2G_LAUNCH(k_pair_to_atom_major<T>,
               dim3((unsigned)div_up(N, 32), (unsigned)std::min<int64_t>(div_up((int64_t)no * nv, 32), 65535)),
               tb, 0, s, o.PovA.ensure((size_t)N * lo * nv), Pia, N, no, nv, lo);
  S2G_LAUNCH(k_mf_convert<T>, grid, 256, 0, s, o.Qs.ensure((size_t)N * nci), Qs,
             (int64_t)N * nci);
  S2G_LAUNCH(k_mf_convert<T>, grid, 256, 0, s, o.Ps.ensure((size_t)N * nci), Ps,
             (int64_t)N * nci);
}

// out (nci x m, FP64) = cK (K X) + cJ (J X) + cX (Kx X) + diag o X  (diag may be NULL),
// products formed in storage type T.
template <typename T>
inline void mf_apply_t(MatFree &mf, MatFreeOps<T> &o, cublasHandle_t h, cudaStream_t s,
                       const double *X, int m, double *out, double cK, double cJ, double cX,
                       const double *diag) {
  const int N = mf.N, maxa = mf.maxa, no = mf.no, nv = mf.nv, nci = mf.nci;
  const int rows = N * maxa, lr = ld8(rows), lo = ld8(no), lv = ld8(nv), lc = ld8(nci);
  const int grid = 148 * 8;
  S2G_CUDA(cudaMemsetAsync(out, 0, sizeof(double) * nci * m, s));
  if (cK != 0.0) {
    // K part: G = Q_S X (N x m); out += cK P_S^T G
    T *Xc = o.Xc.ensure((size_t)lc * m), *Yc = o.Yc.ensure((size_t)lc * m);
    T *G = o.G.ensure((size_t)N * m);
    S2G_LAUNCH(k_mf_convert_ld<T>, grid, 256, 0, s, Xc, lc, X, nci, m);
    mf_gemm(mf, h, s, CUBLAS_OP_N, CUBLAS_OP_N, N, m, nci, 1.0, o.Qs.get(), N, Xc, lc, 0.0, G, N);
    mf_gemm(mf, h, s, CUBLAS_OP_T, CUBLAS_OP_N, nci, m, N, cK, o.Ps.get(), N, G, N, 0.0, Yc, lc);
    S2G_LAUNCH(k_mf_accum_ld<T>, grid, 256, 0, s, out, Yc, lc, nci, m);
  }
  if (cJ != 0.0 || cX != 0.0) {
    const int64_t boxsz = std::max((int64_t)lv * no, (int64_t)lo * nv) * m;
    T *box = o.box.ensure((size_t)boxsz);
    T *Z = o.Z.ensure((size_t)lr * std::max(no, nv) * m);
    T *Zt = o.Zt.ensure((size_t)N * maxa * std::max(lo, lv) * m);
    T *Tm = o.Tm.ensure((size_t)N * maxa * lo * m);
    T *Tacc = o.Tacc.ensure((size_t)lr * no * m);
    auto tgrid = [&](int ncol) {
      return dim3((unsigned)div_up(rows, 32), (unsigned)div_up(ncol, 32), (unsigned)m);
    };
    bool have = false;
    if (cJ != 0.0) {
      S2G_CUDA(cudaMemsetAsync(box, 0, sizeof(T) * boxsz, s));
      // XbT[b + lv*(j + no*r)]
      S2G_LAUNCH(k_mf_scatter<T>, grid, 256, 0, s, box, X, mf.ci, mf.ca, nci, lv,
                 (int64_t)lv * no, m, 1);
      // Z = CvP (rows x nv) * XbT (nv x no*m)
      mf_gemm(mf, h, s, CUBLAS_OP_N, CUBLAS_OP_N, rows, no * m, nv, 1.0, o.CvP.get(), lr, box, lv, 0.0,
              Z, lr);
      S2G_LAUNCH(k_mf_to_atom_major<T>, tgrid(no), dim3(32, 8), 0, s, Zt, Z, N, maxa, no, m, lr,
                 lo);
      // T_A = P^A_oo (no x no) * Zt_A (no x maxa*m), batched over atoms
      mf_gemm_batched(mf, h, s, no, maxa * m, no, o.PooA.get(), lo, (long long)lo * no, Zt, lo,
                      (long long)lo * maxa * m, Tm, lo, (long long)lo * maxa * m, N);
      S2G_LAUNCH(k_mf_from_atom_major<T>, tgrid(no), dim3(32, 8), 0, s, Tacc, Tm, N, maxa, no, m,
                 lr, lo, cJ, 0);
      have = true;
    }
    if (cX != 0.0) {
      S2G_CUDA(cudaMemsetAsync(box, 0, sizeof(T) * boxsz, s));
      // Xb[j + lo*b + lo*nv*r]
      S2G_LAUNCH(k_mf_scatter<T>, grid, 256, 0, s, box, X, mf.ci, mf.ca, nci, lo,
                 (int64_t)lo * nv, m, 0);
      // Z2 = CoP (rows x no) * Xb (no x nv*m)
      mf_gemm(mf, h, s, CUBLAS_OP_N, CUBLAS_OP_N, rows, nv * m, no, 1.0, o.CoP.get(), lr, box, lo, 0.0,
              Z, lr);
      S2G_LAUNCH(k_mf_to_atom_major<T>, tgrid(nv), dim3(32, 8), 0, s, Zt, Z, N, maxa, nv, m, lr,
                 lv);
      // U_A = P^A_ov (no x nv) * Z2t_A (nv x maxa*m)
      mf_gemm_batched(mf, h, s, no, maxa * m, nv, o.PovA.get(), lo, (long long)lo * nv, Zt, lv,
                      (long long)lv * maxa * m, Tm, lo, (long long)lo * maxa * m, N);
      S2G_LAUNCH(k_mf_from_atom_major<T>, tgrid(no), dim3(32, 8), 0, s, Tacc, Tm, N, maxa, no, m,
                 lr, lo, cX, have ? 1 : 0);
    }
    // box[a + lv*(i + no*r)] = CvP^T (nv x rows) * Tacc (rows x no*m)
    mf_gemm(mf, h, s, CUBLAS_OP_T, CUBLAS_OP_N, nv, no * m, rows, 1.0, o.CvP.get(), lr, Tacc, lr, 0.0,
            box, lv);
    S2G_LAUNCH(k_mf_gather<T>, grid, 256, 0, s, out, box, mf.ci, mf.ca, nci, no, lv, m);
  }
  if (diag) S2G_LAUNCH(k_add_diag, grid, 256, 0, s, out, X, diag, nci, m);
}

inline void mf_apply(MatFree &mf, cublasHandle_t h, cudaStream_t s, const double *X, int m,
                     double *out, double cK, double cJ, double cX, const double *diag) {
  if (mf.f32)
    mf_apply_t<float>(mf, mf.f, h, s, X, m, out, cK, cJ, cX, diag);
  else
    mf_apply_t<double>(mf, mf.d, h, s, X, m, out, cK, cJ, cX, diag);
}

}  // namespace std2g
