// Matrix-free J X on the tensor cores (mixed form of the Davidson products).
//
// Same factorisation as matfree.cuh (J X = C_v^T P^A_oo (C_v X^T), per atom A),
// but every GEMM is the split-BF16 tcgen05 contraction of tc_gemm.cuh:
//   G1: Z[(j,r), R]      = sum_b  XbT[(j,r), b] * Cv[R, b]        (one launch)
//   G2: T_A[(s,r), i]    = sum_j  Zt_A[(s,r), j] * P^A[i, j]      (batched over atoms)
//   G3: Y[(i,r), a]      = sum_R  Tt[(i,r), R] * Cv[R, a]^T       (one launch)
// R runs over the padded AO slots (atom A, slot s), j/i over occupied and a/b
// over virtual MOs of the active window, r over the vectors of the block.  The
// layout changes between the GEMMs write the next K-major BF16 hi/lo operand
// directly (tiled transposes).  The K part (p_u . sum_v q_v X_v) is two thin
// FP64 GEMMs.  The exchange-type products K_x X ((ib|ja), the velocity
// correction and A +- B) follow the same pattern with C_o and P^A_ov:
//   G1x: Z2[(b,r), R] = sum_j X[(b,r), j] Co[R, j],
//   G2x: U_A[(s,r), i] = sum_b Z2_A[(s,r), b] P^A_ov[i, b],
// and U joins T before G3.
#pragma once

#include <cuda_bf16.h>

#include "common.cuh"
#include "tc_gemm.cuh"

namespace std2g {

inline int ld64(int64_t x) { return (int)((x + 63) / 64 * 64); }
inline int ld4(int64_t x) { return (int)((x + 3) / 4 * 4); }

__device__ __forceinline__ void split_store(__nv_bfloat16 *hi, __nv_bfloat16 *lo, int64_t o,
                                            double x) {
  __nv_bfloat16 h = __double2bfloat16(x);
  hi[o] = h;
  lo[o] = __double2bfloat16(x - (double)__bfloat162float(h));
}

// Loewdin MO operands: mode 0: out[R*Kp + b] = Cv[R, b] (R < nrow = AO slots);
// mode 1: out[a*Kp + R] = Cv[R, a] (a < nrow = nv); mode 2: out[R*Kp + j] =
// Co[R, j] (R < nrow = AO slots, j < no).  Zero beyond the data.
__global__ void k_tcs_clow(__nv_bfloat16 *__restrict__ hi, __nv_bfloat16 *__restrict__ lo,
                           const double *__restrict__ Clow, int nao, const int *__restrict__ slot,
                           int rows, int no, int nv, int nrow, int Kp, int mode) {
  int64_t total = (int64_t)nrow * Kp;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    int row = (int)(t / Kp), k = (int)(t - (int64_t)row * Kp);
    int R = mode == 1 ? k : row, c = mode == 1 ? row : k;
    double x = 0.0;
    const int ncol = mode == 2 ? no : nv, col0 = mode == 2 ? 0 : no;
    if (R < rows && c < ncol) {
      int ao = slot[R];
      if (ao >= 0) x = Clow[ao + (int64_t)nao * (col0 + c)];
    }
    split_store(hi, lo, t, x);
  }
}

// Atom-major rows of a pair tensor: out[A*n1*K2 + i*K2 + j] = P[A + N*(i*n2 + j)]
// (i < n1, j < n2; P^A_oo with n1 = n2 = no, P^A_ov with n1 = no, n2 = nv;
// padding columns must be zeroed by the caller).  Tiled over (atoms, pairs).
__global__ void k_tcs_pairs(__nv_bfloat16 *__restrict__ hi, __nv_bfloat16 *__restrict__ lo,
                            const double *__restrict__ P, int N, int n1, int n2, int K2) {
  __shared__ double tile[32][33];
  const int64_t np = (int64_t)n1 * n2;
  const int A0 = blockIdx.x * 32, tx = threadIdx.x;
  for (int64_t p0 = (int64_t)blockIdx.y * 32; p0 < np; p0 += (int64_t)gridDim.y * 32) {
    for (int ty = threadIdx.y; ty < 32; ty += 8) {
      int64_t p = p0 + ty;
      int A = A0 + tx;
      if (A < N && p < np) tile[ty][tx] = P[A + (int64_t)N * p];
    }
    __syncthreads();
    for (int ty = threadIdx.y; ty < 32; ty += 8) {
      int A = A0 + ty;
      int64_t p = p0 + tx;
      if (A < N && p < np) {
        int64_t i = p / n2, j = p - i * n2;
        split_store(hi, lo, (int64_t)A * n1 * K2 + i * K2 + j, tile[tx][ty]);
      }
    }
    __syncthreads();
  }
}

// XbT[(j + no*r)*Kv + b] = X[u + nci*r] for the CSF u = (j,b)  (box zeroed first)
__global__ void k_tcs_scatter(__nv_bfloat16 *__restrict__ hi, __nv_bfloat16 *__restrict__ lo,
                              const double *__restrict__ X, const int *__restrict__ ci,
                              const int *__restrict__ ca, int nci, int no, int Kv, int m) {
  int64_t total = (int64_t)nci * m;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    int r = (int)(t / nci), u = (int)(t - (int64_t)r * nci);
    split_store(hi, lo, ((int64_t)ci[u] + (int64_t)no * r) * Kv + ca[u], X[t]);
  }
}

// Xb[(b + nv*r)*Ko + j] = X[u + nci*r] for the CSF u = (j,b)  (box zeroed first)
__global__ void k_tcs_scatter_v(__nv_bfloat16 *__restrict__ hi, __nv_bfloat16 *__restrict__ lo,
                                const double *__restrict__ X, const int *__restrict__ ci,
                                const int *__restrict__ ca, int nci, int nv, int Ko, int m) {
  int64_t total = (int64_t)nci * m;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    int r = (int)(t / nci), u = (int)(t - (int64_t)r * nci);
    split_store(hi, lo, ((int64_t)ca[u] + (int64_t)nv * r) * Ko + ci[u], X[t]);
  }
}

// Z[(j + no*r)*ldR + R] -> Zt[A*(maxa*m*Ko) + (s + maxa*r)*Ko + j], R = A*maxa + s.
// grid (no/32, rows/32, m), block 32x8; padding columns j >= no zeroed by the caller.
__global__ void k_tcs_to_atom(__nv_bfloat16 *__restrict__ hi, __nv_bfloat16 *__restrict__ lo,
                              const float *__restrict__ Z, int ldR, int rows, int maxa, int no,
                              int Ko, int m) {
  __shared__ float tile[32][33];
  const int j0 = blockIdx.x * 32, R0 = blockIdx.y * 32, r = blockIdx.z, tx = threadIdx.x;
  for (int ty = threadIdx.y; ty < 32; ty += 8) {
    int j = j0 + ty, R = R0 + tx;
    if (j < no && R < rows) tile[ty][tx] = Z[((int64_t)j + (int64_t)no * r) * ldR + R];
  }
  __syncthreads();
  for (int ty = threadIdx.y; ty < 32; ty += 8) {
    int R = R0 + ty, j = j0 + tx;
    if (j < no && R < rows) {
      int A = R / maxa, s = R - A * maxa;
      int64_t o = (int64_t)A * maxa * m * Ko + ((int64_t)s + (int64_t)maxa * r) * Ko + j;
      split_store(hi, lo, o, (double)tile[tx][ty]);
    }
  }
}

// f T_A + fU U_A, both [(s + maxa*r)*ldo + i] per atom (stride bst, either
// may be NULL) -> Tt[(i + no*r)*KR + R].
// grid (no/32, rows/32, m), block 32x8; padding columns R >= rows zeroed by the caller.
__global__ void k_tcs_from_atom(__nv_bfloat16 *__restrict__ hi, __nv_bfloat16 *__restrict__ lo,
                                const float *__restrict__ T, const float *__restrict__ U,
                                int64_t bst, int ldo, int rows, int maxa, int no, int KR, int m,
                                double f, double fU) {
  __shared__ float tile[32][33];
  const int i0 = blockIdx.x * 32, R0 = blockIdx.y * 32, r = blockIdx.z, tx = threadIdx.x;
  for (int ty = threadIdx.y; ty < 32; ty += 8) {
    int R = R0 + ty, i = i0 + tx;
    if (i < no && R < rows) {
      int A = R / maxa, s = R - A * maxa;
      const int64_t o = (int64_t)A * bst + ((int64_t)s + (int64_t)maxa * r) * ldo + i;
      float v = 0.f;
      if (T) v += (float)f * T[o];
      if (U) v += (float)fU * U[o];
      tile[ty][tx] = v;
    }
  }
  __syncthreads();
  for (int ty = threadIdx.y; ty < 32; ty += 8) {
    int i = i0 + ty, R = R0 + tx;
    if (i < no && R < rows)
      split_store(hi, lo, ((int64_t)i + (int64_t)no * r) * KR + R, (double)tile[tx][ty]);
  }
}

// out[u + nci*r] += Y[(i_u + no*r)*ldv + a_u]
__global__ void k_tcs_gather(double *__restrict__ out, const float *__restrict__ Y, int ldv,
                             const int *__restrict__ ci, const int *__restrict__ ca, int nci,
                             int no, int m) {
  int64_t total = (int64_t)nci * m;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    int r = (int)(t / nci), u = (int)(t - (int64_t)r * nci);
    out[t] += (double)Y[((int64_t)ci[u] + (int64_t)no * r) * ldv + ca[u]];
  }
}

// A second stream with its own cuBLAS handle, on which the FP64 exchange
// part of the product runs concurrently with the tensor-core Coulomb part.
struct SideStream {
  cudaStream_t s = nullptr;
  cublasHandle_t h = nullptr;
  Dgemm dg;   // FP64 products on this stream (own split-K workspace)
  bool lib_fp64 = false;   // those products through cuBLAS (STD2G_FLAG_LIBRARY_FP64)
  cudaEvent_t fork = nullptr, join = nullptr;
  void init() {
    if (s) return;
    S2G_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    S2G_CUBLAS(cublasCreate(&h));
    S2G_CUBLAS(cublasSetStream(h, s));
    if (lib_fp64) dg.lib = h;
    S2G_CUDA(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
    S2G_CUDA(cudaEventCreateWithFlags(&join, cudaEventDisableTiming));
  }
  ~SideStream() {
    if (h) cublasDestroy(h);
    if (fork) cudaEventDestroy(fork);
    if (join) cudaEventDestroy(join);
    if (s) cudaStreamDestroy(s);
  }
};

struct MatFreeTc {
  int N = 0, maxa = 0, no = 0, nv = 0, nci = 0, rows = 0;
  int Kv = 0, Ko = 0, KR = 0;
  const double *Qs = nullptr, *Ps = nullptr;   // FP64 [csf][atom] charges for the K part
  const int *ci = nullptr, *ca = nullptr;
  TcGemm tc;
  DBuf<__nv_bfloat16> cvt_h, cvt_l, cv2_h, cv2_l, poo_h, poo_l;
  DBuf<__nv_bfloat16> xb_h, xb_l, zt_h, zt_l, tt_h, tt_l;
  DBuf<float> Z, T, Y;
  // exchange chain (K_x X, the (ib|ja) products): C_o rows, P^A_ov rows
  bool has_x = false;
  DBuf<__nv_bfloat16> cot_h, cot_l, pov_h, pov_l, xv_h, xv_l, z2t_h, z2t_l;
  DBuf<float> Z2, U;
  DBuf<double> G, Kt;
  SideStream side;
};

// Operands fixed for the solve: Cv in both K-major orientations, P^A_oo rows.
inline void mftc_setup(MatFreeTc &w, cudaStream_t s, const double *Clow, int nao,
                       const int *slot, const double *Poo, const double *Pia = nullptr) {
  w.rows = w.N * w.maxa;
  w.Kv = ld64(w.nv);
  w.Ko = ld64(w.no);
  w.KR = ld64(w.rows);
  const int g = 148 * 16;
  S2G_LAUNCH(k_tcs_clow, g, 256, 0, s, w.cvt_h.ensure((size_t)w.rows * w.Kv),
             w.cvt_l.ensure((size_t)w.rows * w.Kv), Clow, nao, slot, w.rows, w.no, w.nv, w.rows,
             w.Kv, 0);
  S2G_LAUNCH(k_tcs_clow, g, 256, 0, s, w.cv2_h.ensure((size_t)w.nv * w.KR),
             w.cv2_l.ensure((size_t)w.nv * w.KR), Clow, nao, slot, w.rows, w.no, w.nv, w.nv, w.KR,
             1);
  const size_t np = (size_t)w.N * w.no * w.Ko;
  __nv_bfloat16 *ph = w.poo_h.ensure(np), *pl = w.poo_l.ensure(np);
  S2G_CUDA(cudaMemsetAsync(ph, 0, np * 2, s));
  S2G_CUDA(cudaMemsetAsync(pl, 0, np * 2, s));
  S2G_LAUNCH(k_tcs_pairs,
             dim3((unsigned)div_up(w.N, 32),
                  (unsigned)std::min<int64_t>(div_up((int64_t)w.no * w.no, 32), 65535)),
             dim3(32, 8), 0, s, ph, pl, Poo, w.N, w.no, w.no, w.Ko);
  w.has_x = Pia != nullptr;
  if (w.has_x) {
    S2G_LAUNCH(k_tcs_clow, g, 256, 0, s, w.cot_h.ensure((size_t)w.rows * w.Ko),
               w.cot_l.ensure((size_t)w.rows * w.Ko), Clow, nao, slot, w.rows, w.no, w.nv, w.rows,
               w.Ko, 2);
    const size_t nq = (size_t)w.N * w.no * w.Kv;
    __nv_bfloat16 *qh = w.pov_h.ensure(nq), *ql = w.pov_l.ensure(nq);
    S2G_CUDA(cudaMemsetAsync(qh, 0, nq * 2, s));
    S2G_CUDA(cudaMemsetAsync(ql, 0, nq * 2, s));
    S2G_LAUNCH(k_tcs_pairs,
               dim3((unsigned)div_up(w.N, 32),
                    (unsigned)std::min<int64_t>(div_up((int64_t)w.no * w.nv, 32), 65535)),
               dim3(32, 8), 0, s, qh, ql, Pia, w.N, w.no, w.nv, w.Kv);
  }
}

// out (nci x m, FP64) = cK (K X) + cJ (J X) + cX (K_x X) + diag o X
// (cX != 0 needs the exchange operands of mftc_setup(..., Pia))
inline void mftc_apply(MatFreeTc &w, cublasHandle_t h, cudaStream_t s, const double *X, int m,
                       double *out, double cK, double cJ, double cX, const double *diag) {
  const int N = w.N, no = w.no, nv = w.nv, nci = w.nci, rows = w.rows, maxa = w.maxa;
  const int g = 148 * 8;
  if (cX != 0.0 && !w.has_x) throw Error{STD2G_ESTATE, "mftc_apply: exchange operands not set up"};
  // K part, out = cK Ps^T (Qs X), in FP64 on the side stream
  const bool side = cK != 0.0;
  if (side) {
    w.side.init();
    S2G_CUDA(cudaEventRecord(w.side.fork, s));
    S2G_CUDA(cudaStreamWaitEvent(w.side.s, w.side.fork, 0));
    double *G = w.G.ensure((size_t)N * m);
    const double one = 1.0, zero = 0.0, ck = cK;
    w.side.dg.gemm(w.side.s, CUBLAS_OP_N, CUBLAS_OP_N, N, m, nci, &one, w.Qs, N, X, nci, &zero,
                   G, N);
    w.side.dg.gemm(w.side.s, CUBLAS_OP_T, CUBLAS_OP_N, nci, m, N, &ck, w.Ps, N, G, N, &zero, out,
                   nci);
    S2G_CUDA(cudaEventRecord(w.side.join, w.side.s));
  } else {
    S2G_CUDA(cudaMemsetAsync(out, 0, sizeof(double) * nci * m, s));
  }
  (void)h;
  if (cJ != 0.0 || cX != 0.0) {
    const int64_t mo = (int64_t)no * m, mz = (int64_t)maxa * m;
    const int ldR = ld4(rows), ldo = ld4(no), ldv = ld4(nv);
    const int64_t bst = mz * ldo;
    const dim3 tb(32, 8);
    float *T = nullptr, *U = nullptr;
    if (cJ != 0.0) {
      // G1: Z[(j,r), R] = sum_b X_jb^r Cv[R, b]
      __nv_bfloat16 *xh = w.xb_h.ensure((size_t)mo * w.Kv), *xl = w.xb_l.ensure((size_t)mo * w.Kv);
      S2G_CUDA(cudaMemsetAsync(xh, 0, (size_t)mo * w.Kv * 2, s));
      S2G_CUDA(cudaMemsetAsync(xl, 0, (size_t)mo * w.Kv * 2, s));
      S2G_LAUNCH(k_tcs_scatter, g, 256, 0, s, xh, xl, X, w.ci, w.ca, nci, no, w.Kv, m);
      float *Z = w.Z.ensure((size_t)mo * ldR);
      w.tc.run(s, xh, xl, w.cvt_h.get(), w.cvt_l.get(), (int)mo, rows, w.Kv, Z, ldR,
               2.0 * mo * rows * nv, 1, false, 0, false);
      // G2: T_A[(s,r), i] = sum_j Z_A[(s,r), j] P^A_oo[i, j], batched over atoms
      __nv_bfloat16 *zh = w.zt_h.ensure((size_t)N * mz * w.Ko),
                    *zl = w.zt_l.ensure((size_t)N * mz * w.Ko);
      S2G_CUDA(cudaMemsetAsync(zh, 0, (size_t)N * mz * w.Ko * 2, s));
      S2G_CUDA(cudaMemsetAsync(zl, 0, (size_t)N * mz * w.Ko * 2, s));
      S2G_LAUNCH(k_tcs_to_atom, dim3((unsigned)div_up(no, 32), (unsigned)div_up(rows, 32), (unsigned)m),
                 tb, 0, s, zh, zl, Z, ldR, rows, maxa, no, w.Ko, m);
      T = w.T.ensure((size_t)N * bst);
      w.tc.run(s, zh, zl, w.poo_h.get(), w.poo_l.get(), (int)mz, no, w.Ko, T, ldo,
               2.0 * mz * no * no, N, true, bst, false);
    }
    if (cX != 0.0) {
      // G1x: Z2[(b,r), R] = sum_j X_jb^r Co[R, j]
      const int64_t mv = (int64_t)nv * m;
      __nv_bfloat16 *xh = w.xv_h.ensure((size_t)mv * w.Ko), *xl = w.xv_l.ensure((size_t)mv * w.Ko);
      S2G_CUDA(cudaMemsetAsync(xh, 0, (size_t)mv * w.Ko * 2, s));
      S2G_CUDA(cudaMemsetAsync(xl, 0, (size_t)mv * w.Ko * 2, s));
      S2G_LAUNCH(k_tcs_scatter_v, g, 256, 0, s, xh, xl, X, w.ci, w.ca, nci, nv, w.Ko, m);
      float *Z2 = w.Z2.ensure((size_t)mv * ldR);
      w.tc.run(s, xh, xl, w.cot_h.get(), w.cot_l.get(), (int)mv, rows, w.Ko, Z2, ldR,
               2.0 * mv * rows * no, 1, false, 0, false);
      // G2x: U_A[(s,r), i] = sum_b Z2_A[(s,r), b] P^A_ov[i, b], batched over atoms
      __nv_bfloat16 *zh = w.z2t_h.ensure((size_t)N * mz * w.Kv),
                    *zl = w.z2t_l.ensure((size_t)N * mz * w.Kv);
      S2G_CUDA(cudaMemsetAsync(zh, 0, (size_t)N * mz * w.Kv * 2, s));
      S2G_CUDA(cudaMemsetAsync(zl, 0, (size_t)N * mz * w.Kv * 2, s));
      S2G_LAUNCH(k_tcs_to_atom, dim3((unsigned)div_up(nv, 32), (unsigned)div_up(rows, 32), (unsigned)m),
                 tb, 0, s, zh, zl, Z2, ldR, rows, maxa, nv, w.Kv, m);
      U = w.U.ensure((size_t)N * bst);
      w.tc.run(s, zh, zl, w.pov_h.get(), w.pov_l.get(), (int)mz, no, w.Kv, U, ldo,
               2.0 * mz * no * nv, N, true, bst, false);
    }
    // G3 operand: cJ T + cX U back to (i, r) rows; G3: Y[(i,r), a] = sum_R Tt Cv[R, a]
    __nv_bfloat16 *th = w.tt_h.ensure((size_t)mo * w.KR), *tl = w.tt_l.ensure((size_t)mo * w.KR);
    S2G_CUDA(cudaMemsetAsync(th, 0, (size_t)mo * w.KR * 2, s));
    S2G_CUDA(cudaMemsetAsync(tl, 0, (size_t)mo * w.KR * 2, s));
    S2G_LAUNCH(k_tcs_from_atom, dim3((unsigned)div_up(no, 32), (unsigned)div_up(rows, 32), (unsigned)m),
               tb, 0, s, th, tl, T, U, bst, ldo, rows, maxa, no, w.KR, m, cJ, cX);
    float *Y = w.Y.ensure((size_t)mo * ldv);
    w.tc.run(s, th, tl, w.cv2_h.get(), w.cv2_l.get(), (int)mo, nv, w.KR, Y, ldv,
             2.0 * mo * nv * rows, 1, false, 0, false);
    if (side) S2G_CUDA(cudaStreamWaitEvent(s, w.side.join, 0));
    S2G_LAUNCH(k_tcs_gather, g, 256, 0, s, out, Y, ldv, w.ci, w.ca, nci, no, m);
    w.tc.check(s);
  } else if (side) {
    S2G_CUDA(cudaStreamWaitEvent(s, w.side.join, 0));
  }
  if (diag) S2G_LAUNCH(k_add_diag, g, 256, 0, s, out, X, diag, nci, m);
}

}  // namespace std2g
