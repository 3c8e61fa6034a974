// Mixed-precision form of the linear-response solves (linear_response.f:23-192).
//
// The reference solves, per frequency w and Cartesian component,
//   [(A+B) - w^2 (A-B)^-1] (X+Y) = -2 mu      (linear_response.f:89-131)
// after inverting A-B.  Here the same equations are solved as the coupled
// system in u = X+Y, v = X-Y
//   (A+B) u - w v = -2 mu,     -w u + (A-B) v = 0,
// by iterative refinement: residuals in FP64 from products with the FP64
// A+B and A-B (no inverse is formed), corrections from preconditioned
// conjugate gradients on the same 2n system with lower-precision products
// (dense: FP32 copies of A+B, A-B; matrix-free: the FP32 operator).  For w below the first
// excitation that system is positive definite (its Schur complement is the
// reference's matrix).  The preconditioner is the exact inverse of each 2x2
// block [[p_i, -w], [-w, m_i]] (p, m the diagonals of A+B and A-B).  All
// right-hand sides (frequencies x components) run in lockstep; a column that
// meets negative curvature is flagged and its frequency is solved by the FP64
// form instead.
#pragma once

#include "common.cuh"

namespace std2g {

constexpr int kRespSplit = 32;   // row blocks per column in the reductions

__global__ void k_d2f(float *__restrict__ dst, const double *__restrict__ src, int64_t n) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
       t += (int64_t)gridDim.x * blockDim.x)
    dst[t] = (float)src[t];
}

// B1[:, w*3 + x] = -2 mu_x  (mu = first 3 columns of musel, n rows)
__global__ void k_resp_rhs(double *__restrict__ B1, const double *__restrict__ mu, int n, int nw) {
  const int64_t total = (int64_t)n * nw * 3;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    int64_t col = t / n, i = t - col * n;
    B1[t] = -2.0 * mu[i + (int64_t)n * (col % 3)];
  }
}

// R1 = B1 - PU + w V ; R2 = w U - MV   (PU = (A+B) U, MV = (A-B) V), w per column
__global__ void k_resp_resid(double *__restrict__ R1, double *__restrict__ R2,
                             const double *__restrict__ B1, const double *__restrict__ U,
                             const double *__restrict__ V, const double *__restrict__ PU,
                             const double *__restrict__ MV, const double *__restrict__ wcol,
                             int n, int ncol) {
  const int64_t total = (int64_t)n * ncol;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const double w = wcol[t / n];
    R1[t] = B1[t] - PU[t] + w * V[t];
    R2[t] = w * U[t] - MV[t];
  }
}

__device__ __forceinline__ double resp_block_sum(double s, double *red) {
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) red[warp] = s;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
  return t;   // valid in thread 0
}

// part[j*kRespSplit + b] = sum over row block b of a[:, j] . b[:, j]  (FP64, a/b FP64)
__global__ void k_resp_dot64(const double *__restrict__ a, const double *__restrict__ b, int n,
                             double *__restrict__ part) {
  const int j = blockIdx.y;
  const int64_t chunk = (n + gridDim.x - 1) / gridDim.x;
  const int64_t i0 = chunk * blockIdx.x, i1 = min((int64_t)n, i0 + chunk);
  const double *x = a + (int64_t)n * j, *y = b + (int64_t)n * j;
  double s = 0.0;
  for (int64_t i = i0 + threadIdx.x; i < i1; i += blockDim.x) s += x[i] * y[i];
  __shared__ double red[32];
  s = resp_block_sum(s, red);
  if (threadIdx.x == 0) part[(int64_t)j * gridDim.x + blockIdx.x] = s;
}

// out[j] = sum_b part[j*nsplit + b] in order
__global__ void k_resp_sum(const double *__restrict__ part, int nsplit, int ncol,
                           double *__restrict__ out) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= ncol) return;
  double s = 0.0;
  for (int b = 0; b < nsplit; ++b) s += part[(int64_t)j * nsplit + b];
  out[j] = s;
}

// Diagonals of A+B and A-B from the dense FP64 matrices
__global__ void k_resp_diags(const double *__restrict__ Apb, const double *__restrict__ Amb, int n,
                             float *__restrict__ dp, float *__restrict__ dm) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  dp[i] = (float)Apb[i + (int64_t)n * i];
  dm[i] = (float)Amb[i + (int64_t)n * i];
}

// Matrix-free A+B / A-B (rrpamat stda.f:1893-1928 in operator form): with the
// operator parts K, J, Kx (their own diagonals included),
//   (A+B) x = (2ak K - ax Kx - J) x + d o x,   (A-B) x = (ax Kx - J) x + d o x,
//   d = ed - ak (ia|ia) + (ii|aa);
// for ax = 0, A-B is the diagonal ed - ak (ia|ia).  Also the diagonals of
// A+B and A-B for the preconditioner.
__global__ void k_rpa_mf_diag(double *__restrict__ d, double *__restrict__ dpd,
                              double *__restrict__ dmd, const double *__restrict__ ed,
                              const double *__restrict__ ekd, const double *__restrict__ uci,
                              const int *__restrict__ ci, const int *__restrict__ ca, int nci,
                              int nv, double ak, double ax) {
  int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= nci) return;
  const double e = ekd[u], jd = uci[ca[u] + (int64_t)nv * ci[u]];
  d[u] = ed[u] - ak * e + jd;
  dpd[u] = ed[u] - ax * e + ak * e;
  dmd[u] = ed[u] - ak * e + ax * e;
}

// y[:, j] = d o x[:, j]
__global__ void k_diag_mul(double *__restrict__ y, const double *__restrict__ d,
                           const double *__restrict__ x, int n, int ncol) {
  const int64_t total = (int64_t)n * ncol;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x)
    y[t] = d[t % n] * x[t];
}

// U += du ; V += dv (corrections into the FP64 iterates)
template <typename T>
__global__ void k_resp_accum(double *__restrict__ U, double *__restrict__ V,
                             const T *__restrict__ du, const T *__restrict__ dv, int64_t total) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    U[t] += (double)du[t];
    V[t] += (double)dv[t];
  }
}

// ---- preconditioned CG on the 2n system, ncol independent systems in lockstep ----
// Vectors (type T: FP32 for the dense mixed form, FP64 for the matrix-free
// form) come in halves (u, v), each n x ncol column-major.  Scalars per column
// (FP64): rz, alpha, beta, rr; flag: bit j set on negative curvature.

// z = P r with P the inverse of the 2x2 blocks [[p, -w], [-w, m]]
template <typename T, typename D>
__device__ __forceinline__ void pcg2_prec(T ru, T rv, D p, D m, T w, T &zu, T &zv) {
  const T pp = (T)p, mm = (T)m;
  T det = pp * mm - w * w;
  det = det > (T)1e-12 ? det : (T)1e-12;
  zu = (mm * ru + w * rv) / det;
  zv = (w * ru + pp * rv) / det;
}

// y = 0, r = c, z = P r, p = z; partial r.z and r.r
template <typename T, typename D>
__global__ void k_pcg2_init(T *__restrict__ yu, T *__restrict__ yv, T *__restrict__ ru,
                            T *__restrict__ rv, T *__restrict__ zu, T *__restrict__ zv,
                            T *__restrict__ pu, T *__restrict__ pv, const T *__restrict__ cu,
                            const T *__restrict__ cv, const D *__restrict__ dp,
                            const D *__restrict__ dm, const double *__restrict__ wcol, int n,
                            double *__restrict__ part_rz, double *__restrict__ part_rr) {
  const int j = blockIdx.y;
  const T w = (T)wcol[j];
  const int64_t chunk = (n + gridDim.x - 1) / gridDim.x;
  const int64_t i0 = chunk * blockIdx.x, i1 = min((int64_t)n, i0 + chunk);
  double srz = 0.0, srr = 0.0;
  for (int64_t i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
    const int64_t o = i + (int64_t)n * j;
    const T a = cu[o], b = cv[o];
    T za, zb;
    pcg2_prec(a, b, dp[i], dm[i], w, za, zb);
    yu[o] = (T)0;
    yv[o] = (T)0;
    ru[o] = a;
    rv[o] = b;
    zu[o] = za;
    zv[o] = zb;
    pu[o] = za;
    pv[o] = zb;
    srz += (double)a * za + (double)b * zb;
    srr += (double)a * a + (double)b * b;
  }
  __shared__ double red[32];
  double x = resp_block_sum(srz, red);
  __syncthreads();
  double y = resp_block_sum(srr, red);
  if (threadIdx.x == 0) {
    part_rz[(int64_t)j * gridDim.x + blockIdx.x] = x;
    part_rr[(int64_t)j * gridDim.x + blockIdx.x] = y;
  }
}

// (qu, qv) = ((A+B) pu - w pv, (A-B) pv - w pu), the products given in (qu, qv);
// partial p.q
template <typename T>
__global__ void k_pcg2_pq(T *__restrict__ qu, T *__restrict__ qv, const T *__restrict__ pu,
                          const T *__restrict__ pv, const double *__restrict__ wcol, int n,
                          double *__restrict__ part) {
  const int j = blockIdx.y;
  const T w = (T)wcol[j];
  const int64_t chunk = (n + gridDim.x - 1) / gridDim.x;
  const int64_t i0 = chunk * blockIdx.x, i1 = min((int64_t)n, i0 + chunk);
  double s = 0.0;
  for (int64_t i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
    const int64_t o = i + (int64_t)n * j;
    const T a = qu[o] - w * pv[o], b = qv[o] - w * pu[o];
    qu[o] = a;
    qv[o] = b;
    s += (double)pu[o] * a + (double)pv[o] * b;
  }
  __shared__ double red[32];
  s = resp_block_sum(s, red);
  if (threadIdx.x == 0) part[(int64_t)j * gridDim.x + blockIdx.x] = s;
}

// alpha_j = rz_j / pq_j; 0 for a finished column, 0 and flag bit j on negative curvature
__global__ void k_pcg_alpha(const double *__restrict__ part, int nsplit, int ncol,
                            const double *__restrict__ rz, double *__restrict__ alpha,
                            unsigned *__restrict__ flag) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= ncol) return;
  double pq = 0.0;
  for (int b = 0; b < nsplit; ++b) pq += part[(int64_t)j * nsplit + b];
  if (rz[j] == 0.0 || pq == 0.0) {   // converged (or underflowed) column: frozen
    alpha[j] = 0.0;
  } else if (!(pq > 0.0)) {           // negative curvature: not positive definite
    alpha[j] = 0.0;
    atomicOr(flag, 1u << j);
  } else {
    alpha[j] = rz[j] / pq;
  }
}

// y += a p ; r -= a q ; z = P r ; partial r.z and r.r
template <typename T, typename D>
__global__ void k_pcg2_update(T *__restrict__ yu, T *__restrict__ yv, T *__restrict__ ru,
                              T *__restrict__ rv, T *__restrict__ zu, T *__restrict__ zv,
                              const T *__restrict__ pu, const T *__restrict__ pv,
                              const T *__restrict__ qu, const T *__restrict__ qv,
                              const D *__restrict__ dp, const D *__restrict__ dm,
                              const double *__restrict__ wcol, const double *__restrict__ alpha,
                              int n, double *__restrict__ part_rz, double *__restrict__ part_rr) {
  const int j = blockIdx.y;
  const T a = (T)alpha[j], w = (T)wcol[j];
  const int64_t chunk = (n + gridDim.x - 1) / gridDim.x;
  const int64_t i0 = chunk * blockIdx.x, i1 = min((int64_t)n, i0 + chunk);
  double srz = 0.0, srr = 0.0;
  for (int64_t i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
    const int64_t o = i + (int64_t)n * j;
    yu[o] += a * pu[o];
    yv[o] += a * pv[o];
    const T x = ru[o] - a * qu[o], y = rv[o] - a * qv[o];
    ru[o] = x;
    rv[o] = y;
    T za, zb;
    pcg2_prec(x, y, dp[i], dm[i], w, za, zb);
    zu[o] = za;
    zv[o] = zb;
    srz += (double)x * za + (double)y * zb;
    srr += (double)x * x + (double)y * y;
  }
  __shared__ double red[32];
  double s1 = resp_block_sum(srz, red);
  __syncthreads();
  double s2 = resp_block_sum(srr, red);
  if (threadIdx.x == 0) {
    part_rz[(int64_t)j * gridDim.x + blockIdx.x] = s1;
    part_rr[(int64_t)j * gridDim.x + blockIdx.x] = s2;
  }
}

// rz_new, beta = rz_new / rz, rr; with init != 0 only rz and rr are set
__global__ void k_pcg_beta(const double *__restrict__ part_rz, const double *__restrict__ part_rr,
                           int nsplit, int ncol, double *__restrict__ rz, double *__restrict__ beta,
                           double *__restrict__ rr, int init) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= ncol) return;
  double a = 0.0, b = 0.0;
  for (int q = 0; q < nsplit; ++q) {
    a += part_rz[(int64_t)j * nsplit + q];
    b += part_rr[(int64_t)j * nsplit + q];
  }
  if (!init) beta[j] = rz[j] != 0.0 ? a / rz[j] : 0.0;
  rz[j] = a;
  rr[j] = b;
}

// p = z + beta p, both halves
template <typename T>
__global__ void k_pcg2_dir(T *__restrict__ pu, T *__restrict__ pv, const T *__restrict__ zu,
                           const T *__restrict__ zv, const double *__restrict__ beta, int n,
                           int ncol) {
  const int64_t total = (int64_t)n * ncol;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const T b = (T)beta[t / n];
    pu[t] = zu[t] + b * pu[t];
    pv[t] = zv[t] + b * pv[t];
  }
}

}  // namespace std2g
