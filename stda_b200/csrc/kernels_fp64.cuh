// Element-wise, gather and reduction kernels of the sTDA path (FP64).
//
// Each kernel cites the reference routine whose arithmetic it performs.  Pair
// tensors (transition charges q and gamma-contracted p) are stored as
// [pair][atom] -- column-major N x npairs, the layout of qia(ncent,k) in
// stda.f -- so that contractions over atoms read contiguous memory.
#pragma once

#include "common.cuh"

namespace std2g {

constexpr double kEh2eV_in = 27.211385050;   // stda.f:142

// dst[r + nrows*c] = src[r + lds*cols[c]]
__global__ void k_gather_cols(double *__restrict__ dst, const double *__restrict__ src,
                              int64_t nrows, const int *__restrict__ cols, int64_t ncols,
                              int64_t lds) {
  int64_t total = nrows * ncols;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    int64_t c = t / nrows, r = t - c * nrows;
    dst[t] = src[r + lds * (int64_t)cols[c]];
  }
}

// Packed lower triangle (row-wise, element (i,j) i>=j) -> full n x n
// column-major.  mode 0: symmetric; mode 1: antisymmetric with B(i,j)=A(ij)
// for i>j and B(j,i)=-A(ij), zero diagonal (BLOWSY, onetri.f:62-80).
__global__ void k_unpack(double *__restrict__ full, const double *__restrict__ packed,
                         int n, int mode) {
  int64_t total = (int64_t)n * n;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    int64_t j = t / n, i = t - j * n;   // element (i, j), column-major
    double v;
    if (i >= j) {
      v = packed[i * (i + 1) / 2 + j];
    } else {
      v = packed[j * (j + 1) / 2 + i];
      if (mode == 1) v = -v;
    }
    if (mode == 1 && i == j) v = 0.0;
    full[t] = v;
  }
}

// ---- S^1/2 by a coupled Newton-Schulz iteration (makel, stda.f:1615-1691) ----
// Largest absolute row sum of the symmetric n x n S (a bound on its largest
// eigenvalue): block maxima combined with an atomic max on the bit pattern,
// which orders non-negative doubles like their values.
__global__ void k_row_abs_max(const double *__restrict__ S, int n,
                              unsigned long long *__restrict__ out) {
  double best = 0.0;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    double r = 0.0;
    for (int i = 0; i < n; ++i) r += fabs(S[(int64_t)j * n + i]);   // column j = row j
    best = fmax(best, r);
  }
  for (int o = 16; o > 0; o >>= 1) best = fmax(best, __shfl_xor_sync(0xffffffffu, best, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(best));
}

// A = S / c (c = *cmax as stored by k_row_abs_max), Z = I
__global__ void k_ns_init(double *__restrict__ A, double *__restrict__ Z,
                          const double *__restrict__ S, int n,
                          const unsigned long long *__restrict__ cmax) {
  const double inv = 1.0 / __longlong_as_double((long long)*cmax);
  const int64_t total = (int64_t)n * n;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t j = t / n, i = t - j * n;
    A[t] = S[t] * inv;
    Z[t] = i == j ? 1.0 : 0.0;
  }
}

// in place: Q = Z A Z becomes T = (3 I - Q) / 2, and *err = max |I - Q|
// (bit-pattern max)
__global__ void k_ns_step(double *__restrict__ QT, int n, unsigned long long *__restrict__ err) {
  const int64_t total = (int64_t)n * n;
  double e = 0.0;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t j = t / n, i = t - j * n;
    const double d = (i == j ? 1.0 : 0.0) - QT[t];
    QT[t] = (i == j ? 1.0 : 0.0) + 0.5 * d;
    e = fmax(e, fabs(d));
  }
  for (int o = 16; o > 0; o >>= 1) e = fmax(e, __shfl_xor_sync(0xffffffffu, e, o));
  if ((threadIdx.x & 31) == 0) atomicMax(err, (unsigned long long)__double_as_longlong(e));
}

// *out = max |x| (bit-pattern max; NaN propagates as a huge pattern)
__global__ void k_abs_max(const double *__restrict__ x, int64_t n,
                          unsigned long long *__restrict__ out) {
  double e = 0.0;
  bool nan = false;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
       t += (int64_t)gridDim.x * blockDim.x) {
    const double v = fabs(x[t]);
    nan |= v != v;
    e = fmax(e, v);
  }
  for (int o = 16; o > 0; o >>= 1) {
    e = fmax(e, __shfl_xor_sync(0xffffffffu, e, o));
    nan |= __shfl_xor_sync(0xffffffffu, (int)nan, o) != 0;
  }
  if ((threadIdx.x & 31) == 0)
    atomicMax(out, nan ? 0x7ff8000000000000ull : (unsigned long long)__double_as_longlong(e));
}

// ---- the three dominant CSFs of each root (stda.f:1222-1358) ----
// TDA (Y == nullptr): weights w_j = c_j^2; the reference keeps the first CSF
// whose weight exceeds the running maximum, i.e. the largest weight with the
// lowest CSF index on ties, then the next two the same way excluding the
// ones already taken; the reported value is the coefficient c_j.  One block
// per root, three block-wide arg-max passes.
// sTD-DFT (Y given): u = X + Y, p = X - Y and the first pick follows the
// reference's running comparison |u p| > umax with umax = u p (signed; the
// unrestricted table, sutda.f:1315-1335, compares u p without the absolute
// value: first_abs = 0), the second and third u p > umax; reported value
// X^2 - Y^2.  That comparison is
// order dependent, so one thread of the block scans the CSFs in order.
// out_i / out_a: occupied and virtual MO of the CSF (1-based, virtual
// numbered after the no occupied MOs).
__global__ void k_dominant_csfs(const double *__restrict__ X, const double *__restrict__ Y,
                                int nci, const int *__restrict__ ci, const int *__restrict__ ca,
                                int no, double *__restrict__ out_c, int *__restrict__ out_i,
                                int *__restrict__ out_a, int first_abs) {
  const int r = blockIdx.x;
  const double *x = X + (int64_t)r * nci;
  const double *y = Y ? Y + (int64_t)r * nci : nullptr;
  __shared__ double sv[32];
  __shared__ int si[32];
  __shared__ int pick[3];
  if (y) {
    if (threadIdx.x == 0) {
      int k0 = 0, k1 = 0, k2 = 0;
      double um = -1.0;
      for (int j = 0; j < nci; ++j) {
        const double v = (x[j] + y[j]) * (x[j] - y[j]);
        if ((first_abs ? fabs(v) : v) > um) { um = v; k0 = j; }
      }
      um = -1.0;
      for (int j = 0; j < nci; ++j) {
        const double v = (x[j] + y[j]) * (x[j] - y[j]);
        if (v > um && j != k0) { um = v; k1 = j; }
      }
      um = -1.0;
      for (int j = 0; j < nci; ++j) {
        const double v = (x[j] + y[j]) * (x[j] - y[j]);
        if (v > um && j != k0 && j != k1) { um = v; k2 = j; }
      }
      pick[0] = k0;
      pick[1] = k1;
      pick[2] = k2;
    }
  } else {
    for (int q = 0; q < 3; ++q) {
      double bv = -1.0;
      int bi = nci;
      for (int j = threadIdx.x; j < nci; j += blockDim.x) {
        if ((q > 0 && j == pick[0]) || (q > 1 && j == pick[1])) continue;
        const double v = x[j] * x[j];
        if (v > bv) { bv = v; bi = j; }     // strided scan: the first of equal values kept
      }
      for (int o = 16; o > 0; o >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, bv, o);
        const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
        if (ov > bv || (ov == bv && oi < bi)) { bv = ov; bi = oi; }
      }
      if ((threadIdx.x & 31) == 0) {
        sv[threadIdx.x >> 5] = bv;
        si[threadIdx.x >> 5] = bi;
      }
      __syncthreads();
      if (threadIdx.x < 32) {
        const int nw = blockDim.x >> 5;
        bv = threadIdx.x < nw ? sv[threadIdx.x] : -1.0;
        bi = threadIdx.x < nw ? si[threadIdx.x] : nci;
        for (int o = 16; o > 0; o >>= 1) {
          const double ov = __shfl_xor_sync(0xffffffffu, bv, o);
          const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
          if (ov > bv || (ov == bv && oi < bi)) { bv = ov; bi = oi; }
        }
        if (threadIdx.x == 0) pick[q] = bi < nci ? bi : 0;
      }
      __syncthreads();
    }
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    const int j = pick[threadIdx.x];
    const double v = y ? (x[j] * x[j] - y[j] * y[j]) : x[j];
    out_c[3 * r + threadIdx.x] = nci > threadIdx.x ? v : 0.0;
    out_i[3 * r + threadIdx.x] = nci > threadIdx.x ? ci[j] + 1 : 0;
    out_a[3 * r + threadIdx.x] = nci > threadIdx.x ? ca[j] + no + 1 : 0;
  }
}

// U[:, c] *= sqrt(w[c])   (makel, stda.f:1672-1686)
__global__ void k_scale_cols_sqrt(double *__restrict__ U, const double *__restrict__ w, int n) {
  int64_t total = (int64_t)n * n;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    int64_t c = t / n;
    double e = w[c];
    U[t] *= sqrt(e > 0.0 ? e : 0.0);
  }
}

// MO norm check |sum_k c_k^2 - 1| <= 1e-2 (stda.f:442-452)
__global__ void k_colnorm_check(const double *__restrict__ C, int nao, int ncol, int *flag) {
  int col = blockIdx.x;
  if (col >= ncol) return;
  double s = 0.0;
  for (int k = threadIdx.x; k < nao; k += blockDim.x) {
    double v = C[(int64_t)col * nao + k];
    s += v * v;
  }
  __shared__ double red[256];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0 && fabs(red[0] - 1.0) > 1e-2) atomicExch(flag, col + 1);
}

// gamma^J, gamma^K (stda.f:509-532):
//   gJ = 1/(R^beta + (ax*eta)^-beta)^(1/beta), gK = 1/(R^alpha + eta^-alpha)^(1/alpha)
__global__ void k_gamma(const double *__restrict__ xyz, const double *__restrict__ eta_at, int n,
                        double ax, double alpha, double beta, double *__restrict__ gj,
                        double *__restrict__ gk) {
  int64_t total = (int64_t)n * n;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    int j = (int)(t / n), i = (int)(t - (int64_t)j * n);
    double dx = xyz[4 * i] - xyz[4 * j], dy = xyz[4 * i + 1] - xyz[4 * j + 1],
           dz = xyz[4 * i + 2] - xyz[4 * j + 2];
    double r = sqrt(dx * dx + dy * dy + dz * dz);
    double eb = 0.5 * (eta_at[i] + eta_at[j]);
    double xj = eb * ax;
    double gjv = 0.0;
    if (xj > 0.0) gjv = 1.0 / pow(pow(r, beta) + 1.0 / pow(xj, beta), 1.0 / beta);
    gj[t] = gjv;
    gk[t] = 1.0 / pow(pow(r, alpha) + 1.0 / pow(eb, alpha), 1.0 / alpha);
  }
}

// Loewdin transition charges for a block of MO pairs (lo12pop, stda.f:1727-1744):
//   out[A + N*(x*nq + y)] = sum_{k in atom A} C[k, p0+x] * C[k, q0+y]
// ao_ptr/ao_list list the AOs of each atom (AO -> atom map iaoat inverted).
__global__ void k_charges_block(double *__restrict__ out, const double *__restrict__ C, int nao,
                                int N, const int *__restrict__ ao_ptr,
                                const int *__restrict__ ao_list, int p0, int np, int q0, int nq,
                                int diag_only) {
  int64_t npairs = diag_only ? (int64_t)np : (int64_t)np * nq;
  int64_t total = npairs * N;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    int64_t pr = t / N;
    int A = (int)(t - pr * N);
    int x, y;
    if (diag_only) {
      x = (int)pr;
      y = (int)pr;
    } else {
      x = (int)(pr / nq);
      y = (int)(pr - (int64_t)x * nq);
    }
    const double *cp = C + (int64_t)(p0 + x) * nao;
    const double *cq = C + (int64_t)(q0 + y) * nao;
    double s = 0.0;
    for (int m = ao_ptr[A]; m < ao_ptr[A + 1]; ++m) {
      int k = ao_list[m];
      s += cp[k] * cq[k];
    }
    out[t] = s;
  }
}

// Charges of a full MO block, q^A_(p,q) for p < np, q < nq (lo12pop
// stda.f:1727-1744), out[(p*nq + q)*N + A].  One CTA per 8 x 32 tile of MO
// pairs and one chunk of kChAtoms atoms (grid z): the chunk's AO rows of the
// tile's 40 MO columns are staged in shared memory (so every C element is read
// once per tile and chunk, not once per pair), each thread forms its pair's
// sums for the chunk's atoms, and the results leave as contiguous 128-byte
// segments of the [pair][atom] layout.  Write-bound.  Shared memory:
// 40*max_rows + 256*17 doubles.
constexpr int kChTP = 8, kChTQ = 32, kChAtoms = 16;
__global__ void __launch_bounds__(256)
k_charges_tiled(double *__restrict__ out, const double *__restrict__ C, int nao, int N,
                const int *__restrict__ ao_ptr, const int *__restrict__ ao_list, int p0, int np,
                int q0, int nq, int max_rows, int tri) {
  extern __shared__ double sh[];
  double *cp = sh;                                 // [max_rows][kChTP]
  double *cq = cp + (size_t)max_rows * kChTP;      // [max_rows][kChTQ]
  double *st = cq + (size_t)max_rows * kChTQ;      // [256][kChAtoms + 1]
  const int pt = blockIdx.y * kChTP, qt = blockIdx.x * kChTQ;
  // tri: a symmetric block (p, q over the same MOs) wanted for q <= p only
  if (tri && qt > pt + kChTP - 1) return;
  const int pi = threadIdx.x / kChTQ, qi = threadIdx.x % kChTQ;
  constexpr int kCols = kChTP + kChTQ, kSt = kChAtoms + 1;
  {
    const int A0 = blockIdx.z * kChAtoms;
    const int A1 = min(N, A0 + kChAtoms);
    const int r0 = ao_ptr[A0], nr = ao_ptr[A1] - r0;
    // stage C[rows of the chunk, tile columns]: warp w takes columns w, w + 8,
    // ..., its lanes consecutive rows of one column
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int c = warp; c < kCols; c += 8) {
      const bool isp = c < kChTP;
      const int col = isp ? pt + c : qt + (c - kChTP);
      const bool ok = col < (isp ? np : nq);
      const double *src = C + (int64_t)nao * ((isp ? p0 : q0) + (ok ? col : 0));
      for (int r = lane; r < nr; r += 32) {
        const double v = ok ? src[ao_list[r0 + r]] : 0.0;
        if (isp) cp[r * kChTP + c] = v;
        else cq[r * kChTQ + (c - kChTP)] = v;
      }
    }
    __syncthreads();
    for (int a = A0; a < A1; ++a) {
      double sum = 0.0;
      const int ra = ao_ptr[a] - r0, rb = ao_ptr[a + 1] - r0;
      for (int r = ra; r < rb; ++r) sum += cp[r * kChTP + pi] * cq[r * kChTQ + qi];
      st[threadIdx.x * kSt + (a - A0)] = sum;
    }
    __syncthreads();
    const int na = A1 - A0;
    if (na == kChAtoms) {   // a full chunk: 16 threads write one pair's 128 bytes
      for (int t = threadIdx.x; t < kChTP * kChTQ * kChAtoms; t += blockDim.x) {
        const int pl = t / kChAtoms, a = t % kChAtoms;
        const int p = pt + pl / kChTQ, q = qt + pl % kChTQ;
        if (p < np && q < nq) out[((int64_t)p * nq + q) * N + A0 + a] = st[pl * kSt + a];
      }
    } else {
      for (int t = threadIdx.x; t < kChTP * kChTQ * na; t += blockDim.x) {
        const int pl = t / na, a = t - pl * na;
        const int p = pt + pl / kChTQ, q = qt + pl % kChTQ;
        if (p < np && q < nq) out[((int64_t)p * nq + q) * N + A0 + a] = st[pl * kSt + a];
      }
    }
  }
}

// Unrestricted: zero the charges of pairs (p, q) of mixed spin in a pair array
// [pair][atom] (pair p nq + q; p < psplit and q < qsplit are alpha), so that
// the Coulomb (ij|ab) and exchange (ib|ja) terms vanish between spins
// (utdamat / urpamat, sutda.f:2036-2399)
__global__ void k_zero_cross_spin(double *__restrict__ Q, int N, int np, int nq, int psplit,
                                  int qsplit) {
  const int64_t total = (int64_t)np * nq * N;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t col = t / N;
    const int pp = (int)(col / nq), qq = (int)(col - (int64_t)pp * nq);
    if ((pp < psplit) != (qq < qsplit)) Q[t] = 0.0;
  }
}

// P[:, (i, j)] = P[:, (j, i)] for j > i: the upper pairs of a symmetric pair
// array [pair][atom] (pair (i, j) at column i n + j) from the lower ones
__global__ void k_mirror_pairs(double *__restrict__ P, int N, int n) {
  const int64_t total = (int64_t)n * n * N;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t col = t / N, A = t - col * N;
    const int i = (int)(col / n), j = (int)(col - (int64_t)i * n);
    if (j > i) P[t] = P[((int64_t)j * n + i) * N + A];
  }
}

inline size_t charges_tiled_smem(int max_rows) {
  return sizeof(double) * ((size_t)max_rows * (kChTP + kChTQ) + 256 * (kChAtoms + 1));
}

// Diagonal of A and the energy screen (stda.f:593-668, kshift stda.f:1750-1768):
//   ek = p_ia . q_ia,  de = (e_a - e_i) - (ii|aa) + ak*ek [+ kshift]
//   flag = 1 primary (de <= thr), 2 PT candidate (thr < de < fthr), 0 neither
// One warp per ia pair, fixed-order lane reduction (deterministic).
// Unrestricted (sutda) layout of the active window: occupied = alpha (noa)
// then beta, virtual = alpha (nva) then beta; pairs of mixed spin are no CSFs.
// SOMO shift (somo_shift, sutda.f:2402-2422) of the K-shift path: for a pair
// with 1-based in-spin indices io, iv (iv numbered after the spin's occupied
// MOs), de += sau2 / (1 + (ek / wau2)^steep) when io > nsomo or iv <= nsomo,
// nsomo = noa - nuhf (alpha) or nob + nuhf (beta).
struct UksScreen {
  int uks = 0;                 // 0: restricted
  int noa = 0, nob = 0, nva = 0, nsomo_a = 0, nsomo_b = 0;
  double sau2 = 0.0, wau2 = 1.0;
};

__global__ void k_diag_screen(const double *__restrict__ P, const double *__restrict__ Q, int N,
                              int no, int nv, const double *__restrict__ eps_act,
                              const double *__restrict__ uci, double ak, int kshift,
                              double sau, double wau, double steep, double thr, double fthr,
                              double *__restrict__ de_out, double *__restrict__ ek_out,
                              int *__restrict__ flag, UksScreen us) {
  int64_t npair = (int64_t)no * nv;
  int lane = threadIdx.x & 31;
  int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  int64_t nwarp = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t k = warp; k < npair; k += nwarp) {
    const double *p = P + k * N, *q = Q + k * N;
    double s = 0.0;
    for (int A = lane; A < N; A += 32) s += p[A] * q[A];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) {
      int i = (int)(k / nv), a = (int)(k - (int64_t)i * nv);
      double de = (eps_act[no + a] - eps_act[i]) - uci[a + (int64_t)nv * i] + ak * s;
      if (kshift) de += sau / (1.0 + pow(s / wau, steep));
      bool csf = true;
      if (us.uks) {
        const bool ai = i < us.noa, aa = a < us.nva;
        csf = ai == aa;
        if (csf && kshift) {
          const int io = ai ? i + 1 : i - us.noa + 1;
          const int iv = ai ? us.noa + a + 1 : us.nob + (a - us.nva) + 1;
          const int nsomo = ai ? us.nsomo_a : us.nsomo_b;
          if (io > nsomo || iv <= nsomo) de += us.sau2 / (1.0 + pow(s / us.wau2, steep));
        }
      }
      de_out[k] = de;
      ek_out[k] = s;
      flag[k] = !csf ? 0 : ((de <= thr) ? 1 : ((de > thr && de < fthr) ? 2 : 0));
    }
  }
}

// W[A + N*((i-i0)*nop + s)] = Poo[A + N*(i*no + OP[s])]  for i in [i0, i0+ni)
__global__ void k_gather_occ_pairs(double *__restrict__ W, const double *__restrict__ Poo, int N,
                                   int no, int i0, int ni, const int *__restrict__ OP, int nop) {
  int64_t total = (int64_t)N * ni * nop;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    int64_t col = t / N;
    int A = (int)(t - col * N);
    int ii = (int)(col / nop), s = (int)(col - (int64_t)ii * nop);
    W[t] = Poo[A + (int64_t)N * ((int64_t)(i0 + ii) * no + OP[s])];
  }
}

// V[A + N*(a*nvp + t)] = Qvv[A + N*(a*nv + VP[t])]  for all a < nv
__global__ void k_gather_virt_pairs(double *__restrict__ V, const double *__restrict__ Qvv, int N,
                                    int nv, const int *__restrict__ VP, int nvp) {
  int64_t total = (int64_t)N * nv * nvp;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    int64_t col = t / N;
    int A = (int)(t - col * N);
    int a = (int)(col / nvp), s = (int)(col - (int64_t)a * nvp);
    V[t] = Qvv[A + (int64_t)N * ((int64_t)a * nv + VP[s])];
  }
}

// One PT-selection term (ptselect, stda.f:1812-1826):
//   amat = ak*(ia|jb) - (ij|ab),  pt = amat^2 / (E_k - E_j + 1e-10)
// K: Kbuf[c + nex*r]; J: Jbuf[(a*nvp + vmap[b]) + ldj*((i-i0)*nop + omap[j])]
template <typename TK, typename TJ>
__device__ __forceinline__ double pt_term(const TK *Kbuf, const TJ *Jbuf, int64_t ldj, int64_t ldk,
                                          int nvp, int nop, int r, int c, int iloc, int a,
                                          double de_r, const int *pj, const int *pb,
                                          const int *omap, const int *vmap,
                                          const double *ed, double ak) {
  double kv = (double)Kbuf[(int64_t)c + ldk * r];
  double jv = (double)Jbuf[((int64_t)a * nvp + vmap[pb[c]]) +
                           ldj * ((int64_t)iloc * nop + omap[pj[c]])];
  double amat = ak * kv - jv;
  return amat * amat / (de_r - ed[c] + 1e-10);
}

// Row pass: pert[r] = sum_j pt(r, j) and the selection pert > thrp.
template <typename TK, typename TJ>
__global__ void k_pt_rows(const TK *__restrict__ Kbuf, const TJ *__restrict__ Jbuf, int64_t ldj,
                          int64_t ldk, int nex, int nvp, int nop, int nrows, const int *__restrict__ cand_k,
                          int nv, int i0, const double *__restrict__ de_all,
                          const int *__restrict__ pj, const int *__restrict__ pb,
                          const int *__restrict__ omap, const int *__restrict__ vmap,
                          const double *__restrict__ ed, double ak, double thrp,
                          double *__restrict__ pert_out, unsigned char *__restrict__ sel) {
  int r = blockIdx.x;
  if (r >= nrows) return;
  int k = cand_k[r];
  int i = k / nv, a = k - i * nv;
  double de_r = de_all[k];
  double s = 0.0;
  for (int c = threadIdx.x; c < nex; c += blockDim.x)
    s += pt_term(Kbuf, Jbuf, ldj, ldk, nvp, nop, r, c, i - i0, a, de_r, pj, pb, omap, vmap, ed, ak);
  __shared__ double red[256];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    pert_out[r] = red[0];
    sel[r] = red[0] > thrp ? 1 : 0;
  }
}

// Column pass: colpart[c] = sum over non-selected rows r (in order) of pt(r, c).
template <typename TK, typename TJ>
__global__ void k_pt_cols(const TK *__restrict__ Kbuf, const TJ *__restrict__ Jbuf, int64_t ldj,
                          int64_t ldk, int nex, int nvp, int nop, int nrows, const int *__restrict__ cand_k,
                          int nv, int i0, const double *__restrict__ de_all,
                          const int *__restrict__ pj, const int *__restrict__ pb,
                          const int *__restrict__ omap, const int *__restrict__ vmap,
                          const double *__restrict__ ed, double ak,
                          const unsigned char *__restrict__ sel, double *__restrict__ colpart,
                          int seg_rows) {
  // grid: x over primaries, y over segments of seg_rows candidate rows;
  // colpart[y*nex + c] holds the segment's sum (reduced in fixed order later)
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nex) return;
  const int rbeg = blockIdx.y * seg_rows;
  const int rend = min(nrows, rbeg + seg_rows);
  colpart += (int64_t)blockIdx.y * nex;
  double s = 0.0;
  for (int r = rbeg; r < rend; ++r) {
    if (sel[r]) continue;
    int k = cand_k[r];
    int i = k / nv, a = k - i * nv;
    s += pt_term(Kbuf, Jbuf, ldj, ldk, nvp, nop, r, c, i - i0, a, de_all[k], pj, pb, omap, vmap,
                 ed, ak);
  }
  colpart[c] = s;
}

// pt2[c] = sum_chunks colpart[chunk*nex + c] (fixed order); ed_out[c] = ed[c] - pt2[c]
// (stda.f:1851-1854)
__global__ void k_pt2_finish(const double *__restrict__ colpart, int nchunk, int nex,
                             const double *__restrict__ ed, double *__restrict__ pt2,
                             double *__restrict__ ed_out) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nex) return;
  double s = 0.0;
  for (int q = 0; q < nchunk; ++q) s += colpart[(int64_t)q * nex + c];
  pt2[c] = s;
  ed_out[c] = ed[c] - s;
}

// Direct gathered dot products over atoms for CSF pairs (u, v), one warp per
// element, fixed lane order:
//   mode 0 (J, rtdamat stda.f:2044-2046): sum_A Poo[A,(i_u,i_v)] Qvv[A,(a_u,a_v)]
//   mode 1 (exchange K, rrpamat stda.f:1943-1946):
//          sum_A Pia[A,(i_u,a_v)] Qia[A,(i_v,a_u)]
__global__ void k_pairdot(double *__restrict__ out, int64_t ld, const int *__restrict__ ci,
                          const int *__restrict__ ca, int nci, const double *__restrict__ F,
                          const double *__restrict__ G, int N, int no, int nv, int mode) {
  int lane = threadIdx.x & 31;
  int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  int64_t nwarp = ((int64_t)gridDim.x * blockDim.x) >> 5;
  int64_t total = (int64_t)nci * nci;
  for (int64_t t = warp; t < total; t += nwarp) {
    int v = (int)(t / nci), u = (int)(t - (int64_t)v * nci);
    if (u < v) continue;           // lower triangle, mirrored below
    int64_t fo, go;
    if (mode == 0) {
      fo = (int64_t)N * ((int64_t)ci[u] * no + ci[v]);
      go = (int64_t)N * ((int64_t)ca[u] * nv + ca[v]);
    } else {
      fo = (int64_t)N * ((int64_t)ci[u] * nv + ca[v]);
      go = (int64_t)N * ((int64_t)ci[v] * nv + ca[u]);
    }
    double s = 0.0;
    for (int A = lane; A < N; A += 32) s += F[fo + A] * G[go + A];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) {
      out[u + ld * v] = s;
      out[v + ld * u] = s;
    }
  }
}

// The same couplings gathered from a box of all of them, formed by one GEMM
// (J: box[(i j) + no^2 (a b)] = p_ij . q_ab, the (ij) x (ab) product of the
// gamma^J-contracted occupied pairs with the virtual pairs; mode 1, exchange:
// box[(i b) + nov (j a)] = p_ib . q_ja):
//   mode 0: out[u + ld v] = (i_u j_v | a_u b_v)
//   mode 1: out[u + ld v] = (i_u b_v | j_v a_u)
__global__ void k_box_gather(double *__restrict__ out, int64_t ld, const double *__restrict__ box,
                             const int *__restrict__ ci, const int *__restrict__ ca, int nci,
                             int no, int nv, int mode) {
  const int64_t total = (int64_t)nci * nci;
  const int64_t noo = (int64_t)no * no, nov = (int64_t)no * nv;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int v = (int)(t / nci), u = (int)(t - (int64_t)v * nci);
    const int64_t o = mode == 0
                          ? ((int64_t)ci[u] * no + ci[v]) + noo * ((int64_t)ca[u] * nv + ca[v])
                          : ((int64_t)ci[u] * nv + ca[v]) + nov * ((int64_t)ci[v] * nv + ca[u]);
    out[u + ld * v] = box[o];
  }
}

// A = ak*K - J off the diagonal, A_uu = ed_u (rtdamat stda.f:2044-2051)
__global__ void k_combine_tda(double *__restrict__ A, const double *__restrict__ K,
                              const double *__restrict__ J, int64_t n, double ak,
                              const double *__restrict__ ed) {
  int64_t total = n * n;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    int64_t v = t / n, u = t - v * n;
    A[t] = (u == v) ? ed[u] : ak * K[t] - J[t];
  }
}

// A+B and A-B (rrpamat stda.f:1930-1963) and 0.5*B (rtdacorr apbtrafo.f:618-634)
//   A+B = 2ak K - ax Kx - J ; diag ed - ax ek + ak ek
//   A-B = ax Kx - J         ; diag ed - ak ek + ax ek
//   B/2 = ak K/2 - ax Kx/2  ; diag (ak - ax) ek / 2
__global__ void k_combine_rpa(double *__restrict__ Apb, double *__restrict__ Amb,
                              double *__restrict__ Bh, const double *__restrict__ K,
                              const double *__restrict__ Kx, const double *__restrict__ J,
                              int64_t n, double ak, double ax, const double *__restrict__ ed,
                              const double *__restrict__ ekd) {
  int64_t total = n * n;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    int64_t v = t / n, u = t - v * n;
    if (u == v) {
      double e = ekd[u];
      if (Apb) Apb[t] = ed[u] - ax * e + ak * e;
      if (Amb) Amb[t] = ed[u] - ak * e + ax * e;
      if (Bh) Bh[t] = 0.5 * (ak * e - ax * e);
    } else {
      if (Apb) Apb[t] = 2.0 * ak * K[t] - ax * Kx[t] - J[t];
      if (Amb) Amb[t] = (fabs(ax) < 1e-6) ? 0.0 : ax * Kx[t] - J[t];
      if (Bh) Bh[t] = 0.5 * ak * K[t] - 0.5 * ax * Kx[t];
    }
  }
}

// mu_sel[u + nci*c] = mu_ov[c][i_u + no*a_u], c = 0..8 (L xyz, V xyz, M xyz)
__global__ void k_gather_mu(double *__restrict__ mu_sel, const double *__restrict__ mu_ov, int no,
                            int nv, const int *__restrict__ ci, const int *__restrict__ ca,
                            int nci) {
  int64_t total = (int64_t)nci * 9;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    int c = (int)(t / nci), u = (int)(t - (int64_t)c * nci);
    mu_sel[t] = mu_ov[(int64_t)c * no * nv + ci[u] + (int64_t)no * ca[u]];
  }
}

// Per-root properties (stda.f:1207-1289; velocity corrected apbtrafo.f:180-243).
//   T  [nroot x 9]: contractions of X (or X+Y / X-Y) with mu_L, mu_V, mu_M
//   T2 [nroot x 9]: contractions of X_new = (B/2) X / w (velcorr) or NULL
// out: fL, fV, RL, RV per root
__global__ void k_properties(const double *__restrict__ TL, const double *__restrict__ TVM,
                             const double *__restrict__ T2, int nroot, int ldT,
                             const double *__restrict__ om, double ak, int velcorr,
                             double *__restrict__ fL, double *__restrict__ fV,
                             double *__restrict__ RL, double *__restrict__ RV) {
  int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nroot) return;
  const double rot = -235.7220;
  double w = om[r];
  double ef = 1.0 / (w + 1.0e-8);
  double l[3], v[3], m[3];
  for (int d = 0; d < 3; ++d) {
    l[d] = TL[r + (int64_t)ldT * d];
    v[d] = TVM[r + (int64_t)ldT * (3 + d)];
    m[d] = TVM[r + (int64_t)ldT * (6 + d)];
  }
  if (!velcorr) {
    double sak = sqrt(ak);
    double xl = 0, xv = 0, rl = 0, rv = 0;
    for (int d = 0; d < 3; ++d) {
      double a = sak * l[d], b = sak * v[d], c = sak * m[d];
      xl += a * a;
      xv += b * b;
      rl += a * c;
      rv += b * c;
    }
    fL[r] = w * (2.0 / 3.0) * xl;
    fV[r] = ef * (2.0 / 3.0) * xv;
    RL[r] = rot * rl;
    RV[r] = rot * rv * ef;
  } else {
    double v2[3], m2[3];
    for (int d = 0; d < 3; ++d) {
      v2[d] = T2[r + (int64_t)ldT * (3 + d)];
      m2[d] = T2[r + (int64_t)ldT * (6 + d)];
    }
    double hilf = 1.0 - exp(-150.0 * w * w);
    double efmod = 1.0 / (pow(w, hilf) + 1.0e-8);
    double p23 = ak * 2.0 / 3.0;
    double xl = 0, xv = 0, rl = 0, rv = 0;
    for (int d = 0; d < 3; ++d) {
      xl += l[d] * l[d];
      xv += v[d] * v[d];
      rl += l[d] * m[d];
      rv += v[d] * m[d] + v2[d] * m[d] + v[d] * m2[d];
    }
    fL[r] = xl * p23 * w;
    fV[r] = p23 * ef * xv;
    RL[r] = rot * rl * ak;
    RV[r] = rot * rv * ak * efmod;
  }
}

// X[:, r] *= s[r]  (column scaling, e.g. 1/sqrt(w), 1/w)
__global__ void k_scale_columns(double *__restrict__ X, int64_t n, int ncol,
                                const double *__restrict__ s, int mode) {
  int64_t total = n * ncol;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    int64_t c = t / n;
    double w = s[c];
    double f = mode == 0 ? 1.0 / sqrt(w) : (mode == 1 ? 1.0 / w : 1.0 / (w + 1.0e-8));
    X[t] *= f;
  }
}

// w[r] = sqrt(w[r]) (sRPA omega from omega^2, srpapack.f:110)
__global__ void k_sqrt_inplace(double *__restrict__ w, int n) {
  int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r < n) w[r] = sqrt(w[r]);
}

// X = (XpY + XmY)/2, Y = XpY - X (srpapack.f:146-152)
__global__ void k_xy_from_sums(double *__restrict__ XpY, double *__restrict__ XmY, int64_t total) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    double p = XpY[t], m = XmY[t];
    double x = 0.5 * (p + m);
    XpY[t] = x;
    XmY[t] = p - x;
  }
}

// alpha(0) sum over states (stda.f:1247-1252, doubled at stda.f:1465)
__global__ void k_alpha0(const double *__restrict__ TL, int nroot, int ldT,
                         const double *__restrict__ om, double ak, double *__restrict__ out6) {
  __shared__ double red[6][128];
  double a[6] = {0, 0, 0, 0, 0, 0};
  for (int r = threadIdx.x; r < nroot; r += blockDim.x) {
    double ef = 1.0 / (om[r] + 1.0e-8);
    double x = TL[r] * sqrt(ak), y = TL[r + ldT] * sqrt(ak), z = TL[r + 2 * (int64_t)ldT] * sqrt(ak);
    a[0] += x * x * ef;
    a[1] += x * y * ef;
    a[2] += y * y * ef;
    a[3] += x * z * ef;
    a[4] += y * z * ef;
    a[5] += z * z * ef;
  }
  for (int q = 0; q < 6; ++q) red[q][threadIdx.x] = a[q];
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int q = 0; q < 6; ++q) {
      double s = 0;
      for (int t = 0; t < blockDim.x; ++t) s += red[q][t];
      out6[q] = 2.0 * s;
    }
  }
}

}  // namespace std2g

namespace std2g {

// copy the lower triangle of a column-major n x n matrix to the upper one
__global__ void k_symmetrize_lower(double *__restrict__ A, int64_t n) {
  int64_t total = n * n;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    int64_t j = t / n, i = t - j * n;
    if (i < j) A[t] = A[j + n * i];
  }
}

// M = A + f * B
__global__ void k_axpby_mat(double *__restrict__ M, const double *__restrict__ A,
                            const double *__restrict__ B, int64_t n, double f) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
       t += (int64_t)gridDim.x * blockDim.x)
    M[t] = A[t] + f * B[t];
}

// y = f * x
__global__ void k_scale_copy(double *__restrict__ y, const double *__restrict__ x, int64_t n,
                             double f) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
       t += (int64_t)gridDim.x * blockDim.x)
    y[t] = f * x[t];
}

// out = max_k ||R[:,k]|| / ||B[:,k]||  (one block)
__global__ void k_resid_ratio(const double *__restrict__ R, const double *__restrict__ B, int n,
                              int nrhs, double *__restrict__ out) {
  __shared__ double sr[256], sb[256];
  double worst = 0.0;
  for (int k = 0; k < nrhs; ++k) {
    double a = 0, b = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      double r = R[(int64_t)k * n + i], q = B[(int64_t)k * n + i];
      a += r * r;
      b += q * q;
    }
    sr[threadIdx.x] = a;
    sb[threadIdx.x] = b;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
      if (threadIdx.x < o) {
        sr[threadIdx.x] += sr[threadIdx.x + o];
        sb[threadIdx.x] += sb[threadIdx.x + o];
      }
      __syncthreads();
    }
    if (threadIdx.x == 0) {
      double rr = sb[0] > 0 ? sqrt(sr[0] / sb[0]) : sqrt(sr[0]);
      worst = fmax(worst, rr);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = worst;
}

// box[v*no*nv + i + no*a] = Y[u + nci*v] for the CSF u = (i, a) (box zeroed first)
__global__ void k_box_scatter(double *__restrict__ box, const double *__restrict__ Y,
                              const int *__restrict__ ci, const int *__restrict__ ca, int nci,
                              int no, int nv, int nvec) {
  const int64_t total = (int64_t)nci * nvec;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int v = (int)(t / nci), u = (int)(t - (int64_t)v * nci);
    box[(int64_t)v * no * nv + ci[u] + (int64_t)no * ca[u]] = Y[t];
  }
}

// sel[u + nci*col] = box[col*no*nv + i + no*a] for the CSF u = (i, a)
__global__ void k_box_gather(double *__restrict__ sel, const double *__restrict__ box,
                             const int *__restrict__ ci, const int *__restrict__ ca, int nci,
                             int no, int nv, int ncol) {
  const int64_t total = (int64_t)nci * ncol;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int col = (int)(t / nci), u = (int)(t - (int64_t)col * nci);
    sel[t] = box[(int64_t)col * no * nv + ci[u] + (int64_t)no * ca[u]];
  }
}

// X = f (U + V), Y = f (U - V) from U = X+Y, V = X-Y (f = 1/2; 1/4 also halves
// a response to -2 mu into the response to -mu)
__global__ void k_xy_from_uv(double *__restrict__ X, double *__restrict__ Y,
                             const double *__restrict__ U, const double *__restrict__ V,
                             int64_t n, double f) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
       t += (int64_t)gridDim.x * blockDim.x) {
    X[t] = f * (U[t] + V[t]);
    Y[t] = f * (U[t] - V[t]);
  }
}

// out[i + n*c] += M[i + n*i] * src[i + n*c] * g_c, g_c = 1/sqrt(w_c) (mode 0) or
// 1 (mode 1): the diagonal of M counted once more in a product with src
__global__ void k_add_diag_cols(double *__restrict__ out, const double *__restrict__ M,
                                const double *__restrict__ src, int64_t n, int ncol,
                                const double *__restrict__ w, int mode) {
  const int64_t total = n * ncol;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = t / n, i = t - c * n;
    const double g = mode == 0 ? 1.0 / sqrt(w[c]) : 1.0;
    out[t] += M[i + n * i] * src[t] * g;
  }
}

}  // namespace std2g
