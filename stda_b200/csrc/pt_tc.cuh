// Mixed-precision PT selection (ptselect, stda.f:1773-1863) on the tensor cores.
//
// For a candidate CSF r = (i, a) and a primary CSF q = (j, b) the reference
// forms the coupling A_rq = ak (ia|jb) - (ij|ab) (stda.f:1812-1819) and the
// term t_rq = A_rq^2 / (E_r - E_q + 1e-10); a candidate is kept when
// sum_q t_rq > thrp, and every primary q is lowered by the sum of t_rq over
// the candidates that are not kept (stda.f:1820-1854).
//
// Both couplings are contractions over atoms on the tensor cores (tc_gemm.cuh)
// with split-FP16 operands: every operand vector x is scaled by a power of two
// s (max |s x| < 2^14) and written as hi + lo, hi = fp16(s x),
// lo = fp16(s x - hi), so that |s x - hi - lo| <= 2^-22 |s x| (plus the FP16
// subnormal spacing, 2^-24); the epilogue divides the FP32 result by the two
// scales (exact).  The couplings are written for one chunk of candidate occupied
// indices i in [i0, i0 + ni) into two FP32 buffers of the same layout
//
//     X[((i - i0) * nex + q) * nva + a]          (nva = nv rounded up to 32)
//
// so that both passes over them sweep contiguous memory (rows of nva values
// for consecutive q):
//   (ia|jb): for each i, rows a (p_ia) times columns q (q_jb);
//   (ij|ab): grouped by the primaries' virtual index b -- rows a of the slab
//            q_ab (b fixed) times columns (i, q) with j = j_q (p_ij) -- so
//            only the (i, a, q) combinations the sums need are formed.
// The primaries are taken in (b, j) order so that each group's columns are
// contiguous.
//
// Selection with an error bound: the row pass sums the terms of every
// candidate (FP32 terms, FP64 sums) together with a bound on the error of that
// sum.  The couplings' error is bounded through the Cauchy-Schwarz inequality,
// |delta (p . q)| <= e_c ||p|| ||q||, where e_c covers the split (three of the
// four hi/lo products: 3.05 * 2^-22) and the FP32 accumulation on the tensor
// cores, 3 * Kpad / 16 MMA instructions of 16 exact products each, under the
// stated model that one instruction adds its products to the accumulator with
// an error of at most 4 units in the last place of the larger of |accumulator|
// and the sum of the products' magnitudes (NVIDIA does not document the
// rounding of the accumulation; the model allows truncating alignment with a
// few guard bits and a final round-toward-zero).  Every candidate whose sum
// lies within its bound of thrp is re-decided from FP64 couplings
// (k_pt_recheck), so the selected CSF set is the one FP64 arithmetic gives.
#pragma once

#include <algorithm>
#include <chrono>
#include <cmath>
#include <vector>

#include <cuda_fp16.h>

#include "common.cuh"
#include "tc_gemm.cuh"

namespace std2g {

constexpr float kU32 = 5.9604645e-8f;   // 2^-24

// Relative error of one split-FP16 tensor-core coupling, with respect to the
// product of the operands' 2-norms, for a contraction padded to Kpad.
inline float coupling_error_bound(int Kpad) {
  const double split = 3.05 * std::ldexp(1.0, -22) + std::ldexp(1.0, -30);   // + subnormal floor
  const double accum = (3.0 * Kpad / 16.0) * 4.0 * std::ldexp(1.0, -23);
  return (float)(1.25 * (split + accum));   // 25 % margin
}

// Tile schedule of the two coupling contractions of one chunk (TcTile).
//   mode 0, (ia|jb): tile (ii, ab, qb), qb fastest; A rows ii*nv + ab*128 of the
//     chunk's p_ia, B rows qb*128 of the primaries' q.
//   mode 1, (ij|ab): group g (virtual b of the primaries qs[g] .. qs[g]+nq[g]),
//     tile (ab, nb), nb fastest; A rows g*nv + ab*128 of the q_ab slabs, B rows
//     qs[g]*ni + nb*128 of p_{i j_q}, whose rows are grouped the same way and
//     ordered (ii, q) within a group: row qs[g]*ni + ii*nq[g] + (q - qs[g]).
// Rows of a tile past nv (or past the end of a group's columns) read the next
// rows of the operand or zeros; they are not stored.
struct PairTiles {
  int mode, ni, nv, nva, nex, nab, nqb, ngroups;
  int64_t ntiles;
  const int *g_tile0, *g_qs, *g_nq;   // mode 1: tile prefix [ngroups + 1], first primary, count
  const float *a_inv, *b_inv;         // 1 / scale of every A and B operand row

  __device__ __forceinline__ int64_t count() const { return ntiles; }
  __device__ __forceinline__ TcTile at(int64_t t) const {
    TcTile x{};
    if (mode == 0) {
      const int qb = (int)(t % nqb);
      const int64_t r = t / nqb;
      const int ab = (int)(r % nab), ii = (int)(r / nab);
      x.a_y = ii * nv + ab * tc::BM;
      x.b_y = qb * tc::BN;
      x.m_valid = min(tc::BM, nv - ab * tc::BM);
      x.n_valid = min(tc::BN, nex - qb * tc::BN);
      x.out_base = ((int64_t)ii * nex + qb * tc::BN) * nva + ab * tc::BM;
      x.col_stride = nva;
      x.rs = a_inv + x.a_y;
      x.cs = b_inv + x.b_y;
    } else {
      int lo = 0, hi = ngroups;   // g_tile0[lo] <= t < g_tile0[hi]
      while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if ((int64_t)g_tile0[mid] <= t) lo = mid;
        else hi = mid;
      }
      const int g = lo, qs = g_qs[g], ncol = g_nq[g] * ni;
      const int nnb = (ncol + tc::BN - 1) / tc::BN;
      const int local = (int)(t - g_tile0[g]);
      const int ab = local / nnb, nb = local - ab * nnb;
      x.a_y = g * nv + ab * tc::BM;
      x.b_y = qs * ni + nb * tc::BN;
      x.m_valid = min(tc::BM, nv - ab * tc::BM);
      x.n_valid = min(tc::BN, ncol - nb * tc::BN);
      // column n = ii * nq + (q - qs) of the group
      const int nq = g_nq[g], n0 = nb * tc::BN, ii0 = n0 / nq, qq0 = n0 - ii0 * nq;
      x.out_base = ((int64_t)ii0 * nex + qs + qq0) * nva + ab * tc::BM;
      x.col_stride = nva;
      x.run_len = nq;
      x.run_pos = qq0;
      x.run_skip = ((int64_t)nex - (nq - 1)) * nva;
      x.rs = a_inv + x.a_y;
      x.cs = b_inv + x.b_y;
    }
    return x;
  }
};

// ---------------------------------------------------------------- operands
// scaled split of one value: hi + lo ~= s x
__device__ __forceinline__ void split_f16(double x, double sc, __half &hi, __half &lo) {
  const double y = x * sc;
  hi = __double2half(y);
  lo = __double2half(y - (double)__half2float(hi));
}

// Operand rows c = 0..ncols-1: column idx[c] (or c) of an Nk-row FP64 matrix
// (ld), scaled by 1 / inv[c], as FP16 hi / lo rows of Kpad (zero padded).
// One block of 64 threads per row (grid.x = rows, grid.y covers the rest), two
// consecutive elements per thread and step.
constexpr int kSplitThreads = 64;
__global__ void __launch_bounds__(kSplitThreads)
k_split_f16s(__half *__restrict__ hi, __half *__restrict__ lo, const double *__restrict__ src,
             int64_t ld, const int *__restrict__ idx, const float *__restrict__ inv,
             int64_t ncols, int Nk, int Kpad) {
  for (int64_t c = blockIdx.x + (int64_t)blockIdx.y * gridDim.x; c < ncols;
       c += (int64_t)gridDim.x * gridDim.y) {
    const double *x = src + (idx ? (int64_t)idx[c] : c) * ld;
    const double sc = (double)__frcp_rn(inv[c]);   // exact: inv is a power of 2
    __half2 *h2 = reinterpret_cast<__half2 *>(hi + c * Kpad);
    __half2 *l2 = reinterpret_cast<__half2 *>(lo + c * Kpad);
    for (int k2 = threadIdx.x; 2 * k2 < Kpad; k2 += kSplitThreads) {
      const int k = 2 * k2;
      __half a0, a1, b0, b1;
      split_f16(k < Nk ? x[k] : 0.0, sc, a0, b0);
      split_f16(k + 1 < Nk ? x[k + 1] : 0.0, sc, a1, b1);
      h2[k2] = __halves2half2(a0, a1);
      l2[k2] = __halves2half2(b0, b1);
    }
  }
}

// p_{i j_q} for the chunk, scaled, in the row order of the (ij|ab) tiles:
// row qs[g]*ni + ii*nq[g] + (q - qs[g]) for the primaries q of group g
// (source: column (i0 + ii) * no + j_q of Poo, N values); wsc[row] = 1 / scale
__global__ void __launch_bounds__(kSplitThreads)
k_split_wexp(__half *__restrict__ hi, __half *__restrict__ lo, const double *__restrict__ Poo,
             int N, const int *__restrict__ jq, const float *__restrict__ winv, int nex, int ni,
             int i0, int no, int Kpad, const int *__restrict__ g_qs,
             const int *__restrict__ g_nq, int ngroups, float *__restrict__ wsc) {
  const int64_t rows = (int64_t)nex * ni;
  for (int64_t row = blockIdx.x + (int64_t)blockIdx.y * gridDim.x; row < rows;
       row += (int64_t)gridDim.x * gridDim.y) {
    int lo_g = 0, hi_g = ngroups;   // g_qs[lo_g] * ni <= row < g_qs[hi_g] * ni
    while (hi_g - lo_g > 1) {
      const int mid = (lo_g + hi_g) >> 1;
      if ((int64_t)g_qs[mid] * ni <= row) lo_g = mid;
      else hi_g = mid;
    }
    const int qs = g_qs[lo_g], nq = g_nq[lo_g];
    const int rel = (int)(row - (int64_t)qs * ni), ii = rel / nq, q = qs + (rel - ii * nq);
    const int64_t col = (int64_t)(i0 + ii) * no + jq[q];
    const float iv = winv[col];
    const double sc = (double)__frcp_rn(iv);   // exact: iv is a power of 2
    const double *x = Poo + col * N;
    __half2 *h2 = reinterpret_cast<__half2 *>(hi + row * Kpad);
    __half2 *l2 = reinterpret_cast<__half2 *>(lo + row * Kpad);
    for (int k2 = threadIdx.x; 2 * k2 < Kpad; k2 += kSplitThreads) {
      const int k = 2 * k2;
      __half a0, a1, b0, b1;
      split_f16(k < N ? x[k] : 0.0, sc, a0, b0);
      split_f16(k + 1 < N ? x[k + 1] : 0.0, sc, a1, b1);
      h2[k2] = __halves2half2(a0, a1);
      l2[k2] = __halves2half2(b0, b1);
    }
    if (threadIdx.x == 0) wsc[row] = iv;
  }
}

// grid of the split kernels for `rows` operand rows
inline dim3 split_grid(int64_t rows) {
  const int64_t gx = std::min<int64_t>(rows, 65535);
  const int64_t gy = std::min<int64_t>(div_up(rows, gx), 64);
  return dim3((unsigned)gx, (unsigned)gy);
}

// For column x_c = column idx[c] (or c) of an N-row FP64 matrix (one warp per
// column): nrm[c] = ||x_c||_2 rounded up to FP32, inv[c] = 2^(E - 14) with
// max |x_c| < 2^E, so that the scaled operand s x_c (s = 1 / inv) stays below
// 2^14 and well inside the FP16 range.
__global__ void k_colstats(const double *__restrict__ X, int N, const int *__restrict__ idx,
                           int64_t ncols, float *__restrict__ nrm, float *__restrict__ inv) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t c = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; c < ncols; c += nw) {
    const double *x = X + (idx ? (int64_t)idx[c] : c) * N;
    double s = 0.0, mx = 0.0;
    for (int A = lane; A < N; A += 32) {
      s = fma(x[A], x[A], s);
      mx = fmax(mx, fabs(x[A]));
    }
    for (int o = 16; o > 0; o >>= 1) {
      s += __shfl_xor_sync(0xffffffffu, s, o);
      mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    }
    if (lane == 0) {
      // the FP64 sum is exact to ~N eps relative; 1 + 1e-12 covers it
      nrm[c] = __double2float_ru(sqrt(s) * (1.0 + 1e-12));
      int e = 0;
      if (mx > 0.0) frexp(mx, &e);   // mx < 2^e
      e = max(-100, min(100, e));
      inv[c] = ldexpf(1.f, e - 14);
    }
  }
}

// ---------------------------------------------------------------- row pass
// Per-primary data of the passes, in (b, j) order.
struct PtCols {
  const float *eh, *el;   // E_q as a hi/lo FP32 pair
  const float *qn;        // ||q_q||
  const int *jq;          // occupied index j of q
  const int *gq;          // slab (group) index of b_q
};

// inputs of the column pass's error bound: the row pass's norms, with the
// J-side norms replaced by their maxima over the row's occupied partner j
// (wrow) and over the primary's q_ab slab (vmax)
struct PtColBound {
  const float *pn;     // ||p_ia|| of every (i, a)
  const float *qn;     // ||q_q|| of the primaries
  const int *gq;       // slab of each primary
  const float *wrow;   // max_j ||p_ij|| per occupied i
  const float *vmax;   // max_a ||q_ab|| per slab
  float ecoup;
  int i0;
};

constexpr int kRowThreads = 128;
constexpr int kRowStage = 256;   // primaries staged in shared memory at a time
constexpr int kRowBatch = 8;     // primaries whose loads are issued together

// One PT term t = a^2 / (E_r - E_q) in FP32 and the bound on its error:
//   a = ak K - J from the FP32 couplings kv, jv; the coupling error is
//   dn (the Cauchy-Schwarz term e_c (ak |p_r| |q_q| + |p_ij| |q_ab|), formed by
//   the caller) plus the FP32 rounding of a (2 u (ak |kv| + |jv|));
//   den = (rh - eh) + (rl - el) from hi / lo energy pairs, rden its correctly
//   rounded reciprocal; the relative error of rden is ed = 4 u + 3e-14 rden;
//   bound (2 |a| da + da^2) rden + t (2 ed + cr), cr the rounding allowance of
//   the term's products (6 u) and of the caller's FP32 partial sums.
// The bound is used only while den > 0 and ed < 0.25, i.e. 0 < rden < 8.33e12
// (tested as 0 < rden < 8e12; NaN fails the test): otherwise it is infinite.
__device__ __forceinline__ float2 pt_term(float akf, float kv, float jv, float rh, float rl,
                                          float eh, float el, float dn, float cr) {
  const float am = fmaf(akf, kv, -jv);
  const float den = (rh - eh) + (rl - el);
  const float rden = __frcp_rn(den);
  const float tt = am * am * rden;
  const float da = fmaf(2.f * kU32, fmaf(akf, fabsf(kv), fabsf(jv)), dn);
  const float bt = rden > 0.f && rden < 8.0e12f
                       ? fmaf(da * fmaf(2.f, fabsf(am), da), rden,
                              tt * fmaf(6e-14f, rden, cr + 8.f * kU32))
                       : INFINITY;
  return make_float2(tt, bt);
}

// Partial PT sums of the candidate rows (ii, a) over primaries
// [z * qlen, (z + 1) * qlen): part_t[z][ii * nv + a] = sum of the terms,
// part_b[z][...] = bound on the error of that sum.  Terms are formed in FP32
// and summed in groups of kRowBatch before the FP64 accumulation; each group's
// loads are issued before any of its arithmetic (memory-level parallelism).
__global__ void __launch_bounds__(kRowThreads)
k_ptq_rows(const float *__restrict__ K, const float *__restrict__ J, int ni, int nv, int nva,
           int nex, int qlen, int no, int i0, const double *__restrict__ de_all,
           const int *__restrict__ cand_pos, PtCols cols, const float *__restrict__ pn,
           const float *__restrict__ wn, const float *__restrict__ vn, float akf, float ecoup,
           double *__restrict__ part_t, double *__restrict__ part_b, float2 *__restrict__ rhl) {
  // per staged primary: energy hi / lo, |q_q| and e_c |p_{i j_q}| in one vector
  // load, and the offset of its slab's row of vn
  __shared__ float4 s_c[kRowStage];
  __shared__ int s_go[kRowStage];
  const int a = blockIdx.x * kRowThreads + threadIdx.x;
  const int ii = blockIdx.y, z = blockIdx.z;
  const int q0 = z * qlen, q1 = min(nex, q0 + qlen);
  const bool live = a < nv;
  const int al = live ? a : 0;
  const int64_t k = (int64_t)(i0 + ii) * nv + al;
  const double d = de_all[k] + 1e-10;
  const float rh = (float)d, rl = (float)(d - (double)rh);
  if (z == 0 && live) rhl[ii * nv + a] = make_float2(rh, rl);
  const float apr = ecoup * akf * pn[k];   // e_c ak |p_r|
  double acc_t = 0.0, acc_b = 0.0;
  const float *Kp = K + ((int64_t)ii * nex + q0) * nva + al;
  const float *Jp = J + ((int64_t)ii * nex + q0) * nva + al;
  for (int s0 = q0; s0 < q1; s0 += kRowStage) {
    const int ns = min(kRowStage, q1 - s0);
    __syncthreads();
    for (int t = threadIdx.x; t < ns; t += kRowThreads) {
      const int q = s0 + t;
      s_c[t] = make_float4(cols.eh[q], cols.el[q], cols.qn[q],
                           ecoup * wn[(int64_t)(i0 + ii) * no + cols.jq[q]]);
      s_go[t] = cols.gq[q] * nv;
    }
    __syncthreads();
    for (int t0 = 0; t0 < ns; t0 += kRowBatch) {
      float kv[kRowBatch], jv[kRowBatch], vv[kRowBatch];
      float gt = 0.f, gb = 0.f;
      if (t0 + kRowBatch <= ns) {   // a full batch: no guards
#pragma unroll
        for (int u = 0; u < kRowBatch; ++u) {   // all loads of the batch first
          const int t = t0 + u;
          kv[u] = Kp[(int64_t)t * nva];
          jv[u] = Jp[(int64_t)t * nva];
          vv[u] = vn[s_go[t] + al];
        }
#pragma unroll
        for (int u = 0; u < kRowBatch; ++u) {
          const int t = t0 + u;
          const float4 c = s_c[t];
          const float2 r = pt_term(akf, kv[u], jv[u], rh, rl, c.x, c.y,
                                   fmaf(apr, c.z, c.w * vv[u]), 6.f * kU32);
          gt += r.x;
          gb += r.y;
        }
      } else {
        const int nb = ns - t0;
#pragma unroll
        for (int u = 0; u < kRowBatch; ++u) {
          const int t = t0 + (u < nb ? u : 0);
          kv[u] = Kp[(int64_t)t * nva];
          jv[u] = Jp[(int64_t)t * nva];
          vv[u] = vn[s_go[t] + al];
        }
#pragma unroll
        for (int u = 0; u < kRowBatch; ++u) {
          const int t = t0 + (u < nb ? u : 0);
          const float4 c = s_c[t];
          const float2 r = pt_term(akf, kv[u], jv[u], rh, rl, c.x, c.y,
                                   fmaf(apr, c.z, c.w * vv[u]), 6.f * kU32);
          if (u < nb) {
            gt += r.x;
            gb += r.y;
          }
        }
      }
      acc_t += (double)gt;
      acc_b += (double)gb;
    }
    Kp += (int64_t)ns * nva;
    Jp += (int64_t)ns * nva;
  }
  if (live) {
    part_t[(int64_t)z * ni * nv + ii * nv + a] = acc_t;
    part_b[(int64_t)z * ni * nv + ii * nv + a] = acc_b;
  }
}

// pert[r] = sum_z part_t (in order), bnd[r] = its error bound, sel[r] =
// pert > thrp, for the candidates of the chunk
__global__ void k_ptq_rows_finish(const double *__restrict__ part_t,
                                  const double *__restrict__ part_b, int nz, int ni, int nv,
                                  int i0, const int *__restrict__ cand_pos, double thrp,
                                  double *__restrict__ pert, double *__restrict__ bnd,
                                  unsigned char *__restrict__ sel) {
  const int64_t n = (int64_t)ni * nv;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int r = cand_pos[(int64_t)i0 * nv + e];
    if (r < 0) continue;
    double t = 0.0, b = 0.0;
    for (int z = 0; z < nz; ++z) {
      t += part_t[(int64_t)z * n + e];
      b += part_b[(int64_t)z * n + e];
    }
    // FP32 group sums of non-negative terms (8 each): <= 8 units of 2^-24;
    // the bound itself was formed in FP32: 0.1 % margin
    b = b * 1.001 + t * 1e-6;
    pert[r] = t;
    bnd[r] = b;
    sel[r] = t > thrp ? 1 : 0;
  }
}

// use[ii * nv + a] = 1 for candidates of the chunk that are not selected
__global__ void k_ptq_use(int ni, int nv, int i0, const int *__restrict__ cand_pos,
                          const unsigned char *__restrict__ sel, unsigned char *__restrict__ use) {
  const int64_t n = (int64_t)ni * nv;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int r = cand_pos[(int64_t)i0 * nv + e];
    use[e] = (r >= 0 && !sel[r]) ? 1 : 0;
  }
}

// ---------------------------------------------------------------- column pass
constexpr int kColQ = 4;     // primaries per block
constexpr int kColRows = 2;  // candidate rows per thread and step (loads issued together)

// colpart[q] = sum over the non-selected candidates (ii, a) of the chunk of
// the terms t_(ii,a),q, for kColQ primaries per block: the block's threads
// walk the chunk's (ii, a) rows (a fastest), kColRows at a time with all their
// loads issued first, terms of rows that are not summed multiplied by zero;
// per-thread FP64 sums, then a fixed-order warp and block reduction
// (deterministic).
__global__ void __launch_bounds__(256, 3)
k_ptq_cols(const float *__restrict__ K, const float *__restrict__ J, int ni, int nv, int nva,
           int nex, const unsigned char *__restrict__ use, const float2 *__restrict__ rhl,
           const float *__restrict__ eh, const float *__restrict__ el, float akf,
           double *__restrict__ colpart, PtColBound cb, double *__restrict__ colbnd) {
  const int q0 = blockIdx.x * kColQ;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float ehq[kColQ], elq[kColQ], qnq[kColQ], vmq[kColQ];
  double acc[kColQ], accb[kColQ];
#pragma unroll
  for (int u = 0; u < kColQ; ++u) {
    const int q = min(q0 + u, nex - 1);
    ehq[u] = eh[q];
    elq[u] = el[q];
    qnq[u] = cb.qn[q];
    vmq[u] = cb.vmax[cb.gq[q]];
    acc[u] = accb[u] = 0.0;
  }
  const int64_t nrow = (int64_t)ni * nv;
  for (int64_t e0 = threadIdx.x; e0 < nrow; e0 += (int64_t)blockDim.x * kColRows) {
    float kv[kColRows][kColQ], jv[kColRows][kColQ], w[kColRows], apr[kColRows], wr[kColRows];
    float2 r[kColRows];
#pragma unroll
    for (int v = 0; v < kColRows; ++v) {   // rows e0, e0 + blockDim, ...: coalesced
      const int64_t ev = e0 + (int64_t)v * blockDim.x;
      const int64_t e = min(ev, nrow - 1);
      const int ii = (int)(e / nv), a = (int)(e - (int64_t)ii * nv);
      w[v] = (ev < nrow && use[e]) ? 1.f : 0.f;
      r[v] = rhl[e];
      apr[v] = cb.ecoup * akf * cb.pn[(int64_t)(cb.i0 + ii) * nv + a];
      wr[v] = cb.ecoup * cb.wrow[cb.i0 + ii];
      const int64_t o = ((int64_t)ii * nex + q0) * nva + a;
#pragma unroll
      for (int u = 0; u < kColQ; ++u) {
        const int64_t ou = q0 + u < nex ? o + (int64_t)u * nva : o;
        kv[v][u] = K[ou];
        jv[v][u] = J[ou];
      }
    }
#pragma unroll
    for (int u = 0; u < kColQ; ++u) {
      float t = 0.f, b = 0.f;
#pragma unroll
      for (int v = 0; v < kColRows; ++v) {
        // the row pass's term bound with the coupling's J norms bounded by
        // their row / slab maxima, plus the FP32 partial sum of kColRows terms
        const float2 tb = pt_term(akf, kv[v][u], jv[v][u], r[v].x, r[v].y, ehq[u], elq[u],
                                  fmaf(apr[v], qnq[u], wr[v] * vmq[u]), (6.f + kColRows) * kU32);
        t = fmaf(w[v], tb.x, t);
        b = fmaf(w[v], tb.y, b);
      }
      acc[u] += (double)t;
      accb[u] += (double)b * (1.0 + 8.0 * kU32);
    }
  }
  __shared__ double red[8][kColQ], redb[8][kColQ];
#pragma unroll
  for (int u = 0; u < kColQ; ++u) {
    double v = acc[u], vb = accb[u];
    for (int o = 16; o > 0; o >>= 1) {
      v += __shfl_xor_sync(0xffffffffu, v, o);
      vb += __shfl_xor_sync(0xffffffffu, vb, o);
    }
    if (lane == 0) {
      red[warp][u] = v;
      redb[warp][u] = vb;
    }
  }
  __syncthreads();
  if (threadIdx.x < kColQ && q0 + (int)threadIdx.x < nex) {
    double v = 0.0, vb = 0.0;
    for (int ww = 0; ww < 8; ++ww) {
      v += red[ww][threadIdx.x];
      vb += redb[ww][threadIdx.x];
    }
    colpart[q0 + threadIdx.x] = v;
    colbnd[q0 + threadIdx.x] = vb;
  }
}

// largest entry of each row of a rows x cols FP32 array (row-major)
__global__ void k_rowmax(const float *__restrict__ x, int64_t rows, int cols,
                         float *__restrict__ out) {
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < rows;
       r += (int64_t)gridDim.x * blockDim.x) {
    float m = 0.f;
    for (int c = 0; c < cols; ++c) m = fmaxf(m, x[r * cols + c]);
    out[r] = m;
  }
}

// per primary: the bound of its PT lowering summed over the chunks; *maxb =
// the largest (bit-pattern max of non-negative doubles)
__global__ void k_pt2_bound_finish(const double *__restrict__ colbnd, int nchunk, int nex,
                                   unsigned long long *__restrict__ maxb) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  double s = 0.0;
  if (c < nex)
    for (int q = 0; q < nchunk; ++q) s += colbnd[(int64_t)q * nex + c];
  s *= 1.001;                   // the terms' bounds were formed in FP32
  if (!(s >= 0.0)) s = 1e300;   // INF / NaN: no usable bound
  for (int o = 16; o > 0; o >>= 1) s = fmax(s, __shfl_xor_sync(0xffffffffu, s, o));
  if ((threadIdx.x & 31) == 0) atomicMax(maxb, (unsigned long long)__double_as_longlong(s));
}

// ---------------------------------------------------------------- FP64 recheck
// FP64 PT sum for candidate rows near the threshold (ptselect stda.f:1805-1834),
// couplings as gathered FP64 dot products over atoms.  Grid (nrc, nsplit):
// block (q, y) sums the primaries c = y*8 + warp, + nsplit*8, ...
// rows r in [r0, r1) whose sum lies within its bound of thrp (|pert - thrp| <=
// bnd, NaN included) are appended to list (count *cnt; the order of the
// entries varies, each row's result does not depend on it)
__global__ void k_pt_recheck_rows(const double *__restrict__ pert, const double *__restrict__ bnd,
                                  int r0, int r1, double thrp, int *__restrict__ list,
                                  int *__restrict__ cnt) {
  for (int r = r0 + blockIdx.x * blockDim.x + threadIdx.x; r < r1; r += gridDim.x * blockDim.x)
    if (!(fabs(pert[r] - thrp) > bnd[r])) list[atomicAdd(cnt, 1)] = r;
}

// FP64 PT sums of the listed rows (*nrc of them; blocks x walk the list)
__global__ void k_pt_recheck(const int *__restrict__ rows, const int *__restrict__ nrc,
                             const int *__restrict__ cand_k,
                             const int *__restrict__ pk, int nex, const double *__restrict__ Pia,
                             const double *__restrict__ Qia, const double *__restrict__ Poo,
                             const double *__restrict__ Qvv, int N, int no, int nv,
                             const double *__restrict__ de_all, const double *__restrict__ ed,
                             double ak, double *__restrict__ part) {
  const int n_rows = *nrc;
  for (int q = blockIdx.x; q < n_rows; q += gridDim.x) {
    int r = rows[q];
    int k = cand_k[r];
    int i = k / nv, a = k - i * nv;
    double de_r = de_all[k];
    const double *pr = Pia + (int64_t)N * k;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarp = blockDim.x >> 5;
    double s = 0.0;   // meaningful in lane 0 of each warp
    for (int c = blockIdx.y * nwarp + warp; c < nex; c += gridDim.y * nwarp) {
      int kc = pk[c];
      int j = kc / nv, b = kc - j * nv;
      const double *qc = Qia + (int64_t)N * kc;
      const double *pij = Poo + (int64_t)N * ((int64_t)i * no + j);
      const double *qab = Qvv + (int64_t)N * ((int64_t)a * nv + b);
      double kv = 0.0, jv = 0.0;
      for (int A = lane; A < N; A += 32) {
        kv += pr[A] * qc[A];
        jv += pij[A] * qab[A];
      }
      for (int o = 16; o > 0; o >>= 1) {
        kv += __shfl_xor_sync(0xffffffffu, kv, o);
        jv += __shfl_xor_sync(0xffffffffu, jv, o);
      }
      double amat = ak * kv - jv;
      s += amat * amat / (de_r - ed[c] + 1e-10);
    }
    __shared__ double red[32];
    if (lane == 0) red[warp] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int w = 0; w < nwarp; ++w) t += red[w];
      part[(int64_t)q * gridDim.y + blockIdx.y] = t;
    }
    __syncthreads();
  }
}

// pert[rows[q]] = sum_y part[q][y] (fixed order); selection pert > thrp
__global__ void k_pt_recheck_finish(const int *__restrict__ rows, const int *__restrict__ nrc,
                                    int nsplit, const double *__restrict__ part, double thrp,
                                    double *__restrict__ pert_out, unsigned char *__restrict__ sel) {
  const int n_rows = *nrc;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n_rows; q += gridDim.x * blockDim.x) {
    double t = 0.0;
    for (int y = 0; y < nsplit; ++y) t += part[(int64_t)q * nsplit + y];
    pert_out[rows[q]] = t;
    sel[rows[q]] = t > thrp ? 1 : 0;
  }
}

// ---------------------------------------------------------------- driver
struct MixedWork {
  TcGemm tc;
  DBuf<__half> q_hi, q_lo, v_hi, v_lo, a_hi, a_lo, w_hi, w_lo;
  DBuf<float> K, J, pn, qn, wn, vn, eh, el, pinv, qinv, winv, vinv, wsc;
  DBuf<float2> rhl;
  DBuf<int> pk, ck, cand_pos, jq, gq, vidx, g_tile0, g_qs, g_nq, recheck;
  DBuf<double> ed, part_t, part_b, bnd, colpart, colbnd, recheck_part, ed_bound;
  DBuf<float> wrow, vmax;
  // bound on max_q |PT-lowered diagonal - its FP64 value| of the last selection
  double ed_bound_max = 0.0;
  DBuf<unsigned char> use;
  double *lastX = nullptr;
  int64_t rechecked = 0;
  double ms = 0, flop = 0;
  int64_t launches = 0;
  // per chunk: events around its two contractions (read after the final
  // synchronisation) and its count of FP64-rechecked rows
  std::vector<cudaEvent_t> tev;
  DBuf<int> recheck_cnt;
  // optional per-step timing (synchronises): operands, (ia|jb), (ij|ab), row
  // pass, FP64 recheck, column pass
  bool profile = false;
  double sec_ms[6] = {0, 0, 0, 0, 0, 0};
  ~MixedWork() {
    for (cudaEvent_t e : tev) cudaEventDestroy(e);
  }
};

// Inputs of one PT selection.  Pair tensors are [pair][atom] FP64 with pair
// index i*nv + a (Pia = gamma^K q_ia, Qia), i*no + j (Poo = gamma^J q_ij) and
// a*nv + b (Qvv); de_all: diagonal of every (i, a) pair.
struct PtProblem {
  int N, no, nv;
  const double *Pia, *Qia, *Poo, *Qvv, *de_all;
  double ak, thrp;
  double budget;   // bytes of chunk buffers
};

// Selection of the candidates ck (pair indices, ascending) against the
// primaries pk_bj (pair indices in (b, j) order, energies ed_bj): sel[r] and
// pert[r] per candidate (device, [ck.size()]), and the lowered primary
// energies edp (device, [pk_bj.size()], same order).
inline void mixed_pt_select(MixedWork &mw, cudaStream_t s, const PtProblem &pb,
                            const std::vector<int> &pk_bj, const std::vector<double> &ed_bj,
                            const std::vector<int> &ck, double *pert, unsigned char *sel,
                            double *pt2, double *edp) {
  const int N = pb.N, no = pb.no, nv = pb.nv;
  const int nex = (int)pk_bj.size(), nexpt = (int)ck.size();
  const int64_t nov = (int64_t)no * nv;
  const int Kpad = (int)div_up(N, tc::BK) * tc::BK;
  const int nva = (int)div_up(nv, 32) * 32;
  const int nab = (int)div_up(nv, tc::BM), nqb = (int)div_up(nex, tc::BN);
  mw.rechecked = 0;
  mw.ms = mw.flop = 0;
  mw.launches = 0;
  for (double &v : mw.sec_ms) v = 0;
  auto t_last = std::chrono::steady_clock::now();
  auto tick = [&](int slot) {
    if (!mw.profile) return;
    S2G_CUDA(cudaStreamSynchronize(s));
    const auto t1 = std::chrono::steady_clock::now();
    mw.sec_ms[slot] += std::chrono::duration<double, std::milli>(t1 - t_last).count();
    t_last = t1;
  };
  auto up = [&](DBuf<int> &b, const std::vector<int> &v) {
    int *d = b.ensure(v.size());
    S2G_CUDA(cudaMemcpyAsync(d, v.data(), sizeof(int) * v.size(), cudaMemcpyHostToDevice, s));
    return d;
  };
  // primaries: occupied index, virtual group (slab), energies as hi/lo pairs
  std::vector<int> jq(nex), gq(nex), VP, qs, nq;
  for (int q = 0; q < nex; ++q) {
    const int b = pk_bj[q] % nv;
    jq[q] = pk_bj[q] / nv;
    if (VP.empty() || VP.back() != b) {
      VP.push_back(b);
      qs.push_back(q);
      nq.push_back(0);
    }
    gq[q] = (int)VP.size() - 1;
    ++nq.back();
  }
  const int ng = (int)VP.size();
  std::vector<float> eh(nex), el(nex);
  for (int q = 0; q < nex; ++q) {
    eh[q] = (float)ed_bj[q];
    el[q] = (float)(ed_bj[q] - (double)eh[q]);
  }
  std::vector<int> cand_pos(nov, -1);
  for (int r = 0; r < nexpt; ++r) cand_pos[ck[r]] = r;
  std::vector<int> vidx((size_t)ng * nv);
  for (int g = 0; g < ng; ++g)
    for (int a = 0; a < nv; ++a) vidx[(size_t)g * nv + a] = VP[g] * nv + a;   // q_ba = q_ab
  int *d_pk = up(mw.pk, pk_bj), *d_ck = up(mw.ck, ck), *d_cpos = up(mw.cand_pos, cand_pos);
  int *d_jq = up(mw.jq, jq), *d_gq = up(mw.gq, gq), *d_vidx = up(mw.vidx, vidx);
  int *d_qs = up(mw.g_qs, qs), *d_nq = up(mw.g_nq, nq);
  double *d_ed = mw.ed.ensure(nex);
  S2G_CUDA(cudaMemcpyAsync(d_ed, ed_bj.data(), sizeof(double) * nex, cudaMemcpyHostToDevice, s));
  float *d_eh = mw.eh.ensure(nex), *d_el = mw.el.ensure(nex);
  S2G_CUDA(cudaMemcpyAsync(d_eh, eh.data(), sizeof(float) * nex, cudaMemcpyHostToDevice, s));
  S2G_CUDA(cudaMemcpyAsync(d_el, el.data(), sizeof(float) * nex, cudaMemcpyHostToDevice, s));

  // norms (error bound) and scales (FP16 split) of every operand vector
  auto stats = [&](DBuf<float> &nrm, DBuf<float> &inv, const double *X, const int *idx,
                   int64_t ncols) {
    float *o = nrm.ensure(ncols), *iv = inv.ensure(ncols);
    const int g = (int)std::min<int64_t>(div_up(ncols * 32, 256), 148 * 64);
    S2G_LAUNCH(k_colstats, g, 256, 0, s, X, N, idx, ncols, o, iv);
  };
  stats(mw.pn, mw.pinv, pb.Pia, nullptr, nov);
  stats(mw.qn, mw.qinv, pb.Qia, d_pk, nex);
  stats(mw.wn, mw.winv, pb.Poo, nullptr, (int64_t)no * no);
  stats(mw.vn, mw.vinv, pb.Qvv, d_vidx, (int64_t)ng * nv);
  const float *d_pn = mw.pn.get(), *d_wn = mw.wn.get(), *d_vn = mw.vn.get();
  float *d_wrow = mw.wrow.ensure(no), *d_vmax = mw.vmax.ensure(std::max(ng, 1));
  S2G_LAUNCH(k_rowmax, (int)div_up(no, 128), 128, 0, s, d_wn, (int64_t)no, no, d_wrow);
  if (ng > 0)
    S2G_LAUNCH(k_rowmax, (int)div_up(ng, 128), 128, 0, s, d_vn, (int64_t)ng, nv, d_vmax);
  // operands shared by all chunks: the primaries' q and the q_ab slabs
  auto split = [&](DBuf<__half> &h, DBuf<__half> &l, const double *src, const int *idx,
                   const float *inv, int64_t ncols) {
    __half *ph = h.ensure((size_t)ncols * Kpad + 64), *pl = l.ensure((size_t)ncols * Kpad + 64);
    S2G_LAUNCH(k_split_f16s, split_grid(ncols), kSplitThreads, 0, s, ph, pl, src, (int64_t)N, idx,
               inv, ncols, N, Kpad);
  };
  split(mw.q_hi, mw.q_lo, pb.Qia, d_pk, mw.qinv.get(), nex);
  split(mw.v_hi, mw.v_lo, pb.Qvv, d_vidx, mw.vinv.get(), (int64_t)ng * nv);
  const float ecoup = coupling_error_bound(Kpad);
  const float akf = (float)pb.ak;
  PtCols cols{d_eh, d_el, mw.qn.get(), d_jq, d_gq};

  // chunk of occupied indices: both coupling buffers, the p_{i j_q} operand
  // and the chunk's p_ia operand per occupied index
  const double per_occ = 8.0 * nex * (double)nva + 4.0 * Kpad * ((double)nex + nv) +
                         16.0 * nv + 24.0 * nv;
  const int occ_chunk = std::max(1, (int)std::min<double>(no, pb.budget / per_occ));
  const int nchunk = (int)div_up(no, occ_chunk);
  double *colpart = mw.colpart.ensure((size_t)nchunk * nex);
  double *colbnd = mw.colbnd.ensure((size_t)nchunk * nex);
  double *bnd = mw.bnd.ensure(std::max(nexpt, 1));
  // rows to recheck, listed on the device per chunk (no host round trip
  // between the chunks)
  int *d_rlist = mw.recheck.ensure(std::max(nexpt, 1));
  int *d_rcnt = mw.recheck_cnt.ensure(nchunk);
  S2G_CUDA(cudaMemsetAsync(d_rcnt, 0, sizeof(int) * nchunk, s));
  const int nsplit_rc = (int)std::max<int64_t>(1, std::min<int64_t>(div_up(nex, 64), 128));
  while (mw.tev.size() < 2 * (size_t)nchunk) {
    cudaEvent_t e;
    S2G_CUDA(cudaEventCreate(&e));
    mw.tev.push_back(e);
  }
  int r_begin = 0;
  for (int ch = 0; ch < nchunk; ++ch) {
    const int i0 = ch * occ_chunk, ni = std::min(occ_chunk, no - i0);
    int r_end = r_begin;
    while (r_end < nexpt && ck[r_end] < (int64_t)(i0 + ni) * nv) ++r_end;
    // operands of the chunk
    const float *a_inv = mw.pinv.get() + (int64_t)i0 * nv;
    split(mw.a_hi, mw.a_lo, pb.Pia + (int64_t)i0 * nv * N, nullptr, a_inv, (int64_t)ni * nv);
    const int64_t rows_w = (int64_t)nex * ni;
    float *wsc = mw.wsc.ensure(rows_w);
    {
      __half *h = mw.w_hi.ensure((size_t)rows_w * Kpad + 64),
             *l = mw.w_lo.ensure((size_t)rows_w * Kpad + 64);
      S2G_LAUNCH(k_split_wexp, split_grid(rows_w), kSplitThreads, 0, s, h, l, pb.Poo, N, d_jq,
                 mw.winv.get(), nex, ni, i0, no, Kpad, d_qs, d_nq, ng, wsc);
    }
    std::vector<int> tile0(ng + 1, 0);
    for (int g = 0; g < ng; ++g)
      tile0[g + 1] = tile0[g] + nab * (int)div_up((int64_t)nq[g] * ni, tc::BN);
    int *d_t0 = up(mw.g_tile0, tile0);
    tick(0);
    const size_t nbuf = (size_t)nex * ni * nva;
    float *K = mw.K.ensure(nbuf), *J = mw.J.ensure(nbuf);
    const double fl = 2.0 * ni * (double)nv * nex * N;
    S2G_CUDA(cudaEventRecord(mw.tev[2 * ch], s));
    PairTiles tk{0,       ni,      nv,      nva,   nex,          nab, nqb, 0,
                 (int64_t)ni * nab * nqb, nullptr, nullptr, nullptr, a_inv, mw.qinv.get()};
    mw.tc.run_direct<PairTiles, true>(s, mw.a_hi.get(), mw.a_lo.get(), (int64_t)ni * nv,
                                      mw.q_hi.get(), mw.q_lo.get(), nex, Kpad, tk, tk.ntiles, K,
                                      fl);
    tick(1);
    PairTiles tj{1,    ni,   nv,   nva,  nex,           nab, 0, ng, (int64_t)tile0[ng],
                 d_t0, d_qs, d_nq, mw.vinv.get(), wsc};
    mw.tc.run_direct<PairTiles, true>(s, mw.v_hi.get(), mw.v_lo.get(), (int64_t)ng * nv,
                                      mw.w_hi.get(), mw.w_lo.get(), rows_w, Kpad, tj, tj.ntiles,
                                      J, fl);
    S2G_CUDA(cudaEventRecord(mw.tev[2 * ch + 1], s));
    tick(2);
    mw.flop += 2 * fl;
    mw.launches += 2;
    // row sums and their bounds
    const int nz = (int)std::max<int64_t>(1, std::min<int64_t>(8, div_up(4 * 148 * 4, (int64_t)ni * nab)));
    const int qlen = (int)div_up(nex, nz);
    double *pt = mw.part_t.ensure((size_t)nz * ni * nv), *pbd = mw.part_b.ensure((size_t)nz * ni * nv);
    float2 *rhl = mw.rhl.ensure((size_t)ni * nv);
    S2G_LAUNCH(k_ptq_rows, dim3((unsigned)nab, (unsigned)ni, (unsigned)nz), kRowThreads, 0, s, K, J,
               ni, nv, nva, nex, qlen, no, i0, pb.de_all, d_cpos, cols, d_pn, d_wn, d_vn, akf,
               ecoup, pt, pbd, rhl);
    const int gfin = (int)std::min<int64_t>(div_up((int64_t)ni * nv, 256), 148 * 16);
    S2G_LAUNCH(k_ptq_rows_finish, gfin, 256, 0, s, pt, pbd, nz, ni, nv, i0, d_cpos, pb.thrp, pert,
               bnd, sel);
    // candidates whose sum lies within its bound of thrp: FP64
    const int nr = r_end - r_begin;
    tick(3);
    if (nr > 0) {
      int *rl = d_rlist + r_begin;
      S2G_LAUNCH(k_pt_recheck_rows, (int)std::min<int64_t>(div_up(nr, 256), 148 * 8), 256, 0, s,
                 pert, bnd, r_begin, r_end, pb.thrp, rl, d_rcnt + ch);
      double *part = mw.recheck_part.ensure((size_t)nr * nsplit_rc);
      const int gq = std::min(nr, 1024);
      S2G_LAUNCH(k_pt_recheck, dim3((unsigned)gq, (unsigned)nsplit_rc), 256, 0, s, rl,
                 d_rcnt + ch, d_ck, d_pk, nex, pb.Pia, pb.Qia, pb.Poo, pb.Qvv, N, no, nv,
                 pb.de_all, d_ed, pb.ak, part);
      S2G_LAUNCH(k_pt_recheck_finish, (int)div_up(std::min(nr, 1024 * 128), 128), 128, 0, s, rl,
                 d_rcnt + ch, nsplit_rc, part, pb.thrp, pert, sel);
    }
    tick(4);
    // column sums over the candidates that stay out
    unsigned char *use = mw.use.ensure((size_t)ni * nv);
    S2G_LAUNCH(k_ptq_use, gfin, 256, 0, s, ni, nv, i0, d_cpos, sel, use);
    const PtColBound cb{d_pn, mw.qn.get(), d_gq, d_wrow, d_vmax, ecoup, i0};
    S2G_LAUNCH(k_ptq_cols, (int)div_up(nex, kColQ), 256, 0, s, K, J, ni, nv, nva, nex, use, rhl,
               d_eh, d_el, akf, colpart + (size_t)ch * nex, cb, colbnd + (size_t)ch * nex);
    tick(5);
    r_begin = r_end;
  }
  mw.tc.check(s);
  S2G_LAUNCH(k_pt2_finish, (int)div_up(nex, 128), 128, 0, s, colpart, nchunk, nex, d_ed, pt2, edp);
  auto *mb = (unsigned long long *)mw.ed_bound.ensure(1);
  S2G_CUDA(cudaMemsetAsync(mb, 0, sizeof(unsigned long long), s));
  S2G_LAUNCH(k_pt2_bound_finish, (int)div_up(nex, 128), 128, 0, s, colbnd, nchunk, nex, mb);
  double h_mb = 0.0;
  std::vector<int> h_cnt(nchunk);
  S2G_CUDA(cudaMemcpyAsync(&h_mb, mb, sizeof(double), cudaMemcpyDeviceToHost, s));
  S2G_CUDA(cudaMemcpyAsync(h_cnt.data(), d_rcnt, sizeof(int) * nchunk, cudaMemcpyDeviceToHost, s));
  S2G_CUDA(cudaStreamSynchronize(s));
  mw.ed_bound_max = h_mb;
  for (int ch = 0; ch < nchunk; ++ch) {
    float tms = 0;
    S2G_CUDA(cudaEventElapsedTime(&tms, mw.tev[2 * ch], mw.tev[2 * ch + 1]));
    mw.ms += tms;
    mw.rechecked += h_cnt[ch];
  }
}

}  // namespace std2g
