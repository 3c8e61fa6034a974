// Mixed-precision form of the PT-selection contractions.
//
// The two coupling contractions of ptselect (stda.f:1812-1819) run on the
// tensor cores with split-BF16 operands (tc_gemm.cuh) into FP32 buffers; the
// selection decision of every candidate whose PT sum lies within a relative
// band of the threshold is re-made in FP64 (k_pt_recheck), so the selected CSF
// set is the one the FP64 arithmetic gives.
#pragma once

#include <cmath>
#include <vector>

#include "common.cuh"
#include "tc_gemm.cuh"

namespace std2g {

constexpr double kRecheckBand = 2e-4;   // relative band around thrp decided in FP64

struct MixedWork {
  TcGemm tc;
  DBuf<__nv_bfloat16> bq_hi, bq_lo, bv_hi, bv_lo, a_hi, a_lo, w_hi, w_lo;
  DBuf<float> K, J;
  DBuf<int> recheck;
  DBuf<double> recheck_part;
  DBuf<int64_t> jcol, roff;
  DBuf<float> eh, el, rhl;
  double *lastX = nullptr;
  int Kpad = 0;
  int64_t ldK = 0, ldJ = 0;
  int64_t rechecked = 0;
};

inline int64_t round_up4(int64_t x) { return (x + 3) / 4 * 4; }

inline void split_operand(MixedWork &mw, cudaStream_t s, DBuf<__nv_bfloat16> &h,
                          DBuf<__nv_bfloat16> &l, const double *src, int N, int64_t ncols) {
  const int Kp = mw.Kpad;
  __nv_bfloat16 *ph = h.ensure((size_t)ncols * Kp), *pl = l.ensure((size_t)ncols * Kp);
  int64_t tot = ncols * Kp;
  int g = (int)std::min<int64_t>(div_up(tot, 256), 148 * 32);
  S2G_LAUNCH(k_split_bf16, g, 256, 0, s, ph, pl, src, (int64_t)N, (const int *)nullptr, ncols, N,
             Kp);
}

// B operands of the PT contractions, once per solve: primaries' q (nex x N)
// and the virtual-pair factor q_ab for b in the primaries' virtual set.
inline void mixed_pt_prepare(MixedWork &mw, cudaStream_t s, const double *Qp, const double *QvvP,
                             int N, int nex, int64_t nvcols) {
  mw.Kpad = (int)div_up(N, 64) * 64;
  split_operand(mw, s, mw.bq_hi, mw.bq_lo, Qp, N, nex);
  split_operand(mw, s, mw.bv_hi, mw.bv_lo, QvvP, N, nvcols);
  mw.ldK = round_up4(nex);
  mw.ldJ = round_up4(nvcols);
}

// One candidate chunk: K[r, c] = p_r . q_c  (nr x nex) and the J box
// J[(i,j), (a,b)] = p_ij . q_ab  ((ni*nop) x (nv*nvp)).
inline void mixed_pt_chunk(MixedWork &mw, cudaStream_t s, const double *Pc, const double *W, int N,
                           int nex, int nr, int64_t nvcols, int nwcols) {
  const int Kp = mw.Kpad;
  split_operand(mw, s, mw.a_hi, mw.a_lo, Pc, N, nr);
  split_operand(mw, s, mw.w_hi, mw.w_lo, W, N, nwcols);
  float *K = mw.K.ensure((size_t)nr * mw.ldK);
  float *J = mw.J.ensure((size_t)nwcols * mw.ldJ);
  const int maxrows = 65535 * tc::BM;   // grid y extent of one launch
  for (int r0 = 0; r0 < nr; r0 += maxrows) {
    int rr = std::min(maxrows, nr - r0);
    mw.tc.run(s, mw.a_hi.get() + (size_t)r0 * Kp, mw.a_lo.get() + (size_t)r0 * Kp, mw.bq_hi.get(),
              mw.bq_lo.get(), rr, nex, Kp, K + (size_t)r0 * mw.ldK, mw.ldK,
              2.0 * rr * (double)nex * N);
  }
  for (int r0 = 0; r0 < nwcols; r0 += maxrows) {
    int rr = std::min(maxrows, nwcols - r0);
    mw.tc.run(s, mw.w_hi.get() + (size_t)r0 * Kp, mw.w_lo.get() + (size_t)r0 * Kp, mw.bv_hi.get(),
              mw.bv_lo.get(), rr, (int)nvcols, Kp, J + (size_t)r0 * mw.ldJ, mw.ldJ,
              2.0 * rr * (double)nvcols * N);
  }
}

// ---- PT sums over the FP32 coupling buffers (mixed form) ----
// The couplings K, J carry the split-BF16 GEMM's ~1e-6 relative error, so the
// terms (ak K - J)^2 / (E_r - E_c) are evaluated in FP32 and summed in FP64.
// The energy difference of a candidate r and a primary c, which can cancel,
// is formed from hi/lo FP32 pairs: (rh_r - eh_c) + (rl_r - el_c) keeps ~1e-7
// relative accuracy.  Rows whose sum lands near thrp are re-decided in FP64
// (k_pt_recheck), so the selection is the FP64 one.

// Per primary c (PT order): J column offset and its energy as a hi/lo pair.
// Entries nex <= c < ncol (padding to a multiple of 4) get offset 0 and zero
// energies, so vector loads past the end stay in bounds.
__global__ void k_pt_colinfo(int nex, int ncol, const int *__restrict__ pj,
                             const int *__restrict__ pb, const int *__restrict__ omap,
                             const int *__restrict__ vmap, int64_t ldj,
                             const double *__restrict__ ed, int64_t *__restrict__ jcol,
                             float *__restrict__ eh, float *__restrict__ el) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncol) return;
  if (c >= nex) {
    jcol[c] = 0;
    eh[c] = 0.f;
    el[c] = 0.f;
    return;
  }
  jcol[c] = (int64_t)vmap[pb[c]] + ldj * (int64_t)omap[pj[c]];
  double e = ed[c];
  float h = (float)e;
  eh[c] = h;
  el[c] = (float)(e - (double)h);
}

__device__ __forceinline__ float pt_term32(float kv, float jv, float akf, float rh, float rl,
                                           float ehc, float elc) {
  float amat = akf * kv - jv;
  float den = (rh - ehc) + (rl - elc);
  return __fdividef(amat * amat, den);
}

// Row pass, one warp per candidate row: pert[r] = sum_c term(r, c) and
// sel[r] = pert > thrp; also the row's J offset and energy pair for the column
// pass.  Each lane takes 4 consecutive primaries per step (float4 loads of K,
// ldk a multiple of 4); per-lane partial sums are reduced in a fixed order.
constexpr int kRowWarps = 8;
__global__ void __launch_bounds__(256)
k_pt_rows32(const float *__restrict__ K, const float *__restrict__ J, int64_t ldj, int64_t ldk,
            int nex, int nvp, int nop, int nrows, const int *__restrict__ cand_k, int nv, int i0,
            const double *__restrict__ de_all, const int64_t *__restrict__ jcol,
            const float *__restrict__ eh, const float *__restrict__ el, float akf, double thrp,
            double *__restrict__ pert_out, unsigned char *__restrict__ sel,
            int64_t *__restrict__ roff, float *__restrict__ rhl) {
  const int lane = threadIdx.x & 31;
  const int r = blockIdx.x * kRowWarps + (threadIdx.x >> 5);
  if (r >= nrows) return;
  const int k = cand_k[r];
  const int i = k / nv, a = k - i * nv;
  const int64_t off = (int64_t)a * nvp + ldj * (int64_t)(i - i0) * nop;
  const double d = de_all[k] + 1e-10;
  const float rh = (float)d, rl = (float)(d - (double)rh);
  if (lane == 0) {
    roff[r] = off;
    rhl[2 * r] = rh;
    rhl[2 * r + 1] = rl;
  }
  const float *Kr = K + (int64_t)r * ldk;
  double acc = 0.0;
#pragma unroll 2
  for (int c = lane * 4; c < nex; c += 128) {
    const float4 kv = *reinterpret_cast<const float4 *>(Kr + c);
    const longlong2 j01 = *reinterpret_cast<const longlong2 *>(jcol + c);
    const longlong2 j23 = *reinterpret_cast<const longlong2 *>(jcol + c + 2);
    const float4 e_h = *reinterpret_cast<const float4 *>(eh + c);
    const float4 e_l = *reinterpret_cast<const float4 *>(el + c);
    const float jv0 = J[off + j01.x], jv1 = J[off + j01.y], jv2 = J[off + j23.x],
                jv3 = J[off + j23.y];
    float t = pt_term32(kv.x, jv0, akf, rh, rl, e_h.x, e_l.x);
    if (c + 1 < nex) t += pt_term32(kv.y, jv1, akf, rh, rl, e_h.y, e_l.y);
    if (c + 2 < nex) t += pt_term32(kv.z, jv2, akf, rh, rl, e_h.z, e_l.z);
    if (c + 3 < nex) t += pt_term32(kv.w, jv3, akf, rh, rl, e_h.w, e_l.w);
    acc += (double)t;
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (lane == 0) {
    pert_out[r] = acc;
    sel[r] = acc > thrp ? 1 : 0;
  }
}

// Column pass: colpart[y*nex + c] = sum over the non-selected rows of segment y
// (in row order) of term(r, c).  Rows are taken 8 at a time with all loads
// issued before the arithmetic.
constexpr int kColUnroll = 8;
__global__ void __launch_bounds__(128)
k_pt_cols32(const float *__restrict__ K, const float *__restrict__ J, int64_t ldk, int nex,
            int nrows, const int64_t *__restrict__ jcol, const float *__restrict__ eh,
            const float *__restrict__ el, float akf, const unsigned char *__restrict__ sel,
            const int64_t *__restrict__ roff, const float *__restrict__ rhl,
            double *__restrict__ colpart, int seg_rows) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nex) return;
  const int rbeg = blockIdx.y * seg_rows;
  const int rend = min(nrows, rbeg + seg_rows);
  const int64_t jc = jcol[c];
  const float ehc = eh[c], elc = el[c];
  double s = 0.0;
  for (int r = rbeg; r < rend; r += kColUnroll) {
    float kv[kColUnroll], jv[kColUnroll];
    bool use[kColUnroll];
#pragma unroll
    for (int q = 0; q < kColUnroll; ++q) {
      const int rr = r + q;
      use[q] = rr < rend && !sel[rr];
      kv[q] = 0.f;
      jv[q] = 0.f;
      if (use[q]) {
        kv[q] = K[(int64_t)rr * ldk + c];
        jv[q] = J[roff[rr] + jc];
      }
    }
    float t = 0.f;
#pragma unroll
    for (int q = 0; q < kColUnroll; ++q)
      if (use[q])
        t += pt_term32(kv[q], jv[q], akf, rhl[2 * (r + q)], rhl[2 * (r + q) + 1], ehc, elc);
    s += (double)t;
  }
  colpart[(int64_t)blockIdx.y * nex + c] = s;
}

// FP64 PT sum for candidate rows near the threshold (ptselect stda.f:1805-1834),
// one block per row, couplings as gathered FP64 dot products over atoms.
__global__ void k_pt_recheck(const int *__restrict__ rows, int nrc, const int *__restrict__ cand_k,
                             const int *__restrict__ pk, int nex, const double *__restrict__ Pia,
                             const double *__restrict__ Qia, const double *__restrict__ Poo,
                             const double *__restrict__ Qvv, int N, int no, int nv,
                             const double *__restrict__ de_all, const double *__restrict__ ed,
                             double ak, double *__restrict__ part) {
  // grid (nrc, nsplit): block (q, y) sums couplings c = y*8 + warp (+ nsplit*8 ...)
  int q = blockIdx.x;
  if (q >= nrc) return;
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
}

// pert[rows[q]] = sum_y part[q][y] (fixed order); selection pert > thrp
__global__ void k_pt_recheck_finish(const int *__restrict__ rows, int nrc, int nsplit,
                                    const double *__restrict__ part, double thrp,
                                    double *__restrict__ pert_out, unsigned char *__restrict__ sel) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nrc) return;
  double t = 0.0;
  for (int y = 0; y < nsplit; ++y) t += part[(int64_t)q * nsplit + y];
  pert_out[rows[q]] = t;
  sel[rows[q]] = t > thrp ? 1 : 0;
}

// Rows whose mixed-precision PT sum lies within kRecheckBand of thrp get their
// decision from FP64 arithmetic.
inline void mixed_pt_recheck(MixedWork &mw, cudaStream_t s, double *pert, unsigned char *sel,
                             int nr, double thrp, const int *cand_k, const int *pk, int nex,
                             const double *Pia, const double *Qia, const double *Poo,
                             const double *Qvv, int N, int no, int nv, const double *de_all,
                             const double *ed, double ak) {
  std::vector<double> h(nr);
  S2G_CUDA(cudaMemcpyAsync(h.data(), pert, sizeof(double) * nr, cudaMemcpyDeviceToHost, s));
  S2G_CUDA(cudaStreamSynchronize(s));
  std::vector<int> rows;
  for (int r = 0; r < nr; ++r)
    if (std::fabs(h[r] - thrp) <= kRecheckBand * thrp) rows.push_back(r);
  if (rows.empty()) return;
  int *d = mw.recheck.ensure(rows.size());
  S2G_CUDA(cudaMemcpyAsync(d, rows.data(), sizeof(int) * rows.size(), cudaMemcpyHostToDevice, s));
  const int nrc = (int)rows.size();
  const int nsplit = (int)std::max<int64_t>(1, std::min<int64_t>(div_up(nex, 64), 128));
  double *part = mw.recheck_part.ensure((size_t)nrc * nsplit);
  S2G_LAUNCH(k_pt_recheck, dim3((unsigned)nrc, (unsigned)nsplit), 256, 0, s, d, nrc, cand_k, pk,
             nex, Pia, Qia, Poo, Qvv, N, no, nv, de_all, ed, ak, part);
  S2G_LAUNCH(k_pt_recheck_finish, (int)div_up(nrc, 128), 128, 0, s, d, nrc, nsplit, part, thrp,
             pert, sel);
  mw.rechecked += (int64_t)rows.size();
}

}  // namespace std2g
