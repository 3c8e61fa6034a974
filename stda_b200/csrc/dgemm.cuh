// FP64 matrix products of the engine: C = alpha op(A) op(B) + beta C,
// column-major, op = N or T, optionally batched with fixed strides.
//
// B200 has no FP64 kind of tcgen05; its FP64 tensor path is the warp-level
// DMMA (mma.sync m8n8k4 .f64).  Each CTA (4 warps) computes a 64 x 128 tile
// of C over a K range in steps of 16: the A (64 x 16) and B (16 x 128) tiles
// arrive by 8-byte cp.async in a 4-stage shared-memory ring (three tiles in
// flight while one is multiplied), kept in the global layout's fast order and
// XOR-swizzled so that the fragment reads are conflict-free, and each warp
// owns a 32 x 64 sub-tile = 4 x 8 DMMA tiles (64 accumulators per thread, so
// that an accumulator is reused only every 32 DMMAs).
//
// Tall-skinny products (the Davidson projections V^T W: 300 x 75 outputs over
// 5e4-long sums) split K across CTAs.  The partial tiles go to a workspace and
// a second kernel adds them in a fixed order, so every result is bit-for-bit
// reproducible from run to run (no atomics).  With beta = 0, C is not read.
#pragma once

#include <cublas_v2.h>

#include <vector>

#include "common.cuh"

namespace std2g {

namespace dg {
constexpr int BM = 64, BK = 16, THREADS = 128, STAGES = 4;
constexpr int TILE_A = BM * BK;                              // doubles per A tile
template <int BN> __host__ __device__ constexpr int stage_doubles() { return TILE_A + BN * BK; }
// 64 x 32 tiles: 48 KB (four CTAs per SM); 64 x 64: 64 KB (three); 64 x 128: 96 KB (two)
template <int BN> __host__ __device__ constexpr int smem_bytes() { return STAGES * stage_doubles<BN>() * 8; }
// Shared-memory positions, XOR-swizzled so that the fragment reads of a half
// warp (g = 0..3 along m or n, t = 0..3 along k) hit 16 distinct 8-byte banks:
// operand stored with m (or n) fastest, [BK][W]:
template <int W>
__device__ __forceinline__ int pos_mfast(int k, int m) { return k * W + (m ^ ((k & 3) << 2)); }
// operand stored with k fastest, [rows][BK]:
__device__ __forceinline__ int pos_kfast(int m, int k) { return m * 16 + (k ^ ((m & 3) << 2)); }
}

// D (8x8) += A (8x4, row) * B (4x8, col), FP64.  Fragments: a = A[g][t],
// b = B[t][g], d = {D[g][2t], D[g][2t+1]} with g = lane / 4, t = lane % 4.
__device__ __forceinline__ void dmma_8x8x4(double &d0, double &d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// 8-byte asynchronous global -> shared copy; ok = false fills zeros
__device__ __forceinline__ void cp_async8(double *dst, const double *src, bool ok) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(d), "l"(src),
               "r"(ok ? 8 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Main loop of one CTA tile: acc = op(A) op(B) over the K range [kb, ke) for
// the 64 x BN tile of C at (m0, n0), shared by the strided-batch kernel
// k_dgemm and the grouped kernel k_dgemm_grouped.
// A tiles are kept in the global layout's fast order: m fastest for op(A) = A
// ([k][m]), k fastest for op(A) = A^T ([m][k]); B tiles k fastest for
// op(B) = B ([n][k]), n fastest for op(B) = B^T ([k][n]); swizzled (pos_*).
// CTA tile 64 x BN (BN = 32, 64, 128); warp w owns rows 32 (w & 1) .. +32 and
// columns (BN / 2)(w >> 1) .. +BN / 2: 4 x BN / 16 DMMA tiles.
template <bool TA, bool TB, int BN>
__device__ __forceinline__ void dgemm_mainloop(int M, int N, const double *__restrict__ A,
                                               int64_t lda, const double *__restrict__ B,
                                               int64_t ldb, int m0, int n0, int kb, int ke,
                                               double *smem_d, double (&acc)[4][BN / 16][2]) {
  using namespace dg;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  constexpr int NJ = BN / 16, STAGE = stage_doubles<BN>(), TILE_B = BN * BK;
  const int wm = (warp & 1) * 32, wn = (warp >> 1) * (BN / 2);
  auto As = [&](int st) { return smem_d + (size_t)st * STAGE; };
  auto Bs = [&](int st) { return smem_d + (size_t)st * STAGE + TILE_A; };

  // issue the copies of the K tile starting at k0 into stage st; element q of
  // this thread is idx = tid + 128 q, so along the tile's slow dimension it
  // moves by a fixed stride and one source pointer per operand serves all q
  auto issue = [&](int st, int k0) {
    double *a = As(st), *b = Bs(st);
    if (!TA) {   // m fastest: m = tid % 64, k = tid / 64 + 2 q
      const int m = tid & 63, kq = tid >> 6;
      const bool okm = m0 + m < M;
      const double *src = A + (m0 + m) + (int64_t)(k0 + kq) * lda;
#pragma unroll
      for (int q = 0; q < TILE_A / THREADS; ++q) {
        const int k = kq + 2 * q;
        const bool ok = okm && k0 + k < ke;
        cp_async8(a + pos_mfast<BM>(k, m), ok ? src + (int64_t)(2 * q) * lda : A, ok);
      }
    } else {     // k fastest: k = tid % 16, m = tid / 16 + 8 q
      const int k = tid & 15, mq = tid >> 4;
      const bool okk = k0 + k < ke;
      const double *src = A + (k0 + k) + (int64_t)(m0 + mq) * lda;
#pragma unroll
      for (int q = 0; q < TILE_A / THREADS; ++q) {
        const int m = mq + 8 * q;
        const bool ok = okk && m0 + m < M;
        cp_async8(a + pos_kfast(m, k), ok ? src + (int64_t)(8 * q) * lda : A, ok);
      }
    }
    if (!TB) {   // k fastest: k = tid % 16, n = tid / 16 + 8 q
      const int k = tid & 15, nq = tid >> 4;
      const bool okk = k0 + k < ke;
      const double *src = B + (k0 + k) + (int64_t)(n0 + nq) * ldb;
#pragma unroll
      for (int q = 0; q < TILE_B / THREADS; ++q) {
        const int n = nq + 8 * q;
        const bool ok = okk && n0 + n < N;
        cp_async8(b + pos_kfast(n, k), ok ? src + (int64_t)(8 * q) * ldb : B, ok);
      }
    } else {     // n fastest: n = tid % BN, k = tid / BN + (128 / BN) q
      constexpr int KS = THREADS / BN;
      const int n = tid & (BN - 1), kq = tid / BN;
      const bool okn = n0 + n < N;
      const double *src = B + (n0 + n) + (int64_t)(k0 + kq) * ldb;
#pragma unroll
      for (int q = 0; q < TILE_B / THREADS; ++q) {
        const int k = kq + KS * q;
        const bool ok = okn && k0 + k < ke;
        cp_async8(b + pos_mfast<BN>(k, n), ok ? src + (int64_t)(KS * q) * ldb : B, ok);
      }
    }
  };

#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < NJ; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

  const int nt = ke > kb ? (ke - kb + BK - 1) / BK : 0;
#pragma unroll
  for (int p = 0; p < STAGES - 1; ++p) {
    if (p < nt) issue(p, kb + p * BK);
    cp_async_commit();
  }
  for (int it = 0; it < nt; ++it) {
    cp_async_wait<STAGES - 2>();
    __syncthreads();
    {
      const int nx = it + STAGES - 1;
      if (nx < nt) issue(nx % STAGES, kb + nx * BK);
      cp_async_commit();
    }
    const double *a = As(it % STAGES), *b = Bs(it % STAGES);
#pragma unroll
    for (int ks = 0; ks < BK; ks += 4) {
      double fa[4], fb[NJ];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int m = wm + 8 * i + g, k = ks + t;
        fa[i] = TA ? a[pos_kfast(m, k)] : a[pos_mfast<BM>(k, m)];
      }
#pragma unroll
      for (int j = 0; j < NJ; ++j) {
        const int n = wn + 8 * j + g, k = ks + t;
        fb[j] = TB ? b[pos_mfast<BN>(k, n)] : b[pos_kfast(n, k)];
      }
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < NJ; ++j) dmma_8x8x4(acc[i][j][0], acc[i][j][1], fa[i], fb[j]);
    }
  }
  cp_async_wait<0>();
}

// blockIdx.x: tile of C (m fastest); blockIdx.y: batch * ksplit + split.
// Each split covers K range [split * kchunk, min(K, (split + 1) * kchunk)).
// ksplit == 1: C = alpha acc + beta C;  else work[(b * ksplit + split)][m + n M] = acc.
template <bool TA, bool TB, int BN>
__global__ void __launch_bounds__(dg::THREADS, BN == 32 ? 4 : (BN == 64 ? 3 : 2))
    k_dgemm(int M, int N, int K, double alpha, const double *__restrict__ A, int64_t lda,
            int64_t sA, const double *__restrict__ B, int64_t ldb, int64_t sB, double beta,
            double *__restrict__ C, int64_t ldc, int64_t sC, int ksplit, int kchunk,
            double *__restrict__ work, int tri) {
  using namespace dg;
  extern __shared__ __align__(16) double smem_d[];
  const int tiles_m = (M + BM - 1) / BM;
  const int m0 = (blockIdx.x % tiles_m) * BM, n0 = (blockIdx.x / tiles_m) * BN;
  // tri > 0: column n is the pair (i, j) = (n / tri, n % tri) of a symmetric
  // pair array and only j <= i is wanted: a tile whose columns all lie above
  // the diagonal is skipped (the caller mirrors those columns)
  if (tri > 0) {
    const int i0 = n0 / tri, i1 = min(N - 1, n0 + BN - 1) / tri;
    if (i0 == i1 && n0 - i0 * tri > i0) return;
  }
  const int batch = blockIdx.y / ksplit, split = blockIdx.y % ksplit;
  const int kb = split * kchunk, ke = min(K, kb + kchunk);
  A += batch * sA;
  B += batch * sB;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  constexpr int NJ = BN / 16;
  const int wm = (warp & 1) * 32, wn = (warp >> 1) * (BN / 2);
  double acc[4][NJ][2];
  dgemm_mainloop<TA, TB, BN>(M, N, A, lda, B, ldb, m0, n0, kb, ke, smem_d, acc);

  // epilogue: element (i, j, e) of this thread is C[m0 + wm + 8 i + g][n0 + wn + 8 j + 2 t + e]
  if (ksplit == 1) {
    C += batch * sC;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int row = m0 + wm + 8 * i + g;
      if (row >= M) continue;
#pragma unroll
      for (int j = 0; j < NJ; ++j)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int col = n0 + wn + 8 * j + 2 * t + e;
          if (col >= N) continue;
          double *p = C + row + (int64_t)col * ldc;
          const double v = alpha * acc[i][j][e];
          *p = beta == 0.0 ? v : v + beta * *p;
        }
    }
  } else {
    double *wp = work + (int64_t)blockIdx.y * M * N;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int row = m0 + wm + 8 * i + g;
      if (row >= M) continue;
#pragma unroll
      for (int j = 0; j < NJ; ++j)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int col = n0 + wn + 8 * j + 2 * t + e;
          if (col < N) wp[row + (int64_t)col * M] = acc[i][j][e];
        }
    }
  }
}

// C = alpha sum_s work[b][s] + beta C, splits added in order 0, 1, ...
__global__ void k_dgemm_reduce(int M, int N, int batch, int ksplit, double alpha,
                               const double *__restrict__ work, double beta,
                               double *__restrict__ C, int64_t ldc, int64_t sC) {
  const int64_t mn = (int64_t)M * N, total = mn * batch;
  for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < total;
       x += (int64_t)gridDim.x * blockDim.x) {
    const int64_t b = x / mn, r = x - b * mn;
    const int64_t col = r / M, row = r - col * M;
    const double *w = work + b * ksplit * mn + r;
    double s = 0.0;
    for (int q = 0; q < ksplit; ++q) s += w[q * mn];
    double *p = C + b * sC + row + col * ldc;
    *p = beta == 0.0 ? alpha * s : alpha * s + beta * *p;
  }
}

// One member of a grouped launch: C = alpha op(A) op(B) + beta C with op(A)
// M x K and op(B) K x N (column-major; beta = 0: C is not read).
struct DgProblem {
  int M, N, K;
  double alpha, beta;
  const double *A, *B;
  double *C;
  int64_t lda, ldb, ldc;
  int ks = 1;          // K splits (set by Dgemm::grouped)
  int64_t woff = 0;    // the member's partial tiles in the workspace (ks > 1)
};

// Products of different shapes and operands in one launch (one op(A), op(B)
// and tile width for all): blockIdx.x runs over the tiles of every member,
// member p owning tiles [tile0[p], tile0[p + 1]) (m fastest, then the K
// split); a binary search maps the CTA to its member.  A member with ks > 1
// splits K into ks ranges whose partial tiles go to work + woff and are added
// in split order by k_dgemm_grouped_reduce (deterministic, no atomics).
template <bool TA, bool TB, int BN>
__global__ void __launch_bounds__(dg::THREADS, BN == 32 ? 4 : (BN == 64 ? 3 : 2))
    k_dgemm_grouped(const DgProblem *__restrict__ probs, const int *__restrict__ tile0,
                    int nprob, double *__restrict__ work) {
  using namespace dg;
  extern __shared__ __align__(16) double smem_d[];
  const int tb = blockIdx.x;
  int lo = 0, hi = nprob;   // tile0[lo] <= tb < tile0[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (tile0[mid] <= tb) lo = mid;
    else hi = mid;
  }
  const DgProblem pr = probs[lo];
  const int tiles_m = (pr.M + BM - 1) / BM, tiles_mn = tiles_m * ((pr.N + BN - 1) / BN);
  const int local = (tb - tile0[lo]) % tiles_mn, split = (tb - tile0[lo]) / tiles_mn;
  const int m0 = (local % tiles_m) * BM, n0 = (local / tiles_m) * BN;
  const int kchunk = (((pr.K + pr.ks - 1) / pr.ks + BK - 1) / BK) * BK;
  const int kb = split * kchunk, ke = min(pr.K, kb + kchunk);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  constexpr int NJ = BN / 16;
  const int wm = (warp & 1) * 32, wn = (warp >> 1) * (BN / 2);
  double acc[4][NJ][2];
  dgemm_mainloop<TA, TB, BN>(pr.M, pr.N, pr.A, pr.lda, pr.B, pr.ldb, m0, n0, kb, ke, smem_d,
                             acc);
  double *wp = work + pr.woff + (int64_t)split * pr.M * pr.N;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int row = m0 + wm + 8 * i + g;
    if (row >= pr.M) continue;
#pragma unroll
    for (int j = 0; j < NJ; ++j)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int col = n0 + wn + 8 * j + 2 * t + e;
        if (col >= pr.N) continue;
        if (pr.ks > 1) {
          wp[row + (int64_t)col * pr.M] = acc[i][j][e];
        } else {
          double *p = pr.C + row + (int64_t)col * pr.ldc;
          const double v = pr.alpha * acc[i][j][e];
          *p = pr.beta == 0.0 ? v : v + pr.beta * *p;
        }
      }
  }
}

// C = alpha sum_s work[woff + s M N] + beta C for the members with ks > 1
// (blockIdx.y = member), splits added in order 0, 1, ...
__global__ void k_dgemm_grouped_reduce(const DgProblem *__restrict__ probs,
                                       const double *__restrict__ work) {
  const DgProblem pr = probs[blockIdx.y];
  if (pr.ks <= 1) return;
  const int64_t mn = (int64_t)pr.M * pr.N;
  for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < mn;
       x += (int64_t)gridDim.x * blockDim.x) {
    const double *w = work + pr.woff + x;
    double s = 0.0;
    for (int q = 0; q < pr.ks; ++q) s += w[q * mn];
    const int64_t col = x / pr.M, row = x - col * pr.M;
    double *p = pr.C + row + col * pr.ldc;
    *p = pr.beta == 0.0 ? pr.alpha * s : pr.alpha * s + pr.beta * *p;
  }
}

// Launch wrapper with the split-K workspace.
struct Dgemm {
  DBuf<double> work;
  int nsm = 148;
  int64_t launches = 0;
  // set: the products go to cuBLAS on this handle instead (the library
  // baseline of the plain FP64 form, STD2G_FLAG_LIBRARY_FP64)
  cublasHandle_t lib = nullptr;
  // per-product device time (an event pair around each product) and the
  // algorithmic FLOPs 2 m n k of the products since the last reset()
  bool timed = false;
  std::vector<cudaEvent_t> ev;
  size_t nev = 0;
  double flop = 0;
  int64_t calls = 0;
  ~Dgemm() {
    for (cudaEvent_t e : ev) cudaEventDestroy(e);
  }
  void reset() {
    nev = 0;
    flop = 0;
    calls = 0;
  }
  // device time of the timed products since reset(); the stream must have
  // passed them (the caller synchronises first)
  double elapsed_ms() const {
    double ms = 0;
    for (size_t q = 0; q + 1 < nev; q += 2) {
      float t = 0;
      if (cudaEventElapsedTime(&t, ev[q], ev[q + 1]) == cudaSuccess) ms += t;
    }
    return ms;
  }
  void mark(cudaStream_t s) {
    if (nev == ev.size()) {
      cudaEvent_t e;
      S2G_CUDA(cudaEventCreate(&e));
      ev.push_back(e);
    }
    S2G_CUDA(cudaEventRecord(ev[nev++], s));
  }

  // grouped launch (k_dgemm_grouped, 64 x 32 tiles) of the members with a
  // non-empty output; the descriptors go to `gdesc` / `gtile0` (same stream:
  // a later launch's upload waits for this launch), from `stage` when given
  DBuf<DgProblem> gdesc;
  DBuf<int> gtile0;
  DBuf<double> gwork;   // partial tiles of the split members
  void grouped(cudaStream_t s, bool ta, bool tb, const std::vector<DgProblem> &in,
               PinnedArena *stage = nullptr) {
    std::vector<DgProblem> pr;
    std::vector<int> t0(1, 0);
    int64_t wtot = 0;
    int64_t mnmax = 0;
    for (DgProblem q : in) {
      if (q.M <= 0 || q.N <= 0) continue;
      // long sums over few output tiles (the Davidson's projections, A V of
      // a small block) split K: at least 256 per split, about 128 CTAs
      const int64_t tmn = div_up(q.M, dg::BM) * div_up(q.N, 32);
      q.ks = (int)std::max<int64_t>(
          1, std::min<int64_t>({32, q.K / 256, std::max<int64_t>(1, 128 / tmn)}));
      q.woff = wtot;
      if (q.ks > 1) wtot += (int64_t)q.ks * q.M * q.N;
      mnmax = std::max<int64_t>(mnmax, (int64_t)q.M * q.N);
      pr.push_back(q);
      t0.push_back(t0.back() + (int)(tmn * q.ks));
      flop += 2.0 * q.M * q.N * (double)q.K;
    }
    if (pr.empty()) return;
    ++calls;
    const int np = (int)pr.size();
    double *wk = wtot > 0 ? gwork.ensure((size_t)wtot) : nullptr;
    DgProblem *d = gdesc.ensure(pr.size());
    int *dt = gtile0.ensure(t0.size());
    const void *hp = pr.data(), *ht = t0.data();
    if (stage) {
      hp = stage->put(pr.data(), sizeof(DgProblem) * pr.size());
      ht = stage->put(t0.data(), sizeof(int) * t0.size());
    }
    S2G_CUDA(cudaMemcpyAsync(d, hp, sizeof(DgProblem) * pr.size(), cudaMemcpyHostToDevice, s));
    S2G_CUDA(cudaMemcpyAsync(dt, ht, sizeof(int) * t0.size(), cudaMemcpyHostToDevice, s));
#define S2G_DGEMM_G(TA_, TB_)                                                                   \
  do {                                                                                          \
    S2G_CUDA(cudaFuncSetAttribute(k_dgemm_grouped<TA_, TB_, 32>,                                \
                                  cudaFuncAttributeMaxDynamicSharedMemorySize,                  \
                                  dg::smem_bytes<32>()));                                       \
    S2G_LAUNCH((k_dgemm_grouped<TA_, TB_, 32>), t0.back(), dg::THREADS, dg::smem_bytes<32>(), s, \
               d, dt, np, wk);                                                                  \
  } while (0)
    if (!ta && !tb) S2G_DGEMM_G(false, false);
    else if (ta && !tb) S2G_DGEMM_G(true, false);
    else if (!ta && tb) S2G_DGEMM_G(false, true);
    else S2G_DGEMM_G(true, true);
#undef S2G_DGEMM_G
    ++launches;
    if (wtot > 0) {
      const int g = (int)std::max<int64_t>(1, std::min<int64_t>(div_up(mnmax, 256), 64));
      S2G_LAUNCH(k_dgemm_grouped_reduce, dim3(g, np), 256, 0, s, d, wk);
      ++launches;
    }
  }

  // the argument order of cublasDgemm (alpha / beta by pointer, host values)
  void gemm(cudaStream_t s, cublasOperation_t ta, cublasOperation_t tb, int m, int n, int k,
            const double *alpha, const double *A, int64_t lda, const double *B, int64_t ldb,
            const double *beta, double *C, int64_t ldc) {
    run(s, ta != CUBLAS_OP_N, tb != CUBLAS_OP_N, m, n, k, *alpha, A, lda, 0, B, ldb, 0, *beta, C,
        ldc, 0, 1);
  }

  // op(A) is m x k, op(B) is k x n; strides between batch members (0 for one).
  void run(cudaStream_t s, bool ta, bool tb, int m, int n, int k, double alpha, const double *A,
           int64_t lda, int64_t sA, const double *B, int64_t ldb, int64_t sB, double beta,
           double *C, int64_t ldc, int64_t sC, int batch = 1, int tri = 0) {
    if (m <= 0 || n <= 0 || batch <= 0) return;
    if (k < 0) throw Error{STD2G_EINVAL, "dgemm: negative k"};
    flop += 2.0 * m * n * (double)k * batch;
    ++calls;
    if (timed) mark(s);
    struct EndMark {
      Dgemm &g;
      cudaStream_t s;
      ~EndMark() {
        if (g.timed) g.mark(s);
      }
    } end_mark{*this, s};
    if (lib && tri == 0) {
      const cublasOperation_t oa = ta ? CUBLAS_OP_T : CUBLAS_OP_N, ob = tb ? CUBLAS_OP_T : CUBLAS_OP_N;
      S2G_CUBLAS(cublasSetStream(lib, s));
      if (batch == 1)
        S2G_CUBLAS(cublasDgemm(lib, oa, ob, m, n, k, &alpha, A, (int)lda, B, (int)ldb, &beta, C,
                               (int)ldc));
      else
        S2G_CUBLAS(cublasDgemmStridedBatched(lib, oa, ob, m, n, k, &alpha, A, (int)lda, sA, B,
                                             (int)ldb, sB, &beta, C, (int)ldc, sC, batch));
      return;
    }
    // tile width and split-K: CTAs run in waves (four 64 x 32, three 64 x 64
    // or two 64 x 128 CTAs per SM); for each width pick the split count with
    // the fewest K steps on the busiest SM (each split at least 256 long; a
    // split adds its workspace pass, weighted 3 %), then the width with the
    // lower cost (the time of one K step of a full wave, measured on B200: a
    // 64 x 32 / 64 x 128 wave step takes 0.74 / 1.31 of a 64 x 64 one)
    int bn = 64, ksplit = 1;
    double best = 0.0;
    const int kmax = (int)std::max<int64_t>(1, std::min<int64_t>(64, k / 256));
    for (int w : {32, 64, 128}) {
      const int64_t ctas = div_up(m, dg::BM) * div_up(n, w) * (int64_t)batch;
      const int64_t slots = (w == 32 ? 4 : (w == 64 ? 3 : 2)) * (int64_t)nsm;
      const double per_step = w == 32 ? 0.74 : (w == 64 ? 1.0 : 1.31);
      for (int ks = 1; ks <= kmax; ++ks) {
        const int64_t steps = div_up(ctas * ks, slots) * div_up(div_up(std::max(k, 1), ks), dg::BK);
        const double cost = (double)steps * per_step * (ks > 1 ? 1.03 : 1.0);
        if (best == 0.0 || cost < best) {
          best = cost;
          bn = w;
          ksplit = ks;
        }
      }
    }
    const int tiles = (int)(div_up(m, dg::BM) * div_up(n, bn));
    int kchunk = (int)div_up(div_up(std::max(k, 1), ksplit), dg::BK) * dg::BK;
    ksplit = (int)div_up(std::max(k, 1), kchunk);
    if (batch * ksplit > 65535) throw Error{STD2G_EINVAL, "dgemm: batch too large"};
    double *wk = nullptr;
    if (ksplit > 1) wk = work.ensure((size_t)ksplit * batch * m * n);
    const dim3 grid(tiles, batch * ksplit);
#define S2G_DGEMM(TA_, TB_, BN_)                                                              \
  do {                                                                                        \
    S2G_CUDA(cudaFuncSetAttribute(k_dgemm<TA_, TB_, BN_>,                                     \
                                  cudaFuncAttributeMaxDynamicSharedMemorySize,                \
                                  dg::smem_bytes<BN_>()));                                    \
    S2G_LAUNCH((k_dgemm<TA_, TB_, BN_>), grid, dg::THREADS, dg::smem_bytes<BN_>(), s, m, n, k, \
               alpha, A, lda, sA, B, ldb, sB, beta, C, ldc, sC, ksplit, kchunk, wk, tri);     \
  } while (0)
    if (bn == 32) {
      if (!ta && !tb) S2G_DGEMM(false, false, 32);
      else if (!ta && tb) S2G_DGEMM(false, true, 32);
      else if (ta && !tb) S2G_DGEMM(true, false, 32);
      else S2G_DGEMM(true, true, 32);
    } else if (bn == 64) {
      if (!ta && !tb) S2G_DGEMM(false, false, 64);
      else if (!ta && tb) S2G_DGEMM(false, true, 64);
      else if (ta && !tb) S2G_DGEMM(true, false, 64);
      else S2G_DGEMM(true, true, 64);
    } else {
      if (!ta && !tb) S2G_DGEMM(false, false, 128);
      else if (!ta && tb) S2G_DGEMM(false, true, 128);
      else if (ta && !tb) S2G_DGEMM(true, false, 128);
      else S2G_DGEMM(true, true, 128);
    }
#undef S2G_DGEMM
    ++launches;
    if (ksplit > 1) {
      const int64_t total = (int64_t)m * n * batch;
      const int g = (int)std::min<int64_t>(div_up(total, 256), (int64_t)nsm * 8);
      S2G_LAUNCH(k_dgemm_reduce, g, 256, 0, s, m, n, batch, ksplit, alpha, wk, beta, C, ldc, sC);
      ++launches;
    }
  }
};

}  // namespace std2g
