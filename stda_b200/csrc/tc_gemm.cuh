// Tensor-core (tcgen05 / TMEM / TMA) contraction for sm_100a with split-BF16
// operands:
//
//   D[m, n] (FP32, row-major, ldd) = sum_k A[m, k] * B[n, k]
//
// A and B are given as BF16 pairs (hi, lo) with x ~= hi + lo, stored K-major
// (row-major with K contiguous, K padded to a multiple of 64 with zeros).
// Three MMAs per K step (hi*hi + hi*lo + lo*hi) into one FP32 TMEM
// accumulator recover ~16 mantissa bits of each operand, i.e. products close
// to FP32 accuracy at BF16 tensor-core rate.
//
// This is the contraction over atoms behind the sTDA couplings
// (ptselect stda.f:1812-1819; rtdamat stda.f:2040-2046):
//   (ia|jb) = sum_A p_ia^A q_jb^A    and    (ij|ab) = sum_A p_ij^A q_ab^A.
//
// Persistent CTAs (one per SM) walk 128 x 128 tiles: warp 0 issues TMA loads
// into a 3-stage shared-memory ring, warp 1 issues tcgen05.mma from one thread
// into one of two TMEM accumulators, warp 2 owns the TMEM allocation, warps
// 4-7 drain the other accumulator (tcgen05.ld) through swizzled shared memory
// and TMA bulk stores.  Every mbarrier wait is bounded by
// a ~2 s wall-clock limit; on expiry the CTA records the failure in *err and
// leaves without touching memory further.
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include "common.cuh"

namespace std2g {

namespace tc {

constexpr int BM = 128;
constexpr int BN = 128;
constexpr int BK = 64;          // 64 BF16 = 128 bytes = one 128B swizzle row
constexpr int STAGES = 3;
constexpr int TILE_A = BM * BK * 2;   // bytes per operand tile
constexpr int TILE_B = BN * BK * 2;
constexpr int STAGE_BYTES = 2 * TILE_A + 2 * TILE_B;
// epilogue staging: per epilogue warp two 32 x 32 FP32 blocks (128B-swizzled)
constexpr int EPI_COLS = 32;
constexpr int EPI_BUF = 32 * EPI_COLS * 4;
constexpr int EPI_BYTES = 4 * 2 * EPI_BUF;
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + EPI_BYTES + 1024 + 256;   // + barriers, slack
static_assert(SMEM_BYTES <= 232448, "shared memory budget of one CTA");
constexpr unsigned long long kWaitNs = 2000000000ull;   // 2 s per wait

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ unsigned long long globaltimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// bounded wait; returns false (and flags *err) when the limit expires
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, int *err, int code) {
  if (mbar_try_wait(bar, parity)) return true;
  unsigned long long t0 = globaltimer();
  while (true) {
    for (int q = 0; q < 256; ++q)
      if (mbar_try_wait(bar, parity)) return true;
    if (globaltimer() - t0 > kWaitNs) {
      atomicExch(err, code);
      return false;
    }
    if (*(volatile int *)err) return false;
  }
}

// 3-D tiled TMA load (x = K offset, y = row, z = batch); x is a multiple of 64
// elements, i.e. 128-byte aligned
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, uint64_t *bar,
                                            int x, int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y), "r"(z)
      : "memory");
}

// UMMA shared-memory descriptor: K-major, 128B swizzle, 8-row groups 1024 B apart
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);          // start address
  d |= (uint64_t)1 << 16;                          // leading byte offset (unused, 1)
  d |= (uint64_t)(1024 >> 4) << 32;                // stride byte offset
  d |= (uint64_t)1 << 46;                          // descriptor version (sm_100)
  d |= (uint64_t)2 << 61;                          // SWIZZLE_128B
  return d;
}

// instruction descriptors: BF16 x BF16 (or FP16 x FP16) -> FP32, both
// K-major, M=128, N=BN (A and B always of the same type)
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) |
                            ((uint32_t)(BM >> 4) << 24);
constexpr uint32_t kIdescF16 = (1u << 4) | ((uint32_t)(BN >> 3) << 17) |
                               ((uint32_t)(BM >> 4) << 24);

__device__ __forceinline__ void umma_f16(uint32_t tmem_d, uint64_t da, uint64_t db,
                                         uint32_t accumulate, uint32_t idesc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(
          tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
}

__device__ __forceinline__ void umma_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,"
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int q = 0; q < 16; ++q) v[q] = __uint_as_float(r[q]);
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t *r) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,"
      "%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
        "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
        "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// 3-D tiled TMA store (x = column, y = row, z = batch) from 128B-swizzled smem;
// x is a multiple of 32 FP32 elements and never negative
__device__ __forceinline__ void tma_store_3d(const CUtensorMap *map, const void *src, int x, int y,
                                             int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.global.shared::cta.tile.bulk_group [%0, {%2, %3, %4}], [%1];" ::"l"(
          reinterpret_cast<uint64_t>(map)),
      "r"(smem_u32(src)), "r"(x), "r"(y), "r"(z)
      : "memory");
}

__device__ __forceinline__ void bulk_commit() {
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}

// wait until at most one committed store group still reads shared memory
__device__ __forceinline__ void bulk_wait_read1() {
  asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory");
}

__device__ __forceinline__ void bulk_wait_all() {
  asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
}

}  // namespace tc

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(tc::smem_u32(bar)) : "memory");
}

// One tile of the persistent loop: where its operands are and where its
// output goes.
struct TcTile {
  int a_y, a_z, b_y, b_z;        // TMA row / batch coordinates of the A and B tiles
  int m0, n0, z;                 // TMA-store epilogue: origin of the output tile
  int m_valid, n_valid;          // direct-store epilogue: rows / columns kept
  // direct-store epilogue: column n of the tile goes to D + out_base + m plus
  // n * col_stride, except that the columns form runs of run_len (0: one run):
  // the step from the last column of a run to the first of the next is
  // run_skip instead of col_stride; the tile's first column is run_pos within
  // its run
  int64_t out_base, col_stride, run_skip;
  int run_len, run_pos;
  const float *rs, *cs;          // direct-store epilogue: D *= rs[m] * cs[n] (when set)
};

// Dense (batch, M/128, N/128) tiles; D row-major, stored through TMA.
struct GridTiles {
  int M, N, batch, b_batched;
  __device__ __forceinline__ int64_t count() const {
    return (int64_t)((N + tc::BN - 1) / tc::BN) * ((M + tc::BM - 1) / tc::BM) * batch;
  }
  __device__ __forceinline__ TcTile at(int64_t t) const {
    const int tiles_n = (N + tc::BN - 1) / tc::BN, tiles_m = (M + tc::BM - 1) / tc::BM;
    const int tn = (int)(t % tiles_n);
    const int64_t rest = t / tiles_n;
    const int tm = (int)(rest % tiles_m), z = (int)(rest / tiles_m);
    TcTile x{};
    x.a_y = tm * tc::BM;
    x.a_z = z;
    x.b_y = tn * tc::BN;
    x.b_z = b_batched ? z : 0;
    x.m0 = tm * tc::BM;
    x.n0 = tn * tc::BN;
    x.z = z;
    return x;
  }
};

// Persistent kernel: CTA b handles tiles b, b + gridDim.x, ... of `tiles`.
// The TMEM accumulator is double-buffered (2 x BN columns) so that the
// epilogue of one tile overlaps the MMAs of the next; the TMA producer runs
// ahead across tile boundaries through the 3-stage shared-memory ring.
// Epilogue: kDirect = false stores D[m][n] through 128B-swizzled shared
// memory and TMA (map mD); kDirect = true writes D[out_base + n*col_stride + m]
// from registers (the transposed layout of the PT couplings; a warp's 32 rows
// are 128 contiguous bytes per column).
template <class Tiles, bool kDirect, bool kF16 = false>
__global__ void __launch_bounds__(256, 1)
k_tc_gemm_bf16x3(const __grid_constant__ CUtensorMap mAh, const __grid_constant__ CUtensorMap mAl,
                 const __grid_constant__ CUtensorMap mBh, const __grid_constant__ CUtensorMap mBl,
                 const __grid_constant__ CUtensorMap mD, const Tiles tiles, float *D, int Kpad,
                 int *err) {
  using namespace tc;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char *base = (unsigned char *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  unsigned char *epi = base + STAGES * STAGE_BYTES;   // 1024-aligned staging buffers
  uint64_t *full = (uint64_t *)(epi + EPI_BYTES);
  uint64_t *empty = full + STAGES;
  uint64_t *acc_full = empty + STAGES;     // [2]
  uint64_t *acc_empty = acc_full + 2;      // [2]
  uint32_t *tmem_slot = (uint32_t *)(acc_empty + 2);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nk = Kpad / BK;
  const int64_t ntiles = tiles.count();

  if (threadIdx.x == 0) {
    for (int q = 0; q < STAGES; ++q) {
      mbar_init(&full[q], 1);
      mbar_init(&empty[q], 1);
    }
    for (int q = 0; q < 2; ++q) {
      mbar_init(&acc_full[q], 1);
      mbar_init(&acc_empty[q], 128);   // every epilogue thread arrives
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == 2) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(2 * BN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *(volatile uint32_t *)tmem_slot;

  if (warp == 0 && lane == 0) {
    // ---- TMA producer ----
    int64_t it = 0;
    bool ok = true;
    for (int64_t t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
      const TcTile tl = tiles.at(t);
      for (int kb = 0; kb < nk; ++kb, ++it) {
        const int s = (int)(it % STAGES);
        if (it >= STAGES && !mbar_wait(&empty[s], (uint32_t)(((it / STAGES) - 1) & 1), err, 1)) {
          ok = false;
          break;
        }
        unsigned char *st = base + s * STAGE_BYTES;
        mbar_expect_tx(&full[s], STAGE_BYTES);
        tma_load_3d(st, &mAh, &full[s], kb * BK, tl.a_y, tl.a_z);
        tma_load_3d(st + TILE_A, &mAl, &full[s], kb * BK, tl.a_y, tl.a_z);
        tma_load_3d(st + 2 * TILE_A, &mBh, &full[s], kb * BK, tl.b_y, tl.b_z);
        tma_load_3d(st + 2 * TILE_A + TILE_B, &mBl, &full[s], kb * BK, tl.b_y, tl.b_z);
      }
    }
  } else if (warp == 1 && lane == 0) {
    // ---- MMA issuer ----
    int64_t it = 0, lt = 0;
    bool ok = true;
    for (int64_t t = blockIdx.x; t < ntiles && ok; t += gridDim.x, ++lt) {
      const int ab = (int)(lt & 1);
      if (lt >= 2 && !mbar_wait(&acc_empty[ab], (uint32_t)(((lt >> 1) - 1) & 1), err, 4)) break;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t dacc = tmem + (uint32_t)(ab * BN);
      for (int kb = 0; kb < nk; ++kb, ++it) {
        const int s = (int)(it % STAGES);
        if (!mbar_wait(&full[s], (uint32_t)((it / STAGES) & 1), err, 2)) {
          ok = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t st = smem_u32(base + s * STAGE_BYTES);
        const uint32_t ah = st, al = st + TILE_A, bh = st + 2 * TILE_A,
                       bl = st + 2 * TILE_A + TILE_B;
#pragma unroll
        for (int kk = 0; kk < BK / 16; ++kk) {
          const uint32_t off = kk * 32;   // 16 BF16 = 32 bytes along K
          const uint32_t acc0 = (kb > 0 || kk > 0) ? 1u : 0u;
          constexpr uint32_t id = kF16 ? kIdescF16 : kIdesc;
          umma_f16(dacc, tc::umma_desc(ah + off), tc::umma_desc(bh + off), acc0, id);
          umma_f16(dacc, tc::umma_desc(ah + off), tc::umma_desc(bl + off), 1u, id);
          umma_f16(dacc, tc::umma_desc(al + off), tc::umma_desc(bh + off), 1u, id);
        }
        umma_commit(&empty[s]);   // stage reusable once these MMAs have read it
      }
      if (ok) umma_commit(&acc_full[ab]);   // accumulator complete
    }
  } else if (warp >= 4) {
    // ---- epilogue ----
    // Warp wq owns TMEM lanes (tile rows) 32*wq .. 32*wq+31 and drains them in
    // 32-column blocks.
    const int wq = warp - 4;
    unsigned char *stage0 = epi + (wq * 2) * EPI_BUF;
    int64_t lt = 0;
    uint32_t nblk = 0;
    for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x, ++lt) {
      const int ab = (int)(lt & 1);
      if (!mbar_wait(&acc_full[ab], (uint32_t)((lt >> 1) & 1), err, 3)) break;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const TcTile tl = tiles.at(t);
      if (kDirect) {
        // rows >= m_valid / columns >= n_valid are not stored; a warp whose
        // rows are all out of range skips its loads (the instruction is
        // warp-collective, so the test is warp-uniform)
        if (wq * 32 < tl.m_valid) {
          const int m = wq * 32 + lane;
          float *dst = D + tl.out_base + m;   // column c of the tile (advanced below)
          int rpos = tl.run_pos;
#pragma unroll 1
          for (int c = 0; c < BN && c < tl.n_valid; c += EPI_COLS) {
            uint32_t v[32];
            tc::tmem_ld32(tmem + ((uint32_t)(wq * 32) << 16) + (uint32_t)(ab * BN + c), v);
            const int nend = min(EPI_COLS, tl.n_valid - c);
            // column scales: lane q holds cs[c + q], broadcast by shuffles
            const float csl = (tl.cs && lane < nend) ? tl.cs[c + lane] : 1.f;
            const bool row_ok = m < tl.m_valid;
            const float r = (tl.rs && row_ok) ? tl.rs[m] : 1.f;
#pragma unroll
            for (int q = 0; q < EPI_COLS; ++q) {
              const float cq = __shfl_sync(0xffffffffu, csl, q);
              if (row_ok && q < nend) *dst = __uint_as_float(v[q]) * r * cq;
              if (tl.run_len > 0 && ++rpos == tl.run_len) {
                rpos = 0;
                dst += tl.run_skip;
              } else {
                dst += tl.col_stride;
              }
            }
          }
        }
      } else {
        // TMEM -> registers -> 128B-swizzled smem -> TMA store; the store
        // unit clips rows >= M and columns >= N
#pragma unroll 1
        for (int c = 0; c < BN; c += EPI_COLS, ++nblk) {
          unsigned char *buf = stage0 + (nblk & 1) * EPI_BUF;
          // the store that last used this buffer has finished reading it
          if (lane == 0) tc::bulk_wait_read1();
          __syncwarp();
          uint32_t v[32];
          tc::tmem_ld32(tmem + ((uint32_t)(wq * 32) << 16) + (uint32_t)(ab * BN + c), v);
          // row `lane`: 16-byte chunk q goes to chunk q ^ (lane % 8) (128B swizzle)
          unsigned char *rowp = buf + lane * 128;
#pragma unroll
          for (int q = 0; q < 8; ++q) {
            uint4 w = make_uint4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
            *reinterpret_cast<uint4 *>(rowp + ((q ^ (lane & 7)) << 4)) = w;
          }
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
          __syncwarp();
          if (lane == 0) {
            tc::tma_store_3d(&mD, buf, tl.n0 + c, tl.m0 + wq * 32, tl.z);
            tc::bulk_commit();
          }
        }
      }
      // this thread's reads of the accumulator are complete
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      mbar_arrive(&acc_empty[ab]);
    }
    if (!kDirect && lane == 0) tc::bulk_wait_all();
    __syncwarp();
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 2) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(2 * BN));
  }
}

// x (FP64, column c at src + ld*idx[c] (or ld*c), length Nk) -> hi/lo BF16 rows of Kpad
__global__ void k_split_bf16(__nv_bfloat16 *__restrict__ hi, __nv_bfloat16 *__restrict__ lo,
                             const double *__restrict__ src, int64_t ld, const int *__restrict__ idx,
                             int64_t ncols, int Nk, int Kpad) {
  int64_t total = ncols * Kpad;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    int64_t c = t / Kpad;
    int k = (int)(t - c * Kpad);
    double x = 0.0;
    if (k < Nk) x = src[(idx ? (int64_t)idx[c] : c) * ld + k];
    __nv_bfloat16 h = __double2bfloat16(x);
    __nv_bfloat16 l = __double2bfloat16(x - (double)__bfloat162float(h));
    hi[t] = h;
    lo[t] = l;
  }
}

// ---------------------------------------------------------------- host side
struct TcGemm {
  PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  DBuf<int> err;
  bool ready = false;
  double ms = 0, flop = 0;
  int64_t launches = 0;
  bool armed = false;
  int nsm = 148;
  int max_ctas = 0;   // > 0: at most this many persistent CTAs (SMs shared with other work)
  cudaEvent_t e0 = nullptr, e1 = nullptr;

  void init() {
    if (ready) return;
    cudaDriverEntryPointQueryResult q;
    void *fn = nullptr;
    S2G_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q));
    if (!fn || q != cudaDriverEntryPointSuccess)
      throw Error{STD2G_ECUDA, "cuTensorMapEncodeTiled unavailable"};
    encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
    S2G_CUDA(cudaFuncSetAttribute(k_tc_gemm_bf16x3<GridTiles, false>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, tc::SMEM_BYTES));
    S2G_CUDA(cudaEventCreate(&e0));
    S2G_CUDA(cudaEventCreate(&e1));
    int dev = 0;
    S2G_CUDA(cudaGetDevice(&dev));
    S2G_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    ready = true;
  }

  // rows x Kpad BF16 matrices, `batch` of them `rows*Kpad` elements apart
  CUtensorMap map(const void *p, int64_t rows, int Kpad, int box_rows, int batch = 1,
                  CUtensorMapDataType dt = CU_TENSOR_MAP_DATA_TYPE_BFLOAT16) {
    CUtensorMap m;
    cuuint64_t dims[3] = {(cuuint64_t)Kpad, (cuuint64_t)rows, (cuuint64_t)batch};
    cuuint64_t strides[2] = {(cuuint64_t)Kpad * 2, (cuuint64_t)rows * Kpad * 2};
    cuuint32_t box[3] = {(cuuint32_t)tc::BK, (cuuint32_t)box_rows, 1};
    cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = encode(&m, dt, 3, (void *)p, dims, strides, box,
                        estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
      throw Error{STD2G_ECUDA, "cuTensorMapEncodeTiled failed " + std::to_string((int)r)};
    return m;
  }

  // FP32 output D (rows x cols, row stride ldd elements, `batch` matrices
  // bstride elements apart) stored in 32 x 32 blocks from 128B-swizzled smem
  CUtensorMap map_out(float *p, int64_t rows, int64_t cols, int64_t ldd, int batch,
                      int64_t bstride) {
    CUtensorMap m;
    cuuint64_t dims[3] = {(cuuint64_t)cols, (cuuint64_t)rows, (cuuint64_t)batch};
    cuuint64_t strides[2] = {(cuuint64_t)ldd * 4, (cuuint64_t)bstride * 4};
    cuuint32_t box[3] = {(cuuint32_t)tc::EPI_COLS, 32, 1};
    cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = encode(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, (void *)p, dims, strides, box,
                        estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                        CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
      throw Error{STD2G_ECUDA, "cuTensorMapEncodeTiled (output) failed " + std::to_string((int)r)};
    return m;
  }

  // D (M x N, row-major ldd) = A (M x Kpad) B (N x Kpad)^T, split-BF16 operands,
  // for `batch` independent problems (A, D batched; B batched when b_batched).
  // nflop: algorithmic FLOPs credited to this launch (2 M N K_true per problem).
  void run(cudaStream_t s, const __nv_bfloat16 *Ah, const __nv_bfloat16 *Al,
           const __nv_bfloat16 *Bh, const __nv_bfloat16 *Bl, int M, int N, int Kpad, float *D,
           int64_t ldd, double nflop, int batch = 1, bool b_batched = false,
           int64_t bstride_d = 0, bool sync = true) {
    init();
    if (M <= 0 || N <= 0) return;
    if (Kpad % tc::BK != 0) throw Error{STD2G_EINVAL, "tc_gemm: K not padded to 64"};
    if (((uintptr_t)Ah | (uintptr_t)Al | (uintptr_t)Bh | (uintptr_t)Bl) & 15)
      throw Error{STD2G_EINVAL, "tc_gemm: operands not 16-byte aligned"};
    if ((ldd % 4) != 0 || ((uintptr_t)D & 15))
      throw Error{STD2G_EINVAL, "tc_gemm: output not 16-byte aligned"};
    if (batch < 1 || batch > 65535) throw Error{STD2G_EINVAL, "tc_gemm: bad batch"};
    if (batch > 1 && ((bstride_d % 4) != 0)) throw Error{STD2G_EINVAL, "tc_gemm: batch stride"};
    CUtensorMap ah = map(Ah, M, Kpad, tc::BM, batch), al = map(Al, M, Kpad, tc::BM, batch);
    CUtensorMap bh = map(Bh, N, Kpad, tc::BN, b_batched ? batch : 1);
    CUtensorMap bl = map(Bl, N, Kpad, tc::BN, b_batched ? batch : 1);
    CUtensorMap dm = map_out(D, M, N, ldd, batch, batch > 1 ? bstride_d : (int64_t)M * ldd);
    int *e = err.ensure(1);
    if (!armed) {
      S2G_CUDA(cudaMemsetAsync(e, 0, sizeof(int), s));
      armed = true;
    }
    const int64_t ntiles = div_up(N, tc::BN) * div_up(M, tc::BM) * (int64_t)batch;
    const int cap = max_ctas > 0 ? std::min(max_ctas, nsm) : nsm;
    const int grid = (int)std::min<int64_t>(ntiles, cap);
    if (sync) S2G_CUDA(cudaEventRecord(e0, s));
    const GridTiles tiles{M, N, batch, b_batched ? 1 : 0};
    S2G_LAUNCH((k_tc_gemm_bf16x3<GridTiles, false>), grid, 256, tc::SMEM_BYTES, s, ah, al, bh, bl,
               dm, tiles, (float *)nullptr, Kpad, e);
    ++launches;
    flop += nflop * batch;
    if (sync) {
      S2G_CUDA(cudaEventRecord(e1, s));
      check(s);
      float t = 0;
      S2G_CUDA(cudaEventElapsedTime(&t, e0, e1));
      ms += t;
    }
  }

  // D[tile.out_base + n*tile.col_stride + m] for the tiles of `tiles` (a
  // schedule type with count() / at(), see TcTile): A (a_rows x Kpad) and B
  // (b_rows x Kpad) split-BF16 operands read at the tiles' row coordinates;
  // rows past the end of an operand read as zeros.  No synchronisation: the
  // wait status is read by the next check().
  // kF16: FP16 operands (scaled by the caller; the tiles' rs / cs undo it).
  template <class Tiles, bool kF16 = false>
  void run_direct(cudaStream_t s, const void *Ah, const void *Al, int64_t a_rows,
                  const void *Bh, const void *Bl, int64_t b_rows, int Kpad, const Tiles &tiles,
                  int64_t ntiles, float *D, double nflop) {
    init();
    if (ntiles <= 0) return;
    if (Kpad % tc::BK != 0) throw Error{STD2G_EINVAL, "tc_gemm: K not padded to 64"};
    if (((uintptr_t)Ah | (uintptr_t)Al | (uintptr_t)Bh | (uintptr_t)Bl) & 15)
      throw Error{STD2G_EINVAL, "tc_gemm: operands not 16-byte aligned"};
    if (a_rows >= (int64_t)1 << 31 || b_rows >= (int64_t)1 << 31)
      throw Error{STD2G_EINVAL, "tc_gemm: operand rows beyond the TMA coordinate range"};
    // per device and instantiation; a cheap host call, made every time
    S2G_CUDA(cudaFuncSetAttribute(k_tc_gemm_bf16x3<Tiles, true, kF16>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, tc::SMEM_BYTES));
    const CUtensorMapDataType dt =
        kF16 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16;
    CUtensorMap ah = map(Ah, a_rows, Kpad, tc::BM, 1, dt), al = map(Al, a_rows, Kpad, tc::BM, 1, dt);
    CUtensorMap bh = map(Bh, b_rows, Kpad, tc::BN, 1, dt), bl = map(Bl, b_rows, Kpad, tc::BN, 1, dt);
    int *e = err.ensure(1);
    if (!armed) {
      S2G_CUDA(cudaMemsetAsync(e, 0, sizeof(int), s));
      armed = true;
    }
    const int cap = max_ctas > 0 ? std::min(max_ctas, nsm) : nsm;
    const int grid = (int)std::min<int64_t>(ntiles, cap);
    S2G_LAUNCH((k_tc_gemm_bf16x3<Tiles, true, kF16>), grid, 256, tc::SMEM_BYTES, s, ah, al, bh,
               bl, ah, tiles, D, Kpad, e);
    ++launches;
    flop += nflop;
  }

  // read the error flag of the launches since the last check (synchronises)
  void check(cudaStream_t s) {
    if (!armed) return;
    int h_err = 0;
    S2G_CUDA(cudaMemcpyAsync(&h_err, err.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
    S2G_CUDA(cudaStreamSynchronize(s));
    armed = false;
    if (h_err)
      throw Error{STD2G_ETIMEOUT, "tc_gemm: bounded wait expired (" + std::to_string(h_err) + ")"};
  }
};

}  // namespace std2g
