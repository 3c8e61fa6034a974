// Shared helpers of the std2g engine: status handling, device buffers and the
// kernel-launch counter.
#pragma once

#include <cuda_runtime.h>
#include <cublas_v2.h>
#include <cusolverDn.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <atomic>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/std2g.h"

namespace std2g {

struct Status {
  int code = STD2G_OK;
  std::string msg;
};

// Thrown internally and turned into a status code at the C boundary.
struct Error {
  int code;
  std::string msg;
};

#define S2G_CUDA(x)                                                              \
  do {                                                                           \
    cudaError_t e_ = (x);                                                        \
    if (e_ != cudaSuccess) {                                                     \
      if (e_ == cudaErrorMemoryAllocation)                                       \
        throw ::std2g::Error{STD2G_ENOMEM, std::string(#x) + ": " +              \
                                               cudaGetErrorString(e_)};          \
      throw ::std2g::Error{STD2G_ECUDA,                                          \
                           std::string(#x) + ": " + cudaGetErrorString(e_)};     \
    }                                                                            \
  } while (0)

#define S2G_CUBLAS(x)                                                            \
  do {                                                                           \
    cublasStatus_t s_ = (x);                                                     \
    if (s_ != CUBLAS_STATUS_SUCCESS)                                             \
      throw ::std2g::Error{STD2G_ECUDA,                                          \
                           std::string(#x) + ": cublas " + std::to_string(s_)};  \
  } while (0)

#define S2G_CUSOLVER(x)                                                          \
  do {                                                                           \
    cusolverStatus_t s_ = (x);                                                   \
    if (s_ != CUSOLVER_STATUS_SUCCESS)                                           \
      throw ::std2g::Error{STD2G_ECUDA,                                          \
                           std::string(#x) + ": cusolver " + std::to_string(s_)};\
  } while (0)

// Launch counter shared by all kernels of this library (the number reported
// by std2g_kernel_launches).
extern std::atomic<int64_t> g_launches;

#define S2G_LAUNCH(kernel, grid, block, smem, stream, ...)                       \
  do {                                                                           \
    kernel<<<(grid), (block), (smem), (stream)>>>(__VA_ARGS__);                  \
    ++::std2g::g_launches;                                                       \
    S2G_CUDA(cudaGetLastError());                                                \
  } while (0)

// Device buffer that only grows; reused across solves of one context.
template <typename T>
struct DBuf {
  T *p = nullptr;
  size_t n = 0;
  DBuf() = default;
  DBuf(const DBuf &) = delete;
  DBuf &operator=(const DBuf &) = delete;
  ~DBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  T *ensure(size_t count) {
    if (count <= n && p) return p;
    release();
    size_t c = count ? count : 1;
    S2G_CUDA(cudaMalloc(&p, c * sizeof(T)));
    n = c;
    return p;
  }
  T *get() const { return p; }
};

inline int64_t div_up(int64_t a, int64_t b) { return (a + b - 1) / b; }

// Page-locked host staging memory for small host -> device uploads (launch
// descriptors): a copy from pageable memory may wait for the stream, one from
// here is asynchronous.  Regions are handed out in order and must stay
// untouched until the stream has passed their copies: the owner calls reset()
// only after synchronising the stream.  Grows (freeing the old block after a
// device synchronisation) when a request does not fit.
struct PinnedArena {
  char *base = nullptr;
  size_t cap = 0, off = 0;
  PinnedArena() = default;
  PinnedArena(const PinnedArena &) = delete;
  PinnedArena &operator=(const PinnedArena &) = delete;
  ~PinnedArena() {
    if (base) cudaFreeHost(base);
  }
  void reset() { off = 0; }
  // n bytes of the arena (16-byte aligned), uninitialised
  void *take(size_t n) { return put(nullptr, n); }
  // copy of n bytes at p in the arena (16-byte aligned; p = NULL: no copy)
  void *put(const void *p, size_t n) {
    const size_t at = (off + 15) & ~(size_t)15;
    if (!base || at + n > cap) {
      // a larger block; copies still pending read the old one, so the device
      // is synchronised before it is freed
      const size_t ncap = std::max<size_t>(2 * cap, std::max<size_t>(at + n, 1 << 16));
      char *nb = nullptr;
      S2G_CUDA(cudaMallocHost(&nb, ncap));
      if (base) {
        S2G_CUDA(cudaDeviceSynchronize());
        cudaFreeHost(base);
      }
      base = nb;
      cap = ncap;
      off = 0;
      return put(p, n);
    }
    if (p) std::memcpy(base + at, p, n);
    off = at + n;
    return base + at;
  }
};

}  // namespace std2g
