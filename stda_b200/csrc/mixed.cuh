// Mixed-precision form of the contractions (declarations; filled in by the
// tensor-core kernels).
#pragma once

#include "common.cuh"

namespace std2g {

struct MixedWork {
  DBuf<float> K, J;
  double *lastX = nullptr;
};

inline void mixed_pt_chunk(MixedWork &, cudaStream_t, const double *, const double *,
                           const double *, const double *, int, int, int, int, int) {
  throw Error{STD2G_EINVAL, "mixed form not available in this build"};
}
inline void mixed_pt_recheck(MixedWork &, cudaStream_t, double *, unsigned char *, int, double,
                             const double *, const double *, const double *, const double *, int,
                             int, int, int, const int *, int, int, const double *, const int *,
                             const int *, const int *, const int *, const double *, double, int,
                             int) {
  throw Error{STD2G_EINVAL, "mixed form not available in this build"};
}
inline int mixed_davidson(MixedWork &, cublasHandle_t, cudaStream_t, const double *, int, int,
                          double, double *, double *) {
  throw Error{STD2G_EINVAL, "mixed form not available in this build"};
}

}  // namespace std2g
