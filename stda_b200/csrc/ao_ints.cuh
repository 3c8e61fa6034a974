// One-electron AO integrals on the device: overlap S, dipole length,
// velocity (nabla) and angular momentum (r x nabla) over contracted Cartesian
// Gaussians, written as the packed lower triangles that the engine's load
// path takes.
//
// The reference forms these on the host before it calls stda (main.f:756-797):
// libcint for S, r and nabla (libcint.f:19-352, 653-756) and its own deck for
// r x nabla (intslvm.f:213-300, opam intpack.f90:1207-1284), over the
// primitive list its readers fill (ipty angular type, ipao AO, ipat atom,
// exip exponent, cxip coefficient with every normalisation folded in;
// readbasmold.f:330-517, readxtb.f:150-160).  This file takes that same
// primitive list.
//
// Layout: one thread per packed element (r >= c) of the nao x nao lower
// triangle, k = r (r + 1) / 2 + c; it walks the primitives of AO r and of AO
// c (CSR by AO) and accumulates all ten operators with the 1D Obara-Saika
// recursion of the Gaussian product.  Conventions (origin at 0):
//   S    = <r|c>
//   L_d  = -<r| x_d |c>
//   V_d  = -<r| d/dx_d |c>          (derivative on the ket; 0 on the diagonal)
//   M_d  =  <r| (x x nabla)_d |c>   (derivative on the ket; 0 on the diagonal)
// so that the antisymmetric V, M unpack as B(r,c) = A(rc), B(c,r) = -A(rc)
// (onetri.f:73-79).
#pragma once

#include "common.cuh"

namespace std2g {

// primitive packed for the pair loop (40 bytes, read through the read-only path)
struct AoPrim {
  double x, y, z, alpha, coef;
  int lx, ly, lz, pad;
};

constexpr double kPi = 3.14159265358979323846;

// primitive pairs whose Gaussian product prefactor exp(-mu |AB|^2) falls
// below this contribute nothing at FP64 accuracy
constexpr double kAoPrimScreen = 1e-18;

// 1D Obara-Saika overlap table E[i][j] (i <= a, j <= b + 1) of the Gaussian
// product without its prefactor:
//   E[0][0] = 1,  E[0][j] = PB E[0][j-1] + (j-1)/(2p) E[0][j-2],
//   E[i][j] = PA E[i-1][j] + (i-1)/(2p) E[i-2][j] + j/(2p) E[i-1][j-1];
// built row by row (three live rows of 5, constant indices so that they stay
// in registers).  Returns E[a][b], E[a][b+1] and E[a][b-1] (0 for b = 0).
__device__ __forceinline__ void os1d(int a, int b, double PA, double PB, double inv2p,
                                     double &e0, double &ep, double &em) {
  double r2[5], r1[5], r0[5];
  r1[0] = 1.0;
#pragma unroll
  for (int j = 1; j < 5; ++j) r1[j] = PB * r1[j - 1] + (j >= 2 ? (j - 1) * inv2p * r1[j - 2] : 0.0);
#pragma unroll
  for (int j = 0; j < 5; ++j) r2[j] = 0.0;
#pragma unroll
  for (int i = 1; i < 4; ++i) {
    if (i <= a) {
#pragma unroll
      for (int j = 0; j < 5; ++j) {
        double v = PA * r1[j] + (i - 1) * inv2p * r2[j];
        if (j >= 1) v += j * inv2p * r1[j - 1];
        r0[j] = v;
      }
#pragma unroll
      for (int j = 0; j < 5; ++j) {
        r2[j] = r1[j];
        r1[j] = r0[j];
      }
    }
  }
  e0 = ep = em = 0.0;
#pragma unroll
  for (int j = 0; j < 5; ++j) {
    if (j == b) e0 = r1[j];
    if (j == b + 1) ep = r1[j];
    if (j == b - 1) em = r1[j];
  }
}

// out[q * npk + k], q = 0: S, 1-3: L, 4-6: V, 7-9: M
__global__ void __launch_bounds__(128) k_ao_ints(const AoPrim *__restrict__ prim,
                                                 const int *__restrict__ pptr, int nao,
                                                 double *__restrict__ out) {
  const int64_t npk = (int64_t)nao * (nao + 1) / 2;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < npk;
       k += (int64_t)gridDim.x * blockDim.x) {
    // packed index -> (r, c), c <= r
    int64_t r = (int64_t)((sqrt(8.0 * (double)k + 1.0) - 1.0) * 0.5);
    while (r * (r + 1) / 2 > k) --r;
    while ((r + 1) * (r + 2) / 2 <= k) ++r;
    const int64_t c = k - r * (r + 1) / 2;
    double acc[10];
#pragma unroll
    for (int q = 0; q < 10; ++q) acc[q] = 0.0;
    const int pa0 = pptr[r], pa1 = pptr[r + 1], pb0 = pptr[c], pb1 = pptr[c + 1];
    for (int ia = pa0; ia < pa1; ++ia) {
      const AoPrim A = prim[ia];
      for (int ib = pb0; ib < pb1; ++ib) {
        const AoPrim B = prim[ib];
        const double dx = A.x - B.x, dy = A.y - B.y, dz = A.z - B.z;
        const double p = A.alpha + B.alpha;
        const double ip = 1.0 / p;
        const double K = exp(-A.alpha * B.alpha * ip * (dx * dx + dy * dy + dz * dz));
        if (!(K > kAoPrimScreen)) continue;
        const double pip = kPi * ip;
        const double w = A.coef * B.coef * K * pip * sqrt(pip);
        const double inv2p = 0.5 * ip;
        const double Pd[3] = {(A.alpha * A.x + B.alpha * B.x) * ip,
                              (A.alpha * A.y + B.alpha * B.y) * ip,
                              (A.alpha * A.z + B.alpha * B.z) * ip};
        const double Ad[3] = {A.x, A.y, A.z}, Bd[3] = {B.x, B.y, B.z};
        const int la[3] = {A.lx, A.ly, A.lz}, lb[3] = {B.lx, B.ly, B.lz};
        double s[3], m[3], d[3];
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          double e0, ep, em;
          os1d(la[q], lb[q], Pd[q] - Ad[q], Pd[q] - Bd[q], inv2p, e0, ep, em);
          s[q] = e0;
          m[q] = ep + Bd[q] * e0;                       // <a| x |b>
          d[q] = -2.0 * B.alpha * ep + lb[q] * em;      // <a| d/dx |b>
        }
        acc[0] += w * s[0] * s[1] * s[2];
        acc[1] += w * m[0] * s[1] * s[2];
        acc[2] += w * s[0] * m[1] * s[2];
        acc[3] += w * s[0] * s[1] * m[2];
        acc[4] += w * d[0] * s[1] * s[2];
        acc[5] += w * s[0] * d[1] * s[2];
        acc[6] += w * s[0] * s[1] * d[2];
        acc[7] += w * s[0] * (m[1] * d[2] - m[2] * d[1]);
        acc[8] += w * s[1] * (m[2] * d[0] - m[0] * d[2]);
        acc[9] += w * s[2] * (m[0] * d[1] - m[1] * d[0]);
      }
    }
    const bool diag = r == c;
    out[k] = acc[0];
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      out[(1 + q) * npk + k] = -acc[1 + q];
      out[(4 + q) * npk + k] = diag ? 0.0 : -acc[4 + q];
      out[(7 + q) * npk + k] = diag ? 0.0 : acc[7 + q];
    }
  }
}

// Host side: validates the primitive list, builds the per-AO CSR of
// primitives (stable in input order) and the AO -> atom map
// (iaoat(ipao(i)) = ipat(i), intslvm.f:71-74), uploads, launches k_ao_ints
// into out (10 x npk doubles on the device).
struct AoIntsWork {
  DBuf<AoPrim> prim;
  DBuf<int> pptr;
};

inline std::vector<int> ao_ints(AoIntsWork &w, cudaStream_t s, int ncent, const double *xyz4,
                                int nao, int nprims, const int *ipty, const int *ipao,
                                const int *ipat, const double *exip, const double *cxip,
                                double *out) {
  if (ncent <= 0 || nao <= 0 || nprims < nao || !xyz4 || !ipty || !ipao || !ipat || !exip ||
      !cxip || !out)
    throw Error{STD2G_EINVAL, "ao integrals: bad arguments"};
  std::vector<int> cnt(nao + 1, 0), iaoat(nao, 0);
  for (int i = 0; i < nprims; ++i) {
    if (ipty[i] < 1 || ipty[i] > 20)
      throw Error{STD2G_EINVAL, "ao integrals: primitive type beyond f (ipty 1..20)"};
    if (ipao[i] < 1 || ipao[i] > nao) throw Error{STD2G_EINVAL, "ao integrals: ipao out of range"};
    if (ipat[i] < 1 || ipat[i] > ncent)
      throw Error{STD2G_EINVAL, "ao integrals: ipat out of range"};
    if (!(exip[i] > 0.0)) throw Error{STD2G_EINVAL, "ao integrals: exponent not positive"};
    const int a = ipao[i] - 1;
    if (iaoat[a] != 0 && iaoat[a] != ipat[i])
      throw Error{STD2G_EINVAL, "ao integrals: an AO's primitives sit on two atoms"};
    iaoat[a] = ipat[i];
    ++cnt[a + 1];
  }
  for (int a = 0; a < nao; ++a)
    if (cnt[a + 1] == 0) throw Error{STD2G_EINVAL, "ao integrals: an AO without primitives"};
  // Cartesian exponents of the reference's 20 primitive types (intpack.f90:
  // 1213-1218, lx/my/nz minus one): s; px py pz; xx yy zz xy xz yz;
  // xxx yyy zzz xxy xxz xyy yyz xzz yzz xyz
  static const unsigned char cart[20][3] = {
      {0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {2, 0, 0}, {0, 2, 0}, {0, 0, 2},
      {1, 1, 0}, {1, 0, 1}, {0, 1, 1}, {3, 0, 0}, {0, 3, 0}, {0, 0, 3}, {2, 1, 0},
      {2, 0, 1}, {1, 2, 0}, {0, 2, 1}, {1, 0, 2}, {0, 1, 2}, {1, 1, 1}};
  for (int a = 0; a < nao; ++a) cnt[a + 1] += cnt[a];
  std::vector<int> fill(cnt.begin(), cnt.end() - 1);
  std::vector<AoPrim> hp(nprims);
  for (int i = 0; i < nprims; ++i) {
    const int at = ipat[i] - 1, t = ipty[i] - 1;
    AoPrim q;
    q.x = xyz4[4 * at];
    q.y = xyz4[4 * at + 1];
    q.z = xyz4[4 * at + 2];
    q.alpha = exip[i];
    q.coef = cxip[i];
    q.lx = cart[t][0];
    q.ly = cart[t][1];
    q.lz = cart[t][2];
    q.pad = 0;
    hp[fill[ipao[i] - 1]++] = q;
  }
  AoPrim *dp = w.prim.ensure(nprims);
  int *dptr = w.pptr.ensure(nao + 1);
  S2G_CUDA(cudaMemcpyAsync(dp, hp.data(), sizeof(AoPrim) * nprims, cudaMemcpyHostToDevice, s));
  S2G_CUDA(cudaMemcpyAsync(dptr, cnt.data(), sizeof(int) * (nao + 1), cudaMemcpyHostToDevice, s));
  const int64_t npk = (int64_t)nao * (nao + 1) / 2;
  const int grid = (int)std::min<int64_t>(div_up(npk, 128), 148 * 16);
  S2G_LAUNCH(k_ao_ints, grid, 128, 0, s, dp, dptr, nao, out);
  // the host arrays above must outlive the copies
  S2G_CUDA(cudaStreamSynchronize(s));
  return iaoat;
}

}  // namespace std2g
