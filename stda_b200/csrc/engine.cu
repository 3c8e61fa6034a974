// std2g engine: context, inputs, and the sTDA / sTD-DFT solve.
//
// The solve follows SUBROUTINE stda (stda.f:53-1606) phase by phase; each
// phase runs on the context's stream.  Dense FP64 contractions that are plain
// library GEMMs (AO->MO transforms, gamma*Q) go to cuBLAS; the symmetric
// eigen-decompositions of S and of the small dense CI matrices go to cuSOLVER;
// the charge formation, the screen, the PT selection and the A build use the
// kernels of this library (kernels_fp64.cuh, tc_gemm.cuh).
#include <algorithm>
#include <dlfcn.h>
#include <functional>
#include <chrono>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>

#include <cub/cub.cuh>

#include "common.cuh"
#include "eta_table.cuh"
#include "kernels_fp64.cuh"
#include "davidson.cuh"
#include "davidson_rpa.cuh"
#include "ao_ints.cuh"
#include "dgemm.cuh"
#include "matfree.cuh"
#include "matfree_tc.cuh"
#include "pt_tc.cuh"
#include "response_mixed.cuh"
#include "symeig_small.cuh"
#include "batch_davidson.cuh"

namespace std2g {

std::atomic<int64_t> g_launches{0};


enum Phase {
  PH_SETUP = 0, PH_SQRTS, PH_MOINT, PH_CHARGES, PH_SCREEN, PH_PT, PH_BUILD, PH_EIGEN, PH_PROPS,
  PH_RESPONSE, PH_COUNT
};
static const char *kPhaseNames[PH_COUNT] = {"setup", "sqrt_S", "mo_integrals", "charges",
                                            "screen", "pt_select", "build", "eigen",
                                            "properties", "response"};

struct Ctx {
  std2g_opts opts{};
  cudaStream_t stream = nullptr;
  cublasHandle_t blas = nullptr;
  cusolverDnHandle_t solver = nullptr;
  cusolverDnParams_t solver_params = nullptr;   // 64-bit cuSOLVER API (large n)
  std::vector<char> host_work;
  bool loaded = false;
  int ncent = 0, nmo = 0, nao = 0;
  std::vector<double> h_eps, h_occ, h_xyz;
  AoIntsWork aoi;   // primitive list of the device AO integrals (ao_ints.cuh)
  DBuf<double> w_Ares, w_Rres, w_part, w_rn, w_domc;   // dense residuals, dominant CSFs
  DBuf<int> w_domi;
  Dgemm dg;         // the engine's FP64 matrix products (dgemm.cuh)
  int dev_sms = 148;   // SMs of the context's device
  // device inputs
  DBuf<double> d_xyz, d_C, d_eps_act, d_eta, d_Sfull, d_sqrtS, d_ao9;
  DBuf<int> d_ao_ptr, d_ao_list, d_iaoat, d_slot_ao;
  int maxa = 1;
  int chunk_rows = 1;   // largest AO count of kChAtoms consecutive atoms
  bool sqrtS_ready = false;
  // unrestricted wavefunction (std2g_set_spins): spin of each MO, 1 alpha / 2 beta
  bool uks = false;
  std::vector<int> h_csp;
  int ns_iters = 0;            // Newton-Schulz steps of the last S^1/2
  DBuf<double> w_ns;           // its scale / error words
  // work buffers
  DBuf<double> w_Cact, w_Clow, w_T, w_mu_ov, w_gj, w_gk, w_Qii, w_Qaa, w_Pii, w_uci;
  DBuf<double> w_Qia, w_Pia, w_Qoo, w_Poo, w_Qvv, w_de, w_ek;
  DBuf<int> w_flag, w_act_idx, w_pk, w_ck, w_tmpi, w_pj, w_pb, w_omap, w_vmap, w_OP, w_VP, w_ci,
      w_ca, w_allk, w_status;
  DBuf<double> w_ed, w_edsorted, w_Qp, w_QvvP, w_W, w_Pc, w_Kbuf, w_Jbuf, w_pert, w_colpart,
      w_pt2, w_edp;
  DBuf<unsigned char> w_sel;
  DBuf<double> w_Qs, w_Ps, w_K, w_J, w_Kx, w_A, w_Apb, w_Amb, w_Bh, w_Ambh, w_M, w_eval, w_X,
      w_Y, w_tmp, w_musel, w_TL, w_TVM, w_T2, w_props, w_work;
  // quadratic response: length dipoles in the occupied and virtual blocks,
  // response vectors, and the work arrays of the M Y products
  DBuf<double> w_To, w_moo, w_mvv, w_Uall, w_Vall, w_qx, w_qy, w_qbox, w_qmy, w_qsel, w_qg,
      w_tpx, w_tpy;
  DBuf<double> w_jbox;   // (ij|ab) / (ib|ja) box of the dense build
  DBuf<int> w_info;
  DBuf<char> w_cub;
  MixedWork mixed;
  struct RespWork {
    DBuf<float> Apb32, Amb32, dp, dm;
    DBuf<double> B1, U, V, PU, MV, R1, R2, pa, pb, wcol, rz, alpha, beta, rr, nrm, nrm2, dmf, dpd,
        dmd;
    DBuf<char> vecs[12];
    DBuf<unsigned> flag;
    int outer = 0, inner = 0;
  } rw;
  DavidsonWork dav;
  DavidsonRpaWork davr;
  MatFree mf;
  MatFreeTc mftc;
  // tensor-core contraction statistics of the last solve
  double tc_ms = 0, tc_flop = 0;
  int64_t tc_launches = 0;
  int dav_iters = 0;
  int64_t dav_matvecs = 0, dav_fp64_matvecs = 0;
  // last results
  int last_nci = 0, last_nroot = 0, last_no = 0, last_nv = 0;
  bool last_rpa = false;
  double ph_ms[PH_COUNT] = {0};
  cudaEvent_t ev[PH_COUNT + 1];
  // shared batched eigensolver (std2g_attach_batch) and the events that order
  // this context's stream with the batch's
  BatchDavidson *batch = nullptr;
  cudaEvent_t ev_bready = nullptr, ev_bdone = nullptr;
  bool last_batched = false;
};

// --------------------------------------------------------------------------
// FP64 C = alpha op(A) op(B) + beta C through the engine's DMMA kernel
// (dgemm.cuh); batch > 1: members at fixed strides sA, sB, sC.
static void gemm(Ctx &c, cublasOperation_t ta, cublasOperation_t tb, int m, int n, int k,
                 double alpha, const double *A, int64_t lda, const double *B, int64_t ldb,
                 double beta, double *C, int64_t ldc, int batch = 1, int64_t sA = 0,
                 int64_t sB = 0, int64_t sC = 0) {
  if (m == 0 || n == 0) return;
  c.dg.run(c.stream, ta != CUBLAS_OP_N, tb != CUBLAS_OP_N, m, n, k, alpha, A, lda, sA, B, ldb,
           sB, beta, C, ldc, sC, batch);
}

static int grid_for(int64_t n, int block = 256) {
  int64_t g = div_up(n, block);
  return (int)std::max<int64_t>(1, std::min<int64_t>(g, 148 * 64));
}

static void record(Ctx &c, int ph) { S2G_CUDA(cudaEventRecord(c.ev[ph], c.stream)); }

// Dense symmetric eigen-decomposition with an eigenvalue window (vl, vu]
// (ssyevr 'V' range, stda.f:1143-1147) or the lowest k (range 'I').
// A (n x n) is overwritten by the eigenvectors; returns the number found.
static void dense_eig_full(Ctx &c, double *A, int n, double *w);
static int dense_eig(Ctx &c, double *A, int n, double vl, double vu, int kmax, double *w) {
  if (kmax > 0) {   // lowest kmax roots: full decomposition, eigenvectors in the leading columns
    dense_eig_full(c, A, n, w);
    return std::min(kmax, n);
  }
  int meig = 0, lwork = 0;
  cusolverEigRange_t range = kmax > 0 ? CUSOLVER_EIG_RANGE_I : CUSOLVER_EIG_RANGE_V;
  int il = 1, iu = kmax > 0 ? std::min(kmax, n) : n;
  S2G_CUSOLVER(cusolverDnDsyevdx_bufferSize(c.solver, CUSOLVER_EIG_MODE_VECTOR, range,
                                            CUBLAS_FILL_MODE_LOWER, n, A, n, vl, vu, il, iu,
                                            &meig, w, &lwork));
  double *work = c.w_work.ensure((size_t)lwork + 1);
  int *info = c.w_info.ensure(1);
  S2G_CUSOLVER(cusolverDnDsyevdx(c.solver, CUSOLVER_EIG_MODE_VECTOR, range,
                                 CUBLAS_FILL_MODE_LOWER, n, A, n, vl, vu, il, iu, &meig, w, work,
                                 lwork, info));
  int h_info = 0;
  S2G_CUDA(cudaMemcpyAsync(&h_info, info, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
  S2G_CUDA(cudaStreamSynchronize(c.stream));
  if (h_info != 0) throw Error{STD2G_ECUDA, "syevdx info " + std::to_string(h_info)};
  return meig;
}

// Full symmetric eigen-decomposition (makel stda.f:1615-1691, smatpow srpapack.f:201-256),
// through the 64-bit cuSOLVER interface: the workspace of n >~ 11000 exceeds
// 2^31 bytes.
static void dense_eig_full(Ctx &c, double *A, int n, double *w) {
  if (!c.solver_params) S2G_CUSOLVER(cusolverDnCreateParams(&c.solver_params));
  size_t dbytes = 0, hbytes = 0;
  S2G_CUSOLVER(cusolverDnXsyevd_bufferSize(c.solver, c.solver_params, CUSOLVER_EIG_MODE_VECTOR,
                                           CUBLAS_FILL_MODE_LOWER, n, CUDA_R_64F, A, n,
                                           CUDA_R_64F, w, CUDA_R_64F, &dbytes, &hbytes));
  double *work = c.w_work.ensure(dbytes / sizeof(double) + 1);
  if (c.host_work.size() < hbytes + 1) c.host_work.resize(hbytes + 1);
  int *info = c.w_info.ensure(1);
  S2G_CUSOLVER(cusolverDnXsyevd(c.solver, c.solver_params, CUSOLVER_EIG_MODE_VECTOR,
                                CUBLAS_FILL_MODE_LOWER, n, CUDA_R_64F, A, n, CUDA_R_64F, w,
                                CUDA_R_64F, work, dbytes, c.host_work.data(), hbytes, info));
  int h_info = 0;
  S2G_CUDA(cudaMemcpyAsync(&h_info, info, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
  S2G_CUDA(cudaStreamSynchronize(c.stream));
  if (h_info != 0) throw Error{STD2G_ECUDA, "syevd info " + std::to_string(h_info)};
}

// X = U diag(sqrt(w)) U^T, U overwritten (tmp n*n)
static void sym_sqrt(Ctx &c, double *U, const double *w, int n, double *out, double *tmp) {
  S2G_CUDA(cudaMemcpyAsync(tmp, U, sizeof(double) * n * n, cudaMemcpyDeviceToDevice, c.stream));
  S2G_LAUNCH(k_scale_cols_sqrt, grid_for((int64_t)n * n), 256, 0, c.stream, tmp, w, n);
  gemm(c, CUBLAS_OP_N, CUBLAS_OP_T, n, n, n, 1.0, tmp, n, U, n, 0.0, out, n);
}

// S^1/2 of the AO overlap (makel, stda.f:1615-1691) without an eigensolver:
// with A = S / c (c = largest absolute row sum >= lambda_max, so the spectrum
// of A lies in (0, 1]), the coupled Newton-Schulz iteration
//   T_k = (3 I - Z_k A Z_k) / 2,   Z_{k+1} = T_k Z_k,   Z_0 = I
// converges quadratically to A^-1/2 (every iterate is a polynomial in A, so
// Y_k = A Z_k is the companion sequence that converges to A^1/2), and
// S^1/2 = sqrt(c) A Z.  Stops when max |I - Z A Z| < 1e-14 or stagnates at the
// rounding level below 1e-10.  A spectrum that is
// not positive (makel's negative-eigenvalue stop, stda.f:1658-1670) makes
// the iteration fail its final check ||Y Y - A||_max < 1e-10 ||A||_max.
// Three FP64 products per step on the engine's DMMA kernel.
static void sqrt_overlap(Ctx &c, const double *S, int n, double *out) {
  cudaStream_t s = c.stream;
  const size_t nn = (size_t)n * n;
  double *A = c.w_tmp.ensure(nn * 4), *Z = A + nn, *P = A + 2 * nn, *T = A + 3 * nn;
  // steps run in groups of kGroup between host reads of their errors (one
  // synchronisation per group); steps past convergence stay at the fixed
  // point Z A Z = I to rounding and are harmless
  constexpr int kGroup = 3;
  auto *flags = (unsigned long long *)c.w_ns.ensure(1 + kGroup);
  S2G_CUDA(cudaMemsetAsync(flags, 0, (1 + kGroup) * sizeof(unsigned long long), s));
  S2G_LAUNCH(k_row_abs_max, (int)div_up(n, 256), 256, 0, s, S, n, flags);
  S2G_LAUNCH(k_ns_init, grid_for((int64_t)nn), 256, 0, s, A, Z, S, n, flags);
  unsigned long long h[1 + kGroup] = {0};
  double err = 1.0, prev = 2.0;
  int it = 0;
  // quadratic convergence ends at the rounding level of the products: stop at
  // 1e-14, or once below 1e-10 a step no longer halves the error
  bool done = false;
  while (!done && it < 99) {
    S2G_CUDA(cudaMemsetAsync(flags + 1, 0, kGroup * sizeof(unsigned long long), s));
    for (int q = 0; q < kGroup; ++q) {
      gemm(c, CUBLAS_OP_N, CUBLAS_OP_N, n, n, n, 1.0, A, n, Z, n, 0.0, P, n);   // P = A Z
      gemm(c, CUBLAS_OP_N, CUBLAS_OP_N, n, n, n, 1.0, Z, n, P, n, 0.0, T, n);   // T = Z A Z
      S2G_LAUNCH(k_ns_step, grid_for((int64_t)nn), 256, 0, s, T, n, flags + 1 + q);
      gemm(c, CUBLAS_OP_N, CUBLAS_OP_N, n, n, n, 1.0, T, n, Z, n, 0.0, P, n);   // Z <- T Z
      std::swap(Z, P);
    }
    S2G_CUDA(cudaMemcpyAsync(h, flags, sizeof(h), cudaMemcpyDeviceToHost, s));
    S2G_CUDA(cudaStreamSynchronize(s));
    for (int q = 0; q < kGroup && !done; ++q) {
      prev = err;
      std::memcpy(&err, &h[1 + q], sizeof(double));
      ++it;
      if (!std::isfinite(err) || err > 1e6 || err < 1e-14 || (err < 1e-10 && err > 0.5 * prev))
        done = true;
    }
  }
  it = (it + kGroup - 1) / kGroup * kGroup;   // steps executed
  c.ns_iters = it;
  double cmax;
  std::memcpy(&cmax, &h[0], sizeof(double));
  // Y = A Z (= A^1/2); check Y Y = A, then S^1/2 = sqrt(c) Y
  gemm(c, CUBLAS_OP_N, CUBLAS_OP_N, n, n, n, 1.0, A, n, Z, n, 0.0, P, n);
  S2G_CUDA(cudaMemcpyAsync(T, A, sizeof(double) * nn, cudaMemcpyDeviceToDevice, s));
  gemm(c, CUBLAS_OP_N, CUBLAS_OP_N, n, n, n, 1.0, P, n, P, n, -1.0, T, n);   // T = Y Y - A
  S2G_CUDA(cudaMemsetAsync(flags + 1, 0, sizeof(unsigned long long), s));
  S2G_LAUNCH(k_abs_max, grid_for((int64_t)nn), 256, 0, s, T, (int64_t)nn, flags + 1);
  S2G_CUDA(cudaMemcpyAsync(h, flags, sizeof(h), cudaMemcpyDeviceToHost, s));
  S2G_CUDA(cudaStreamSynchronize(s));
  double resid;
  std::memcpy(&resid, &h[1], sizeof(double));
  // ||A||_max <= 1 by the scaling
  if (!(err < 1e-10) || !(resid < 1e-10))
    throw Error{STD2G_ES_NOT_PD, "S^1/2: overlap matrix not positive definite (Newton-Schulz "
                                 "did not converge)"};
  S2G_LAUNCH(k_scale_copy, grid_for((int64_t)nn), 256, 0, s, out, P, (int64_t)nn, std::sqrt(cmax));
}

static uint64_t fnv1a(const std::vector<int> &a, const std::vector<int> &b) {
  uint64_t h = 1469598103934665603ull;
  for (size_t k = 0; k < a.size(); ++k) {
    int v[2] = {a[k], b[k]};
    const unsigned char *p = (const unsigned char *)v;
    for (int q = 0; q < 8; ++q) {
      h ^= p[q];
      h *= 1099511628211ull;
    }
  }
  return h;
}

// --------------------------------------------------------------------------
// Inputs of one molecule.  The packed integrals come either from the host
// (S, muL, muV, muM) or, with pk_dev, already on the device in the layout of
// k_ao_ints (10 x npk: S, L, V, M).
static void load(Ctx &c, int ncent, int nmo, int nao, const double *xyz, const double *C,
                 const double *eps, const double *occ, const int *iaoat, const double *S,
                 const double *muL, const double *muV, const double *muM,
                 const double *pk_dev = nullptr) {
  if (ncent <= 0 || nmo <= 0 || nao <= 0 || !xyz || !C || !eps || !occ || !iaoat ||
      (!pk_dev && (!S || !muL || !muV || !muM)))
    throw Error{STD2G_EINVAL, "load: bad arguments"};
  c.ncent = ncent;
  c.nmo = nmo;
  c.nao = nao;
  c.h_eps.assign(eps, eps + nmo);
  c.h_occ.assign(occ, occ + nmo);
  c.h_xyz.assign(xyz, xyz + 4 * (size_t)ncent);
  std::vector<double> eta(ncent);
  for (int a = 0; a < ncent; ++a) {
    int z = (int)std::lround(xyz[4 * a + 3]);
    if (z < 1 || z > 94) throw Error{STD2G_EINVAL, "load: nuclear charge out of range"};
    eta[a] = kEta[z - 1];
  }
  std::vector<int> cnt(ncent + 1, 0), ptr(ncent + 1, 0), list(nao);
  for (int k = 0; k < nao; ++k) {
    int a = iaoat[k] - 1;
    if (a < 0 || a >= ncent) throw Error{STD2G_EINVAL, "load: iaoat out of range"};
    cnt[a]++;
  }
  for (int a = 0; a < ncent; ++a) ptr[a + 1] = ptr[a] + cnt[a];
  std::vector<int> fill(ptr.begin(), ptr.end() - 1);
  for (int k = 0; k < nao; ++k) list[fill[iaoat[k] - 1]++] = k;
  int maxa = 1;
  for (int a = 0; a < ncent; ++a) maxa = std::max(maxa, cnt[a]);
  std::vector<int> slot((size_t)ncent * maxa, -1);
  for (int a = 0; a < ncent; ++a)
    for (int q = 0; q < cnt[a]; ++q) slot[(size_t)a * maxa + q] = list[ptr[a] + q];
  c.maxa = maxa;
  c.chunk_rows = 1;
  for (int a0 = 0; a0 < ncent; a0 += kChAtoms)
    c.chunk_rows = std::max(c.chunk_rows, ptr[std::min(ncent, a0 + kChAtoms)] - ptr[a0]);
  size_t npk = (size_t)nao * (nao + 1) / 2;
  cudaStream_t s = c.stream;
  S2G_CUDA(cudaMemcpyAsync(c.d_slot_ao.ensure(slot.size()), slot.data(), sizeof(int) * slot.size(),
                           cudaMemcpyHostToDevice, s));
  S2G_CUDA(cudaMemcpyAsync(c.d_xyz.ensure(4 * ncent), xyz, sizeof(double) * 4 * ncent,
                           cudaMemcpyHostToDevice, s));
  S2G_CUDA(cudaMemcpyAsync(c.d_eta.ensure(ncent), eta.data(), sizeof(double) * ncent,
                           cudaMemcpyHostToDevice, s));
  S2G_CUDA(cudaMemcpyAsync(c.d_C.ensure((size_t)nao * nmo), C, sizeof(double) * nao * nmo,
                           cudaMemcpyHostToDevice, s));
  S2G_CUDA(cudaMemcpyAsync(c.d_ao_ptr.ensure(ncent + 1), ptr.data(), sizeof(int) * (ncent + 1),
                           cudaMemcpyHostToDevice, s));
  S2G_CUDA(cudaMemcpyAsync(c.d_ao_list.ensure(nao), list.data(), sizeof(int) * nao,
                           cudaMemcpyHostToDevice, s));
  // packed integrals -> full AO matrices (BLOWSY, onetri.f:62-80)
  const double *pk = pk_dev;
  if (!pk) {
    double *h2d = c.w_work.ensure(npk * 10);
    S2G_CUDA(cudaMemcpyAsync(h2d, S, sizeof(double) * npk, cudaMemcpyHostToDevice, s));
    S2G_CUDA(cudaMemcpyAsync(h2d + npk, muL, sizeof(double) * npk * 3, cudaMemcpyHostToDevice, s));
    S2G_CUDA(cudaMemcpyAsync(h2d + 4 * npk, muV, sizeof(double) * npk * 3, cudaMemcpyHostToDevice,
                             s));
    S2G_CUDA(cudaMemcpyAsync(h2d + 7 * npk, muM, sizeof(double) * npk * 3, cudaMemcpyHostToDevice,
                             s));
    pk = h2d;
  }
  size_t nn = (size_t)nao * nao;
  double *Sf = c.d_Sfull.ensure(nn);
  double *ao9 = c.d_ao9.ensure(nn * 9);
  int g = grid_for((int64_t)nn);
  S2G_LAUNCH(k_unpack, g, 256, 0, s, Sf, pk, nao, 0);
  for (int q = 0; q < 9; ++q)
    S2G_LAUNCH(k_unpack, g, 256, 0, s, ao9 + nn * q, pk + npk * (1 + q), nao, q < 3 ? 0 : 1);
  S2G_CUDA(cudaStreamSynchronize(s));
  c.sqrtS_ready = false;
  c.uks = false;
  c.h_csp.clear();
  c.loaded = true;
}

// Quadratic-response consumers of the linear-response vectors (lresp1,
// linear_response.f:196-908; lresp_2PA_SP, :4604-4938).
struct QuadReq {
  // beta(-2w; w, w): the response frequencies are (w_k, -2 w_k) pairs
  double *beta = nullptr;       // [nbeta*27] row-major beta[k][x][y][z]
  double *beta_hrs = nullptr;   // [nbeta]
  int nbeta = 0;
  // two-photon absorption of the lowest ntpa sTD-DFT states
  double *tpa = nullptr;        // [ntpa*6] rows (n, w_n eV, delta_par, delta_perp, delta_circ, rho)
  int ntpa = 0;
};

// A dynamic-polarizability request (lresp, linear_response.f:23-192).  With U
// and V set (device, n x 3 per frequency slot), the solvers also leave the
// vectors X+Y (U) and X-Y (V) of every frequency there; slot[w] (NULL: w)
// names the slot of frequency w.
struct RespReq {
  const double *omega;
  int n;
  double *alpha;   // [n*9]
  double *resid;   // [n] or NULL
  double *U = nullptr, *V = nullptr;
  const int *slot = nullptr;
  const QuadReq *quad = nullptr;
};

// (A-B)^-1 by Cholesky (ssptrf/ssptri, linear_response.f:89-95), then per omega
// [(A+B) - w^2 (A-B)^-1] (X+Y) = -2 mu (linear_response.f:104-131) and
// alpha_xy = -2 sum_j mu_x,j (X+Y)_y,j (linear_response.f:153-171).
static void response(Ctx &c, double *Apb, double *Amb, int nci, const double *musel,
                     const RespReq &rq) {
  cudaStream_t s = c.stream;
  const size_t n2 = (size_t)nci * nci;
  int *info = c.w_info.ensure(1);
  int h_info = 0;
  auto check_info = [&](int code, const char *what) {
    S2G_CUDA(cudaMemcpyAsync(&h_info, info, sizeof(int), cudaMemcpyDeviceToHost, s));
    S2G_CUDA(cudaStreamSynchronize(s));
    if (h_info != 0) throw Error{code, std::string(what) + " info " + std::to_string(h_info)};
  };
  double *Ainv = c.w_Ambh.ensure(n2);
  S2G_CUDA(cudaMemcpyAsync(Ainv, Amb, sizeof(double) * n2, cudaMemcpyDeviceToDevice, s));
  int lwork = 0;
  S2G_CUSOLVER(cusolverDnDpotrf_bufferSize(c.solver, CUBLAS_FILL_MODE_LOWER, nci, Ainv, nci, &lwork));
  int lw2 = 0;
  S2G_CUSOLVER(cusolverDnDpotri_bufferSize(c.solver, CUBLAS_FILL_MODE_LOWER, nci, Ainv, nci, &lw2));
  int lw3 = 0;
  S2G_CUSOLVER(cusolverDnDgetrf_bufferSize(c.solver, nci, nci, Ainv, nci, &lw3));
  double *work = c.w_work.ensure((size_t)std::max(lwork, std::max(lw2, lw3)) + 1);
  S2G_CUSOLVER(cusolverDnDpotrf(c.solver, CUBLAS_FILL_MODE_LOWER, nci, Ainv, nci, work, lwork, info));
  check_info(STD2G_EAMB_NOT_PD, "A-B Cholesky");
  S2G_CUSOLVER(cusolverDnDpotri(c.solver, CUBLAS_FILL_MODE_LOWER, nci, Ainv, nci, work, lw2, info));
  check_info(STD2G_EAMB_NOT_PD, "A-B inverse");
  S2G_LAUNCH(k_symmetrize_lower, grid_for((int64_t)n2), 256, 0, s, Ainv, (int64_t)nci);
  double *Mw = c.w_M.ensure(n2);
  double *B = c.w_TL.ensure((size_t)nci * 3 * 3);
  double *Xs = B + (size_t)nci * 3;
  double *R = Xs + (size_t)nci * 3;
  int *ipiv = c.w_tmpi.ensure(std::max<size_t>(nci, 1));
  double *a9 = c.w_props.ensure(16);
  for (int w = 0; w < rq.n; ++w) {
    double om = rq.omega[w];
    S2G_LAUNCH(k_axpby_mat, grid_for((int64_t)n2), 256, 0, s, Mw, Apb, Ainv, (int64_t)n2, -om * om);
    // B = -2 mu_L ; Xs = B
    S2G_LAUNCH(k_scale_copy, grid_for((int64_t)nci * 3), 256, 0, s, B, musel, (int64_t)nci * 3, -2.0);
    S2G_CUDA(cudaMemcpyAsync(Xs, B, sizeof(double) * nci * 3, cudaMemcpyDeviceToDevice, s));
    double *F = c.w_Apb.get() == Apb ? c.w_Kx.ensure(n2) : c.w_Kx.ensure(n2);
    S2G_CUDA(cudaMemcpyAsync(F, Mw, sizeof(double) * n2, cudaMemcpyDeviceToDevice, s));
    S2G_CUSOLVER(cusolverDnDpotrf(c.solver, CUBLAS_FILL_MODE_LOWER, nci, F, nci, work, lwork, info));
    S2G_CUDA(cudaMemcpyAsync(&h_info, info, sizeof(int), cudaMemcpyDeviceToHost, s));
    S2G_CUDA(cudaStreamSynchronize(s));
    if (h_info == 0) {
      S2G_CUSOLVER(cusolverDnDpotrs(c.solver, CUBLAS_FILL_MODE_LOWER, nci, 3, F, nci, Xs, nci, info));
    } else {
      // omega above the lowest excitation: indefinite, use LU (ssptrf is Bunch-Kaufman)
      S2G_CUDA(cudaMemcpyAsync(F, Mw, sizeof(double) * n2, cudaMemcpyDeviceToDevice, s));
      S2G_CUSOLVER(cusolverDnDgetrf(c.solver, nci, nci, F, nci, work, ipiv, info));
      check_info(STD2G_ENOCONV, "response LU");
      S2G_CUSOLVER(cusolverDnDgetrs(c.solver, CUBLAS_OP_N, nci, 3, F, nci, ipiv, Xs, nci, info));
    }
    check_info(STD2G_ENOCONV, "response solve");
    // residual R = B - M X
    S2G_CUDA(cudaMemcpyAsync(R, B, sizeof(double) * nci * 3, cudaMemcpyDeviceToDevice, s));
    gemm(c, CUBLAS_OP_N, CUBLAS_OP_N, nci, 3, nci, -1.0, Mw, nci, Xs, nci, 1.0, R, nci);
    // alpha = -2 mu^T (X+Y): a9[x + 3y]
    gemm(c, CUBLAS_OP_T, CUBLAS_OP_N, 3, 3, nci, -2.0, musel, nci, Xs, nci, 0.0, a9, 3);
    S2G_LAUNCH(k_resid_ratio, 1, 256, 0, s, R, B, nci, 3, a9 + 9);
    double h[10];
    S2G_CUDA(cudaMemcpyAsync(h, a9, sizeof(double) * 10, cudaMemcpyDeviceToHost, s));
    S2G_CUDA(cudaStreamSynchronize(s));
    for (int x = 0; x < 3; ++x)
      for (int y = 0; y < 3; ++y) rq.alpha[(size_t)w * 9 + 3 * x + y] = h[x + 3 * y];
    if (rq.resid) rq.resid[w] = h[9];
    if (rq.U) {
      // X+Y and X-Y = w (A-B)^-1 (X+Y) (linear_response.f:312-327)
      const size_t off = (size_t)nci * 3 * (rq.slot ? rq.slot[w] : w);
      S2G_CUDA(cudaMemcpyAsync(rq.U + off, Xs, sizeof(double) * nci * 3, cudaMemcpyDeviceToDevice,
                               s));
      gemm(c, CUBLAS_OP_N, CUBLAS_OP_N, nci, 3, nci, om, Ainv, nci, Xs, nci, 0.0, rq.V + off, nci);
    }
  }
}

// Iterative refinement of the coupled (u, v) response equations
// (response_mixed.cuh).  fp64(U, V, PU, MV) forms PU = (A+B) U and MV = (A-B) V
// in FP64; inner(pu, pv, qu, qv) the same products for the CG vectors (type T)
// in lower precision.  dp, dm: diagonals of A+B, A-B for the preconditioner.
// Frequencies whose system is not positive definite (or that do not converge)
// are returned in `fallback` (their alpha entries are left untouched).
template <typename T, typename D, class Fp64Products, class InnerProducts>
static void response_ir(Ctx &c, int n, const double *musel, const RespReq &rq,
                        std::vector<int> &fallback, const D *dp, const D *dm,
                        const Fp64Products &fp64, const InnerProducts &inner) {
  cudaStream_t s = c.stream;
  auto &w = c.rw;
  const int nw = rq.n, ncol = 3 * nw;
  if (ncol > 32) throw Error{STD2G_EINVAL, "response: at most 10 frequencies per call"};
  const size_t nc = (size_t)n * ncol;
  const int g = grid_for((int64_t)nc);
  const double tol = 1e-10;   // relative FP64 residual of every right-hand side
  const int kMaxOuter = 12, kMaxInner = 400;
  const bool prof = c.opts.verbose >= 2;
  const auto t0 = std::chrono::steady_clock::now();
  std::vector<double> hw(ncol);
  for (int j = 0; j < ncol; ++j) hw[j] = rq.omega[j / 3];
  double *wcol = w.wcol.ensure(ncol);
  S2G_CUDA(cudaMemcpyAsync(wcol, hw.data(), sizeof(double) * ncol, cudaMemcpyHostToDevice, s));
  double *B1 = w.B1.ensure(nc), *U = w.U.ensure(nc), *V = w.V.ensure(nc);
  double *PU = w.PU.ensure(nc), *MV = w.MV.ensure(nc), *R1 = w.R1.ensure(nc),
         *R2 = w.R2.ensure(nc);
  double *pa = w.pa.ensure((size_t)ncol * kRespSplit), *pb = w.pb.ensure((size_t)ncol * kRespSplit);
  double *nrm = w.nrm.ensure(ncol), *nrm2 = w.nrm2.ensure(ncol);
  S2G_LAUNCH(k_resp_rhs, g, 256, 0, s, B1, musel, n, nw);
  S2G_CUDA(cudaMemsetAsync(U, 0, sizeof(double) * nc, s));
  S2G_CUDA(cudaMemsetAsync(V, 0, sizeof(double) * nc, s));
  const dim3 rgrid(kRespSplit, (unsigned)ncol);
  const int sgrid = (int)div_up(ncol, 32);
  auto coldot64 = [&](const double *a, const double *b, double *out) {
    S2G_LAUNCH(k_resp_dot64, rgrid, 256, 0, s, a, b, n, pa);
    S2G_LAUNCH(k_resp_sum, sgrid, 32, 0, s, pa, kRespSplit, ncol, out);
  };
  std::vector<double> hb(ncol), hr(ncol), hr2(ncol), hrel(ncol, 1.0);
  coldot64(B1, B1, nrm);
  S2G_CUDA(cudaMemcpyAsync(hb.data(), nrm, sizeof(double) * ncol, cudaMemcpyDeviceToHost, s));
  // CG vectors, halves (u, v)
  T *vec[12];
  for (int q = 0; q < 12; ++q) vec[q] = (T *)w.vecs[q].ensure(nc * sizeof(T));
  T *yu = vec[0], *yv = vec[1], *ru = vec[2], *rv = vec[3], *zu = vec[4], *zv = vec[5],
    *pu = vec[6], *pv = vec[7], *qu = vec[8], *qv = vec[9], *cu = vec[10], *cv = vec[11];
  double *rz = w.rz.ensure(ncol), *al = w.alpha.ensure(ncol), *be = w.beta.ensure(ncol),
         *rr = w.rr.ensure(ncol);
  unsigned *flag = w.flag.ensure(1);
  S2G_CUDA(cudaMemsetAsync(flag, 0, sizeof(unsigned), s));
  auto pcg = [&]() {
    S2G_LAUNCH((k_pcg2_init<T, D>), rgrid, 256, 0, s, yu, yv, ru, rv, zu, zv, pu, pv, cu, cv, dp,
               dm, wcol, n, pa, pb);
    S2G_LAUNCH(k_pcg_beta, sgrid, 32, 0, s, pa, pb, kRespSplit, ncol, rz, be, rr, 1);
    std::vector<double> rr0(ncol), rrn(ncol);
    S2G_CUDA(cudaMemcpyAsync(rr0.data(), rr, sizeof(double) * ncol, cudaMemcpyDeviceToHost, s));
    S2G_CUDA(cudaStreamSynchronize(s));
    for (int it = 1; it <= kMaxInner; ++it) {
      inner(pu, pv, qu, qv);
      S2G_LAUNCH(k_pcg2_pq<T>, rgrid, 256, 0, s, qu, qv, pu, pv, wcol, n, pa);
      S2G_LAUNCH(k_pcg_alpha, sgrid, 32, 0, s, pa, kRespSplit, ncol, rz, al, flag);
      S2G_LAUNCH((k_pcg2_update<T, D>), rgrid, 256, 0, s, yu, yv, ru, rv, zu, zv, pu, pv, qu, qv,
                 dp, dm, wcol, al, n, pa, pb);
      S2G_LAUNCH(k_pcg_beta, sgrid, 32, 0, s, pa, pb, kRespSplit, ncol, rz, be, rr, 0);
      S2G_LAUNCH(k_pcg2_dir<T>, g, 256, 0, s, pu, pv, zu, zv, be, n, ncol);
      ++w.inner;
      if (it % 8 == 0) {
        S2G_CUDA(cudaMemcpyAsync(rrn.data(), rr, sizeof(double) * ncol, cudaMemcpyDeviceToHost,
                                 s));
        S2G_CUDA(cudaStreamSynchronize(s));
        bool done_all = true;
        for (int j = 0; j < ncol; ++j)
          if (rrn[j] > 1e-11 * rr0[j]) done_all = false;
        if (done_all) break;
      }
    }
  };
  w.outer = w.inner = 0;
  for (int outer = 0; outer <= kMaxOuter; ++outer) {
    // FP64 residuals of the coupled equations
    fp64(U, V, PU, MV);
    S2G_LAUNCH(k_resp_resid, g, 256, 0, s, R1, R2, B1, U, V, PU, MV, wcol, n, ncol);
    coldot64(R1, R1, nrm);
    coldot64(R2, R2, nrm2);
    S2G_CUDA(cudaMemcpyAsync(hr.data(), nrm, sizeof(double) * ncol, cudaMemcpyDeviceToHost, s));
    S2G_CUDA(cudaMemcpyAsync(hr2.data(), nrm2, sizeof(double) * ncol, cudaMemcpyDeviceToHost, s));
    unsigned hflag = 0;
    S2G_CUDA(cudaMemcpyAsync(&hflag, flag, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    S2G_CUDA(cudaStreamSynchronize(s));
    double worst = 0.0;
    for (int j = 0; j < ncol; ++j) {
      hrel[j] = hb[j] > 0 ? std::sqrt((hr[j] + hr2[j]) / hb[j]) : 0.0;
      if (!(hflag >> j & 1u)) worst = std::max(worst, hrel[j]);
    }
    w.outer = outer;
    if (worst <= tol || outer == kMaxOuter) {
      for (int fw = 0; fw < nw; ++fw) {
        bool bad = false;
        for (int x = 0; x < 3; ++x) {
          const int j = 3 * fw + x;
          bad |= (hflag >> j & 1u) != 0 || hrel[j] > tol;
        }
        if (bad) fallback.push_back(fw);
      }
      break;
    }
    // correction from the lower-precision solve of the same system
    if (sizeof(T) == sizeof(float)) {
      S2G_LAUNCH(k_d2f, g, 256, 0, s, (float *)cu, R1, (int64_t)nc);
      S2G_LAUNCH(k_d2f, g, 256, 0, s, (float *)cv, R2, (int64_t)nc);
    } else {
      S2G_CUDA(cudaMemcpyAsync(cu, R1, sizeof(double) * nc, cudaMemcpyDeviceToDevice, s));
      S2G_CUDA(cudaMemcpyAsync(cv, R2, sizeof(double) * nc, cudaMemcpyDeviceToDevice, s));
    }
    pcg();
    S2G_LAUNCH(k_resp_accum<T>, g, 256, 0, s, U, V, yu, yv, (int64_t)nc);
  }
  if (prof) {
    S2G_CUDA(cudaStreamSynchronize(s));
    std::fprintf(stderr, "response (refined): %d refinement steps, %d CG steps, %.2f ms\n",
                 w.outer, w.inner,
                 std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0)
                     .count());
  }
  // alpha = -2 mu^T (X+Y) per frequency
  double *a9 = c.w_props.ensure(16);
  for (int fw = 0; fw < nw; ++fw) {
    if (std::find(fallback.begin(), fallback.end(), fw) != fallback.end()) continue;
    if (rq.U) {
      const size_t off = (size_t)n * 3 * (rq.slot ? rq.slot[fw] : fw);
      S2G_CUDA(cudaMemcpyAsync(rq.U + off, U + (size_t)n * 3 * fw, sizeof(double) * n * 3,
                               cudaMemcpyDeviceToDevice, s));
      S2G_CUDA(cudaMemcpyAsync(rq.V + off, V + (size_t)n * 3 * fw, sizeof(double) * n * 3,
                               cudaMemcpyDeviceToDevice, s));
    }
    gemm(c, CUBLAS_OP_T, CUBLAS_OP_N, 3, 3, n, -2.0, musel, n, U + (size_t)n * 3 * fw, n, 0.0,
         a9, 3);
    double ha[9];
    S2G_CUDA(cudaMemcpyAsync(ha, a9, sizeof(double) * 9, cudaMemcpyDeviceToHost, s));
    S2G_CUDA(cudaStreamSynchronize(s));
    for (int x = 0; x < 3; ++x)
      for (int yy = 0; yy < 3; ++yy) rq.alpha[(size_t)fw * 9 + 3 * x + yy] = ha[x + 3 * yy];
    if (rq.resid) {
      double wf = 0;
      for (int x = 0; x < 3; ++x) wf = std::max(wf, hrel[3 * fw + x]);
      rq.resid[fw] = wf;
    }
  }
}

// Mixed form with the dense matrices: FP64 residual products with A+B, A-B,
// FP32 copies of both for the CG products.
static void response_mixed(Ctx &c, const double *Apb, const double *Amb, int n,
                           const double *musel, const RespReq &rq, std::vector<int> &fallback) {
  cudaStream_t s = c.stream;
  auto &w = c.rw;
  const size_t n2 = (size_t)n * n;
  const int ncol = 3 * rq.n;
  float *Apb32 = w.Apb32.ensure(n2), *Amb32 = w.Amb32.ensure(n2);
  S2G_LAUNCH(k_d2f, grid_for((int64_t)n2), 256, 0, s, Apb32, Apb, (int64_t)n2);
  S2G_LAUNCH(k_d2f, grid_for((int64_t)n2), 256, 0, s, Amb32, Amb, (int64_t)n2);
  float *dp = w.dp.ensure(n), *dm = w.dm.ensure(n);
  S2G_LAUNCH(k_resp_diags, (int)div_up(n, 256), 256, 0, s, Apb, Amb, n, dp, dm);
  cublasHandle_t h = c.blas;
  const float one = 1.f, zero = 0.f;
  const double done = 1.0, dzero = 0.0;
  auto fp64 = [&](const double *U, const double *V, double *PU, double *MV) {
    c.dg.gemm(s, CUBLAS_OP_N, CUBLAS_OP_N, n, ncol, n, &done, Apb, n, U, n, &dzero, PU, n);
    c.dg.gemm(s, CUBLAS_OP_N, CUBLAS_OP_N, n, ncol, n, &done, Amb, n, V, n, &dzero, MV, n);
  };
  auto inner = [&](const float *pu, const float *pv, float *qu, float *qv) {
    S2G_CUBLAS(cublasSgemm(h, CUBLAS_OP_N, CUBLAS_OP_N, n, ncol, n, &one, Apb32, n, pu, n, &zero,
                           qu, n));
    S2G_CUBLAS(cublasSgemm(h, CUBLAS_OP_N, CUBLAS_OP_N, n, ncol, n, &one, Amb32, n, pv, n, &zero,
                           qv, n));
  };
  response_ir<float, float>(c, n, musel, rq, fallback, dp, dm, fp64, inner);
}

// Matrix-free form (no n x n storage): products with A+B, A-B through the
// Loewdin-MO operators (k_rpa_mf_diag), FP64 (matfree.cuh) for the residuals
// and, in the mixed form, the split-BF16 tensor-core operators
// (matfree_tc.cuh) for the CG.
static void response_matfree(Ctx &c, int n, const double *musel, const RespReq &rq,
                             std::vector<int> &fallback, const double *ed, const double *ekd,
                             const double *uci, double ak, double ax, bool mixed) {
  cudaStream_t s = c.stream;
  auto &w = c.rw;
  const int ncol = 3 * rq.n;
  double *d = w.dmf.ensure(n), *dpd = w.dpd.ensure(n), *dmd = w.dmd.ensure(n);
  S2G_LAUNCH(k_rpa_mf_diag, (int)div_up(n, 128), 128, 0, s, d, dpd, dmd, ed, ekd, uci, c.mf.ci,
             c.mf.ca, n, c.mf.nv, ak, ax);
  const bool amb_diag = std::fabs(ax) < 1e-6;
  auto products = [&](const double *U, const double *V, double *PU, double *MV, bool tc) {
    if (tc)
      mftc_apply(c.mftc, c.blas, s, U, ncol, PU, 2.0 * ak, -1.0, -ax, d);
    else
      mf_apply(c.mf, c.blas, s, U, ncol, PU, 2.0 * ak, -1.0, -ax, d);
    if (amb_diag)
      S2G_LAUNCH(k_diag_mul, grid_for((int64_t)n * ncol), 256, 0, s, MV, dmd, V, n, ncol);
    else if (tc)
      mftc_apply(c.mftc, c.blas, s, V, ncol, MV, 0.0, -1.0, ax, d);
    else
      mf_apply(c.mf, c.blas, s, V, ncol, MV, 0.0, -1.0, ax, d);
  };
  auto fp64 = [&](const double *U, const double *V, double *PU, double *MV) {
    products(U, V, PU, MV, false);
  };
  auto inner = [&](const double *pu, const double *pv, double *qu, double *qv) {
    products(pu, pv, qu, qv, mixed);
  };
  response_ir<double, double>(c, n, musel, rq, fallback, dpd, dmd, fp64, inner);
}

// --------------------------------------------------------------------------
// Quadratic-response dot products G[x + nx*(y*ny + v)] = X_x . (M_y Y_v) for
// the sums of lresp1 / lresp_2PA_SP (List_A / List_B, linear_response.f:
// 1089-1167), where M_y couples CSFs that share their virtual (through
// -mu^y_ij) or their occupied MO (through mu^y_ab):
//   (M_y Y)_(i,a) = -sum_j mu^y_ij Y_(j,a) + sum_b mu^y_ab Y_(i,b)
// over the selected CSFs.  Y is scattered into (no x nv) boxes, M_y applied as
// two GEMMs with the occupied / virtual dipole blocks, gathered back at the
// CSFs and dotted with X.  X: nci x nx, Y: nci x ny (device, column-major).
static std::vector<double> quad_dots(Ctx &c, int nci, int no, int nv, const int *ci,
                                     const int *ca, const double *X, int nx, const double *Y,
                                     int ny) {
  cudaStream_t s = c.stream;
  const int64_t box = (int64_t)no * nv;
  double *bx = c.w_qbox.ensure((size_t)box * ny);
  S2G_CUDA(cudaMemsetAsync(bx, 0, sizeof(double) * box * ny, s));
  S2G_LAUNCH(k_box_scatter, grid_for((int64_t)nci * ny), 256, 0, s, bx, Y, ci, ca, nci, no, nv,
             ny);
  double *my = c.w_qmy.ensure((size_t)box * ny * 3);
  for (int y = 0; y < 3; ++y) {
    double *out = my + (size_t)box * ny * y;
    gemm(c, CUBLAS_OP_N, CUBLAS_OP_N, no, nv * ny, no, -1.0, c.w_moo.get() + (size_t)no * no * y,
         no, bx, no, 0.0, out, no);
    gemm(c, CUBLAS_OP_N, CUBLAS_OP_N, no, nv, nv, 1.0, bx, no, c.w_mvv.get() + (size_t)nv * nv * y,
         nv, 1.0, out, no, ny, box, 0, box);
  }
  double *sel = c.w_qsel.ensure((size_t)nci * 3 * ny);
  S2G_LAUNCH(k_box_gather, grid_for((int64_t)nci * 3 * ny), 256, 0, s, sel, my, ci, ca, nci, no,
             nv, 3 * ny);
  double *G = c.w_qg.ensure((size_t)nx * 3 * ny);
  gemm(c, CUBLAS_OP_T, CUBLAS_OP_N, nx, 3 * ny, nci, 1.0, X, nci, sel, nci, 0.0, G, nx);
  std::vector<double> h((size_t)nx * 3 * ny);
  S2G_CUDA(cudaMemcpyAsync(h.data(), G, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, s));
  S2G_CUDA(cudaStreamSynchronize(s));
  return h;
}

// <beta^2_ZZZ> + <beta^2_XZZ> of the hyper-Rayleigh orientational average
// (linear_response.f:1489-1662); i, j, k run over distinct axes
static double beta_hrs_value(const double b[3][3][3]) {
  double s_iii = 0, s_iij = 0, s_jii = 0, s_ijj = 0, s_ijk = 0, iii_ijj = 0, jii_iij = 0,
         iii_jji = 0, iij_jii = 0, iij_jkk = 0, jii_jkk = 0, iij_kkj = 0, ijk_jik = 0,
         ijj_ikk = 0, iik_jjk = 0;
  for (int i = 0; i < 3; ++i) {
    s_iii += b[i][i][i] * b[i][i][i];
    for (int j = 0; j < 3; ++j) {
      if (j == i) continue;
      s_iij += b[i][i][j] * b[i][i][j];
      s_jii += b[j][i][i] * b[j][i][i];
      s_ijj += b[i][j][j] * b[i][j][j];
      iii_ijj += b[i][i][i] * b[i][j][j];
      jii_iij += b[j][i][i] * b[i][i][j];
      iii_jji += b[i][i][i] * b[j][j][i];
      iij_jii += b[i][i][j] * b[j][i][i];
      for (int k = 0; k < 3; ++k) {
        if (k == i || k == j) continue;
        s_ijk += b[i][j][k] * b[i][j][k];
        iij_jkk += b[i][i][j] * b[j][k][k];
        jii_jkk += b[j][i][i] * b[j][k][k];
        iij_kkj += b[i][i][j] * b[k][k][j];
        ijk_jik += b[i][j][k] * b[j][i][k];
        ijj_ikk += b[i][j][j] * b[i][k][k];
        iik_jjk += b[i][i][k] * b[j][j][k];
      }
    }
  }
  const double zzz = s_iii / 7 + 4 * s_iij / 35 + s_jii / 35 + 2 * s_ijk / 105 + 2 * iii_ijj / 35 +
                     4 * jii_iij / 35 + 4 * iii_jji / 35 + 4 * iij_jkk / 105 + jii_jkk / 105 +
                     4 * iij_kkj / 105 + 4 * ijk_jik / 105;
  const double xzz = s_iii / 35 + 4 * iii_ijj / 105 - 2 * iii_jji / 35 + 8 * s_iij / 105 -
                     2 * iij_jkk / 105 + 2 * s_ijk / 35 - 2 * ijk_jik / 105 + 3 * s_ijj / 35 -
                     2 * iij_jii / 35 + ijj_ikk / 35 - 2 * iik_jjk / 105;
  return std::sqrt(zzz + xzz);
}

// beta(-2w; w, w) from the response vectors of the frequency pairs
// (w_k, -2 w_k) in slots (2k, 2k+1) of U = X+Y, V = X-Y (lresp1,
// linear_response.f:196-700: beta = A - B summed over the six assignments of
// the axes to the -2w X vector, the dipole and the w Y vector).
static void hyperpolarizability(Ctx &c, int nci, int no, int nv, const int *ci, const int *ca,
                                const double *U, const double *V, const QuadReq &q) {
  cudaStream_t s = c.stream;
  double *Xa = c.w_qx.ensure((size_t)nci * 6), *Ya = c.w_qy.ensure((size_t)nci * 6);
  for (int kk = 0; kk < q.nbeta; ++kk) {
    // columns (w-1)*3 + x of X and Y: w = 1 the +w vectors, w = 2 the -2w ones
    for (int w = 0; w < 2; ++w) {
      const size_t off = (size_t)nci * 3 * (2 * kk + w);
      S2G_LAUNCH(k_xy_from_uv, grid_for((int64_t)nci * 3), 256, 0, s, Xa + (size_t)nci * 3 * w,
                 Ya + (size_t)nci * 3 * w, U + off, V + off, (int64_t)nci * 3, 0.5);
    }
    const std::vector<double> G = quad_dots(c, nci, no, nv, ci, ca, Xa, 6, Ya, 6);
    // T(x, wx, y, z, wz) = X_wx[:, x] . M_y . Y_wz[:, z]
    auto T = [&](int x, int wx, int y, int z, int wz) {
      return G[(size_t)((wx - 1) * 3 + x) + 6 * (size_t)(y * 6 + (wz - 1) * 3 + z)];
    };
    double b[3][3][3];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j)
        for (int k = 0; k < 3; ++k) {
          b[i][j][k] = T(i, 2, j, k, 1) + T(i, 2, k, j, 1) + T(j, 1, k, i, 2) + T(j, 1, i, k, 1) +
                       T(k, 1, i, j, 1) + T(k, 1, j, i, 2);
          q.beta[(size_t)kk * 27 + 9 * i + 3 * j + k] = b[i][j][k];
        }
    if (q.beta_hrs) q.beta_hrs[kk] = beta_hrs_value(b);
  }
}

static void response(Ctx &c, double *Apb, double *Amb, int nci, const double *musel,
                     const RespReq &rq);

// Two-photon absorption of the lowest q.ntpa sTD-DFT states (lresp_2PA_SP,
// linear_response.f:4604-4938; TPA_resp_fast_SP :4940-5025): for state n the
// response to -mu at w = -w_n / 2 gives X, Y per axis, and
//   sigma_xy = -1/2 [X_x M_y Yn + X_y M_x Yn + Xn M_x Y_y + Xn M_y Y_x]
// with the state vectors Xn, Yn (w_tpx, w_tpy); F, G, H (each / 30) give
// delta_par = 2F+2G+2H, delta_perp = -F+4G-H, delta_circ = -2F+3G+3H and
// rho = delta_par / delta_perp.  The responses are the FP64 form's dense
// solves of the A+B, A-B built for the states.
static void two_photon(Ctx &c, int nci, int no, int nv, const int *ci, const int *ca,
                       const double *musel, const std::vector<double> &w, const QuadReq &q) {
  cudaStream_t s = c.stream;
  const int nt = q.ntpa;
  double *Xq = c.w_qx.ensure((size_t)nci * 4), *Yq = c.w_qy.ensure((size_t)nci * 4);
  for (int n0 = 0; n0 < nt; n0 += 10) {
    const int ng = std::min(10, nt - n0);
    std::vector<double> om(ng), al((size_t)ng * 9), rs(ng);
    for (int k = 0; k < ng; ++k) om[k] = -0.5 * w[n0 + k];
    RespReq sub{om.data(), ng, al.data(), rs.data()};
    sub.U = c.w_Uall.ensure((size_t)nci * 3 * ng);
    sub.V = c.w_Vall.ensure((size_t)nci * 3 * ng);
    response(c, c.w_Apb.get(), c.w_Amb.get(), nci, musel, sub);
    for (int k = 0; k < ng; ++k) {
      const int n = n0 + k;
      const size_t off = (size_t)nci * 3 * k;
      // the solver answers -2 mu: a quarter of U +- V is X, Y for -mu
      S2G_LAUNCH(k_xy_from_uv, grid_for((int64_t)nci * 3), 256, 0, s, Xq, Yq, sub.U + off,
                 sub.V + off, (int64_t)nci * 3, 0.25);
      S2G_CUDA(cudaMemcpyAsync(Xq + (size_t)nci * 3, c.w_tpx.get() + (size_t)nci * n,
                               sizeof(double) * nci, cudaMemcpyDeviceToDevice, s));
      S2G_CUDA(cudaMemcpyAsync(Yq + (size_t)nci * 3, c.w_tpy.get() + (size_t)nci * n,
                               sizeof(double) * nci, cudaMemcpyDeviceToDevice, s));
      const std::vector<double> G = quad_dots(c, nci, no, nv, ci, ca, Xq, 4, Yq, 4);
      auto T = [&](int a, int y, int v) { return G[(size_t)a + 4 * (size_t)(y * 4 + v)]; };
      double sg[3][3], tr = 0.0, g2 = 0.0, h2 = 0.0;
      for (int x = 0; x < 3; ++x)
        for (int y = 0; y < 3; ++y)
          sg[x][y] = -0.5 * (T(x, y, 3) + T(y, x, 3) + T(3, x, y) + T(3, y, x));
      for (int x = 0; x < 3; ++x) {
        tr += sg[x][x];
        for (int y = 0; y < 3; ++y) {
          g2 += sg[x][y] * sg[x][y];
          h2 += sg[x][y] * sg[y][x];
        }
      }
      const double F = tr * tr / 30.0, Gs = g2 / 30.0, H = h2 / 30.0;
      const double par = 2 * F + 2 * Gs + 2 * H, perp = -F + 4 * Gs - H;
      double *row = q.tpa + (size_t)6 * n;
      row[0] = n + 1;
      row[1] = w[n] * 27.21139;
      row[2] = par;
      row[3] = perp;
      row[4] = -2 * F + 3 * Gs + 3 * H;
      row[5] = par / perp;
    }
  }
}

static void solve(Ctx &c, const std2g_params &p_in, std2g_result *res, const RespReq *resp,
                  const QuadReq *tpa = nullptr) {
  if (!c.loaded) throw Error{STD2G_ESTATE, "solve before load"};
  std2g_params p = p_in;
  if (resp) {
    if (p.triplet) throw Error{STD2G_EINVAL, "response: triplet not available"};
    p.rpa = 1;
    p.velcorr = 0;
  }
  cudaStream_t s = c.stream;
  const int N = c.ncent, nao = c.nao;
  const bool mixed = c.opts.precision == 1;
  c.tc_ms = 0;
  c.tc_flop = 0;
  c.tc_launches = 0;
  c.dg.reset();
  c.mftc.side.dg.reset();
  c.mixed.rechecked = 0;
  c.mixed.ed_bound_max = 0.0;   // the FP64 PT path lowers the diagonal in FP64
  c.dav_iters = 0;
  c.dav_matvecs = 0;
  c.dav_fp64_matvecs = 0;
  record(c, PH_SETUP);
  const double thr = p.e_thr_ev / kEh2eV_in;
  const double fthr = p.fthr_ev < 1.79e308 ? p.fthr_ev / kEh2eV_in : INFINITY;
  if (c.uks) {
    if (p.triplet) throw Error{STD2G_EINVAL, "unrestricted input: no triplet keyword (sutda)"};
    if (resp || tpa)
      throw Error{STD2G_EINVAL, "unrestricted input: response and 2PA are restricted-only"};
  }
  // UCIS scaling of (ia|jb): 1 unrestricted (sutda.f:625), 2 singlet, 0 triplet
  const double ak = c.uks ? 1.0 : (p.triplet ? 0.0 : 2.0);
  const double beta_j = p.beta_j >= -99.0 ? p.beta_j : 0.20 + 1.830 * p.ax;
  const double alpha_k = p.alpha_k >= -99.0 ? p.alpha_k : 1.420 + 0.480 * p.ax;
  const bool want_quad = (resp && resp->quad) || (tpa && tpa->ntpa > 0);

  // ---- orbital window and energy sort (stda.f:145-192, 261-308, 333) ----
  const double deps = 2.0 * (1.0 + 0.8 * p.ax) * thr;
  // occupation limits: closed shell 2 / 0; unrestricted 1 / 0 per spin MO
  // (sutda.f:169-174: occ > 0.99, occ < 0.01)
  const double occ_hi = c.uks ? 0.99 : 1.990;
  double omax = -1e42, vmin = 1e42;
  for (int i = 0; i < c.nmo; ++i) {
    if (c.h_occ[i] > occ_hi && c.h_eps[i] > omax) omax = c.h_eps[i];
    if (c.h_occ[i] < 0.010 && c.h_eps[i] < vmin) vmin = c.h_eps[i];
  }
  auto by_eps = [&](int a, int b) { return c.h_eps[a] < c.h_eps[b]; };
  std::vector<int> oidx, vidx;
  UksScreen us;
  if (!c.uks) {
    for (int i = 0; i < c.nmo; ++i) {
      if (c.h_occ[i] > 1.990 && c.h_eps[i] > vmin - deps) oidx.push_back(i);
      if (c.h_occ[i] < 0.010 && c.h_eps[i] < omax + deps) vidx.push_back(i);
    }
    std::stable_sort(oidx.begin(), oidx.end(), by_eps);
    std::stable_sort(vidx.begin(), vidx.end(), by_eps);
  } else {
    // sutda.f:178-360: per spin, occupied then virtual, each sorted by energy;
    // the window's occupied MOs are alpha then beta, its virtual ones alike
    int nocc_a = 0, nocc_b = 0;
    std::vector<int> o[2], v[2];
    for (int i = 0; i < c.nmo; ++i) {
      const int sp = c.h_csp[i] - 1;
      if (c.h_occ[i] > 0.99) (sp == 0 ? nocc_a : nocc_b)++;
      if (c.h_occ[i] > 0.99 && c.h_eps[i] > vmin - deps) o[sp].push_back(i);
      if (c.h_occ[i] < 0.010 && c.h_eps[i] < omax + deps) v[sp].push_back(i);
    }
    for (int sp = 0; sp < 2; ++sp) {
      std::stable_sort(o[sp].begin(), o[sp].end(), by_eps);
      std::stable_sort(v[sp].begin(), v[sp].end(), by_eps);
    }
    oidx = o[0];
    oidx.insert(oidx.end(), o[1].begin(), o[1].end());
    vidx = v[0];
    vidx.insert(vidx.end(), v[1].begin(), v[1].end());
    const int nuhf = nocc_a - nocc_b;
    us.uks = 1;
    us.noa = (int)o[0].size();
    us.nob = (int)o[1].size();
    us.nva = (int)v[0].size();
    us.nsomo_a = us.noa - nuhf;
    us.nsomo_b = us.nob + nuhf;
    us.sau2 = p.shftmax_somo * 0.036749320;
    us.wau2 = p.shftwidth * 0.036749320 * 5.0;
    if ((o[0].empty() || v[0].empty()) && (o[1].empty() || v[1].empty()))
      throw Error{STD2G_ENOCSF, "no CSF, increase energy threshold"};
  }
  const int no = (int)oidx.size(), nv = (int)vidx.size(), moci = no + nv;
  if (no == 0 || nv == 0) throw Error{STD2G_ENOCSF, "no CSF, increase energy threshold"};
  std::vector<int> act(oidx);
  act.insert(act.end(), vidx.begin(), vidx.end());
  std::vector<double> eps_act(moci);
  for (int m = 0; m < moci; ++m) eps_act[m] = c.h_eps[act[m]];
  S2G_CUDA(cudaMemcpyAsync(c.w_act_idx.ensure(moci), act.data(), sizeof(int) * moci,
                           cudaMemcpyHostToDevice, s));
  S2G_CUDA(cudaMemcpyAsync(c.d_eps_act.ensure(moci), eps_act.data(), sizeof(double) * moci,
                           cudaMemcpyHostToDevice, s));
  double *Cact = c.w_Cact.ensure((size_t)nao * moci);
  S2G_LAUNCH(k_gather_cols, grid_for((int64_t)nao * moci), 256, 0, s, Cact, c.d_C.get(),
             (int64_t)nao, c.w_act_idx.get(), (int64_t)moci, (int64_t)nao);

  // ---- S^1/2 (makel stda.f:1615-1691), once per load ----
  record(c, PH_SQRTS);
  if (!c.sqrtS_ready) {
    sqrt_overlap(c, c.d_Sfull.get(), nao, c.d_sqrtS.ensure((size_t)nao * nao));
    c.sqrtS_ready = true;
  }
  double *Clow = c.w_Clow.ensure((size_t)nao * moci);
  gemm(c, CUBLAS_OP_N, CUBLAS_OP_N, nao, moci, nao, 1.0, c.d_sqrtS.get(), nao, Cact, nao, 0.0,
       Clow, nao);
  int *status = c.w_status.ensure(4);
  S2G_CUDA(cudaMemsetAsync(status, 0, sizeof(int) * 4, s));
  S2G_LAUNCH(k_colnorm_check, moci, 256, 0, s, Clow, nao, moci, status);

  // ---- MO property integrals, occ-virt block (ONETRI, stda.f:351-412) ----
  record(c, PH_MOINT);
  {
    size_t nn = (size_t)nao * nao;
    double *T = c.w_T.ensure((size_t)nao * nv * 9);
    double *mu = c.w_mu_ov.ensure((size_t)no * nv * 9);
    // T_q = O_q C_v, mu_q = C_o^T T_q for the nine AO operators (batched)
    gemm(c, CUBLAS_OP_N, CUBLAS_OP_N, nao, nv, nao, 1.0, c.d_ao9.get(), nao,
         Cact + (size_t)nao * no, nao, 0.0, T, nao, 9, (int64_t)nn, 0, (int64_t)nao * nv);
    gemm(c, CUBLAS_OP_T, CUBLAS_OP_N, no, nv, nao, 1.0, Cact, nao, T, nao, 0.0, mu, no, 9, 0,
         (int64_t)nao * nv, (int64_t)no * nv);
    if (want_quad) {
      // length dipoles of the occupied-occupied and virtual-virtual blocks
      // (the same packed moci x moci transform, stda.f:351-412; lresp1 reads them)
      double *To = c.w_To.ensure((size_t)nao * no * 3);
      gemm(c, CUBLAS_OP_N, CUBLAS_OP_N, nao, no, nao, 1.0, c.d_ao9.get(), nao, Cact, nao, 0.0, To,
           nao, 3, (int64_t)nn, 0, (int64_t)nao * no);
      gemm(c, CUBLAS_OP_T, CUBLAS_OP_N, no, no, nao, 1.0, Cact, nao, To, nao, 0.0,
           c.w_moo.ensure((size_t)no * no * 3), no, 3, 0, (int64_t)nao * no, (int64_t)no * no);
      gemm(c, CUBLAS_OP_T, CUBLAS_OP_N, nv, nv, nao, 1.0, Cact + (size_t)nao * no, nao, T, nao,
           0.0, c.w_mvv.ensure((size_t)nv * nv * 3), nv, 3, 0, (int64_t)nao * nv,
           (int64_t)nv * nv);
    }
  }

  // ---- gamma and charges (stda.f:465-479, 509-532, 558-590, 728-763) ----
  record(c, PH_CHARGES);
  double *gj = c.w_gj.ensure((size_t)N * N), *gk = c.w_gk.ensure((size_t)N * N);
  S2G_LAUNCH(k_gamma, grid_for((int64_t)N * N), 256, 0, s, c.d_xyz.get(), c.d_eta.get(), N, p.ax,
             alpha_k, beta_j, gj, gk);
  const int64_t nov = (int64_t)no * nv;
  double *Qii = c.w_Qii.ensure((size_t)N * no), *Qaa = c.w_Qaa.ensure((size_t)N * nv);
  double *Qia = c.w_Qia.ensure((size_t)N * nov), *Pia = c.w_Pia.ensure((size_t)N * nov);
  double *Qoo = c.w_Qoo.ensure((size_t)N * no * no), *Poo = c.w_Poo.ensure((size_t)N * no * no);
  double *Qvv = c.w_Qvv.ensure((size_t)N * nv * nv);
  const int *aop = c.d_ao_ptr.get(), *aol = c.d_ao_list.get();
  S2G_LAUNCH(k_charges_block, grid_for((int64_t)N * no), 256, 0, s, Qii, Clow, nao, N, aop, aol,
             0, no, 0, no, 1);
  S2G_LAUNCH(k_charges_block, grid_for((int64_t)N * nv), 256, 0, s, Qaa, Clow, nao, N, aop, aol,
             no, nv, no, nv, 1);
  {
    // full MO blocks: ia, ij, ab pairs
    const size_t shb = charges_tiled_smem(c.chunk_rows);
    if (shb > 227 * 1024) throw Error{STD2G_EINVAL, "charges: too many AOs per atom"};
    // the limit is a per-function setting shared by every context and thread:
    // always the same (maximum) value, never a size of this molecule
    S2G_CUDA(cudaFuncSetAttribute(k_charges_tiled, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  227 * 1024));
    auto tiled = [&](double *out, int p0, int np, int q0, int nq, int tri) {
      const dim3 g((unsigned)div_up(nq, kChTQ), (unsigned)div_up(np, kChTP),
                   (unsigned)div_up(N, kChAtoms));
      S2G_LAUNCH(k_charges_tiled, g, 256, shb, s, out, Clow, nao, N, aop, aol, p0, np, q0, nq,
                 c.chunk_rows, tri);
    };
    tiled(Qia, 0, no, no, nv, 0);
    tiled(Qoo, 0, no, 0, no, 1);   // only q_ij, j <= i: it feeds P_oo alone
    tiled(Qvv, no, nv, no, nv, 0);
    if (c.uks) {
      S2G_LAUNCH(k_zero_cross_spin, grid_for((int64_t)N * no * nv), 256, 0, s, Qia, N, no, nv,
                 us.noa, us.nva);
      S2G_LAUNCH(k_zero_cross_spin, grid_for((int64_t)N * no * no), 256, 0, s, Qoo, N, no, no,
                 us.noa, us.noa);
      S2G_LAUNCH(k_zero_cross_spin, grid_for((int64_t)N * nv * nv), 256, 0, s, Qvv, N, nv, nv,
                 us.nva, us.nva);
    }
  }
  // p = gamma q (ssymm, stda.f:558-590, 742-743)
  double *Pii = c.w_Pii.ensure((size_t)N * no), *uci = c.w_uci.ensure((size_t)nv * no);
  gemm(c, CUBLAS_OP_N, CUBLAS_OP_N, N, no, N, 1.0, gj, N, Qii, N, 0.0, Pii, N);
  gemm(c, CUBLAS_OP_T, CUBLAS_OP_N, nv, no, N, 1.0, Qaa, N, Pii, N, 0.0, uci, nv);
  gemm(c, CUBLAS_OP_N, CUBLAS_OP_N, N, (int)nov, N, 1.0, gk, N, Qia, N, 0.0, Pia, N);
  // P_oo is symmetric in (i, j): the product over the pairs j <= i, then the
  // upper pairs mirrored
  c.dg.run(s, false, false, N, no * no, N, 1.0, gj, N, 0, Qoo, N, 0, 0.0, Poo, N, 0, 1, no);
  S2G_LAUNCH(k_mirror_pairs, grid_for((int64_t)no * no * N), 256, 0, s, Poo, N, no);

  // ---- diagonal + energy screen (stda.f:593-668) ----
  record(c, PH_SCREEN);
  double *de = c.w_de.ensure(nov), *ek = c.w_ek.ensure(nov);
  int *flag = c.w_flag.ensure(nov);
  S2G_LAUNCH(k_diag_screen, grid_for(nov * 32), 256, 0, s, Pia, Qia, N, no, nv,
             c.d_eps_act.get(), uci, ak, p.kshift, p.shftmax * 0.036749320,
             p.shftwidth * 0.036749320, p.shftsteep, thr, fthr, de, ek, flag, us);
  std::vector<int> h_flag(nov);
  int h_status[4];
  S2G_CUDA(cudaMemcpyAsync(h_flag.data(), flag, sizeof(int) * nov, cudaMemcpyDeviceToHost, s));
  S2G_CUDA(cudaMemcpyAsync(h_status, status, sizeof(int) * 4, cudaMemcpyDeviceToHost, s));
  S2G_CUDA(cudaStreamSynchronize(s));
  if (h_status[0] != 0) throw Error{STD2G_EMONORM, "internal MO norm error"};
  std::vector<int> pk_unsorted, ck;
  for (int64_t k = 0; k < nov; ++k) {
    if (h_flag[k] == 1) pk_unsorted.push_back((int)k);
    else if (h_flag[k] == 2) ck.push_back((int)k);
  }
  const int nex = (int)pk_unsorted.size(), nexpt = (int)ck.size();
  if (nex < 1) throw Error{STD2G_ENOCSF, "no CSF, increase energy threshold"};
  // energy sort of primaries, stable in (i,a) enumeration order (stda.f:651-668)
  std::vector<int> pk(nex);
  std::vector<double> ed(nex);
  {
    int *d_in = c.w_tmpi.ensure(2 * (size_t)nex);
    S2G_CUDA(cudaMemcpyAsync(d_in, pk_unsorted.data(), sizeof(int) * nex, cudaMemcpyHostToDevice, s));
    double *keys_in = c.w_ed.ensure(2 * (size_t)nex);
    // gather keys on device
    S2G_LAUNCH(k_gather_cols, grid_for(nex), 256, 0, s, keys_in, de, (int64_t)1, d_in,
               (int64_t)nex, (int64_t)1);
    size_t tmpb = 0;
    S2G_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmpb, keys_in, keys_in + nex, d_in,
                                             d_in + nex, nex, 0, 64, s));
    char *tmp = c.w_cub.ensure(tmpb + 16);
    S2G_CUDA(cub::DeviceRadixSort::SortPairs(tmp, tmpb, keys_in, keys_in + nex, d_in, d_in + nex,
                                             nex, 0, 64, s));
    S2G_CUDA(cudaMemcpyAsync(pk.data(), d_in + nex, sizeof(int) * nex, cudaMemcpyDeviceToHost, s));
    S2G_CUDA(cudaMemcpyAsync(ed.data(), keys_in + nex, sizeof(double) * nex,
                             cudaMemcpyDeviceToHost, s));
    S2G_CUDA(cudaStreamSynchronize(s));
  }

  // ---- PT selection (ptselect, stda.f:1773-1863) ----
  record(c, PH_PT);
  std::vector<int> newk;
  std::vector<double> ed_lowered(ed);
  if (nexpt > 0) {
    // Mixed form: the couplings go to the tensor cores once there are enough
    // of them (candidates x primaries); smaller problems are latency-bound and
    // use the FP64 GEMMs, which give the FP64 selection directly.
    const bool tc_pt = mixed && ((c.opts.flags & STD2G_FLAG_TENSOR_ALWAYS) ||
                                 (double)nexpt * (double)nex >= 2.5e8);
    std::vector<int> kpos(nov, -1);
    for (int q = 0; q < nex; ++q) kpos[pk[q]] = q;
    unsigned char *sel = c.w_sel.ensure(nexpt);
    double *pert = c.w_pert.ensure(nexpt);
    double *pt2 = c.w_pt2.ensure(nex), *edp = c.w_edp.ensure(nex);
    // The PT kernels see the primaries in (j,b) enumeration order (FP64 form:
    // contiguous coupling reads) or (b,j) order (mixed form: the J
    // contraction grouped by virtual index); pt2 is mapped back to the energy
    // order afterwards.
    std::vector<int> pko = pk_unsorted;
    if (tc_pt)
      std::stable_sort(pko.begin(), pko.end(),
                       [&](int x, int y) { return x % nv < y % nv; });   // (b, j)
    std::vector<double> edo(nex);
    for (int q = 0; q < nex; ++q) edo[q] = ed[kpos[pko[q]]];
    if (tc_pt) {
      PtProblem pb{N, no, nv, Pia, Qia, Poo, Qvv, de, ak, p.thrp, 6.0e9};
      c.mixed.profile = c.opts.verbose >= 2;
      mixed_pt_select(c.mixed, s, pb, pko, edo, ck, pert, sel, pt2, edp);
      if (c.mixed.profile)
        std::fprintf(stderr,
                     "pt select (mixed): operands %.2f, (ia|jb) %.2f, (ij|ab) %.2f, rows %.2f, "
                     "recheck %.2f (%lld rows), columns %.2f ms\n",
                     c.mixed.sec_ms[0], c.mixed.sec_ms[1], c.mixed.sec_ms[2], c.mixed.sec_ms[3],
                     c.mixed.sec_ms[4], (long long)c.mixed.rechecked, c.mixed.sec_ms[5]);
      c.tc_ms = c.mixed.ms;
      c.tc_flop = c.mixed.flop;
      c.tc_launches = c.mixed.launches;
    } else {
      // FP64 form: explicit K (candidates x primaries) and the (i,j) x (a,b)
      // box of J per chunk of candidate occupied indices, FP64 GEMMs
      std::vector<int> omap(no, -1), vmap(nv, -1), OP, VP, pj(nex), pb(nex);
      for (int q = 0; q < nex; ++q) {
        pj[q] = pko[q] / nv;
        pb[q] = pko[q] % nv;
        omap[pj[q]] = 1;
        vmap[pb[q]] = 1;
      }
      for (int i = 0; i < no; ++i)
        if (omap[i] >= 0) { omap[i] = (int)OP.size(); OP.push_back(i); }
      for (int a = 0; a < nv; ++a)
        if (vmap[a] >= 0) { vmap[a] = (int)VP.size(); VP.push_back(a); }
      const int nop = (int)OP.size(), nvp = (int)VP.size();
      auto up = [&](DBuf<int> &b, const std::vector<int> &v) {
        int *d = b.ensure(v.size());
        S2G_CUDA(cudaMemcpyAsync(d, v.data(), sizeof(int) * v.size(), cudaMemcpyHostToDevice, s));
        return d;
      };
      int *d_pk = up(c.w_pk, pko), *d_ck = up(c.w_ck, ck), *d_pj = up(c.w_pj, pj),
          *d_pb = up(c.w_pb, pb), *d_omap = up(c.w_omap, omap), *d_vmap = up(c.w_vmap, vmap),
          *d_OP = up(c.w_OP, OP), *d_VP = up(c.w_VP, VP);
      double *d_ed = c.w_edsorted.ensure(nex);
      S2G_CUDA(cudaMemcpyAsync(d_ed, edo.data(), sizeof(double) * nex, cudaMemcpyHostToDevice, s));
      // primaries' charges and the virtual-pair factor
      double *Qp = c.w_Qp.ensure((size_t)N * nex);
      S2G_LAUNCH(k_gather_cols, grid_for((int64_t)N * nex), 256, 0, s, Qp, Qia, (int64_t)N, d_pk,
                 (int64_t)nex, (int64_t)N);
      double *QvvP = c.w_QvvP.ensure((size_t)N * nv * nvp);
      S2G_LAUNCH(k_gather_virt_pairs, grid_for((int64_t)N * nv * nvp), 256, 0, s, QvvP, Qvv, N, nv,
                 d_VP, nvp);
      // chunk candidates by occupied index (candidates are in (i,a) order)
      const int64_t ldj = (int64_t)nv * nvp;
      const double budget = 6.0e9;   // bytes of K/J buffers per chunk
      const double per_occ = 8.0 * ((double)nex * nv + (double)ldj * nop) + 8.0 * (double)N * (nv + nop);
      int occ_chunk = std::max(1, (int)std::min<double>(no, budget / per_occ));
      std::vector<int> first_of_occ(no + 1, nexpt);
      {
        int q = 0;
        for (int i = 0; i <= no; ++i) {
          while (q < nexpt && ck[q] / nv < i) ++q;
          first_of_occ[i] = q;
        }
      }
      int nchunk = (int)div_up(no, occ_chunk);
      // column sums of the PT terms by segments of candidate rows (deterministic order)
      const int kSeg = 2048;
      std::vector<int> seg_off(nchunk + 1, 0);
      for (int q = 0; q < nchunk; ++q) {
        int a0 = q * occ_chunk, a1 = std::min(no, a0 + occ_chunk);
        int nrq = first_of_occ[a1] - first_of_occ[a0];
        seg_off[q + 1] = seg_off[q] + (int)div_up(nrq, kSeg);
      }
      const int nseg_total = std::max(1, seg_off[nchunk]);
      double *colpart = c.w_colpart.ensure((size_t)nseg_total * nex);
      for (int q = 0; q < nchunk; ++q) {
        int i0 = q * occ_chunk, i1 = std::min(no, i0 + occ_chunk), ni = i1 - i0;
        int r0 = first_of_occ[i0], r1 = first_of_occ[i1], nr = r1 - r0;
        if (nr == 0) continue;
        const dim3 cgrid((unsigned)div_up(nex, 128), (unsigned)(seg_off[q + 1] - seg_off[q]));
        double *cpart = colpart + (size_t)seg_off[q] * nex;
        double *Pc = c.w_Pc.ensure((size_t)N * nr);
        S2G_LAUNCH(k_gather_cols, grid_for((int64_t)N * nr), 256, 0, s, Pc, Pia, (int64_t)N,
                   d_ck + r0, (int64_t)nr, (int64_t)N);
        double *W = c.w_W.ensure((size_t)N * ni * nop);
        S2G_LAUNCH(k_gather_occ_pairs, grid_for((int64_t)N * ni * nop), 256, 0, s, W, Poo, N, no,
                   i0, ni, d_OP, nop);
        double *Kb = c.w_Kbuf.ensure((size_t)nex * nr);
        double *Jb = c.w_Jbuf.ensure((size_t)ldj * ni * nop);
        gemm(c, CUBLAS_OP_T, CUBLAS_OP_N, nex, nr, N, 1.0, Qp, N, Pc, N, 0.0, Kb, nex);
        gemm(c, CUBLAS_OP_T, CUBLAS_OP_N, (int)ldj, ni * nop, N, 1.0, QvvP, N, W, N, 0.0, Jb,
             (int)ldj);
        S2G_LAUNCH((k_pt_rows<double, double>), nr, 256, 0, s, Kb, Jb, ldj, (int64_t)nex, nex,
                   nvp, nop, nr, d_ck + r0, nv, i0, de, d_pj, d_pb, d_omap, d_vmap, d_ed, ak,
                   p.thrp, pert + r0, sel + r0);
        S2G_LAUNCH((k_pt_cols<double, double>), cgrid, 128, 0, s, Kb, Jb, ldj, (int64_t)nex, nex,
                   nvp, nop, nr, d_ck + r0, nv, i0, de, d_pj, d_pb, d_omap, d_vmap, d_ed, ak,
                   sel + r0, cpart, kSeg);
      }
      if (seg_off[nchunk] == 0) S2G_CUDA(cudaMemsetAsync(colpart, 0, sizeof(double) * nex, s));
      S2G_LAUNCH(k_pt2_finish, (int)div_up(nex, 128), 128, 0, s, colpart, nseg_total, nex, d_ed,
                 pt2, edp);
    }
    std::vector<unsigned char> h_sel(nexpt);
    std::vector<double> h_edp(nex);
    S2G_CUDA(cudaMemcpyAsync(h_sel.data(), sel, nexpt, cudaMemcpyDeviceToHost, s));
    S2G_CUDA(cudaMemcpyAsync(h_edp.data(), edp, sizeof(double) * nex, cudaMemcpyDeviceToHost, s));
    S2G_CUDA(cudaStreamSynchronize(s));
    for (int q = 0; q < nex; ++q) ed_lowered[kpos[pko[q]]] = h_edp[q];
    for (int q = 0; q < nexpt; ++q)
      if (h_sel[q]) newk.push_back(ck[q]);
  }
  const int nnew = (int)newk.size();
  const int nci = nex + nnew;
  std::vector<int> allk(pk);
  allk.insert(allk.end(), newk.begin(), newk.end());
  std::vector<double> ed_all(ed_lowered);
  if (nnew > 0) {
    int *d_new = c.w_tmpi.ensure(std::max<size_t>(2 * (size_t)nex, nnew));
    S2G_CUDA(cudaMemcpyAsync(d_new, newk.data(), sizeof(int) * nnew, cudaMemcpyHostToDevice, s));
    double *d_denew = c.w_pert.ensure(std::max<size_t>(nexpt, nnew));
    S2G_LAUNCH(k_gather_cols, grid_for(nnew), 256, 0, s, d_denew, de, (int64_t)1, d_new,
               (int64_t)nnew, (int64_t)1);
    std::vector<double> h_de(nnew);
    S2G_CUDA(cudaMemcpyAsync(h_de.data(), d_denew, sizeof(double) * nnew, cudaMemcpyDeviceToHost, s));
    S2G_CUDA(cudaStreamSynchronize(s));
    ed_all.insert(ed_all.end(), h_de.begin(), h_de.end());
  }
  if (c.uks) {
    // sutda's CSF order: alpha primaries (energy order), alpha PT-selected
    // (candidate order), then the same for beta (ptselect_uks, sutda.f:1929-2007)
    std::vector<int> order;
    for (int sp = 0; sp < 2; ++sp)
      for (int part = 0; part < 2; ++part)
        for (int u = part ? nex : 0; u < (part ? nci : nex); ++u)
          if ((allk[u] / nv < us.noa) == (sp == 0)) order.push_back(u);
    std::vector<int> k2(nci);
    std::vector<double> e2(nci);
    for (int u = 0; u < nci; ++u) {
      k2[u] = allk[order[u]];
      e2[u] = ed_all[order[u]];
    }
    allk.swap(k2);
    ed_all.swap(e2);
  }
  std::vector<int> ci(nci), ca(nci);
  for (int u = 0; u < nci; ++u) {
    ci[u] = allk[u] / nv;
    ca[u] = allk[u] % nv;
  }

  // ---- A / A+-B build (rtdamat stda.f:2010-2056, rrpamat stda.f:1870-2004) ----
  record(c, PH_BUILD);
  auto up = [&](DBuf<int> &b, const std::vector<int> &v) {
    int *d = b.ensure(v.size());
    S2G_CUDA(cudaMemcpyAsync(d, v.data(), sizeof(int) * v.size(), cudaMemcpyHostToDevice, s));
    return d;
  };
  int *d_ci = up(c.w_ci, ci), *d_ca = up(c.w_ca, ca), *d_allk = up(c.w_allk, allk);
  double *d_edall = c.w_ed.ensure(std::max<size_t>(2 * (size_t)nex, nci));
  S2G_CUDA(cudaMemcpyAsync(d_edall, ed_all.data(), sizeof(double) * nci, cudaMemcpyHostToDevice, s));
  const size_t n2 = (size_t)nci * nci;
  double *Qs = c.w_Qs.ensure((size_t)N * nci), *Ps = c.w_Ps.ensure((size_t)N * nci);
  S2G_LAUNCH(k_gather_cols, grid_for((int64_t)N * nci), 256, 0, s, Qs, Qia, (int64_t)N, d_allk,
             (int64_t)nci, (int64_t)N);
  S2G_LAUNCH(k_gather_cols, grid_for((int64_t)N * nci), 256, 0, s, Ps, Pia, (int64_t)N, d_allk,
             (int64_t)nci, (int64_t)N);
  double *ekd = c.w_tmp.ensure(std::max<size_t>(nci, (size_t)2 * nao * nao));
  S2G_LAUNCH(k_gather_cols, grid_for(nci), 256, 0, s, ekd, ek, (int64_t)1, d_allk, (int64_t)nci,
             (int64_t)1);
  // TDA problems with a root count above 320 CSFs use the matrix-free operators
  // and the blocked Davidson solver (a dense eigen-decomposition of 320-1024
  // CSFs took longer: 48 molecules of 20-150 atoms, 20 roots, 723 against
  // 735 ms); everything else builds the matrices explicitly.
  // (sTD-DFT roots: the matrix-free A+B, A-B products and the Davidson of
  // davidson_rpa.cuh, FP64 products in both forms)
  // A context attached to a shared batched eigensolver (std2g_attach_batch):
  // TDA root requests of 321 to kBatchMaxCsf CSFs build the dense A and join
  // the batch's lockstep Davidson (batch_davidson.cuh) instead of running
  // their own; the batch is FP64 in both forms.
  constexpr int kBatchMaxCsf = 6144;
  const bool batch_eig = c.batch != nullptr && !resp && !p.rpa && p.nroots > 0 &&
                         p.solver == 0 && nci > 320 && nci <= kBatchMaxCsf &&
                         bd_fits(nci, std::min(p.nroots, nci)) &&
                         !(c.opts.flags & STD2G_FLAG_TENSOR_ALWAYS);
  c.last_batched = batch_eig;
  const bool use_mf = !batch_eig && !resp && p.nroots > 0 &&
                      (p.solver == 2 || (p.solver == 0 && nci > 320));
  // Mixed form: the tensor-core first Davidson stage pays off once the
  // products dominate; below kTcDavidsonMin CSFs (solver auto) the solve is
  // latency-bound and runs the single FP64 stage.  The tensor-core stage
  // reaches residuals of ~1e-6; for tighter tolerances the FP64 second stage,
  // restarted from the Ritz vectors alone, would do most of the work, so those
  // also run the single FP64 stage.
  constexpr int kTcDavidsonMin = 16384;
  const bool tc_dav =
      mixed && !p.rpa && ((c.opts.flags & STD2G_FLAG_TENSOR_ALWAYS) ||
                ((p.solver == 2 || nci >= kTcDavidsonMin) && !(p.conv_tol > 0 && p.conv_tol < 1e-6)));
  // alpha(w) through the matrix-free operators and the refined iterative solve:
  // when requested (solver == 2), when the dense A+B, A-B and their work copies
  // would exceed ~24 GB, and in the mixed form from 4096 CSFs (its tensor-core
  // operator products beat the dense build there: 38 vs 80 ms for 12457 CSFs)
  const bool resp_mf =
      resp != nullptr && (p.solver == 2 || (double)nci * nci * 8.0 * 10.0 > 24e9 ||
                          (mixed && p.solver == 0 && nci > 4096));
  // the mixed form's inner products of that solve go to the tensor cores once
  // atoms x CSFs (the size of one operator product) reaches 1.5e6; below that
  // the FP64 products are as fast or faster (measured alpha at 3 w: 7.5 vs 10.1
  // ms for 20 atoms / 713 CSFs, 18.0 vs 18.4 ms for 90 / 13645, but 23.9 vs
  // 30.7 ms for 130 / 23567 and 38 vs 77 ms for 200 / 12457) and the solve is
  // the FP64 form's, which converges in its first refinement step
  constexpr double kTcResponseMinWork = 1.5e6;
  const bool tc_resp = resp_mf && mixed &&
                       ((c.opts.flags & STD2G_FLAG_TENSOR_ALWAYS) ||
                        (double)N * nci >= kTcResponseMinWork);
  double *K = nullptr, *J = nullptr, *Kx = nullptr;
  if (!use_mf && !resp_mf) {
    K = c.w_K.ensure(n2);
    J = c.w_J.ensure(n2);
    gemm(c, CUBLAS_OP_T, CUBLAS_OP_N, nci, nci, N, 1.0, Ps, N, Qs, N, 0.0, K, nci);
    // J (and the exchange couplings Kx) gathered from the box of all
    // (ij|ab) ((ib|ja)) formed by one FP64 GEMM (an (i j) x (a b) product of
    // N-long dots) while the box stays within kBoxMax doubles and within 16x
    // the nci^2 elements wanted; otherwise one gathered dot (2N loads) per
    // element
    constexpr double kBoxMax = 1.5e8;
    const int64_t noo = (int64_t)no * no, nvv = (int64_t)nv * nv;
    auto box_pays = [&](double cells) { return cells <= kBoxMax && cells <= 16.0 * (double)n2; };
    if (box_pays((double)noo * (double)nvv)) {
      double *box = c.w_jbox.ensure((size_t)(noo * nvv));
      gemm(c, CUBLAS_OP_T, CUBLAS_OP_N, (int)noo, (int)nvv, N, 1.0, Poo, N, Qvv, N, 0.0, box,
           (int)noo);
      S2G_LAUNCH(k_box_gather, grid_for(n2), 256, 0, s, J, (int64_t)nci, box, d_ci, d_ca, nci,
                 no, nv, 0);
    } else {
      S2G_LAUNCH(k_pairdot, grid_for(n2 * 32), 256, 0, s, J, (int64_t)nci, d_ci, d_ca, nci, Poo,
                 Qvv, N, no, nv, 0);
    }
    if (p.rpa || p.velcorr) {
      Kx = c.w_Kx.ensure(n2);
      if (box_pays((double)nov * (double)nov)) {
        double *box = c.w_jbox.ensure((size_t)(nov * nov));
        gemm(c, CUBLAS_OP_T, CUBLAS_OP_N, (int)nov, (int)nov, N, 1.0, Pia, N, Qia, N, 0.0, box,
             (int)nov);
        S2G_LAUNCH(k_box_gather, grid_for(n2), 256, 0, s, Kx, (int64_t)nci, box, d_ci, d_ca,
                   nci, no, nv, 1);
      } else {
        S2G_LAUNCH(k_pairdot, grid_for(n2 * 32), 256, 0, s, Kx, (int64_t)nci, d_ci, d_ca, nci,
                   Pia, Qia, N, no, nv, 1);
      }
    }
  } else {
    // matrix-free operators (matfree.cuh): padded Loewdin MOs, atom-major P
    MatFree &mf = c.mf;
    mf.N = N;
    mf.maxa = c.maxa;
    mf.no = no;
    mf.nv = nv;
    mf.nci = nci;
    mf.nao = nao;
    mf.f32 = false;
    if (resp_mf || tc_dav) {
      // tensor-core products (mixed form): the first Davidson stage, the
      // velocity correction and the CG products of the refined alpha(w) solve
      MatFreeTc &w = c.mftc;
      w.N = N;
      w.maxa = c.maxa;
      w.no = no;
      w.nv = nv;
      w.nci = nci;
      w.Qs = Qs;
      w.Ps = Ps;
      w.ci = d_ci;
      w.ca = d_ca;
    }
    if (resp_mf) {
      mf_setup_ops<double>(mf, mf.d, s, Clow, c.d_slot_ao.get(), Poo, Pia, Qs, Ps, true);
      if (tc_resp) mftc_setup(c.mftc, s, Clow, nao, c.d_slot_ao.get(), Poo, Pia);
    } else if (tc_dav) {
      // tensor-core products for the first Davidson stage (and the velocity
      // correction's exchange products)
      mftc_setup(c.mftc, s, Clow, nao, c.d_slot_ao.get(), Poo, p.velcorr ? Pia : nullptr);
    } else {
      mf_setup_ops<double>(mf, mf.d, s, Clow, c.d_slot_ao.get(), Poo, Pia, Qs, Ps,
                           p.velcorr || p.rpa);
    }
    mf.ci = d_ci;
    mf.ca = d_ca;
    S2G_LAUNCH(k_mf_diag, (int)div_up(nci, 128), 128, 0, s, mf.dA.ensure(nci), d_edall, ekd, uci,
               d_ci, d_ca, nci, nv, ak);
  }
  int nroot = 0;
  double *X = nullptr, *Yv = nullptr, *om = nullptr;
  double *Bh = nullptr;
  // FP64 residual norms of the returned roots and the eigenvalue estimates
  // around them (the error estimates of the result); empty: not formed
  std::vector<double> root_resid, root_ritz;
  if (p.rpa && use_mf) {
    // sTD-DFT roots by the subspace form of srpapack (davidson_rpa.cuh)
    record(c, PH_EIGEN);
    om = c.w_eval.ensure(std::max(nci, nao));
    const double tol = p.conv_tol > 0 ? p.conv_tol : 1e-6;
    double *d = c.rw.dmf.ensure(nci), *dpd = c.rw.dpd.ensure(nci), *dmd = c.rw.dmd.ensure(nci);
    S2G_LAUNCH(k_rpa_mf_diag, (int)div_up(nci, 128), 128, 0, s, d, dpd, dmd, d_edall, ekd, uci,
               d_ci, d_ca, nci, nv, ak, p.ax);
    const bool amb_diag = std::fabs(p.ax) < 1e-6;
    MatVec mv_p = [&](const double *V, int nb, double *W) {
      mf_apply(c.mf, c.blas, s, V, nb, W, 2.0 * ak, -1.0, -p.ax, d);
    };
    MatVec mv_m = [&](const double *V, int nb, double *W) {
      if (amb_diag)   // ax = 0: A-B is its diagonal ed - ak (ia|ia)
        S2G_LAUNCH(k_diag_mul, grid_for((int64_t)nci * nb), 256, 0, s, W, dmd, V, nci, nb);
      else
        mf_apply(c.mf, c.blas, s, V, nb, W, 0.0, -1.0, p.ax, d);
    };
    nroot = std::min(p.nroots, nci);
    X = c.w_X.ensure((size_t)nci * nroot);
    Yv = c.w_Y.ensure((size_t)nci * nroot);
    const int conv = davidson_rpa(c.dav, c.davr, c.blas, c.solver, s, mv_p, mv_m, dpd, dmd, nci,
                                  p.nroots, tol, 300, om, X, Yv);
    c.dav_iters = c.davr.iters;
    c.dav_matvecs = 0;
    c.dav_fp64_matvecs = c.davr.matvecs;
    if (conv < nroot)
      throw Error{STD2G_ENOCONV, "sTD-DFT Davidson: " + std::to_string(conv) + " of " +
                                     std::to_string(nroot) + " roots converged"};
    root_resid = c.davr.final_resid;
    root_ritz = c.davr.final_omega;
  } else if (!p.rpa && use_mf) {
    record(c, PH_EIGEN);
    om = c.w_eval.ensure(std::max(nci, nao));
    // residual norm tolerance of the final (FP64) stage; the tensor-core stage
    // stops at 1e-6 at the least, about as far as its FP32-accurate products reach
    const double tol = p.conv_tol > 0 ? p.conv_tol : 1e-6;
    const double tol1 = std::max(tol, 1e-6);
    double *Xd = c.w_X.ensure((size_t)nci * p.nroots);
    MatVec mv = [&](const double *V, int nb, double *W) {
      mf_apply(c.mf, c.blas, s, V, nb, W, ak, -1.0, 0.0, c.mf.dA.get());
    };
    int conv = 0;
    if (tc_dav) {
      // stage 1: tensor-core (split-BF16 FP32) products; stage 2: FP64 products
      // from those Ritz vectors until the FP64 residuals meet tol
      MatVec mv_tc = [&](const double *V, int nb, double *W) {
        mftc_apply(c.mftc, c.blas, s, V, nb, W, ak, -1.0, 0.0, c.mf.dA.get());
      };
      c.dav.profile = c.opts.verbose >= 2;
      for (double &v : c.dav.sec_ms) v = 0;
      davidson(c.dav, c.blas, c.solver, s, mv_tc, d_edall, nci, p.nroots, tol1, 300, om, Xd);
      c.dav_iters = c.dav.iters;
      c.dav_matvecs = c.dav.matvecs;
      if (c.dav.profile)
        std::fprintf(stderr,
                     "davidson stage 1: %d iters, sigma %.2f, H %.2f, eig %.2f, ritz %.2f, "
                     "ortho %.2f ms\n",
                     c.dav.iters, c.dav.sec_ms[0], c.dav.sec_ms[1], c.dav.sec_ms[2],
                     c.dav.sec_ms[3], c.dav.sec_ms[4]);
      for (double &v : c.dav.sec_ms) v = 0;
      SectionClock sc(c.dav, s);
      // (the velocity correction uses the tensor-core exchange products, so the
      // FP64 operators need no P^A_ov)
      mf_setup_ops<double>(c.mf, c.mf.d, s, Clow, c.d_slot_ao.get(), Poo, Pia, Qs, Ps, false);
      c.mf.f32 = false;
      sc.tick(0);
      if (c.dav.profile) std::fprintf(stderr, "FP64 operator setup %.2f ms\n", c.dav.sec_ms[0]);
      for (double &v : c.dav.sec_ms) v = 0;
      conv = davidson(c.dav, c.blas, c.solver, s, mv, d_edall, nci, p.nroots, tol, 100, om, Xd,
                      true, false);
      c.dav_iters += c.dav.iters;
      c.dav_fp64_matvecs = c.dav.matvecs;   // B X of the velocity correction also in FP64
      if (c.dav.profile)
        std::fprintf(stderr,
                     "davidson stage 2: %d iters, sigma %.2f, H %.2f, eig %.2f, ritz %.2f, "
                     "ortho %.2f ms\n",
                     c.dav.iters, c.dav.sec_ms[0], c.dav.sec_ms[1], c.dav.sec_ms[2],
                     c.dav.sec_ms[3], c.dav.sec_ms[4]);
    } else {
      conv = davidson(c.dav, c.blas, c.solver, s, mv, d_edall, nci, p.nroots, tol, 300, om, Xd);
      c.dav_iters = c.dav.iters;
      c.dav_matvecs = 0;
      c.dav_fp64_matvecs = c.dav.matvecs;
    }
    if (conv < std::min(p.nroots, nci))
      throw Error{STD2G_ENOCONV, "Davidson: " + std::to_string(conv) + " of " +
                                     std::to_string(p.nroots) + " roots converged"};
    nroot = std::min(p.nroots, nci);
    X = Xd;
    c.mixed.lastX = X;
    root_resid = c.dav.final_resid;
    root_ritz = c.dav.final_theta;
  } else if (!p.rpa) {
    double *A = c.w_A.ensure(n2);
    S2G_LAUNCH(k_combine_tda, grid_for(n2), 256, 0, s, A, K, J, (int64_t)nci, ak, d_edall);
    if (p.velcorr) {
      Bh = c.w_Bh.ensure(n2);
      S2G_LAUNCH(k_combine_rpa, grid_for(n2), 256, 0, s, (double *)nullptr, (double *)nullptr, Bh,
                 K, Kx, J, (int64_t)nci, ak, p.ax, d_edall, ekd);
    }
    record(c, PH_EIGEN);
    om = c.w_eval.ensure(std::max(nci, nao));
    if (batch_eig) {
      // the lowest p.nroots roots, as the matrix-free Davidson of an unbatched
      // solve gives them, from the shared batch
      BatchProblem bp;
      bp.dw = &c.dav;
      bp.blas = c.blas;
      bp.sol = c.solver;
      bp.A = A;
      bp.diag = d_edall;
      bp.n = nci;
      bp.kwant = std::min(p.nroots, nci);
      bp.tol = p.conv_tol > 0 ? p.conv_tol : 1e-6;
      bp.max_iter = 300;
      bd_prepare(bp);
      nroot = bp.kwant;
      bp.omega_out = om;
      bp.X_out = c.w_X.ensure((size_t)nci * nroot);
      std::vector<int> order(nci);
      std::iota(order.begin(), order.end(), 0);
      std::stable_sort(order.begin(), order.end(),
                       [&](int x, int y) { return ed_all[x] < ed_all[y]; });
      bp.init_idx.assign(order.begin(), order.begin() + bp.k);
      if (!c.ev_bready) {
        S2G_CUDA(cudaEventCreateWithFlags(&c.ev_bready, cudaEventDisableTiming));
        S2G_CUDA(cudaEventCreateWithFlags(&c.ev_bdone, cudaEventDisableTiming));
      }
      bp.ready = c.ev_bready;
      bp.done = c.ev_bdone;
      S2G_CUDA(cudaEventRecord(c.ev_bready, s));
      c.batch->solve(bp);
      S2G_CUDA(cudaStreamWaitEvent(s, c.ev_bdone, 0));
      if (bp.status != STD2G_OK) throw Error{bp.status, bp.msg};
      c.dav_iters = bp.iters;
      c.dav_matvecs = 0;
      c.dav_fp64_matvecs = bp.matvecs;
      if (bp.nconv < nroot)
        throw Error{STD2G_ENOCONV, "Davidson (batched): " + std::to_string(bp.nconv) + " of " +
                                       std::to_string(nroot) + " roots converged"};
      X = bp.X_out;
      c.mixed.lastX = X;
      root_resid = bp.final_resid;
      root_ritz = bp.final_theta;
    } else {
      nroot = dense_eig(c, A, nci, 0.0, thr, p.nroots, om);
      X = A;
      c.mixed.lastX = X;
      if (nroot < 1) throw Error{STD2G_ENOROOT, "no root below the energy threshold"};
      // FP64 residuals ||A x - w x|| of the returned eigenvectors: A rebuilt
      // from K, J and the diagonal (its storage now holds the eigenvectors)
      {
        double *Ar = c.w_Ares.ensure(n2), *Rr = c.w_Rres.ensure((size_t)nci * nroot);
        S2G_LAUNCH(k_combine_tda, grid_for(n2), 256, 0, s, Ar, K, J, (int64_t)nci, ak, d_edall);
        gemm(c, CUBLAS_OP_N, CUBLAS_OP_N, nci, nroot, nci, 1.0, Ar, nci, X, nci, 0.0, Rr, nci);
        double *part = c.w_part.ensure((size_t)nroot * kColSplit), *rn = c.w_rn.ensure(nroot);
        S2G_LAUNCH(k_dav_resid, dim3(kColSplit, (unsigned)nroot), 256, 0, s, Rr, X, om, nci, part);
        S2G_LAUNCH(k_colnorm_finish, (int)div_up(nroot, 128), 128, 0, s, part, kColSplit, nroot,
                   rn);
        root_resid.assign(nroot, 0.0);
        root_ritz.assign(nroot, 0.0);
        S2G_CUDA(cudaMemcpyAsync(root_resid.data(), rn, sizeof(double) * nroot,
                                 cudaMemcpyDeviceToHost, s));
        S2G_CUDA(cudaMemcpyAsync(root_ritz.data(), om, sizeof(double) * nroot,
                                 cudaMemcpyDeviceToHost, s));
      }
    }
  } else {
    double *Apb = nullptr, *Amb = nullptr;
    if (!resp_mf) {
      Apb = c.w_Apb.ensure(n2);
      Amb = c.w_Amb.ensure(n2);
      // J holds (ij|ab); A+B and A-B from K, Kx, J
      S2G_LAUNCH(k_combine_rpa, grid_for(n2), 256, 0, s, Apb, Amb, (double *)nullptr, K, Kx, J,
                 (int64_t)nci, ak, p.ax, d_edall, ekd);
    }
    if (resp) {
      record(c, PH_EIGEN);
      record(c, PH_PROPS);
      record(c, PH_RESPONSE);
      double *musel = c.w_musel.ensure((size_t)nci * 9);
      S2G_LAUNCH(k_gather_mu, grid_for((int64_t)nci * 9), 256, 0, s, musel, c.w_mu_ov.get(), no,
                 nv, d_ci, d_ca, nci);
      RespReq rq = *resp;
      if (want_quad && rq.quad->nbeta > 0) {
        rq.U = c.w_Uall.ensure((size_t)nci * 3 * rq.n);
        rq.V = c.w_Vall.ensure((size_t)nci * 3 * rq.n);
      }
      if (resp_mf) {
        std::vector<int> fb;
        response_matfree(c, nci, musel, rq, fb, d_edall, ekd, uci, ak, p.ax, tc_resp);
        if (!fb.empty())
          throw Error{STD2G_ENOCONV,
                      "alpha(w): a frequency above the first excitation needs the dense form, "
                      "which does not fit for this CSF space"};
      } else if (mixed) {
        std::vector<int> fb;
        response_mixed(c, Apb, Amb, nci, musel, rq, fb);
        if (!fb.empty()) {
          // frequencies above the first excitation: the FP64 form's factorisations
          std::vector<double> om(fb.size()), al(fb.size() * 9), rs(fb.size());
          for (size_t q = 0; q < fb.size(); ++q) om[q] = resp->omega[fb[q]];
          RespReq sub{om.data(), (int)fb.size(), al.data(), rs.data()};
          std::vector<int> slots(fb.begin(), fb.end());
          if (rq.U) {
            sub.U = rq.U;
            sub.V = rq.V;
            sub.slot = slots.data();
          }
          response(c, Apb, Amb, nci, musel, sub);
          for (size_t q = 0; q < fb.size(); ++q) {
            std::copy(al.begin() + 9 * q, al.begin() + 9 * q + 9, resp->alpha + 9 * fb[q]);
            if (resp->resid) resp->resid[fb[q]] = rs[q];
          }
        }
      } else {
        response(c, Apb, Amb, nci, musel, rq);
      }
      if (want_quad && rq.quad->nbeta > 0)
        hyperpolarizability(c, nci, no, nv, d_ci, d_ca, rq.U, rq.V, *rq.quad);
      record(c, PH_COUNT);
      S2G_CUDA(cudaStreamSynchronize(s));
      for (int q = 0; q < PH_COUNT; ++q) {
        float ms = 0;
        cudaEventElapsedTime(&ms, c.ev[q], c.ev[q + 1]);
        c.ph_ms[q] = ms;
      }
      float tot = 0;
      cudaEventElapsedTime(&tot, c.ev[PH_SETUP], c.ev[PH_COUNT]);
      (void)cudaGetLastError();
      c.last_nci = nci;
      c.last_nroot = 0;
      c.last_no = no;
      c.last_nv = nv;
      c.last_rpa = true;
      if (res) {
        res->nroot = 0;
        res->no = no;
        res->nv = nv;
        res->nex = nex;
        res->nexpt = nexpt;
        res->new_pt = nnew;
        res->nci = nci;
        res->ms_total = tot;
        res->csf_hash = fnv1a(ci, ca);
      }
      return;
    }
    record(c, PH_EIGEN);
    // (A-B)^1/2 (smatpow srpapack.f:201-256)
    double *U = c.w_Ambh.ensure(n2);
    S2G_CUDA(cudaMemcpyAsync(U, Amb, sizeof(double) * n2, cudaMemcpyDeviceToDevice, s));
    double *w = c.w_eval.ensure(std::max(nci, nao));
    dense_eig_full(c, U, nci, w);
    double wmin = 0;
    S2G_CUDA(cudaMemcpyAsync(&wmin, w, sizeof(double), cudaMemcpyDeviceToHost, s));
    S2G_CUDA(cudaStreamSynchronize(s));
    if (wmin < 0) throw Error{STD2G_EAMB_NOT_PD, "matrix power impossible (A-B)"};
    double *Ambh = c.w_M.ensure(n2);
    double *tmp2 = c.w_Kx.ensure(n2);   // Kx no longer needed
    sym_sqrt(c, U, w, nci, Ambh, tmp2);
    // M = (A-B)^1/2 (A+B) (A-B)^1/2 (srpapack.f:58-71)
    gemm(c, CUBLAS_OP_N, CUBLAS_OP_N, nci, nci, nci, 1.0, Apb, nci, Ambh, nci, 0.0, tmp2, nci);
    double *Mm = U;
    gemm(c, CUBLAS_OP_N, CUBLAS_OP_N, nci, nci, nci, 1.0, Ambh, nci, tmp2, nci, 0.0, Mm, nci);
    om = c.w_eval.ensure(std::max(nci, nao));
    nroot = dense_eig(c, Mm, nci, 0.0, thr * thr, p.nroots, om);
    if (nroot < 1) throw Error{STD2G_ENOROOT, "RPA diag failed"};
    S2G_LAUNCH(k_sqrt_inplace, (int)div_up(nroot, 128), 128, 0, s, om, nroot);
    // X+Y = (A-B)^1/2 Z / sqrt(w); X-Y = (A+B)(X+Y)/w (srpapack.f:108-143)
    X = c.w_X.ensure((size_t)nci * nroot);
    Yv = c.w_Y.ensure((size_t)nci * nroot);
    gemm(c, CUBLAS_OP_N, CUBLAS_OP_N, nci, nroot, nci, 1.0, Ambh, nci, Mm, nci, 0.0, X, nci);
    S2G_LAUNCH(k_scale_columns, grid_for((int64_t)nci * nroot), 256, 0, s, X, (int64_t)nci, nroot,
               om, 0);
    gemm(c, CUBLAS_OP_N, CUBLAS_OP_N, nci, nroot, nci, 1.0, Apb, nci, X, nci, 0.0, Yv, nci);
    S2G_LAUNCH(k_scale_columns, grid_for((int64_t)nci * nroot), 256, 0, s, Yv, (int64_t)nci,
               nroot, om, 1);
    if (tpa && tpa->ntpa > 0) {
      // The state vectors lresp_2PA_SP contracts: under its keyword srpapack
      // skips the halving of the packed diagonals of (A-B)^1/2 and A+B before
      // its packed products (srpapack.f:99-106, 116-133), so each diagonal
      // enters twice: X+Y = (S + diag S) Z / sqrt(w), X-Y = (P + diag P)(X+Y) / w
      // with S = (A-B)^1/2, P = A+B.  Only the two-photon sums use them.
      if (tpa->ntpa > nroot)
        throw Error{STD2G_EINVAL, "number of 2PA excitations too large (more than the roots "
                                  "below the energy threshold)"};
      const int nt = tpa->ntpa;
      double *U2 = c.w_Uall.ensure((size_t)nci * nt), *V2 = c.w_Vall.ensure((size_t)nci * nt);
      S2G_CUDA(cudaMemcpyAsync(U2, X, sizeof(double) * nci * nt, cudaMemcpyDeviceToDevice, s));
      S2G_LAUNCH(k_add_diag_cols, grid_for((int64_t)nci * nt), 256, 0, s, U2, Ambh, Mm,
                 (int64_t)nci, nt, om, 0);
      gemm(c, CUBLAS_OP_N, CUBLAS_OP_N, nci, nt, nci, 1.0, Apb, nci, U2, nci, 0.0, V2, nci);
      S2G_LAUNCH(k_add_diag_cols, grid_for((int64_t)nci * nt), 256, 0, s, V2, Apb, U2,
                 (int64_t)nci, nt, om, 1);
      S2G_LAUNCH(k_scale_columns, grid_for((int64_t)nci * nt), 256, 0, s, V2, (int64_t)nci, nt,
                 om, 1);
      S2G_LAUNCH(k_xy_from_uv, grid_for((int64_t)nci * nt), 256, 0, s,
                 c.w_tpx.ensure((size_t)nci * nt), c.w_tpy.ensure((size_t)nci * nt), U2, V2,
                 (int64_t)nci * nt, 0.5);
    }
  }

  // ---- properties (stda.f:1207-1289, apbtrafo.f:23-243) ----
  record(c, PH_PROPS);
  double *musel = c.w_musel.ensure((size_t)nci * 9);
  S2G_LAUNCH(k_gather_mu, grid_for((int64_t)nci * 9), 256, 0, s, musel, c.w_mu_ov.get(), no, nv,
             d_ci, d_ca, nci);
  double *TL = c.w_TL.ensure((size_t)nroot * 9), *TVM = c.w_TVM.ensure((size_t)nroot * 9);
  double *props = c.w_props.ensure((size_t)nroot * 4 + 8);
  double *T2 = nullptr;
  if (!p.rpa) {
    gemm(c, CUBLAS_OP_T, CUBLAS_OP_N, nroot, 9, nci, 1.0, X, nci, musel, nci, 0.0, TL, nroot);
    S2G_CUDA(cudaMemcpyAsync(TVM, TL, sizeof(double) * nroot * 9, cudaMemcpyDeviceToDevice, s));
    if (p.velcorr) {
      // X_new = (B/2) X / w (apbtrafo.f:51-65)
      double *Xn = c.w_Y.ensure((size_t)nci * nroot);
      if (use_mf && tc_dav)   // mixed form: tensor-core exchange products
        mftc_apply(c.mftc, c.blas, s, X, nroot, Xn, 0.5 * ak, 0.0, -0.5 * p.ax, nullptr);
      else if (use_mf)
        mf_apply(c.mf, c.blas, s, X, nroot, Xn, 0.5 * ak, 0.0, -0.5 * p.ax, nullptr);
      else
        gemm(c, CUBLAS_OP_N, CUBLAS_OP_N, nci, nroot, nci, 1.0, Bh, nci, X, nci, 0.0, Xn, nci);
      S2G_LAUNCH(k_scale_columns, grid_for((int64_t)nci * nroot), 256, 0, s, Xn, (int64_t)nci,
                 nroot, om, 2);
      T2 = c.w_T2.ensure((size_t)nroot * 9);
      gemm(c, CUBLAS_OP_T, CUBLAS_OP_N, nroot, 9, nci, 1.0, Xn, nci, musel, nci, 0.0, T2, nroot);
    }
  } else {
    // uu = X+Y for the length form, pp = X-Y for velocity / magnetic
    gemm(c, CUBLAS_OP_T, CUBLAS_OP_N, nroot, 9, nci, 1.0, X, nci, musel, nci, 0.0, TL, nroot);
    gemm(c, CUBLAS_OP_T, CUBLAS_OP_N, nroot, 9, nci, 1.0, Yv, nci, musel, nci, 0.0, TVM, nroot);
    int64_t tot = (int64_t)nci * nroot;
    S2G_LAUNCH(k_xy_from_sums, grid_for(tot), 256, 0, s, X, Yv, tot);
  }
  S2G_LAUNCH(k_properties, (int)div_up(nroot, 128), 128, 0, s, TL, TVM, T2, nroot, nroot, om, ak,
             (!p.rpa && p.velcorr) ? 1 : 0, props, props + nroot, props + 2 * nroot,
             props + 3 * nroot);
  S2G_LAUNCH(k_alpha0, 1, 128, 0, s, TL, nroot, nroot, om, ak, props + 4 * nroot);
  // the three dominant CSFs of each root (stda.f:1222-1358)
  double *dom_c = c.w_domc.ensure((size_t)3 * nroot);
  int *dom_ia = c.w_domi.ensure((size_t)6 * nroot);
  S2G_LAUNCH(k_dominant_csfs, nroot, 256, 0, s, X, p.rpa ? Yv : (const double *)nullptr, nci,
             d_ci, d_ca, no, dom_c, dom_ia, dom_ia + 3 * nroot, c.uks ? 0 : 1);
  record(c, PH_RESPONSE);
  record(c, PH_COUNT);

  // ---- results ----
  std::vector<double> h_props((size_t)nroot * 4 + 6), h_om(nroot), h_domc((size_t)3 * nroot);
  std::vector<int> h_domi((size_t)6 * nroot);
  S2G_CUDA(cudaMemcpyAsync(h_props.data(), props, sizeof(double) * (nroot * 4 + 6),
                           cudaMemcpyDeviceToHost, s));
  S2G_CUDA(cudaMemcpyAsync(h_domc.data(), dom_c, sizeof(double) * 3 * nroot,
                           cudaMemcpyDeviceToHost, s));
  S2G_CUDA(cudaMemcpyAsync(h_domi.data(), dom_ia, sizeof(int) * 6 * nroot, cudaMemcpyDeviceToHost,
                           s));
  S2G_CUDA(cudaMemcpyAsync(h_om.data(), om, sizeof(double) * nroot, cudaMemcpyDeviceToHost, s));
  S2G_CUDA(cudaStreamSynchronize(s));
  for (int q = 0; q < PH_COUNT; ++q) {
    float ms = 0;
    cudaEventElapsedTime(&ms, c.ev[q], c.ev[q + 1]);
    c.ph_ms[q] = ms;
  }
  float tot = 0;
  cudaEventElapsedTime(&tot, c.ev[PH_SETUP], c.ev[PH_COUNT]);
  (void)cudaGetLastError();
  c.last_nci = nci;
  c.last_nroot = nroot;
  c.last_no = no;
  c.last_nv = nv;
  c.last_rpa = p.rpa;
  if (res) {
    res->nroot = nroot;
    res->no = no;
    res->nv = nv;
    res->nex = nex;
    res->nexpt = nexpt;
    res->new_pt = nnew;
    res->nci = nci;
    res->ms_total = tot;
    res->csf_hash = fnv1a(ci, ca);
    int m = std::min(nroot, res->cap);
    for (int r = 0; r < m; ++r) {
      if (res->omega) res->omega[r] = h_om[r];
      if (res->fL) res->fL[r] = h_props[r];
      if (res->fV) res->fV[r] = h_props[nroot + r];
      if (res->RL) res->RL[r] = h_props[2 * nroot + r];
      if (res->RV) res->RV[r] = h_props[3 * nroot + r];
      const bool have = r < (int)root_resid.size();
      const double rr = have ? root_resid[r] : -1.0;
      if (res->resid) res->resid[r] = rr;
      if (res->err_est) {
        // |w - w(A)| <= min(||r||, ||r||^2 / gap) (Kato-Temple), the gap
        // from the other eigenvalue estimates less their own residuals
        double gap = 1e300;
        for (size_t q = 0; q < root_ritz.size(); ++q)
          if ((int)q != r)
            gap = std::min(gap, std::fabs(root_ritz[q] - h_om[r]) -
                                    (q < root_resid.size() ? root_resid[q] : 0.0));
        // plus (Weyl) the bound on the PT-lowered diagonal's deviation from
        // its FP64 value, nonzero where the tensor-core selection formed it
        res->err_est[r] = !have ? -1.0
                                : (gap > 0 ? std::min(rr, rr * rr / gap) : rr) +
                                      c.mixed.ed_bound_max;
      }
      for (int q = 0; q < 3; ++q) {
        if (res->dom_coef) res->dom_coef[3 * r + q] = h_domc[3 * r + q];
        if (res->dom_i) res->dom_i[3 * r + q] = h_domi[3 * r + q];
        if (res->dom_a) res->dom_a[3 * r + q] = h_domi[3 * nroot + 3 * r + q];
      }
    }
    for (int q = 0; q < 6; ++q) res->alpha0[q] = h_props[4 * nroot + q];
    if (nroot > res->cap) throw Error{STD2G_ECAP, "result capacity too small"};
  }
  if (tpa && tpa->ntpa > 0) {
    if (!p.rpa) throw Error{STD2G_EINVAL, "two-photon absorption needs the sTD-DFT states"};
    two_photon(c, nci, no, nv, d_ci, d_ca, musel, h_om, *tpa);
  }
}

}  // namespace std2g

// ============================ C boundary =================================
using std2g::Ctx;
using std2g::Error;
using std2g::BatchDavidson;

static thread_local std::string g_last_error;

static int guard(const std::function<void()> &f) {
  try {
    f();
    return STD2G_OK;
  } catch (const Error &e) {
    g_last_error = e.msg;
    return e.code;
  } catch (const std::bad_alloc &) {
    g_last_error = "host allocation failed";
    return STD2G_ENOMEM;
  } catch (...) {
    g_last_error = "unknown error";
    return STD2G_ECUDA;
  }
}

extern "C" {

int std2g_create(void **ctx, const std2g_opts *opts) {
  if (!ctx) return STD2G_EINVAL;
  return guard([&] {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
      throw Error{STD2G_ENODEV, "no CUDA device"};
    std2g_opts o{};
    if (opts) o = *opts;
    if (o.device < 0 || o.device >= ndev) throw Error{STD2G_EINVAL, "bad device ordinal"};
    cudaDeviceProp prop;
    S2G_CUDA(cudaGetDeviceProperties(&prop, o.device));
    if (prop.major != 10) throw Error{STD2G_ENODEV, "an sm_100 (B200) device is required"};
    S2G_CUDA(cudaSetDevice(o.device));
    auto *c = new Ctx();
    c->opts = o;
    c->dev_sms = prop.multiProcessorCount;
    c->dg.nsm = prop.multiProcessorCount;
    c->dav.dg = &c->dg;
    c->mf.dg = &c->dg;
    c->mftc.side.dg.nsm = prop.multiProcessorCount;
    S2G_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    S2G_CUBLAS(cublasCreate(&c->blas));
    S2G_CUBLAS(cublasSetStream(c->blas, c->stream));
    // FP32 GEMMs of this handle (the mixed form's dense response products) run
    // on the tensor cores as split-BF16 products (FP32 emulation) where the
    // cuBLAS in the process has that mode (12.9 and later; a host that loaded
    // an older cuBLAS first keeps plain FP32 GEMMs, which the FP64 refinement
    // of those solves accepts as well)
    using SetEmulation = cublasStatus_t (*)(cublasHandle_t, cublasEmulationStrategy_t);
    auto set_emulation = (SetEmulation)dlsym(RTLD_DEFAULT, "cublasSetEmulationStrategy");
    if (set_emulation &&
        cublasSetMathMode(c->blas, CUBLAS_FP32_EMULATED_BF16X9_MATH) == CUBLAS_STATUS_SUCCESS)
      set_emulation(c->blas, CUBLAS_EMULATION_STRATEGY_EAGER);
    S2G_CUSOLVER(cusolverDnCreate(&c->solver));
    S2G_CUSOLVER(cusolverDnSetStream(c->solver, c->stream));
    if (o.flags & STD2G_FLAG_LIBRARY_FP64) {
      c->dg.lib = c->blas;
      c->mftc.side.lib_fp64 = true;
    }
    for (auto &e : c->ev) S2G_CUDA(cudaEventCreate(&e));
    *ctx = c;
  });
}

int std2g_load(void *ctx, int ncent, int nmo, int nao, const double *xyz, const double *C,
               const double *eps, const double *occ, const int *iaoat, const double *S,
               const double *mu_L, const double *mu_V, const double *mu_M) {
  if (!ctx) return STD2G_EINVAL;
  auto *c = (Ctx *)ctx;
  return guard([&] {
    S2G_CUDA(cudaSetDevice(c->opts.device));
    std2g::load(*c, ncent, nmo, nao, xyz, C, eps, occ, iaoat, S, mu_L, mu_V, mu_M);
  });
}

int std2g_ao_integrals(void *ctx, int ncent, const double *xyz, int nao, int nprims,
                       const int *ipty, const int *ipao, const int *ipat, const double *exip,
                       const double *cxip, double *S, double *mu_L, double *mu_V, double *mu_M) {
  if (!ctx) return STD2G_EINVAL;
  auto *c = (Ctx *)ctx;
  return guard([&] {
    S2G_CUDA(cudaSetDevice(c->opts.device));
    cudaStream_t s = c->stream;
    const size_t npk = (size_t)nao * (nao + 1) / 2;
    double *pk = c->w_work.ensure(npk * 10);
    std2g::ao_ints(c->aoi, s, ncent, xyz, nao, nprims, ipty, ipao, ipat, exip, cxip, pk);
    double *dst[4] = {S, mu_L, mu_V, mu_M};
    const size_t off[4] = {0, npk, 4 * npk, 7 * npk}, cnt[4] = {npk, 3 * npk, 3 * npk, 3 * npk};
    for (int q = 0; q < 4; ++q)
      if (dst[q])
        S2G_CUDA(cudaMemcpyAsync(dst[q], pk + off[q], sizeof(double) * cnt[q],
                                 cudaMemcpyDeviceToHost, s));
    S2G_CUDA(cudaStreamSynchronize(s));
  });
}

int std2g_load_prims(void *ctx, int ncent, int nmo, int nao, const double *xyz, const double *C,
                     const double *eps, const double *occ, int nprims, const int *ipty,
                     const int *ipao, const int *ipat, const double *exip, const double *cxip) {
  if (!ctx) return STD2G_EINVAL;
  auto *c = (Ctx *)ctx;
  return guard([&] {
    S2G_CUDA(cudaSetDevice(c->opts.device));
    const size_t npk = (size_t)nao * (nao + 1) / 2;
    double *pk = c->w_work.ensure(npk * 10);
    const std::vector<int> iaoat = std2g::ao_ints(c->aoi, c->stream, ncent, xyz, nao, nprims,
                                                  ipty, ipao, ipat, exip, cxip, pk);
    std2g::load(*c, ncent, nmo, nao, xyz, C, eps, occ, iaoat.data(), nullptr, nullptr, nullptr,
                nullptr, pk);
  });
}

int std2g_set_spins(void *ctx, const int *csp) {
  if (!ctx || !csp) return STD2G_EINVAL;
  auto *c = (Ctx *)ctx;
  if (!c->loaded) return STD2G_ESTATE;
  for (int i = 0; i < c->nmo; ++i)
    if (csp[i] != 1 && csp[i] != 2) return STD2G_EINVAL;
  c->h_csp.assign(csp, csp + c->nmo);
  c->uks = true;
  return STD2G_OK;
}

int std2g_solve(void *ctx, const std2g_params *par, std2g_result *res) {
  if (!ctx || !par) return STD2G_EINVAL;
  auto *c = (Ctx *)ctx;
  return guard([&] {
    S2G_CUDA(cudaSetDevice(c->opts.device));
    if (par->e_thr_ev <= 0) throw Error{STD2G_EINVAL, "e_thr_ev must be positive"};
    std2g::solve(*c, *par, res, nullptr);
  });
}

int std2g_polarizability(void *ctx, const std2g_params *par, const double *omega, int nomega,
                         double *alpha, double *resid) {
  if (!ctx || !par || !omega || nomega <= 0 || !alpha) return STD2G_EINVAL;
  auto *c = (Ctx *)ctx;
  return guard([&] {
    S2G_CUDA(cudaSetDevice(c->opts.device));
    std2g::RespReq rq{omega, nomega, alpha, resid};
    std2g::solve(*c, *par, nullptr, &rq);
  });
}

int std2g_hyperpolarizability(void *ctx, const std2g_params *par, const double *omega,
                              int nomega, double *beta, double *beta_hrs) {
  if (!ctx || !par || !omega || nomega <= 0 || !beta) return STD2G_EINVAL;
  auto *c = (Ctx *)ctx;
  return guard([&] {
    S2G_CUDA(cudaSetDevice(c->opts.device));
    // at most 5 (w, -2w) pairs per refined solve: its CG runs 3 columns per frequency
    for (int k0 = 0; k0 < nomega; k0 += 5) {
      const int nk = std::min(5, nomega - k0);
      std::vector<double> om(2 * nk), al(2 * nk * 9), rs(2 * nk);
      for (int k = 0; k < nk; ++k) {
        om[2 * k] = omega[k0 + k];
        om[2 * k + 1] = -2.0 * omega[k0 + k];
      }
      std2g::QuadReq q;
      q.beta = beta + (size_t)27 * k0;
      q.beta_hrs = beta_hrs ? beta_hrs + k0 : nullptr;
      q.nbeta = nk;
      std2g::RespReq rq{om.data(), 2 * nk, al.data(), rs.data()};
      rq.quad = &q;
      std2g::solve(*c, *par, nullptr, &rq);
    }
  });
}

int std2g_two_photon(void *ctx, const std2g_params *par, int ntrans, double *rows) {
  if (!ctx || !par || ntrans <= 0 || !rows) return STD2G_EINVAL;
  auto *c = (Ctx *)ctx;
  return guard([&] {
    S2G_CUDA(cudaSetDevice(c->opts.device));
    std2g_params p = *par;
    p.rpa = 1;
    p.velcorr = 0;
    p.nroots = 0;      // the states come from the dense sRPA window (srpapack)
    p.solver = 1;
    std2g::QuadReq q;
    q.tpa = rows;
    q.ntpa = ntrans;
    std2g::solve(*c, p, nullptr, nullptr, &q);
  });
}

int std2g_get_csf(void *ctx, int *iconf, double *ed, int cap, int *nci) {
  if (!ctx || !nci) return STD2G_EINVAL;
  auto *c = (Ctx *)ctx;
  return guard([&] {
    int n = c->last_nci;
    *nci = n;
    if (n == 0) throw Error{STD2G_ESTATE, "no solve yet"};
    if (cap < n) throw Error{STD2G_ECAP, "capacity too small"};
    std::vector<int> ci(n), ca(n);
    std::vector<double> h_ed(n);
    S2G_CUDA(cudaMemcpy(ci.data(), c->w_ci.get(), sizeof(int) * n, cudaMemcpyDeviceToHost));
    S2G_CUDA(cudaMemcpy(ca.data(), c->w_ca.get(), sizeof(int) * n, cudaMemcpyDeviceToHost));
    S2G_CUDA(cudaMemcpy(h_ed.data(), c->w_ed.get(), sizeof(double) * n, cudaMemcpyDeviceToHost));
    for (int u = 0; u < n; ++u) {
      if (iconf) {
        iconf[2 * u] = ci[u] + 1;
        iconf[2 * u + 1] = c->last_no + ca[u] + 1;
      }
      if (ed) ed[u] = h_ed[u];
    }
  });
}

int std2g_get_vectors(void *ctx, double *X, double *Y, int cap, int *nroot, int *nci) {
  if (!ctx || !nroot || !nci) return STD2G_EINVAL;
  auto *c = (Ctx *)ctx;
  return guard([&] {
    *nroot = c->last_nroot;
    *nci = c->last_nci;
    if (c->last_nci == 0) throw Error{STD2G_ESTATE, "no solve yet"};
    if (cap < c->last_nroot) throw Error{STD2G_ECAP, "capacity too small"};
    size_t bytes = sizeof(double) * (size_t)c->last_nci * c->last_nroot;
    const double *src = c->last_rpa ? c->w_X.get() : c->mixed.lastX;
    if (X) S2G_CUDA(cudaMemcpy(X, src, bytes, cudaMemcpyDeviceToHost));
    if (Y && c->last_rpa) S2G_CUDA(cudaMemcpy(Y, c->w_Y.get(), bytes, cudaMemcpyDeviceToHost));
  });
}

int std2g_phase_times(void *ctx, double *ms, int cap) {
  if (!ctx) return 0;
  auto *c = (Ctx *)ctx;
  int n = std::min(cap, (int)std2g::PH_COUNT);
  for (int q = 0; q < n; ++q) ms[q] = c->ph_ms[q];
  return std2g::PH_COUNT;
}

const char *std2g_phase_name(int q) {
  return (q >= 0 && q < std2g::PH_COUNT) ? std2g::kPhaseNames[q] : "";
}

int64_t std2g_kernel_launches(void *) { return std2g::g_launches.load(); }

int std2g_set_sm_limit(void *ctx, int max_sms) {
  if (!ctx || max_sms < 0) return STD2G_EINVAL;
  auto *c = (std2g::Ctx *)ctx;
  c->mixed.tc.max_ctas = max_sms;
  c->mftc.tc.max_ctas = max_sms;
  // (the FP64 products keep sizing their split-K for all SMs: they are short
  // and latency-bound, and a share of the SMs made the server's batches
  // slower, 61 against 83 solves/s)
  return STD2G_OK;
}

int std2g_batch_create(int device, void **batch) {
  if (!batch) return STD2G_EINVAL;
  *batch = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev)
    return STD2G_ENODEV;
  return guard([&] { *batch = new BatchDavidson(device); });
}

int std2g_attach_batch(void *ctx, void *batch) {
  if (!ctx) return STD2G_EINVAL;
  auto *c = (Ctx *)ctx;
  auto *b = (BatchDavidson *)batch;
  if (b && b->device() != c->opts.device) return STD2G_EINVAL;
  c->batch = b;
  return STD2G_OK;
}

int std2g_batch_stats(void *batch, int64_t *problems, int64_t *iterations, int64_t *members,
                      double *ms) {
  if (!batch || !problems || !iterations || !members) return STD2G_EINVAL;
  ((BatchDavidson *)batch)->stats(problems, iterations, members, ms);
  return STD2G_OK;
}

void std2g_batch_destroy(void *batch) { delete (BatchDavidson *)batch; }

int std2g_last_batched(void *ctx) { return ctx ? (int)((Ctx *)ctx)->last_batched : 0; }

int std2g_kernel_stats(void *ctx, double *ms, int64_t *launches, double *flop) {
  if (!ctx) return STD2G_EINVAL;
  auto *c = (Ctx *)ctx;
  if (ms) *ms = c->tc_ms;
  if (launches) *launches = c->tc_launches;
  if (flop) *flop = c->tc_flop;
  return STD2G_OK;
}

int std2g_set_gemm_timing(void *ctx, int on) {
  if (!ctx) return STD2G_EINVAL;
  auto *c = (Ctx *)ctx;
  c->dg.timed = on != 0;
  c->mftc.side.dg.timed = on != 0;
  return STD2G_OK;
}

int std2g_gemm_stats(void *ctx, double *ms, int64_t *calls, double *flop) {
  if (!ctx) return STD2G_EINVAL;
  auto *c = (Ctx *)ctx;
  return guard([&] {
    S2G_CUDA(cudaSetDevice(c->opts.device));
    S2G_CUDA(cudaDeviceSynchronize());
    if (ms) *ms = c->dg.elapsed_ms() + c->mftc.side.dg.elapsed_ms();
    if (calls) *calls = c->dg.calls + c->mftc.side.dg.calls;
    if (flop) *flop = c->dg.flop + c->mftc.side.dg.flop;
  });
}

int std2g_solver_stats(void *ctx, int *iters, int64_t *matvecs, int64_t *matvecs_fp64,
                       int64_t *pt_rechecked) {
  if (!ctx) return STD2G_EINVAL;
  auto *c = (Ctx *)ctx;
  if (iters) *iters = c->dav_iters;
  if (matvecs) *matvecs = c->dav_matvecs;
  if (matvecs_fp64) *matvecs_fp64 = c->dav_fp64_matvecs;
  if (pt_rechecked) *pt_rechecked = c->opts.precision == 1 ? c->mixed.rechecked : 0;
  return STD2G_OK;
}

int std2g_symeig_check(int device, int n, int k, const double *A, double *w, double *Z,
                       double *w_ref) {
  if (n < 1 || k < 1 || k > n || !A || !w || !Z || !w_ref) return STD2G_EINVAL;
  return guard([&] {
    using namespace std2g;
    S2G_CUDA(cudaSetDevice(device));
    cudaStream_t s;
    S2G_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    DBuf<double> dA, dw, dZ, dwork, dref, dA2, dlw;
    DBuf<int> dinfo;
    const size_t n2 = (size_t)n * n;
    S2G_CUDA(cudaMemcpyAsync(dA.ensure(n2), A, sizeof(double) * n2, cudaMemcpyHostToDevice, s));
    S2G_CUDA(cudaMemsetAsync(dinfo.ensure(2), 0, 2 * sizeof(int), s));
    symeig_small(s, dA.get(), n, n, k, dw.ensure(k), dZ.ensure((size_t)n * k), n,
                 dwork.ensure(symeig_work_doubles(n, k)), dinfo.get());
    // cuSOLVER on a copy
    cusolverDnHandle_t h;
    S2G_CUSOLVER(cusolverDnCreate(&h));
    S2G_CUSOLVER(cusolverDnSetStream(h, s));
    S2G_CUDA(cudaMemcpyAsync(dA2.ensure(n2), A, sizeof(double) * n2, cudaMemcpyHostToDevice, s));
    int lw = 0;
    S2G_CUSOLVER(cusolverDnDsyevd_bufferSize(h, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER,
                                             n, dA2.get(), n, dref.ensure(n), &lw));
    S2G_CUSOLVER(cusolverDnDsyevd(h, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, n,
                                  dA2.get(), n, dref.get(), dlw.ensure((size_t)lw + 1), lw,
                                  dinfo.get() + 1));
    int hinfo[2] = {0, 0};
    S2G_CUDA(cudaMemcpyAsync(w, dw.get(), sizeof(double) * k, cudaMemcpyDeviceToHost, s));
    S2G_CUDA(cudaMemcpyAsync(Z, dZ.get(), sizeof(double) * n * k, cudaMemcpyDeviceToHost, s));
    S2G_CUDA(cudaMemcpyAsync(w_ref, dref.get(), sizeof(double) * n, cudaMemcpyDeviceToHost, s));
    S2G_CUDA(cudaMemcpyAsync(hinfo, dinfo.get(), 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
    S2G_CUDA(cudaStreamSynchronize(s));
    cusolverDnDestroy(h);
    cudaStreamDestroy(s);
    if (hinfo[0] != 0) throw Error{STD2G_ECUDA, "symeig_small: non-finite result"};
    if (hinfo[1] != 0) throw Error{STD2G_ECUDA, "syevd info " + std::to_string(hinfo[1])};
  });
}

int std2g_dgemm_check(int device, int ta, int tb, int m, int n, int k, double alpha,
                      const double *A, int64_t lda, const double *B, int64_t ldb, double beta,
                      double *C, int64_t ldc, int batch, double *ms) {
  if (m < 1 || n < 1 || k < 0 || batch < 1 || !A || !B || !C) return STD2G_EINVAL;
  const int64_t ar = ta ? k : m, ac = ta ? m : k, br = tb ? n : k, bc = tb ? k : n;
  if (lda < std::max<int64_t>(1, ar) || ldb < std::max<int64_t>(1, br) || ldc < m)
    return STD2G_EINVAL;
  return guard([&] {
    using namespace std2g;
    S2G_CUDA(cudaSetDevice(device));
    cudaStream_t s;
    S2G_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    const size_t na = (size_t)lda * ac, nb = (size_t)ldb * bc, nc = (size_t)ldc * n;
    DBuf<double> dA, dB, dC;
    S2G_CUDA(cudaMemcpyAsync(dA.ensure(na * batch), A, sizeof(double) * na * batch,
                             cudaMemcpyHostToDevice, s));
    S2G_CUDA(cudaMemcpyAsync(dB.ensure(nb * batch), B, sizeof(double) * nb * batch,
                             cudaMemcpyHostToDevice, s));
    S2G_CUDA(cudaMemcpyAsync(dC.ensure(nc * batch), C, sizeof(double) * nc * batch,
                             cudaMemcpyHostToDevice, s));
    Dgemm g;
    cudaDeviceProp prop;
    S2G_CUDA(cudaGetDeviceProperties(&prop, device));
    g.nsm = prop.multiProcessorCount;
    // an untimed run into a scratch copy of C sizes the split-K workspace
    DBuf<double> dW;
    S2G_CUDA(cudaMemcpyAsync(dW.ensure(nc * batch), dC.get(), sizeof(double) * nc * batch,
                             cudaMemcpyDeviceToDevice, s));
    g.run(s, ta != 0, tb != 0, m, n, k, alpha, dA.get(), lda, (int64_t)na, dB.get(), ldb,
          (int64_t)nb, beta, dW.get(), ldc, (int64_t)nc, batch);
    cudaEvent_t e0, e1;
    S2G_CUDA(cudaEventCreate(&e0));
    S2G_CUDA(cudaEventCreate(&e1));
    S2G_CUDA(cudaEventRecord(e0, s));
    g.run(s, ta != 0, tb != 0, m, n, k, alpha, dA.get(), lda, (int64_t)na, dB.get(), ldb,
          (int64_t)nb, beta, dC.get(), ldc, (int64_t)nc, batch);
    S2G_CUDA(cudaEventRecord(e1, s));
    S2G_CUDA(cudaMemcpyAsync(C, dC.get(), sizeof(double) * nc * batch, cudaMemcpyDeviceToHost, s));
    S2G_CUDA(cudaStreamSynchronize(s));
    float t = 0;
    S2G_CUDA(cudaEventElapsedTime(&t, e0, e1));
    if (ms) *ms = t;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaStreamDestroy(s);
  });
}

const char *std2g_error_string(int status) {
  switch (status) {
    case STD2G_OK: return "ok";
    case STD2G_EINVAL: return "invalid argument";
    case STD2G_ECUDA: return g_last_error.empty() ? "CUDA error" : g_last_error.c_str();
    case STD2G_ENOMEM: return "out of device memory";
    case STD2G_ENOCSF: return "no CSF, increase energy threshold (-e option)";
    case STD2G_ES_NOT_PD: return "S^1/2: overlap matrix not positive definite";
    case STD2G_EMONORM: return "internal MO norm error";
    case STD2G_ENOROOT: return "no root below the energy threshold";
    case STD2G_ENOCONV: return "iterative solver did not converge";
    case STD2G_EAMB_NOT_PD: return "matrix power impossible (A-B not positive definite)";
    case STD2G_ESTATE: return "call order";
    case STD2G_ECAP: return "caller buffer too small";
    case STD2G_ENODEV: return "no sm_100 CUDA device";
    case STD2G_ETIMEOUT: return "device wait timed out";
    default: return "unknown status";
  }
}

void std2g_destroy(void *ctx) {
  if (!ctx) return;
  auto *c = (Ctx *)ctx;
  cudaSetDevice(c->opts.device);
  cudaStreamSynchronize(c->stream);
  for (auto &e : c->ev) cudaEventDestroy(e);
  if (c->ev_bready) cudaEventDestroy(c->ev_bready);
  if (c->ev_bdone) cudaEventDestroy(c->ev_bdone);
  if (c->solver_params) cusolverDnDestroyParams(c->solver_params);
  if (c->solver) cusolverDnDestroy(c->solver);
  if (c->blas) cublasDestroy(c->blas);
  delete c;   // buffers free themselves
}

}  // extern "C"
