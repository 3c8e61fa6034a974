// Diagonal screen of the sTDA path for callers that cannot allocate device memory.
//
// std2g_screen_noalloc computes, for every occupied/virtual pair (i,a) of an
// active window, the diagonal element of A and its screen flag -- the same
// quantities std2g_solve forms internally before the PT selection (charges
// q_ia, gamma^J / gamma^K, (ii|aa), (ia|ia)).  Unlike std2g_solve it calls no
// cudaMalloc, cudaFree or library routine that allocates: its working arrays
// live in one file-scope __device__ array of fixed size (kScratchDoubles,
// 64 MiB) that every GPU loading this library keeps until the process exits.
// It is meant for hosts whose device memory is owned by another allocator (a
// framework that has reserved the GPU's memory for its own pool) or that must
// not call cudaMalloc at this point (it synchronises the device), and who hand
// in device buffers they already own.  The array's device address is looked
// up once per device and kept; a cudaDeviceReset by the host invalidates it,
// so the entry point does not support hosts that reset the device.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "../../include/std2g.h"
#include "eta_table.cuh"

namespace {

constexpr size_t kScratchDoubles = 8u << 20;   // 64 MiB
constexpr int kMaxDevices = 64;

// Shared by every call on a device; it keeps the last call's contents.
static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

// Device address of g_noalloc_scratch per device, looked up once per device
// (std::call_once: several host threads may make the first call at once).
static double *g_scratch_ptr[kMaxDevices] = {nullptr};
static cudaError_t g_setup_status[kMaxDevices];
static std::once_flag g_setup_once[kMaxDevices];

// hardness table in constant memory, initialised with the module
__constant__ double c_eta[std2g::kEtaElements] = {STD2G_ETA_VALUES};

// Restores the caller's current device when the entry point returns.
struct DeviceGuard {
  int prev = -1;
  DeviceGuard() {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

// gamma^J and gamma^K (stda.f:509-532) from xyz(4,ncent)
__global__ void na_gamma(const double *__restrict__ xyz, int n, double ax, double alpha,
                         double beta, double *__restrict__ gj, double *__restrict__ gk) {
  int64_t total = (int64_t)n * n;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    int j = (int)(t / n), i = (int)(t - (int64_t)j * n);
    double dx = xyz[4 * i] - xyz[4 * j], dy = xyz[4 * i + 1] - xyz[4 * j + 1],
           dz = xyz[4 * i + 2] - xyz[4 * j + 2];
    double r = sqrt(dx * dx + dy * dy + dz * dz);
    int zi = (int)llrint(xyz[4 * i + 3]), zj = (int)llrint(xyz[4 * j + 3]);
    zi = zi < 1 ? 1 : (zi > std2g::kEtaElements ? std2g::kEtaElements : zi);   // table range
    zj = zj < 1 ? 1 : (zj > std2g::kEtaElements ? std2g::kEtaElements : zj);
    double eb = 0.5 * (c_eta[zi - 1] + c_eta[zj - 1]);
    double xj = eb * ax;
    gj[t] = xj > 0.0 ? 1.0 / pow(pow(r, beta) + 1.0 / pow(xj, beta), 1.0 / beta) : 0.0;
    gk[t] = 1.0 / pow(pow(r, alpha) + 1.0 / pow(eb, alpha), 1.0 / alpha);
  }
}

// Loewdin charges q^A_pq (lo12pop, stda.f:1727-1744) straight from the 1-based
// AO -> atom map: out[A + N*x] for pair x = (p0 + x/nq, q0 + x%nq) or, with
// diag, x = (p0 + x, q0 + x).
__global__ void na_charges(double *__restrict__ out, const double *__restrict__ C, int nao, int N,
                           const int *__restrict__ iaoat, int p0, int np, int q0, int nq,
                           int diag) {
  int64_t npairs = diag ? (int64_t)np : (int64_t)np * nq;
  int64_t total = npairs * N;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    int64_t pr = t / N;
    int A = (int)(t - pr * N);
    int x = diag ? (int)pr : (int)(pr / nq);
    int y = diag ? (int)pr : (int)(pr - (int64_t)x * nq);
    const double *cp = C + (int64_t)(p0 + x) * nao;
    const double *cq = C + (int64_t)(q0 + y) * nao;
    double s = 0.0;
    for (int k = 0; k < nao; ++k)
      if (iaoat[k] - 1 == A) s += cp[k] * cq[k];
    out[t] = s;
  }
}

// P[:, c] = gamma Q[:, c]  (ssymm, stda.f:558-565, 589-590)
__global__ void na_gamma_apply(double *__restrict__ P, const double *__restrict__ g,
                               const double *__restrict__ Q, int N, int64_t ncol) {
  int64_t total = (int64_t)N * ncol;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    int64_t c = t / N;
    int A = (int)(t - c * N);
    const double *q = Q + c * N;
    double s = 0.0;
    for (int B = 0; B < N; ++B) s += g[A + (int64_t)N * B] * q[B];
    P[t] = s;
  }
}

// de_ia = (e_a - e_i) - (ii|aa) + ak (ia|ia) [+ kshift]; flag 1 primary, 2 PT
// candidate, 0 neither (stda.f:593-640)
__global__ void na_screen(const double *__restrict__ Pia, const double *__restrict__ Qia,
                          const double *__restrict__ Pii, const double *__restrict__ Qaa, int N,
                          int no, int nv, const double *__restrict__ eps, double ak, int kshift,
                          double sau, double wau, double steep, double thr, double fthr,
                          double *__restrict__ de_out, int *__restrict__ flag) {
  int64_t npair = (int64_t)no * nv;
  int lane = threadIdx.x & 31;
  int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  int64_t nwarp = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t k = warp; k < npair; k += nwarp) {
    int i = (int)(k / nv), a = (int)(k - (int64_t)i * nv);
    const double *p = Pia + k * N, *q = Qia + k * N;
    const double *pi = Pii + (int64_t)i * N, *qa = Qaa + (int64_t)a * N;
    double ek = 0.0, jd = 0.0;
    for (int A = lane; A < N; A += 32) {
      ek += p[A] * q[A];
      jd += qa[A] * pi[A];
    }
    for (int o = 16; o > 0; o >>= 1) {
      ek += __shfl_xor_sync(0xffffffffu, ek, o);
      jd += __shfl_xor_sync(0xffffffffu, jd, o);
    }
    if (lane == 0) {
      double de = (eps[no + a] - eps[i]) - jd + ak * ek;
      if (kshift) de += sau / (1.0 + pow(ek / wau, steep));
      de_out[k] = de;
      flag[k] = (de <= thr) ? 1 : ((de > thr && de < fthr) ? 2 : 0);
    }
  }
}

int grid_of(int64_t n) {
  int64_t g = (n + 255) / 256;
  if (g < 1) g = 1;
  if (g > 148 * 32) g = 148 * 32;
  return (int)g;
}

}  // namespace

extern "C" int std2g_screen_noalloc(int device, int ncent, int nao, int no, int nv,
                                    const double *d_xyz, const int *d_iaoat, const double *d_clow,
                                    const double *d_eps, const std2g_params *par, double *d_de,
                                    int *d_flag, void *stream) {
  if (!par || !d_xyz || !d_iaoat || !d_clow || !d_eps || !d_de || !d_flag) return STD2G_EINVAL;
  if (device < 0 || device >= kMaxDevices || ncent <= 0 || nao <= 0 || no <= 0 || nv <= 0 ||
      par->e_thr_ev <= 0)
    return STD2G_EINVAL;
  const int N = ncent;
  const int64_t nov = (int64_t)no * nv;
  // scratch layout (doubles): gj, gk (N^2 each), Qii, Pii (N*no), Qaa (N*nv), Qia, Pia (N*nov)
  const int64_t need = 2 * (int64_t)N * N + 2 * (int64_t)N * no + (int64_t)N * nv + 2 * N * nov;
  if (need > (int64_t)kScratchDoubles) return STD2G_ECAP;   // larger than the fixed scratch
  DeviceGuard guard;   // the caller's current device is restored on every return
  if (cudaSetDevice(device) != cudaSuccess) return STD2G_ENODEV;
  // an error the caller left pending is not ours to report or to clear
  if (cudaPeekAtLastError() != cudaSuccess) return STD2G_ECUDA;
  std::call_once(g_setup_once[device], [device] {
    // one-time set-up on this device, with the device current: the device
    // address of the scratch array (the first call on a device does it; make
    // that call before any stream capture)
    double *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress((void **)&p, g_noalloc_scratch);
    if (e == cudaSuccess && !p) e = cudaErrorInvalidSymbol;
    g_setup_status[device] = e;
    if (e == cudaSuccess) g_scratch_ptr[device] = p;
  });
  if (g_setup_status[device] != cudaSuccess) return STD2G_ECUDA;
  cudaStream_t s = (cudaStream_t)stream;
  double *base = g_scratch_ptr[device];
  double *gj = base, *gk = gj + (int64_t)N * N, *Qii = gk + (int64_t)N * N;
  double *Pii = Qii + (int64_t)N * no, *Qaa = Pii + (int64_t)N * no, *Qia = Qaa + (int64_t)N * nv;
  double *Pia = Qia + N * nov;
  // every scratch element read below is written earlier in this call, so
  // nothing has to be cleared; calls that overlap on the GPU race on it
  const double ax = par->ax;
  const double beta = par->beta_j >= -99.0 ? par->beta_j : 0.20 + 1.830 * ax;
  const double alpha = par->alpha_k >= -99.0 ? par->alpha_k : 1.420 + 0.480 * ax;
  const double ak = par->triplet ? 0.0 : 2.0;
  const double thr = par->e_thr_ev / 27.211385050;
  const double fthr = par->fthr_ev < 1.79e308 ? par->fthr_ev / 27.211385050 : INFINITY;
  // each launch's configuration error is checked where it happens
#define NA_CHECK()                                                               \
  do {                                                                           \
    if (cudaGetLastError() != cudaSuccess) return STD2G_ECUDA;                   \
  } while (0)
  na_gamma<<<grid_of((int64_t)N * N), 256, 0, s>>>(d_xyz, N, ax, alpha, beta, gj, gk);
  NA_CHECK();
  na_charges<<<grid_of((int64_t)N * no), 256, 0, s>>>(Qii, d_clow, nao, N, d_iaoat, 0, no, 0, no, 1);
  NA_CHECK();
  na_charges<<<grid_of((int64_t)N * nv), 256, 0, s>>>(Qaa, d_clow, nao, N, d_iaoat, no, nv, no, nv,
                                                      1);
  NA_CHECK();
  na_charges<<<grid_of(N * nov), 256, 0, s>>>(Qia, d_clow, nao, N, d_iaoat, 0, no, no, nv, 0);
  NA_CHECK();
  na_gamma_apply<<<grid_of((int64_t)N * no), 256, 0, s>>>(Pii, gj, Qii, N, no);
  NA_CHECK();
  na_gamma_apply<<<grid_of(N * nov), 256, 0, s>>>(Pia, gk, Qia, N, nov);
  NA_CHECK();
  na_screen<<<grid_of(nov * 32), 256, 0, s>>>(Pia, Qia, Pii, Qaa, N, no, nv, d_eps, ak, par->kshift,
                                              par->shftmax * 0.036749320,
                                              par->shftwidth * 0.036749320, par->shftsteep, thr,
                                              fthr, d_de, d_flag);
  NA_CHECK();
#undef NA_CHECK
  return STD2G_OK;
}
