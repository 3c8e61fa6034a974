// Diagonal screen of the sTDA path for callers that cannot allocate device memory.
//
// std2g_screen_noalloc computes, for every occupied/virtual pair (i,a) of an
// active window, the diagonal element of A and its screen flag -- the same
// quantities std2g_solve forms internally before the PT selection (charges
// q_ia, gamma^J / gamma^K, (ii|aa), (ia|ia)).  Unlike std2g_solve it calls no
// cudaMalloc, cudaFree or library routine that allocates: its working arrays
// live in one file-scope __device__ array of fixed size (kScratchBytes) that
// every GPU loading this library keeps until the process exits.  It is meant
// for hosts whose device memory is owned by another allocator (a framework
// that has reserved the GPU's memory for its own pool) or that must not call
// cudaMalloc at this point (it synchronises the device), and who hand in
// device buffers they already own.
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/std2g.h"

namespace {

constexpr size_t kScratchDoubles = 8u << 20;   // 64 MiB
constexpr size_t kScratchBytes = kScratchDoubles * sizeof(double);
constexpr int kMaxDevices = 64;

// Shared by every call on a device; it keeps the last call's contents.
static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

// Device address of g_noalloc_scratch per device (set-up on first use).
static double *g_scratch_ptr[kMaxDevices] = {nullptr};

const double kEta[94] = {
    0.472592880, 0.922033910, 0.174528880, 0.257007330, 0.339490860, 0.421954120, 0.504381930,
    0.586918630, 0.669313510, 0.751916070, 0.179641050, 0.221572760, 0.263485780, 0.305396450,
    0.347340140, 0.389247250, 0.431156700, 0.473082690, 0.171054690, 0.202762440, 0.210073220,
    0.217396470, 0.224710390, 0.232015010, 0.239339690, 0.246656380, 0.253982550, 0.261288630,
    0.268594760, 0.275925650, 0.307629990, 0.339315800, 0.372359850, 0.402735490, 0.434457760,
    0.466117080, 0.155850790, 0.186493240, 0.193562100, 0.200633110, 0.207705220, 0.214772540,
    0.221846140, 0.228918720, 0.235986210, 0.243056120, 0.250130180, 0.257199370, 0.287847800,
    0.318486730, 0.349124310, 0.379765930, 0.410408080, 0.441057770, 0.050193320, 0.067625700,
    0.085044450, 0.102477360, 0.119911050, 0.137327720, 0.154762970, 0.172182650, 0.189612880,
    0.207047600, 0.224467520, 0.241896450, 0.259325030, 0.276760940, 0.294182310, 0.311595870,
    0.329022740, 0.345922980, 0.363880480, 0.381305860, 0.398774760, 0.416142980, 0.433645100,
    0.451040140, 0.468489860, 0.485845500, 0.125267300, 0.142686770, 0.160116150, 0.177558890,
    0.194975570, 0.212407780, 0.072635250, 0.094221580, 0.099202950, 0.104186210, 0.142356330,
    0.163942940, 0.185519410, 0.223701390};

__constant__ double c_eta[94];

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
    zi = zi < 1 ? 1 : (zi > 94 ? 94 : zi);   // table range; callers pass Z in 1..94
    zj = zj < 1 ? 1 : (zj > 94 ? 94 : zj);
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
  if (cudaSetDevice(device) != cudaSuccess) return STD2G_ENODEV;
  cudaStream_t s = (cudaStream_t)stream;
  if (!g_scratch_ptr[device]) {
    // one-time set-up on this device: device address of the scratch array and
    // the hardness table (first call on a device; make it before any capture)
    double *p = nullptr;
    if (cudaGetSymbolAddress((void **)&p, g_noalloc_scratch) != cudaSuccess || !p)
      return STD2G_ECUDA;
    if (cudaMemcpyToSymbol(c_eta, kEta, sizeof(kEta)) != cudaSuccess) return STD2G_ECUDA;
    g_scratch_ptr[device] = p;
  }
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
  na_gamma<<<grid_of((int64_t)N * N), 256, 0, s>>>(d_xyz, N, ax, alpha, beta, gj, gk);
  na_charges<<<grid_of((int64_t)N * no), 256, 0, s>>>(Qii, d_clow, nao, N, d_iaoat, 0, no, 0, no, 1);
  na_charges<<<grid_of((int64_t)N * nv), 256, 0, s>>>(Qaa, d_clow, nao, N, d_iaoat, no, nv, no, nv,
                                                      1);
  na_charges<<<grid_of(N * nov), 256, 0, s>>>(Qia, d_clow, nao, N, d_iaoat, 0, no, no, nv, 0);
  na_gamma_apply<<<grid_of((int64_t)N * no), 256, 0, s>>>(Pii, gj, Qii, N, no);
  na_gamma_apply<<<grid_of(N * nov), 256, 0, s>>>(Pia, gk, Qia, N, nov);
  na_screen<<<grid_of(nov * 32), 256, 0, s>>>(Pia, Qia, Pii, Qaa, N, no, nv, d_eps, ak, par->kshift,
                                              par->shftmax * 0.036749320,
                                              par->shftwidth * 0.036749320, par->shftsteep, thr,
                                              fthr, d_de, d_flag);
  return cudaGetLastError() == cudaSuccess ? STD2G_OK : STD2G_ECUDA;
}
