/*
 * std2g -- B200 (sm_100a) engine for the sTDA / sTD-DFT excited-state path of
 * std2.  Plain C ABI: plain pointers and sizes, integer status codes, no
 * C++ or framework types, so that the Fortran host can bind it with
 * iso_c_binding and any other host through its FFI.
 *
 * The boundary replaces one Fortran call of the reference,
 *
 *   call stda(ncent,nmo,nao,xyz,cc,eps,occ,iaoat,thre,thrp,ax,alpha,beta,
 *             ptlim,nvec,nprims)                      (main.f:928-929)
 *   SUBROUTINE stda(...)                              (stda.f:53-54)
 *
 * together with the scratch files the reference passes between its phases
 * (AO integrals sint/x?lint/x?vint/x?mint written at main.f:756-797 and read at
 * stda.f:351-425; amb/apbmat/bmat, stda.f:1926-1995 and apbtrafo.f:603).  The
 * split into create / load / solve keeps inputs resident on the device so that
 * several solves (sTDA, sTD-DFT, alpha(omega)) reuse them.
 *
 * All arrays are caller-owned and follow the Fortran layout of the reference:
 * column-major matrices, packed lower triangles enumerated row by row
 * (k = i*(i-1)/2 + j for i >= j, 1-based as in lin(), stda.f:2174-2181).
 *
 * Error convention: every entry point returns 0 on success and a positive
 * STD2G_E* code otherwise; it never calls exit() or stop.  The reference's
 * equivalents are Fortran `stop` statements (e.g. stda.f:316-318, 644, 1150,
 * 1658-1670; srpapack.f:92,229).
 *
 * Threading: one context is used by one host thread at a time.  Separate
 * contexts may share a device; each owns a CUDA stream.
 */
#ifndef STD2G_H
#define STD2G_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
enum {
  STD2G_OK = 0,
  STD2G_EINVAL = 1,        /* bad argument (null pointer, size <= 0, bad index) */
  STD2G_ECUDA = 2,         /* CUDA runtime / driver error */
  STD2G_ENOMEM = 3,        /* device allocation failed or budget exceeded */
  STD2G_ENOCSF = 4,        /* 'no CSF, increase energy threshold' (stda.f:316-318,644) */
  STD2G_ES_NOT_PD = 5,     /* negative overlap eigenvalue in S^1/2 (stda.f:1658-1670) */
  STD2G_EMONORM = 6,       /* 'internal MO norm error' (stda.f:448-451) */
  STD2G_ENOROOT = 7,       /* no root below E_thr ('internal error in diag', stda.f:1150) */
  STD2G_ENOCONV = 8,       /* Davidson / iterative solve did not converge */
  STD2G_EAMB_NOT_PD = 9,   /* A-B not positive definite ('matrix power impossible', srpapack.f:229) */
  STD2G_ESTATE = 10,       /* call order (solve before load, response before sTD-DFT) */
  STD2G_ECAP = 11,         /* caller buffer too small */
  STD2G_ENODEV = 12,       /* no CUDA device / not an sm_100 device */
  STD2G_ETIMEOUT = 13      /* a bounded device-side wait ran out */
};

/* ---- engine options (per context) -------------------------------------- */
/* Mixed form: tensor-core PT couplings and Davidson products at any problem
   size (by default they are used from ~2.5e8 PT couplings and 16384 CSFs, below
   which the solve is latency-bound and the FP64 GEMMs serve it). */
#define STD2G_FLAG_TENSOR_ALWAYS 1
/* FP64 matrix products through cuBLAS instead of the engine's own DMMA kernel
   (the library baseline that the plain FP64 form is compared with). */
#define STD2G_FLAG_LIBRARY_FP64 2
/* Request server only (std2g_server_opts.flags): the slots' contexts share one
   batched eigensolver (std2g_batch_create / std2g_attach_batch). */
#define STD2G_FLAG_BATCH_EIGEN 4

typedef struct {
  int device;            /* CUDA device ordinal */
  int precision;         /* 0: FP64 form (all contractions FP64)
                            1: mixed form (BF16-split tensor-core contractions,
                               FP32 A storage, FP64 screen / Rayleigh-Ritz) */
  int verbose;           /* 0 silent; 1 per-phase timings to stderr */
  int flags;             /* STD2G_FLAG_* */
  int64_t max_device_bytes; /* 0 = no limit */
} std2g_opts;

/* ---- keywords of the sTDA path (main.f:84-131, stda.f:53-54) ------------ */
typedef struct {
  double ax;         /* -ax  Fock exchange mixing */
  double e_thr_ev;   /* -e   energy threshold / spectral range (eV) */
  double thrp;       /* -p   PT selection threshold (already 10**-x) */
  double alpha_k;    /* -al  (-100: default 1.42+0.48 ax, stda.f:497-500) */
  double beta_j;     /* -be  (-100: default 0.20+1.83 ax, stda.f:494-496) */
  double fthr_ev;    /* -lpt PT limit (eV); >= 1.79e308 means off */
  int triplet;       /* -t   */
  int rpa;           /* -rpa sTD-DFT (A+B, A-B) instead of TDA */
  int velcorr;       /* velocity correction of R_V (default on for sTDA) */
  int kshift;        /* K(ia,ia)-dependent diagonal shift (-xtb / -kshift) */
  double shftmax, shftwidth, shftsteep;   /* kshiftcommon, eV */
  int nroots;        /* 0: every root in (0, E_thr] as ssyevr's window does;
                        k > 0: the lowest k roots (Davidson) */
  int solver;        /* 0 auto, 1 dense diagonalisation, 2 iterative: blocked
                        Davidson for roots (in the mixed form with its tensor-core
                        first stage at any size; auto uses that stage from 16384
                        CSFs), matrix-free refined solve for alpha(w) (auto uses
                        it when the dense A+B, A-B would exceed ~24 GB, and in
                        the mixed form from 4096 CSFs; the mixed form's inner
                        products use the tensor cores from 1.5e6 atoms x CSFs) */
  double conv_tol;   /* Davidson residual norm tolerance (0: 1e-6) */
  double shftmax_somo; /* unrestricted K-shift path: extra shift of SOMO
                          excitations, eV (somo_shift, sutda.f:2402-2422; the
                          -xtb default 1.0, main.f:208) */
} std2g_params;

/* ---- results of one solve ---------------------------------------------- */
typedef struct {
  int cap;           /* capacity of the per-root arrays below (in) */
  int nroot;         /* roots returned (out) */
  int no, nv;        /* active occupied / virtual MOs */
  int nex;           /* primary CSFs (diagonal <= E_thr) */
  int nexpt;         /* CSFs considered in PT */
  int new_pt;        /* CSFs added by PT selection */
  int nci;           /* total CSFs */
  double *omega;     /* [cap] excitation energies (Eh) */
  double *fL, *fV;   /* [cap] oscillator strengths, length / velocity */
  double *RL, *RV;   /* [cap] rotatory strengths (R_V velocity-corrected for sTDA) */
  double *resid;     /* [cap] FP64 residual norm of each returned root's vector
                        (||A x - w x||, or the sTD-DFT pair's residual); -1
                        where none is formed (dense sTD-DFT); may be NULL */
  double alpha0[6];  /* alpha(0) sum over states, xx xy yy xz yz zz (stda.f:1247-1252) */
  uint64_t csf_hash; /* FNV-1a hash of the selected CSF list (i,a) in order */
  double ms_total;   /* device time of the solve (ms) */
  /* the three dominant CSFs of each root, as the reference's state table
     prints them (stda.f:1222-1358, 1456-1462): value (TDA coefficient, or
     X^2 - Y^2 for sTD-DFT) and the CSF's occupied / virtual MO (1-based,
     virtual numbered after the occupied ones as in std2g_get_csf); may be NULL */
  double *dom_coef;  /* [3*cap] */
  int *dom_i, *dom_a;/* [3*cap] */
  /* per-root bound on |omega - omega_FP64-exact| (Eh): from the FP64 residual
     r of the returned vector, min(||r||, ||r||^2 / gap) with the gap to the
     other eigenvalue estimates (Kato-Temple), plus, in the mixed form, the
     bound on the PT-lowered diagonal's deviation from its FP64 value (Weyl);
     -1 where no residual is formed (dense sTD-DFT); may be NULL */
  double *err_est;   /* [cap] */
} std2g_result;

/* Create a context on opts->device.  Replaces the allocation part of stda.f
   (stda.f:195-206); no reference counterpart otherwise. */
int std2g_create(void **ctx, const std2g_opts *opts);

/* Copy one wavefunction and its AO integrals to the device.
   Arguments mirror stda(ncent,nmo,nao,xyz,c,eps,occ,iaoat,...) (stda.f:53-66):
     xyz    [4*ncent]        x,y,z (Bohr) and nuclear charge per atom (xyz(4,ncent))
     C      [nao*nmo]        MO coefficients, column-major (c(nao*nmo))
     eps    [nmo], occ [nmo] orbital energies (Eh) and occupations
     iaoat  [nao]            AO -> atom, 1-based
   plus the AO integrals the reference reads from scratch files
   (stda.f:351-425), packed lower triangles of nao*(nao+1)/2 each:
     S        overlap (sint)
     mu_L     [3*npk] dipole length  -<a|r|b>   (xlint, ylint, zlint)
     mu_V     [3*npk] velocity       -<a|d|b>, element (a>=b) (xvint ...)
     mu_M     [3*npk] angular mom.  <a|r x d|b>, element (a>=b) (xmint ...) */
int std2g_load(void *ctx, int ncent, int nmo, int nao,
               const double *xyz, const double *C, const double *eps,
               const double *occ, const int *iaoat, const double *S,
               const double *mu_L, const double *mu_V, const double *mu_M);

/* Mark the loaded wavefunction as unrestricted (UKS): csp[k] = 1 (alpha) or
   2 (beta) for each of the nmo MOs, occupations 1 / 0 per spin MO, as the
   reference passes csp to sutda (main.f:933, sutda.f:54).  std2g_solve then
   runs UKS sTDA / sTD-DFT: per-spin windows, (ia|jb) between all CSFs and
   (ij|ab) within a spin (ak = 1), ptselect_uks, the SOMO shift with the
   K-shift, no spin factor in the properties.  The CSF list is the alpha block
   then the beta block; std2g_get_csf indexes the window's occupied MOs as
   [alpha, beta] and its virtual MOs likewise.  Response, beta and 2PA stay
   restricted-only (STD2G_EINVAL).  A new std2g_load / std2g_load_prims
   returns the context to restricted input. */
int std2g_set_spins(void *ctx, const int *csp);

/* AO one-electron integrals on the device from the primitive list the
   reference's readers fill (readbasmold.f:330-517, readxtb.f:150-160) and its
   integral step consumes (intslvm.f:21-210; libcint.f:19-352, 653-756):
     ipty [nprims]  Cartesian type 1..20: s; px py pz; xx yy zz xy xz yz;
                    xxx yyy zzz xxy xxz xyy yyz xzz yzz xyz (intpack.f90:1213-1218)
     ipao [nprims]  AO of the primitive, 1-based
     ipat [nprims]  atom of the primitive, 1-based
     exip [nprims]  exponent;  cxip [nprims] coefficient, all normalisation folded in
   Writes the packed S, mu_L, mu_V, mu_M of std2g_load (host arrays; any may be
   NULL to skip it).  Replaces the host precompute of main.f:756-797. */
int std2g_ao_integrals(void *ctx, int ncent, const double *xyz, int nao, int nprims,
                       const int *ipty, const int *ipao, const int *ipat,
                       const double *exip, const double *cxip, double *S,
                       double *mu_L, double *mu_V, double *mu_M);

/* std2g_load with the AO integrals formed on the device from the primitive
   list (as std2g_ao_integrals); iaoat follows from iaoat(ipao(i)) = ipat(i)
   (intslvm.f:71-74).  No integral array crosses the host link. */
int std2g_load_prims(void *ctx, int ncent, int nmo, int nao, const double *xyz,
                     const double *C, const double *eps, const double *occ,
                     int nprims, const int *ipty, const int *ipao, const int *ipat,
                     const double *exip, const double *cxip);

/* Run the excitation path: orbital window, S^1/2, Loewdin charges, gamma,
   diagonal screen, PT selection, A (or A+B / A-B), eigen-solve, properties and
   (sTDA) the velocity correction.  Replaces stda.f:142-1471 for the RKS
   singlet/triplet sTDA branch and the sTD-DFT branch (srpapack.f:32-197). */
int std2g_solve(void *ctx, const std2g_params *par, std2g_result *res);

/* Dynamic polarizability alpha(omega) from the A+B / A-B matrices of the last
   sTD-DFT build (params.rpa=1 path of std2g_solve, or built here if needed).
   Replaces lresp (linear_response.f:23-192).  omega in Eh (the reference reads
   wavelengths and converts with 45.56335/lambda, linear_response.f:85).
   alpha: [nomega*9] row-major 3x3 tensors.  resid: [nomega] max relative
   residual of the solves (may be NULL). */
int std2g_polarizability(void *ctx, const std2g_params *par, const double *omega,
                         int nomega, double *alpha, double *resid);

/* First hyperpolarizability beta(-2w; w, w) of sTD-DFT, the second-harmonic
   tensor that lresp1 prints (linear_response.f:196-700; the -resp keyword),
   at the frequencies omega [nomega] (Eh; the reference reads wavelengths and
   prepends w = 0, linear_response.f:283-287).  The linear responses at +w and
   -2w come from the same solver as std2g_polarizability (FP64 residuals below
   1e-10 in both forms) and are contracted with the occupied-occupied and
   virtual-virtual dipole couplings (List_A / List_B, :1089-1167).
   beta [nomega*27]: row-major beta[w][x][y][z] (atomic units); beta_hrs
   [nomega] (may be NULL): the hyper-Rayleigh value sqrt(<beta^2_ZZZ> +
   <beta^2_XZZ>) (:1489-1662). */
int std2g_hyperpolarizability(void *ctx, const std2g_params *par, const double *omega,
                              int nomega, double *beta, double *beta_hrs);

/* Two-photon absorption of the lowest ntrans sTD-DFT states in the
   single-photon-resonance form (lresp_2PA_SP, linear_response.f:4604-4938;
   the -2PA keyword): rows [ntrans*6] = (n, w_n in eV, delta_par, delta_perp,
   delta_circ, rho = delta_par / delta_perp) as in the reference's 2PA-abs
   file.  The states are those of the dense sTD-DFT solve of par's window, with
   the reference's -2PA state vectors (srpapack.f:99-106 skips the halving of
   the packed diagonals under that keyword, so each diagonal enters twice);
   the responses at -w_n / 2 are the FP64 form's dense solves.  STD2G_EINVAL
   when ntrans exceeds the roots below E_thr. */
int std2g_two_photon(void *ctx, const std2g_params *par, int ntrans, double *rows);

/* Selected CSF list of the last solve: iconf [2*cap] as (i,a) pairs, 1-based
   MO indices within the active window (occupied 1..no, virtual no+1..no+nv,
   as iconf(:,1:2) in stda.f), and the diagonal ed [cap] after PT lowering. */
int std2g_get_csf(void *ctx, int *iconf, double *ed, int cap, int *nci);

/* Eigenvectors of the last solve: X [nci*cap] column-major (TDA X, or sTD-DFT
   X with Y in the second array when non-NULL). */
int std2g_get_vectors(void *ctx, double *X, double *Y, int cap, int *nroot, int *nci);

/* Per-phase device timings of the last solve in ms (names via
   std2g_phase_name); returns the number of phases. */
int std2g_phase_times(void *ctx, double *ms, int cap);
const char *std2g_phase_name(int phase);

/* Number of kernels this library launched since the context was created. */
int64_t std2g_kernel_launches(void *ctx);

/* Tensor-core contraction statistics of the last solve: total device time
   (ms), number of launches and algorithmic FLOPs (used for the roofline). */
int std2g_kernel_stats(void *ctx, double *ms, int64_t *launches, double *flop);

/* FP64 matrix-product statistics of the last solve.  With timing on, every
   product is bracketed by an event pair on its stream (off by default: the
   events add a host call per product); std2g_gemm_stats returns the summed
   device time of the timed products (0 with timing off), their number and
   their algorithmic FLOPs 2 m n k.  The first solve after a load also
   counts the products of the overlap's square root (formed once per load). */
int std2g_set_gemm_timing(void *ctx, int on);
int std2g_gemm_stats(void *ctx, double *ms, int64_t *calls, double *flop);

/* Statistics of the last solve: Davidson iterations, sigma vectors formed
   with tensor-core (mixed) products and with FP64 products, and the number of
   PT candidates whose selection was re-decided in FP64 (mixed form). */
int std2g_solver_stats(void *ctx, int *iters, int64_t *matvecs, int64_t *matvecs_fp64,
                       int64_t *pt_rechecked);

/* Diagonal screen without any device allocation.  This entry point has no
   counterpart in the reference.  It is for callers that cannot allocate device
   memory: hosts whose GPU memory is owned by another allocator (a framework
   that has reserved it for its own pool), or that must not call cudaMalloc at
   this point because it synchronises the device.  They pass device buffers
   they already own:
     d_xyz   [4*ncent]        x,y,z (Bohr), Z (1..94) per atom
     d_iaoat [nao]            AO -> atom, 1-based
     d_clow  [nao*(no+nv)]    Loewdin-orthogonalised MOs of the active window,
                              occupied then virtual, each block energy-sorted
     d_eps   [no+nv]          their orbital energies (Eh)
   and receive, for k = i*nv + a (0-based i < no, a < nv),
     d_de    [no*nv]          diagonal element of A ((e_a-e_i) - (ii|aa) + ak (ia|ia))
     d_flag  [no*nv]          1 primary (<= E_thr), 2 PT candidate, 0 neither
   from par: ax, e_thr_ev, alpha_k, beta_j, fthr_ev, triplet, kshift(+shift).
   Work arrays live in one fixed 64 MiB __device__ array that every GPU using
   this library keeps until the process exits; sizes with
   2N^2 + N(2no + nv) + 2 N no nv > 8 Mi doubles return STD2G_ECAP.  The first
   call on a device looks up that array's address (make it before any stream
   capture; several host threads may make it at once).  All calls share the
   array, so calls whose kernels overlap on the GPU race.  Kernels are queued
   on `stream` (a cudaStream_t, NULL = default).  The caller's current device
   is restored on return; an error the caller left pending in the CUDA context
   makes the call return STD2G_ECUDA without launching anything (the error is
   left in place).  Not supported after a cudaDeviceReset by the host. */
int std2g_screen_noalloc(int device, int ncent, int nao, int no, int nv, const double *d_xyz,
                         const int *d_iaoat, const double *d_clow, const double *d_eps,
                         const std2g_params *par, double *d_de, int *d_flag, void *stream);

/* ---- served / batched form ---------------------------------------------
   Many molecules through a pool of contexts (continuous batching).  The
   reference runs one molecule per process (main.f:928-929); this layer has no
   counterpart there.  A request is admitted when one of `slots` contexts is
   free and its estimated device footprint fits `hbm_budget` beside the
   requests in flight (FIFO; a request that alone exceeds the budget runs when
   nothing else does).  Requests that arrive while others run start as soon as
   a slot and memory free up; their kernels overlap on the device.  Each
   context keeps its device work buffers between requests.  The server owns
   one host thread per slot; submit / wait / poll are thread-safe. */
typedef struct {
  int device;
  int precision;        /* as std2g_opts.precision, for every slot */
  int slots;            /* concurrent solves (1..64) */
  int trace;            /* > 0: one line per finished request on stderr (slot,
                           times, phase times of its solve and alpha(omega)) */
  int64_t hbm_budget;   /* bytes the admitted requests may use (0: 80 % of free memory) */
  int flags;            /* STD2G_FLAG_* of every slot's context */
} std2g_server_opts;

typedef struct {
  int ncent, nmo, nao;  /* as std2g_load; every array is copied at submit */
  const double *xyz, *C, *eps, *occ;
  const int *iaoat;
  const double *S, *mu_L, *mu_V, *mu_M;
  std2g_params params;  /* the excitation solve (std2g_solve) */
  int nomega;           /* > 0: also alpha(omega) (std2g_polarizability) */
  const double *omega;  /* [nomega] Eh */
  /* optional primitive list (as std2g_load_prims): with nprims > 0 the AO
     integrals are formed on the device and iaoat, S, mu_L, mu_V, mu_M may be
     NULL */
  int nprims;
  const int *ipty, *ipao, *ipat;
  const double *exip, *cxip;
} std2g_request;

int std2g_server_create(void **srv, const std2g_server_opts *opts);
/* Queue one request; *ticket identifies it for poll / wait.  If every slot
   has lost its context (a replacement context could not be created), queued
   requests finish with that status and submit returns it. */
int std2g_server_submit(void *srv, const std2g_request *rq, int64_t *ticket);
/* *done = 1 once the request has finished (successfully or not). */
int std2g_server_poll(void *srv, int64_t ticket, int *done);
/* Block until the request has finished; returns its status and, on success,
   fills res (caller arrays of res->cap), alpha [nomega*9], alpha_resid
   [nomega] and timing_ms [3] = queued, running, total (submit to finish).
   The ticket is released, except on STD2G_ECAP (res->cap below the number of
   roots): then res->nroot holds that number and the caller waits again on
   the same ticket with more room. */
int std2g_server_wait(void *srv, int64_t ticket, std2g_result *res, double *alpha,
                      double *alpha_resid, double *timing_ms);
/* stats[7]: submitted, completed, in flight, peak in flight, bytes in flight
   (estimated), peak bytes in flight, budget. */
int std2g_server_stats(void *srv, int64_t *stats);
/* With STD2G_FLAG_BATCH_EIGEN: std2g_batch_stats of the server's batch (zeros
   without it). */
int std2g_server_batch_stats(void *srv, int64_t *problems, int64_t *iterations,
                             int64_t *members, double *ms);
/* Stop the workers after their current requests (queued ones are dropped) and
   free the contexts; call after the last wait. */
void std2g_server_destroy(void *srv);

/* Cap the persistent tensor-core kernels of this context at max_sms CTAs (one
   per SM; 0 = all SMs), so that several contexts sharing a device (the
   request server's slots) leave SMs to each other's kernels.  No reference
   counterpart. */
int std2g_set_sm_limit(void *ctx, int max_sms);

/* ---- batched eigensolves across contexts ---------------------------------
   Many molecules' excitation solves share one lockstep Davidson: contexts
   attached to a batch, each solving on its own host thread, hand the TDA
   eigenproblem of a std2g_solve (321 to 6144 CSFs, a root request of
   p.nroots > 0 with solver 0, roots + buffer roots <= 112) to the batch, whose
   coordinator thread runs one Davidson iteration of every waiting problem per
   round of launches (grouped FP64 products, batched Rayleigh-Ritz, batched
   residual and Cholesky-QR kernels; three host synchronisations per round for
   the whole batch).  Problems join at the next iteration and leave when their
   roots converge (continuous batching).  Results are those of the unbatched
   Davidson (same algorithm, FP64 throughout; dense A instead of matrix-free
   products) to the convergence tolerance.  No reference counterpart: the
   reference solves one molecule per process with ssyevr (stda.f:1133-1150).
   std2g_batch_destroy: after every attached context has finished its solves. */
int std2g_batch_create(int device, void **batch);
/* Attach (batch) or detach (NULL) a context; same device as the batch. */
int std2g_attach_batch(void *ctx, void *batch);
/* Problems solved, batched iterations run, members summed over iterations;
   ms (NULL or [2]): wall time of the iterations, total and up to their first
   host synchronisation (products, Rayleigh-Ritz, residuals). */
int std2g_batch_stats(void *batch, int64_t *problems, int64_t *iterations, int64_t *members,
                      double *ms);
void std2g_batch_destroy(void *batch);
/* 1 when the last std2g_solve of ctx took its eigensolve from a batch. */
int std2g_last_batched(void *ctx);

/* Diagnostic: the engine's FP64 matrix product (DMMA kernel with split-K,
   used for ONETRI, the Loewdin transform, gamma.q and the property
   contractions): C = alpha op(A) op(B) + beta C on host arrays, column-major,
   op = transpose when ta / tb; batch members follow one another at sizes
   lda*cols(A), ldb*cols(B), ldc*n.  *ms (may be NULL): device time of the
   product alone.  No reference counterpart (the reference calls BLAS). */
int std2g_dgemm_check(int device, int ta, int tb, int m, int n, int k, double alpha,
                      const double *A, int64_t lda, const double *B, int64_t ldb,
                      double beta, double *C, int64_t ldc, int batch, double *ms);

/* Diagnostic: lowest k eigenpairs of the symmetric n x n matrix A (host,
   column-major, lower triangle used) by the engine's single-block eigensolver
   of the Davidson Rayleigh-Ritz step (n <= 320), and all eigenvalues by
   cuSOLVER syevd for comparison.  w [k], Z [n*k], w_ref [n] (host).  No
   reference counterpart (the reference diagonalises with LAPACK ssyevr). */
int std2g_symeig_check(int device, int n, int k, const double *A, double *w, double *Z,
                       double *w_ref);

const char *std2g_error_string(int status);
void std2g_destroy(void *ctx);

#ifdef __cplusplus
}
#endif
#endif /* STD2G_H */
