/* TEST INFRASTRUCTURE ONLY: the CPU baseline's restatement of the reference's
 * two pair loops, with the reference's arithmetic.  The product never links
 * or calls this file; the oracle's CPU timing sample does.
 *
 *   ptselect (stda.f:1773-1863): for every PT candidate k = (i,a) and every
 *     primary j = (jo,b): ek = sdot(N, p_ia, q_jb), ej = sdot(N, p_ij, q_ab)
 *     in real*4, pt(j) = (ak ek - ej)^2 / (E_k - E_j + 1e-10) in real*8;
 *     the candidate is selected when sum_j pt(j) > thrp, otherwise pt is added
 *     to pt2.  OpenMP over candidates, as there.
 *   rtdamat (stda.f:2010-2056): A(j,i) = ak sdot(N, p_ia, q_jb) -
 *     sdot(N, p_ij, q_ab) for j < i, A(i,i) = ed(i), real*4.  OpenMP over rows.
 *
 * Layout (0-based): p_ia, q_ia [N x no*nv] column (i*nv + a); p_ij [N x
 * no(no+1)/2] and q_ab [N x nv(nv+1)/2] column lin(x,y) = max(max+1)/2 + min.
 * The dot product is compiled once per instruction set (target_clones) and
 * picked at load time, as an optimised BLAS sdot would be.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

static inline int64_t lin0(int64_t x, int64_t y) {
  const int64_t hi = x > y ? x : y, lo = x > y ? y : x;
  return hi * (hi + 1) / 2 + lo;
}

__attribute__((target_clones("avx512f", "avx2", "default")))
static float sdot_n(int n, const float *x, const float *y) {
  float s = 0.0f;
#pragma omp simd reduction(+ : s)
  for (int t = 0; t < n; ++t) s += x[t] * y[t];
  return s;
}

/* PT selection over candidates (kio, kiv) with energies edpt against the
 * primaries (jo, jv) with energies ed.  incl[k] = 1 when selected; pt2[j]
 * accumulates the unselected candidates' terms.  Returns the number selected. */
int pairloops_ptselect(int N, int nv, const float *pia, const float *qia, const float *pij,
                       const float *qab, int nk, const int *kio, const int *kiv,
                       const double *edpt, int nex, const int *jo, const int *jv,
                       const double *ed, double dak, double thrp, unsigned char *incl,
                       double *pt2) {
  const float ak = (float)dak;
  int nsel = 0;
  memset(pt2, 0, sizeof(double) * (size_t)nex);
#pragma omp parallel reduction(+ : nsel)
  {
    double *pt = (double *)malloc(sizeof(double) * (size_t)(nex > 0 ? nex : 1));
    double *acc = (double *)calloc((size_t)(nex > 0 ? nex : 1), sizeof(double));
#pragma omp for schedule(dynamic, 1)
    for (int k = 0; k < nk; ++k) {
      const int io = kio[k], iv = kiv[k];
      const float *qk = pia + (int64_t)N * ((int64_t)io * nv + iv);
      const double de = edpt[k];
      double pert = 0.0;
      for (int j = 0; j < nex; ++j) {
        const float ek = sdot_n(N, qk, qia + (int64_t)N * ((int64_t)jo[j] * nv + jv[j]));
        const float ej = sdot_n(N, pij + (int64_t)N * lin0(io, jo[j]),
                                qab + (int64_t)N * lin0(iv, jv[j]));
        const double amat = (double)(ak * ek - ej);
        pt[j] = amat * amat / (de - ed[j] + 1e-10);
        pert += pt[j];
      }
      if (pert > thrp) {
        incl[k] = 1;
        ++nsel;
      } else {
        incl[k] = 0;
        for (int j = 0; j < nex; ++j) acc[j] += pt[j];
      }
    }
#pragma omp critical
    for (int j = 0; j < nex; ++j) pt2[j] += acc[j];
    free(acc);
    free(pt);
  }
  return nsel;
}

/* Rows r0..r1-1 of the lower triangle of A (rtdamat) into rows [r1-r0 x nci]
 * (row r holds A(r, 0..r), the rest untouched). */
void pairloops_rtdamat_rows(int N, int nv, const float *pia, const float *qia, const float *pij,
                            const float *qab, int nci, const int *io, const int *iv,
                            const double *ed, double dak, int r0, int r1, float *rows) {
  const float ak = (float)dak;
#pragma omp parallel for schedule(dynamic, 4)
  for (int i = r0; i < r1; ++i) {
    const float *qk = pia + (int64_t)N * ((int64_t)io[i] * nv + iv[i]);
    float *row = rows + (int64_t)(i - r0) * nci;
    for (int j = 0; j < i; ++j) {
      const float ek = sdot_n(N, qk, qia + (int64_t)N * ((int64_t)io[j] * nv + iv[j]));
      const float ej = sdot_n(N, pij + (int64_t)N * lin0(io[i], io[j]),
                              qab + (int64_t)N * lin0(iv[i], iv[j]));
      row[j] = ak * ek - ej;
    }
    row[i] = (float)ed[i];
  }
}
