/* gjx_pp80.c -- accuracy post-processor of (H)SVD results, in x87 extended
 * precision (long double, 64-bit significand), following the reference's
 * var/pp80.f90 (the non-MAGMA build, REAL(10) arithmetic, no FMA):
 *
 *   gjx_pp80_jorth   || X^T J X - J ||_M and _F       pp80.f90:187-263 (U),
 *                    || X J X^T - J ||_M and _F       pp80.f90:265-339 (U U^T),
 *                                                     pp80.f90:469-646 (V, J)
 *   gjx_pp80_resid   || A U - U D ||_M, _F and _R     pp80.f90:660-760
 *                    (rows of U back-permuted by IPIV first, QBAKCP,
 *                    pp80.f90:876-901)
 *   gjx_pp80_derr    ABSERR and RELERR of D against the exact LAMBDA after
 *                    both are sorted descending        pp80.f90:800-880
 *
 * Every sum runs in the order of the Fortran loops, so the results are the
 * reference tool's to the last bit where the inputs are the same.  The
 * matrix products run over OpenMP threads (one output column per iteration,
 * as the reference's !$OMP PARALLEL DO), which does not change any sum.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef long double ld_t;

/* element (k, j) of X (column major, leading dimension ldx), read as column j
 * of X (trans = 0) or as row j (trans != 0) */
static inline ld_t xel(const double *X, unsigned ldx, int trans, unsigned k, unsigned j)
{
  return (ld_t)(trans ? X[(size_t)k * ldx + j] : X[(size_t)j * ldx + k]);
}

/* E = X^T Js X - Jr (trans = 0; X is nk x nr) or X Js X^T - Jr (trans != 0;
 * X is nr x nk), Js = diag(+1 x psum, -1 ...), Jr = diag(+1 x pres, -1 ...).
 * out[0] = max |E_ij| (i >= j), out[1] = || E ||_F. */
int gjx_pp80_jorth(const unsigned rows, const unsigned cols, const double *const X, const unsigned ldx,
                   const int trans, const unsigned psum, const unsigned pres, double *const out)
{
  const unsigned nk = trans ? cols : rows, nr = trans ? rows : cols;
  if (!X || !out || ldx < rows || psum > nk || pres > nr)
    return -1;
  ld_t *const MM = (ld_t *)malloc(sizeof(ld_t) * (size_t)nr * nr);
  if (!MM && nr)
    return -2;
#pragma omp parallel for schedule(dynamic, 1)
  for (unsigned j = 0u; j < nr; ++j) {
    ld_t s = (j < pres) ? -1.0L : 1.0L;
    for (unsigned k = 0u; k < psum; ++k) {
      const ld_t x = xel(X, ldx, trans, k, j);
      s = s + x * x;
    }
    for (unsigned k = psum; k < nk; ++k) {
      const ld_t x = xel(X, ldx, trans, k, j);
      s = s - x * x;
    }
    MM[(size_t)j * nr + j] = fabsl(s);
    for (unsigned i = j + 1u; i < nr; ++i) {
      ld_t t = 0.0L;
      for (unsigned k = 0u; k < psum; ++k)
        t = t + xel(X, ldx, trans, k, j) * xel(X, ldx, trans, k, i);
      for (unsigned k = psum; k < nk; ++k)
        t = t - xel(X, ldx, trans, k, j) * xel(X, ldx, trans, k, i);
      MM[(size_t)j * nr + i] = fabsl(t);
    }
  }
  ld_t qmax = 0.0L, off = 0.0L, diag = 0.0L;
  for (unsigned j = 0u; j < nr; ++j)
    for (unsigned i = j; i < nr; ++i)
      if (MM[(size_t)j * nr + i] > qmax)
        qmax = MM[(size_t)j * nr + i];
  for (unsigned j = 0u; j < nr; ++j) {
    diag = diag + MM[(size_t)j * nr + j] * MM[(size_t)j * nr + j];
    for (unsigned i = j + 1u; i < nr; ++i)
      off = off + MM[(size_t)j * nr + i] * MM[(size_t)j * nr + i];
  }
  diag = 2.0L * off + diag;
  out[0] = (double)qmax;
  out[1] = (double)sqrtl(diag);
  free(MM);
  return 0;
}

/* Residual of the eigenproblem A = G J G^T: R = U diag(D) - A U with the rows
 * of U back-permuted by ipiv (1-based LAPACK-style interchanges, sign ignored;
 * NULL: none).  out[0] = max |R_ij|, out[1] = || R ||_F, out[2] = max of
 * |R_ij| / (sqrt|D_i| sqrt|D_j|) over the first n rows and |R_ij| below them,
 * as the reference tool scales only rows 1..n. */
int gjx_pp80_resid(const unsigned m, const unsigned n, const double *const A, const unsigned lda,
                   const double *const U, const unsigned ldu, const double *const D, const int *const ipiv,
                   double *const out)
{
  if (!A || !U || !D || !out || lda < m || ldu < m || n > m)
    return -1;
  ld_t *const Uq = (ld_t *)malloc(sizeof(ld_t) * (size_t)m * n);
  ld_t *const R = (ld_t *)malloc(sizeof(ld_t) * (size_t)m * n);
  if ((!Uq || !R) && m && n) {
    free(Uq);
    free(R);
    return -2;
  }
  for (unsigned j = 0u; j < n; ++j)
    for (unsigned i = 0u; i < m; ++i)
      Uq[(size_t)j * m + i] = (ld_t)U[(size_t)j * ldu + i];
  if (ipiv)
    for (unsigned kk = n; kk-- > 0u;) {
      const unsigned kp = (unsigned)abs(ipiv[kk]) - 1u;
      if (kp != kk && kp < m)
        for (unsigned j = 0u; j < n; ++j) {
          const ld_t t = Uq[(size_t)j * m + kk];
          Uq[(size_t)j * m + kk] = Uq[(size_t)j * m + kp];
          Uq[(size_t)j * m + kp] = t;
        }
    }
#pragma omp parallel for schedule(dynamic, 1)
  for (unsigned j = 0u; j < n; ++j)
    for (unsigned i = 0u; i < m; ++i) {
      ld_t v = Uq[(size_t)j * m + i] * (ld_t)D[j];
      for (unsigned k = 0u; k < m; ++k)
        v = v - (ld_t)A[(size_t)k * lda + i] * Uq[(size_t)j * m + k];
      R[(size_t)j * m + i] = fabsl(v);
    }
  ld_t qmax = 0.0L, ss = 0.0L;
  for (unsigned j = 0u; j < n; ++j)
    for (unsigned i = 0u; i < m; ++i)
      if (R[(size_t)j * m + i] > qmax)
        qmax = R[(size_t)j * m + i];
  out[0] = (double)qmax;
  for (unsigned j = 0u; j < n; ++j)
    for (unsigned i = 0u; i < m; ++i)
      ss = ss + R[(size_t)j * m + i] * R[(size_t)j * m + i];
  out[1] = (double)sqrtl(ss);
  for (unsigned j = 0u; j < n; ++j) {
    const ld_t qj = sqrtl(fabsl((ld_t)D[j]));
    for (unsigned i = 0u; i < n; ++i)
      R[(size_t)j * m + i] = R[(size_t)j * m + i] / (sqrtl(fabsl((ld_t)D[i])) * qj);
  }
  qmax = 0.0L;
  for (unsigned j = 0u; j < n; ++j)
    for (unsigned i = 0u; i < m; ++i)
      if (R[(size_t)j * m + i] > qmax)
        qmax = R[(size_t)j * m + i];
  out[2] = (double)qmax;
  free(R);
  free(Uq);
  return 0;
}

static int desc(const void *a, const void *b)
{
  const double x = *(const double *)a, y = *(const double *)b;
  return (x < y) - (x > y);
}

/* abserr[i] = lambda_i - D_i and relerr[i] = abserr[i] / lambda_i after
 * both vectors are sorted descending; element n of each holds the entry of
 * largest magnitude (its sign kept, the first one on ties). */
int gjx_pp80_derr(const unsigned n, const double *const D, const double *const lambda, double *const abserr,
                  double *const relerr)
{
  if (!D || !lambda || !abserr || !relerr)
    return -1;
  double *const dd = (double *)malloc(sizeof(double) * (n ? n : 1u));
  double *const ll = (double *)malloc(sizeof(double) * (n ? n : 1u));
  if (!dd || !ll) {
    free(dd);
    free(ll);
    return -2;
  }
  memcpy(dd, D, sizeof(double) * n);
  memcpy(ll, lambda, sizeof(double) * n);
  qsort(dd, n, sizeof(double), desc);
  qsort(ll, n, sizeof(double), desc);
  double scl = 0.0;
  for (unsigned i = 0u; i < n; ++i) {
    abserr[i] = ll[i] - dd[i];
    if (fabs(scl) < fabs(abserr[i]))
      scl = abserr[i];
  }
  abserr[n] = scl;
  scl = 0.0;
  for (unsigned i = 0u; i < n; ++i) {
    relerr[i] = abserr[i] / ll[i];
    if (fabs(scl) < fabs(relerr[i]))
      scl = relerr[i];
  }
  relerr[n] = scl;
  free(ll);
  free(dd);
  return 0;
}
