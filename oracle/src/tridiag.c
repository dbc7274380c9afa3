/*
 * ORACLE (test infrastructure only; never linked into the product).
 *
 * Batched tridiagonal solves as ops_tridMultiDimBatch / _Inc hand them to
 * the Tridsolver library (ops/c/src/tridiag/ops_tridiag.cpp:78-165 and
 * :168-249): every line along `solvedim` of an ndim-dimensional array with
 * extents dims[] and padded extents pads[] (element (i0,i1,i2) at
 * i0 + i1*pads[0] + i2*pads[0]*pads[1]) is the system
 *     a_i x_{i-1} + b_i x_i + c_i x_{i+1} = d_i,   a_0 and c_{n-1} unused.
 * Tridsolver (github.com/OP-DSL/tridsolver, not vendored in the reference
 * and not pinned to a version) solves each line with the Thomas algorithm;
 * this restates the textbook Thomas elimination (forward elimination with
 * c'_i = c_i / (b_i - a_i c'_{i-1}), back substitution). The non-Inc form
 * overwrites d with x; the Inc form adds x to u and leaves d untouched
 * (ops_tridiag.cpp:168-249). Parity is unpinned at the Tridsolver boundary:
 * no reference vector exists for it, so tests hold both sides to the FP64
 * residual of the system and to each other within rounding.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

static void line_geometry(int ndim, int solvedim, const int *dims, const int *pads, long *stride, long *nlines) {
  long s = 1;
  for (int d = 0; d < solvedim; d++) s *= pads[d];
  *stride = s;
  long n = 1;
  for (int d = 0; d < ndim; d++)
    if (d != solvedim) n *= dims[d];
  *nlines = n;
}

/* Offset of the first element of line `l` (lines enumerate the non-solve
 * dimensions, fastest dimension first). */
static long line_offset(int ndim, int solvedim, const int *dims, const int *pads, long l) {
  long off = 0, mult = 1;
  for (int d = 0; d < ndim; d++) {
    if (d == solvedim) {
      mult *= pads[d];
      continue;
    }
    long idx = l % dims[d];
    l /= dims[d];
    off += idx * mult;
    mult *= pads[d];
  }
  return off;
}

/* Lines are independent: OpenMP splits them over the host threads (the
 * CPU baseline uses all cores; tests run it single-threaded or not, with
 * identical results since each line is solved by one thread). */
#define THOMAS_BODY(T)                                                                     \
  long stride, nlines;                                                                     \
  line_geometry(ndim, solvedim, dims, pads, &stride, &nlines);                             \
  const int n = dims[solvedim];                                                            \
  _Pragma("omp parallel")                                                                  \
  {                                                                                        \
  T *cp = (T *)malloc(sizeof(T) * (n > 0 ? n : 1));                                        \
  T *dp = (T *)malloc(sizeof(T) * (n > 0 ? n : 1));                                        \
  _Pragma("omp for schedule(static)")                                                      \
  for (long l = 0; l < nlines; l++) {                                                      \
    if (n <= 0) continue;                                                                  \
    const long o = line_offset(ndim, solvedim, dims, pads, l);                             \
    cp[0] = c[o] / b[o];                                                                   \
    dp[0] = d[o] / b[o];                                                                   \
    for (int i = 1; i < n; i++) {                                                          \
      const long k = o + i * stride;                                                       \
      T r = (T)1 / (b[k] - a[k] * cp[i - 1]);                                              \
      cp[i] = c[k] * r;                                                                    \
      dp[i] = (d[k] - a[k] * dp[i - 1]) * r;                                               \
    }                                                                                      \
    for (int i = n - 2; i >= 0; i--) dp[i] = dp[i] - cp[i] * dp[i + 1];                    \
    for (int i = 0; i < n; i++) {                                                          \
      const long k = o + i * stride;                                                       \
      if (u) u[k] += dp[i];                                                                \
      else d[k] = dp[i];                                                                   \
    }                                                                                      \
  }                                                                                        \
  free(cp);                                                                                \
  free(dp);                                                                                \
  }

/* tridDmtsvStridedBatch / tridDmtsvStridedBatchInc (u != NULL). */
void oracle_trid_batch_d(const double *a, const double *b, const double *c, double *d, double *u, int ndim,
                         int solvedim, const int *dims, const int *pads) {
  THOMAS_BODY(double)
}

/* tridSmtsvStridedBatch / tridSmtsvStridedBatchInc (u != NULL). */
void oracle_trid_batch_s(const float *a, const float *b, const float *c, float *d, float *u, int ndim, int solvedim,
                         const int *dims, const int *pads) {
  THOMAS_BODY(float)
}
