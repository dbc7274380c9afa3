/*
 * ORACLE (test infrastructure only; never linked into the product).
 *
 * Plain-C restatement of the reference's Laplace Jacobi app:
 *   apps/c/laplace2d_tutorial/step7/laplace2d.cpp:113-124 (iteration loop)
 *   apps/c/laplace2d_tutorial/step7/laplace_kernels.h:10-12 (copy)
 *   apps/c/laplace2d_tutorial/step7/laplace_kernels.h:22-26 (apply_stencil)
 * The per-cell expression keeps the reference's operation order, and the
 * max reduction is order-independent, so results are bit-identical to the
 * reference's CPU build (checked by tests against oracle/_ref and golden
 * vectors produced by it).
 *
 * Layout: a field is its full extent (imax+2) x (jmax+2) doubles, x fastest,
 * logical index (x, y) at [(y+1)*(imax+2) + (x+1)], halo ring = boundary.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "seeded_rng.h"

/* Runs `iters` Jacobi iterations in place on A (full extent); writes the
 * max |delta| of iteration k to err[k] when err is non-NULL. */
void oracle_laplace_run(int imax, int jmax, int iters, double *A, double *err) {
  const long W = imax + 2;
  double *Anew = (double *)malloc(sizeof(double) * W * (jmax + 2));
  memcpy(Anew, A, sizeof(double) * W * (jmax + 2));
  for (int it = 0; it < iters; it++) {
    double error = -1.0;  /* reduction handle first use: any value < |delta| */
    int first = 1;
    for (int y = 0; y < jmax; y++) {
      for (int x = 0; x < imax; x++) {
        const long c = (y + 1) * W + (x + 1);
        /* Anew(0,0) = 0.25f * (A(1,0) + A(-1,0) + A(0,-1) + A(0,1)) */
        Anew[c] = 0.25f * (A[c + 1] + A[c - 1] + A[c - W] + A[c + W]);
        double d = fabs(Anew[c] - A[c]);
        if (first) { error = d; first = 0; }
        else error = fmax(error, d);
      }
    }
    if (err) err[it] = (imax > 0 && jmax > 0) ? error : -1.7976931348623157e308;
    for (int y = 0; y < jmax; y++)
      for (int x = 0; x < imax; x++) {
        const long c = (y + 1) * W + (x + 1);
        A[c] = Anew[c];
      }
  }
  free(Anew);
}

/* Seeded initial field: zero interior, ring cell (x, y) = u01(seed, k) with
 * k = (y+1)*(imax+2) + (x+1) (the same rule as the reference-side driver
 * oracle/ref_drivers/laplace_seeded.cpp). */
void oracle_laplace_seed(int imax, int jmax, uint64_t seed, double *A) {
  const long W = imax + 2;
  for (int y = -1; y <= jmax; y++)
    for (int x = -1; x <= imax; x++) {
      long k = (long)(y + 1) * W + (x + 1);
      int ring = (x == -1 || x == imax || y == -1 || y == jmax);
      A[k] = ring ? sm64_u01(seed, (uint64_t)k) : 0.0;
    }
}

/* The reference step7 boundary (laplace_kernels.h:14-20 with the driver's
 * ranges, laplace2d.cpp:69-91): sine on the left column, damped sine on the
 * right, zero elsewhere; used for the golden known-answer test. */
void oracle_laplace_step7_init(int imax, int jmax, double *A) {
  const long W = imax + 2;
  const double pi = 2.0 * asin(1.0);
  memset(A, 0, sizeof(double) * W * (jmax + 2));
  for (int y = -1; y <= jmax; y++) {
    A[(y + 1) * W + 0] = sin(pi * (y + 1) / (jmax + 1));
    A[(y + 1) * W + (imax + 1)] = sin(pi * (y + 1) / (jmax + 1)) * exp(-pi);
  }
}

uint64_t oracle_sm64_at(uint64_t seed, uint64_t k) { return sm64_at(seed, k); }
double oracle_sm64_u01(uint64_t seed, uint64_t k) { return sm64_u01(seed, k); }
