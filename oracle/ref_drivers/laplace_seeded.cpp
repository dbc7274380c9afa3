/*
 * Test infrastructure (oracle side only): seeded Laplace driver for the
 * reference OPS library. Built by oracle/build_ref.sh into oracle/_ref with
 * the reference's own kernels (apps/c/laplace2d_tutorial/step7/
 * laplace_kernels.h) and the reference's legacy translator, exactly like the
 * reference builds its step7 app (apps/c/laplace2d_tutorial/step7/
 * laplace2d.cpp:41-124), with three differences:
 *   - grid size, iteration count and seed come from the command line;
 *   - the boundary ring holds seeded U[0,1) values instead of the sine
 *     profile; cell (x, y) of the ring, x in [-1, imax], y in [-1, jmax],
 *     takes sm64_u01(seed, (y+1)*(imax+2) + (x+1));
 *   - a fixed number of iterations runs (no tolerance exit), and the max
 *     |delta| of every iteration is printed with 17 digits.
 * usage: laplace2d_seeded <imax> <jmax> <iters> <seed> [dump.bin]
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <stdint.h>

int imax, jmax;
double pi = 2.0 * asin(1.0);

#define OPS_2D
#include <ops_seq_v2.h>
#include "laplace_kernels.h"
#include "seeded_rng.h"

static void seed_ring(ops_dat dat, ops_stencil sten, uint64_t seed) {
  ops_memspace ms = OPS_HOST;
  double *p = (double *)ops_dat_get_raw_pointer(dat, 0, sten, &ms);
  int disp[OPS_MAX_DIM], size[OPS_MAX_DIM], stride[OPS_MAX_DIM], dm[OPS_MAX_DIM], dp[OPS_MAX_DIM];
  ops_dat_get_raw_metadata(dat, 0, disp, size, stride, dm, dp);
  for (int y = -1; y <= jmax; y++)
    for (int x = -1; x <= imax; x++)
      if (x == -1 || x == imax || y == -1 || y == jmax)
        p[x + y * stride[0]] =
            sm64_u01(seed, (uint64_t)(y + 1) * (uint64_t)(imax + 2) + (uint64_t)(x + 1));
  ops_dat_release_raw_data(dat, 0, OPS_WRITE);
}

int main(int argc, const char **argv) {
  if (argc < 5) {
    fprintf(stderr, "usage: %s imax jmax iters seed [dump.bin]\n", argv[0]);
    return 2;
  }
  imax = atoi(argv[1]);
  jmax = atoi(argv[2]);
  int iter_max = atoi(argv[3]);
  uint64_t seed = strtoull(argv[4], NULL, 10);
  ops_init(argc, argv, 1);

  double *A = NULL, *Anew = NULL;
  ops_block block = ops_decl_block(2, "my_grid");
  int size[] = {imax, jmax};
  int base[] = {0, 0};
  int d_m[] = {-1, -1};
  int d_p[] = {1, 1};
  ops_dat d_A = ops_decl_dat(block, 1, size, base, d_m, d_p, A, "double", "A");
  ops_dat d_Anew = ops_decl_dat(block, 1, size, base, d_m, d_p, Anew, "double", "Anew");
  int s2d_00[] = {0, 0};
  ops_stencil S2D_00 = ops_decl_stencil(2, 1, s2d_00, "0,0");
  int s2d_5pt[] = {0, 0, 1, 0, -1, 0, 0, 1, 0, -1};
  ops_stencil S2D_5pt = ops_decl_stencil(2, 5, s2d_5pt, "5pt");
  ops_reduction h_err = ops_decl_reduction_handle(sizeof(double), "double", "error");
  ops_decl_const("imax", 1, "int", &imax);
  ops_decl_const("jmax", 1, "int", &jmax);
  ops_decl_const("pi", 1, "double", &pi);
  ops_partition("");

  int full_range[] = {-1, imax + 1, -1, jmax + 1};
  ops_par_loop(set_zero, "set zero", block, 2, full_range,
               ops_arg_dat(d_A, 1, S2D_00, "double", OPS_WRITE));
  ops_par_loop(set_zero, "set zero", block, 2, full_range,
               ops_arg_dat(d_Anew, 1, S2D_00, "double", OPS_WRITE));
  seed_ring(d_A, S2D_00, seed);
  seed_ring(d_Anew, S2D_00, seed);

  double error = 1.0;
  double ct0, ct1, et0, et1;
  ops_timers(&ct0, &et0);
  int interior_range[] = {0, imax, 0, jmax};
  for (int iter = 0; iter < iter_max; iter++) {
    ops_par_loop(apply_stencil, "apply stencil", block, 2, interior_range,
                 ops_arg_dat(d_A, 1, S2D_5pt, "double", OPS_READ),
                 ops_arg_dat(d_Anew, 1, S2D_00, "double", OPS_WRITE),
                 ops_arg_reduce(h_err, 1, "double", OPS_MAX));
    ops_reduction_result(h_err, &error);
    ops_par_loop(copy, "copy", block, 2, interior_range,
                 ops_arg_dat(d_A, 1, S2D_00, "double", OPS_WRITE),
                 ops_arg_dat(d_Anew, 1, S2D_00, "double", OPS_READ));
    printf("iter %d err %.17E\n", iter, error);
  }
  ops_timers(&ct1, &et1);
  printf("wall_seconds %.9f\n", et1 - et0);
  printf("final_error %.17E\n", error);

  if (argc > 5) {
    /* full field, halo included, row-major with x fastest: (imax+2)*(jmax+2) */
    ops_memspace ms = OPS_HOST;
    double *p = (double *)ops_dat_get_raw_pointer(d_A, 0, S2D_00, &ms);
    int disp[OPS_MAX_DIM], sz[OPS_MAX_DIM], stride[OPS_MAX_DIM], dm[OPS_MAX_DIM], dp[OPS_MAX_DIM];
    ops_dat_get_raw_metadata(d_A, 0, disp, sz, stride, dm, dp);
    FILE *f = fopen(argv[5], "wb");
    for (int y = -1; y <= jmax; y++) fwrite(p + (-1) + y * stride[0], sizeof(double), imax + 2, f);
    fclose(f);
    ops_dat_release_raw_data(d_A, 0, OPS_READ);
  }
  ops_exit();
  return 0;
}
