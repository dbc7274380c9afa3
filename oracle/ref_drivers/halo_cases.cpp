// Test infrastructure: drives the reference OPS library's own
// ops_decl_halo / ops_decl_halo_group / ops_halo_transfer
// (ops/c/src/sequential/ops_host_singlenode.cpp:172) on two 2D blocks and
// writes both dats (full extent, x fastest) after each halo group, so that the
// B200 implementation can be compared with the reference bit for bit.
//
// Cases (one per group, each starting from freshly filled dats): matching
// orientation across x and across y, the second block flipped in y and in x,
// x and y swapped, and a double -> float exchange (mixed precision).
// usage: halo_cases <out_dir>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define OPS_2D
#include "ops_seq_v2.h"

static void fill_d(ACC<double> &v, const int *idx, const double *tag) {
  v(0, 0) = *tag + 100.0 * idx[0] + idx[1] + 0.25;
}
static void fill_f(ACC<float> &v, const int *idx, const double *tag) {
  v(0, 0) = (float)(*tag + 100.0 * idx[0] + idx[1] + 0.5);
}

static void dump(ops_dat d, const char *dir, int c, const char *tag) {
  char path[512];
  snprintf(path, sizeof(path), "%s/case%d_%s.bin", dir, c, tag);
  FILE *f = fopen(path, "wb");
  if (!f) exit(2);
  const int nx = d->size[0], ny = d->size[1];
  fwrite(&nx, 4, 1, f);
  fwrite(&ny, 4, 1, f);
  fwrite(d->data, d->elem_size, (size_t)nx * ny, f);
  fclose(f);
}

int main(int argc, char **argv) {
  if (argc < 2) return 1;
  const char *out = argv[1];
  ops_init(1, argv, 1);
  ops_block g0 = ops_decl_block(2, "g0");
  ops_block g1 = ops_decl_block(2, "g1");
  int s0[] = {0, 0};
  ops_stencil S0 = ops_decl_stencil(2, 1, s0, "00");
  int size[] = {20, 20}, base[] = {0, 0}, dm[] = {-2, -2}, dp[] = {2, 2};
  double *nil = NULL;
  float *nilf = NULL;
  ops_dat a = ops_decl_dat(g0, 1, size, base, dm, dp, nil, "double", "a");
  ops_dat b = ops_decl_dat(g1, 1, size, base, dm, dp, nil, "double", "b");
  ops_dat bf = ops_decl_dat(g1, 1, size, base, dm, dp, nilf, "float", "bf");
  int rng[] = {0, 20, 0, 20};

  // {iter, from_base, to_base, from_dir, to_dir} for the a -> b halo and the b -> a halo of each case
  struct H { int it[2], fb[2], tb[2], fd[2], td[2]; };
  const H cases[6][2] = {
      {{{2, 20}, {18, 0}, {-2, 0}, {1, 2}, {1, 2}}, {{2, 20}, {0, 0}, {20, 0}, {1, 2}, {1, 2}}},
      {{{20, 2}, {0, 18}, {0, -2}, {1, 2}, {1, 2}}, {{20, 2}, {0, 0}, {0, 20}, {1, 2}, {1, 2}}},
      {{{2, 20}, {0, 0}, {20, 0}, {1, 2}, {1, -2}}, {{2, 20}, {18, 0}, {-2, 0}, {1, -2}, {1, 2}}},
      {{{20, 2}, {0, 0}, {0, 20}, {1, 2}, {-1, 2}}, {{20, 2}, {0, 18}, {0, -2}, {-1, 2}, {1, 2}}},
      {{{2, 20}, {18, 0}, {0, -2}, {1, 2}, {2, 1}}, {{2, 20}, {0, 0}, {20, 0}, {2, 1}, {1, 2}}},
      {{{3, 20}, {17, 0}, {-2, 0}, {1, 2}, {1, 2}}, {{0, 0}, {0, 0}, {0, 0}, {0, 0}, {0, 0}}},
  };
  for (int c = 0; c < 6; c++) {
    const double ta = 10000.0, tb = 20000.0;
    ops_par_loop(fill_d, "fill", g0, 2, rng, ops_arg_dat(a, 1, S0, "double", OPS_WRITE), ops_arg_idx(),
                 ops_arg_gbl(&ta, 1, "double", OPS_READ));
    ops_par_loop(fill_d, "fill", g1, 2, rng, ops_arg_dat(b, 1, S0, "double", OPS_WRITE), ops_arg_idx(),
                 ops_arg_gbl(&tb, 1, "double", OPS_READ));
    ops_par_loop(fill_f, "fill", g1, 2, rng, ops_arg_dat(bf, 1, S0, "float", OPS_WRITE), ops_arg_idx(),
                 ops_arg_gbl(&tb, 1, "double", OPS_READ));
    ops_halo hs[2];
    int nh = 0;
    if (c < 5) {
      H h0 = cases[c][0], h1 = cases[c][1];
      hs[nh++] = ops_decl_halo(a, b, h0.it, h0.fb, h0.tb, h0.fd, h0.td);
      hs[nh++] = ops_decl_halo(b, a, h1.it, h1.fb, h1.tb, h1.fd, h1.td);
    } else {
      H h0 = cases[c][0];
      hs[nh++] = ops_decl_halo(a, bf, h0.it, h0.fb, h0.tb, h0.fd, h0.td);
    }
    ops_halo_group grp = ops_decl_halo_group(nh, hs);
    ops_halo_transfer(grp);
    ops_execute();
    dump(a, out, c, "a");
    dump(b, out, c, "b");
    dump(bf, out, c, "bf");
  }
  ops_exit();
  printf("halo cases written\n");
  return 0;
}
