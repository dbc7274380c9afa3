// TeaLeaf 2D implicit heat conduction loop kernels.
//
// Each functor restates one reference kernel with the same operation order
// (apps/c/TeaLeaf/*kernel*.h, cited per functor); compiled with
// --fmad=false the cell updates round like the reference's CPU build. Loop
// names are "tealeaf/<reference kernel name>".
#include <cstddef>

#include "clover_common.h"
#include "runtime.h"

namespace opsb {
namespace tea {

using clover::field_type;
using clover::grid_type;
using clover::kMaxStates;
using clover::state_type;

enum { FIELD_DENSITY = 0, FIELD_ENERGY0, FIELD_ENERGY1, FIELD_U, FIELD_P, FIELD_SD, FIELD_R, FIELD_Z, NUM_FIELDS };

struct Consts {
  field_type field;
  grid_type grid;
  int number_of_states;
  int g_circ, g_point, g_rect;
  state_type states[kMaxStates];
};
__constant__ Consts tc;

using D = ACC2<double>;
using I = ACC2<int>;

#define TL_LOOP(NAME) static constexpr const char *kname = "tealeaf/" #NAME

// ---- initialise_chunk_kernel.h -------------------------------------------
struct initialise_chunk_kernel_zero {  // :8
  TL_LOOP(initialise_chunk_kernel_zero);
  __device__ void operator()(D &var) const { var(0, 0) = 0.0; }
};
struct initialise_chunk_kernel_zero_x {  // :12
  TL_LOOP(initialise_chunk_kernel_zero_x);
  __device__ void operator()(D &var) const { var(0, 0) = 0.0; }
};
struct initialise_chunk_kernel_zero_y {  // :16
  TL_LOOP(initialise_chunk_kernel_zero_y);
  __device__ void operator()(D &var) const { var(0, 0) = 0.0; }
};
struct initialise_chunk_kernel_x {  // :20
  TL_LOOP(initialise_chunk_kernel_x);
  __device__ void operator()(D &vertexx, const I &xx, D &vertexdx) const {
    int x_min = tc.field.x_min - 2;
    double d_x = (tc.grid.xmax - tc.grid.xmin) / (double)tc.grid.x_cells;
    double min_x = tc.grid.xmin + d_x * tc.field.left;
    vertexx(0, 0) = min_x + d_x * (xx(0, 0) - x_min);
    vertexdx(0, 0) = (double)d_x;
  }
};
struct initialise_chunk_kernel_y {  // :32
  TL_LOOP(initialise_chunk_kernel_y);
  __device__ void operator()(D &vertexy, const I &yy, D &vertexdy) const {
    int y_min = tc.field.y_min - 2;
    double d_y = (tc.grid.ymax - tc.grid.ymin) / (double)tc.grid.y_cells;
    double min_y = tc.grid.ymin + d_y * tc.field.bottom;
    vertexy(0, 0) = min_y + d_y * (yy(0, 0) - y_min);
    vertexdy(0, 0) = (double)d_y;
  }
};
struct initialise_chunk_kernel_xx {  // :44
  TL_LOOP(initialise_chunk_kernel_xx);
  __device__ void operator()(I &xx, const IDX &idx) const { xx(0, 0) = idx[0] - 2; }
};
struct initialise_chunk_kernel_yy {  // :48
  TL_LOOP(initialise_chunk_kernel_yy);
  __device__ void operator()(I &yy, const IDX &idx) const { yy(0, 0) = idx[1] - 2; }
};
struct initialise_chunk_kernel_cellx {  // :53
  TL_LOOP(initialise_chunk_kernel_cellx);
  __device__ void operator()(const D &vertexx, D &cellx, D &celldx) const {
    double d_x = (tc.grid.xmax - tc.grid.xmin) / (double)tc.grid.x_cells;
    cellx(0, 0) = 0.5 * (vertexx(0, 0) + vertexx(1, 0));
    celldx(0, 0) = d_x;
  }
};
struct initialise_chunk_kernel_celly {  // :63
  TL_LOOP(initialise_chunk_kernel_celly);
  __device__ void operator()(const D &vertexy, D &celly, D &celldy) const {
    double d_y = (tc.grid.ymax - tc.grid.ymin) / (double)tc.grid.y_cells;
    celly(0, 0) = 0.5 * (vertexy(0, 0) + vertexy(0, 1));
    celldy(0, 0) = d_y;
  }
};
struct initialise_chunk_kernel_volume {  // :75
  TL_LOOP(initialise_chunk_kernel_volume);
  __device__ void operator()(D &volume, const D &celldy, D &xarea, const D &celldx, D &yarea) const {
    double d_x = (tc.grid.xmax - tc.grid.xmin) / (double)tc.grid.x_cells;
    double d_y = (tc.grid.ymax - tc.grid.ymin) / (double)tc.grid.y_cells;
    volume(0, 0) = d_x * d_y;
    xarea(0, 0) = celldy(0, 0);
    yarea(0, 0) = celldx(0, 0);
  }
};

// ---- generate_chunk_kernel.h:9 (rectangles, circles, points) ----------------
struct generate_chunk_kernel {
  TL_LOOP(generate_chunk_kernel);
  __device__ void operator()(const D &vertexx, const D &vertexy, D &energy0, D &density0, D &u0, const D &cellx,
                             const D &celly) const {
    double radius = 0.0, x_cent, y_cent;
    energy0(0, 0) = tc.states[0].energy;
    density0(0, 0) = tc.states[0].density;
    for (int i = 1; i < tc.number_of_states; i++) {
      const state_type &s = tc.states[i];
      x_cent = s.xmin;
      y_cent = s.ymin;
      int is_in2 = 0;
      if (s.geometry == tc.g_rect) {
        if (vertexx(1, 0) >= s.xmin && vertexx(0, 0) < s.xmax)
          if (vertexy(0, 1) >= s.ymin && vertexy(0, 0) < s.ymax) is_in2 = 1;
      } else if (s.geometry == tc.g_circ) {
        for (int i1 = -1; i1 <= 0; i1++)
          for (int j1 = -1; j1 <= 0; j1++)
            radius = sqrt((cellx(i1, 0) - x_cent) * (cellx(i1, 0) - x_cent) +
                          (celly(0, j1) - y_cent) * (celly(0, j1) - y_cent));
        if (radius <= s.radius) is_in2 = 1;
      } else if (s.geometry == tc.g_point) {
        if (vertexx(0, 0) == x_cent && vertexy(0, 0) == y_cent) is_in2 = 1;
      }
      if (is_in2) {
        energy0(0, 0) = s.energy;
        density0(0, 0) = s.density;
      }
    }
    u0(0, 0) = energy0(0, 0) * density0(0, 0);
  }
};

// ---- set_field_kernels.h:4 ----------------------------------------------------
struct set_field_kernel {
  TL_LOOP(set_field_kernel);
  __device__ void operator()(const D &energy0, D &energy1) const { energy1(0, 0) = energy0(0, 0); }
};

// ---- update_halo_kernels.h: reflective copies of the six halo fields ---------
template <int OX, int OY>
struct uh_tea {
  static CopyLoopSpec copy_spec() {
    CopyLoopSpec c;
    c.nfields = 6;
    for (int f = 0; f < 6; f++) c.arg[f] = f, c.flag[f] = FIELD_DENSITY + f;
    c.flags_arg = 6;
    c.off[0] = OX; c.off[1] = OY;
    return c;
  }
  __device__ void operator()(D &density, D &energy0, D &energy1, D &u, D &p, D &sd, const int *fields) const {
    if (fields[FIELD_DENSITY] == 1) density(0, 0) = density(OX, OY);
    if (fields[FIELD_ENERGY0] == 1) energy0(0, 0) = energy0(OX, OY);
    if (fields[FIELD_ENERGY1] == 1) energy1(0, 0) = energy1(OX, OY);
    if (fields[FIELD_U] == 1) u(0, 0) = u(OX, OY);
    if (fields[FIELD_P] == 1) p(0, 0) = p(OX, OY);
    if (fields[FIELD_SD] == 1) sd(0, 0) = sd(OX, OY);
  }
};
#define UH_TEA(NAME, OX, OY)                     \
  struct NAME : uh_tea<OX, OY> { TL_LOOP(NAME); }; \
  OPSB_REGISTER_COPY_LOOP(NAME);
UH_TEA(update_halo_kernel1_b2, 0, 3)
UH_TEA(update_halo_kernel1_b1, 0, 1)
UH_TEA(update_halo_kernel1_t2, 0, -3)
UH_TEA(update_halo_kernel1_t1, 0, -1)
UH_TEA(update_halo_kernel1_l2, 3, 0)
UH_TEA(update_halo_kernel1_l1, 1, 0)
UH_TEA(update_halo_kernel1_r2, -3, 0)
UH_TEA(update_halo_kernel1_r1, -1, 0)

// ---- tea_leaf_common_kernels.h -------------------------------------------------
struct tea_leaf_common_init_u_u0_kernel {  // :7
  TL_LOOP(tea_leaf_common_init_u_u0_kernel);
  __device__ void operator()(D &u, D &u0, const D &energy, const D &density) const {
    u(0, 0) = energy(0, 0) * density(0, 0);
    u0(0, 0) = energy(0, 0) * density(0, 0);
  }
};
struct tea_leaf_common_init_Kx_Ky_kernel {  // :12
  TL_LOOP(tea_leaf_common_init_Kx_Ky_kernel);
  __device__ void operator()(D &Kx, D &Ky, const D &w) const {
    Kx(0, 0) = (w(-1, 0) + w(0, 0)) / (2.0 * w(-1, 0) * w(0, 0));
    Ky(0, 0) = (w(0, -1) + w(0, 0)) / (2.0 * w(0, -1) * w(0, 0));
  }
};
// A u with the 5-point conduction operator (shared by :17, :27, cg_calc_w).
__device__ __forceinline__ double tea_smvp(const D &Kx, const D &Ky, const D &u, double rx, double ry) {
  return (1.0 + ry * (Ky(0, 1) + Ky(0, 0)) + rx * (Kx(1, 0) + Kx(0, 0))) * u(0, 0) -
         ry * (Ky(0, 1) * u(0, 1) + Ky(0, 0) * u(0, -1)) - rx * (Kx(1, 0) * u(1, 0) + Kx(0, 0) * u(-1, 0));
}
struct tea_leaf_common_init_kernel {  // :17
  TL_LOOP(tea_leaf_common_init_kernel);
  __device__ void operator()(D &w, D &r, const D &Kx, const D &Ky, const D &u, const double *rx,
                             const double *ry) const {
    w(0, 0) = tea_smvp(Kx, Ky, u, *rx, *ry);
    r(0, 0) = u(0, 0) - w(0, 0);
  }
};
struct tea_leaf_common_residual_kernel {  // :27
  TL_LOOP(tea_leaf_common_residual_kernel);
  __device__ void operator()(D &r, const D &Kx, const D &Ky, const D &u, const D &u0, const double *rx,
                             const double *ry) const {
    double smvp = 0.0;
    smvp = tea_smvp(Kx, Ky, u, *rx, *ry);
    r(0, 0) = u0(0, 0) - smvp;
  }
};
struct tea_leaf_common_init_diag_init_kernel {  // :38
  TL_LOOP(tea_leaf_common_init_diag_init_kernel);
  __device__ void operator()(D &Mi, const D &Kx, const D &Ky, const double *rx, const double *ry) const {
    Mi(0, 0) = 1.0 / (1.0 + (*ry) * (Ky(0, 1) + Ky(0, 0)) + (*rx) * (Kx(1, 0) + Kx(0, 0)));
  }
};

// ---- tea_leaf_kernels.h ----------------------------------------------------------
struct tea_leaf_init_zero2_kernel {  // :7
  TL_LOOP(tea_leaf_init_zero2_kernel);
  __device__ void operator()(D &p, D &z) const {
    p(0, 0) = 0.0;
    z(0, 0) = 0.0;
  }
};
struct tea_leaf_init_zero_kernel {  // :12
  TL_LOOP(tea_leaf_init_zero_kernel);
  __device__ void operator()(D &p) const { p(0, 0) = 0.0; }
};
struct tea_leaf_yeqx_kernel {  // :16
  TL_LOOP(tea_leaf_yeqx_kernel);
  __device__ void operator()(D &p, const D &x) const { p(0, 0) = x(0, 0); }
};
struct tea_leaf_dot_kernel {  // :22
  TL_LOOP(tea_leaf_dot_kernel);
  __device__ void operator()(const D &r, const D &p, RED<double> &rro) const { *rro = *rro + r(0, 0) * p(0, 0); }
};
struct tea_leaf_axpy_kernel {  // :26
  TL_LOOP(tea_leaf_axpy_kernel);
  __device__ void operator()(D &u, const D &p, const double *alpha) const { u(0, 0) = u(0, 0) + (*alpha) * p(0, 0); }
};
struct tea_leaf_axpby_kernel {  // :34
  TL_LOOP(tea_leaf_axpby_kernel);
  __device__ void operator()(D &u, const D &p, const double *alpha, const double *beta) const {
    u(0, 0) = (*alpha) * u(0, 0) + (*beta) * p(0, 0);
  }
};
struct tea_leaf_zeqxty_kernel {  // :38
  TL_LOOP(tea_leaf_zeqxty_kernel);
  __device__ void operator()(D &z, const D &x, const D &y) const { z(0, 0) = x(0, 0) * y(0, 0); }
};
struct tea_leaf_recip_kernel {  // :42
  TL_LOOP(tea_leaf_recip_kernel);
  __device__ void operator()(D &u, const D &p) const { u(0, 0) = 1.0 / p(0, 0); }
};
struct tea_leaf_recip2_kernel {  // :46
  TL_LOOP(tea_leaf_recip2_kernel);
  __device__ void operator()(D &z, const D &x, const D &y) const { z(0, 0) = x(0, 0) / y(0, 0); }
};
struct tea_leaf_norm2_kernel {  // :54
  TL_LOOP(tea_leaf_norm2_kernel);
  __device__ void operator()(const D &x, RED<double> &norm) const { *norm = *norm + x(0, 0) * x(0, 0); }
};

// ---- tea_leaf_cg_kernels.h -------------------------------------------------------
struct tea_leaf_cg_calc_w_reduce_kernel {  // :8
  TL_LOOP(tea_leaf_cg_calc_w_reduce_kernel);
  __device__ void operator()(D &w, const D &Kx, const D &Ky, const D &p, const double *rx, const double *ry,
                             RED<double> &pw) const {
    w(0, 0) = tea_smvp(Kx, Ky, p, *rx, *ry);
    *pw = *pw + w(0, 0) * p(0, 0);
  }
};
struct tea_leaf_cg_calc_ur_r_reduce_kernel {  // :17
  TL_LOOP(tea_leaf_cg_calc_ur_r_reduce_kernel);
  __device__ void operator()(D &r, const D &w, const double *alpha, RED<double> &rnn) const {
    r(0, 0) = r(0, 0) - (*alpha) * w(0, 0);
    *rnn = *rnn + r(0, 0) * r(0, 0);
  }
};

// ---- tea_leaf_kernels.h:30, :50 (Chebyshev and PPCG helpers) --------------------
struct tea_leaf_xpy_kernel {  // :30
  TL_LOOP(tea_leaf_xpy_kernel);
  __device__ void operator()(D &u, const D &p) const { u(0, 0) = u(0, 0) + p(0, 0); }
};
struct tea_leaf_recip3_kernel {  // :50
  TL_LOOP(tea_leaf_recip3_kernel);
  __device__ void operator()(D &z, const D &x, const double *theta) const { z(0, 0) = x(0, 0) / (*theta); }
};

// ---- tea_leaf_cheby_kernels.h:7 ------------------------------------------------------
struct tea_leaf_cheby_init_kernel {
  TL_LOOP(tea_leaf_cheby_init_kernel);
  __device__ void operator()(D &w, D &r, const D &Kx, const D &Ky, const D &u, const D &u0, const double *rx,
                             const double *ry) const {
    w(0, 0) = tea_smvp(Kx, Ky, u, *rx, *ry);
    r(0, 0) = u0(0, 0) - w(0, 0);
  }
};

// ---- tea_leaf_ppcg_kernels.h ----------------------------------------------------------
struct tea_leaf_ppcg_init1_kernel {  // :7
  TL_LOOP(tea_leaf_ppcg_init1_kernel);
  __device__ void operator()(D &sd, D &rtemp, D &utemp, const D &z, const D &r, const double *theta_r) const {
    sd(0, 0) = z(0, 0) * (*theta_r);
    rtemp(0, 0) = r(0, 0);
    utemp(0, 0) = sd(0, 0);
  }
};
struct tea_leaf_ppcg_init2_kernel {  // :13
  TL_LOOP(tea_leaf_ppcg_init2_kernel);
  __device__ void operator()(D &sd, D &rtemp, D &utemp, const D &r, const double *theta_r) const {
    sd(0, 0) = r(0, 0) * (*theta_r);
    rtemp(0, 0) = r(0, 0);
    utemp(0, 0) = sd(0, 0);
  }
};
struct tea_leaf_ppcg_inner1_kernel {  // :19
  TL_LOOP(tea_leaf_ppcg_inner1_kernel);
  __device__ void operator()(D &rtemp, const D &Kx, const D &Ky, const D &sd, const double *rx,
                             const double *ry) const {
    double smvp = 0.0;
    smvp = tea_smvp(Kx, Ky, sd, *rx, *ry);
    rtemp(0, 0) = rtemp(0, 0) - smvp;
  }
};
struct tea_leaf_ppcg_inner2_kernel {  // :30
  TL_LOOP(tea_leaf_ppcg_inner2_kernel);
  __device__ void operator()(D &sd, D &utemp, const D &z, const double *alpha, const double *beta) const {
    sd(0, 0) = (*alpha) * sd(0, 0) + (*beta) * z(0, 0);
    utemp(0, 0) = utemp(0, 0) + sd(0, 0);
  }
};
struct tea_leaf_ppcg_reduce_kernel {  // :35
  TL_LOOP(tea_leaf_ppcg_reduce_kernel);
  __device__ void operator()(const D &rstore, const D &r, const D &z, RED<double> &rnn) const {
    *rnn = *rnn + (r(0, 0) - rstore(0, 0)) * z(0, 0);
  }
};

// ---- tea_leaf_jacobi_kernels.h:8 ---------------------------------------------------
struct tea_leaf_jacobi_kernel {
  TL_LOOP(tea_leaf_jacobi_kernel);
  __device__ void operator()(D &u1, const D &Kx, const D &Ky, const D &un, const D &u0, const double *rx,
                             const double *ry, RED<double> &error) const {
    u1(0, 0) = (u0(0, 0) + (*rx) * (Kx(1, 0) * un(1, 0) + Kx(0, 0) * un(-1, 0)) +
                (*ry) * (Ky(0, 1) * un(0, 1) + Ky(0, 0) * un(0, -1))) /
               (1.0 + (*rx) * (Kx(1, 0) + Kx(0, 0)) + (*ry) * (Ky(0, 1) + Ky(0, 0)));
    *error = *error + fabs(u1(0, 0) - un(0, 0));
  }
};

// ---- field_summary_kernel.h:4 ---------------------------------------------------------
struct field_summary_kernel {
  TL_LOOP(field_summary_kernel);
  __device__ void operator()(const D &volume, const D &density, const D &energy, const D &u, RED<double> &vol,
                             RED<double> &mass, RED<double> &ie, RED<double> &temp) const {
    double cell_vol = volume(0, 0);
    double cell_mass = cell_vol * density(0, 0);
    *vol = *vol + cell_vol;
    *mass = *mass + cell_mass;
    *ie = *ie + cell_mass * energy(0, 0);
    *temp = *temp + cell_mass * u(0, 0);
  }
};

#define REG(K) OPSB_REGISTER_LOOP(K);
REG(initialise_chunk_kernel_zero) REG(initialise_chunk_kernel_zero_x) REG(initialise_chunk_kernel_zero_y)
REG(initialise_chunk_kernel_x) REG(initialise_chunk_kernel_y) REG(initialise_chunk_kernel_xx)
REG(initialise_chunk_kernel_yy) REG(initialise_chunk_kernel_cellx) REG(initialise_chunk_kernel_celly)
REG(initialise_chunk_kernel_volume) REG(generate_chunk_kernel) REG(set_field_kernel)
REG(update_halo_kernel1_b2) REG(update_halo_kernel1_b1) REG(update_halo_kernel1_t2) REG(update_halo_kernel1_t1)
REG(update_halo_kernel1_l2) REG(update_halo_kernel1_l1) REG(update_halo_kernel1_r2) REG(update_halo_kernel1_r1)
REG(tea_leaf_common_init_u_u0_kernel) REG(tea_leaf_common_init_Kx_Ky_kernel) REG(tea_leaf_common_init_kernel)
REG(tea_leaf_common_residual_kernel) REG(tea_leaf_common_init_diag_init_kernel) REG(tea_leaf_init_zero2_kernel)
REG(tea_leaf_init_zero_kernel) REG(tea_leaf_yeqx_kernel) REG(tea_leaf_dot_kernel) REG(tea_leaf_axpy_kernel)
REG(tea_leaf_axpby_kernel) REG(tea_leaf_zeqxty_kernel) REG(tea_leaf_recip_kernel) REG(tea_leaf_recip2_kernel)
REG(tea_leaf_norm2_kernel) REG(tea_leaf_cg_calc_w_reduce_kernel) REG(tea_leaf_cg_calc_ur_r_reduce_kernel)
REG(tea_leaf_jacobi_kernel) REG(field_summary_kernel) REG(tea_leaf_xpy_kernel) REG(tea_leaf_recip3_kernel)
REG(tea_leaf_cheby_init_kernel) REG(tea_leaf_ppcg_init1_kernel) REG(tea_leaf_ppcg_init2_kernel)
REG(tea_leaf_ppcg_inner1_kernel) REG(tea_leaf_ppcg_inner2_kernel) REG(tea_leaf_ppcg_reduce_kernel)

struct ConstReg {
  ConstReg() {
#define C(name, member) Runtime::register_const("tealeaf/" name, &tc, offsetof(Consts, member), sizeof(Consts::member))
    C("field", field); C("grid", grid); C("number_of_states", number_of_states); C("g_circ", g_circ);
    C("g_point", g_point); C("g_rect", g_rect); C("states", states);
#undef C
  }
};
static ConstReg const_reg;

}  // namespace tea
}  // namespace opsb
