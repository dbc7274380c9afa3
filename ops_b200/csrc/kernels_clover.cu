// CloverLeaf 2D hydro loop kernels (compressible Euler, Lagrangian step plus
// advective remap; ideal gas, gamma = 1.4).
//
// Each functor restates one reference kernel with the same operation order
// (apps/c/CloverLeaf/*_kernel.h, cited per functor); with --fmad=false the
// cell updates round exactly like the reference's x86-64 CPU build.
// Divisions whose numerator is often exactly zero (velocities, fluxes and
// viscosity of quiescent regions) go through qdiv, which returns the same
// IEEE quotient without the division for a zero numerator, and the
// advection limiter's cell-width ratio through qratio (exactly 1 for equal
// widths). Loop names are "cloverleaf/<reference kernel name>".
#include <cstddef>

#include "clover_common.h"
#include "fused_exec.cuh"
#include "runtime.h"

namespace opsb {
namespace clover {

__constant__ Consts cc;

using D = ACC2<double>;
using I = ACC2<int>;

#define CL_LOOP(NAME) static constexpr const char *kname = "cloverleaf/" #NAME
// Resident CTAs per SM (register budget) where the default of 8 (32
// registers) spills more than the extra occupancy gains; measured per
// kernel on the 3840^2 deck.

// ---- initialise_chunk_kernel.h -------------------------------------------
struct initialise_chunk_kernel_xx {  // :30
  CL_LOOP(initialise_chunk_kernel_xx);
  __device__ void operator()(I &xx, const IDX &idx) const { xx(0, 0) = idx[0] - 2; }
};
struct initialise_chunk_kernel_yy {  // :34
  CL_LOOP(initialise_chunk_kernel_yy);
  __device__ void operator()(I &yy, const IDX &idx) const { yy(0, 0) = idx[1] - 2; }
};
struct initialise_chunk_kernel_x {  // :7
  CL_LOOP(initialise_chunk_kernel_x);
  __device__ void operator()(D &vertexx, const I &xx, D &vertexdx) const {
    int x_min = cc.field.x_min - 2;
    double d_x = (cc.grid.xmax - cc.grid.xmin) / (double)cc.grid.x_cells;
    double min_x = cc.grid.xmin + d_x * cc.field.left;
    vertexx(0, 0) = min_x + d_x * (xx(0, 0) - x_min);
    vertexdx(0, 0) = (double)d_x;
  }
};
struct initialise_chunk_kernel_y {  // :19
  CL_LOOP(initialise_chunk_kernel_y);
  __device__ void operator()(D &vertexy, const I &yy, D &vertexdy) const {
    int y_min = cc.field.y_min - 2;
    double d_y = (cc.grid.ymax - cc.grid.ymin) / (double)cc.grid.y_cells;
    double min_y = cc.grid.ymin + d_y * cc.field.bottom;
    vertexy(0, 0) = min_y + d_y * (yy(0, 0) - y_min);
    vertexdy(0, 0) = (double)d_y;
  }
};
struct initialise_chunk_kernel_cellx {  // :39
  CL_LOOP(initialise_chunk_kernel_cellx);
  __device__ void operator()(const D &vertexx, D &cellx, D &celldx) const {
    double d_x = (cc.grid.xmax - cc.grid.xmin) / (double)cc.grid.x_cells;
    cellx(0, 0) = 0.5 * (vertexx(0, 0) + vertexx(1, 0));
    celldx(0, 0) = d_x;
  }
};
struct initialise_chunk_kernel_celly {  // :49
  CL_LOOP(initialise_chunk_kernel_celly);
  __device__ void operator()(const D &vertexy, D &celly, D &celldy) const {
    double d_y = (cc.grid.ymax - cc.grid.ymin) / (double)cc.grid.y_cells;
    celly(0, 0) = 0.5 * (vertexy(0, 0) + vertexy(0, 1));
    celldy(0, 0) = d_y;
  }
};
struct initialise_chunk_kernel_volume {  // :61
  CL_LOOP(initialise_chunk_kernel_volume);
  __device__ void operator()(D &volume, const D &celldy, D &xarea, const D &celldx, D &yarea) const {
    double d_x = (cc.grid.xmax - cc.grid.xmin) / (double)cc.grid.x_cells;
    double d_y = (cc.grid.ymax - cc.grid.ymin) / (double)cc.grid.y_cells;
    volume(0, 0) = d_x * d_y;
    xarea(0, 0) = celldy(0, 0);
    yarea(0, 0) = celldx(0, 0);
  }
};

// ---- generate_chunk_kernel.h:9 ---------------------------------------------
struct generate_chunk_kernel {
  CL_LOOP(generate_chunk_kernel);
  __device__ void operator()(const D &vertexx, const D &vertexy, D &energy0, D &density0, D &xvel0, D &yvel0,
                             const D &cellx, const D &celly) const {
    double radius = 0.0, x_cent, y_cent;
    energy0(0, 0) = cc.states[0].energy;
    density0(0, 0) = cc.states[0].density;
    xvel0(0, 0) = cc.states[0].xvel;
    yvel0(0, 0) = cc.states[0].yvel;
    for (int i = 1; i < cc.number_of_states; i++) {
      const state_type &s = cc.states[i];
      x_cent = s.xmin;
      y_cent = s.ymin;
      int is_in = 0, is_in2 = 0;
      if (s.geometry == cc.g_rect) {
        for (int i1 = -1; i1 <= 0; i1++)
          for (int j1 = -1; j1 <= 0; j1++)
            if (vertexx(1 + i1, 0) >= s.xmin && vertexx(0 + i1, 0) < s.xmax)
              if (vertexy(0, 1 + j1) >= s.ymin && vertexy(0, 0 + j1) < s.ymax) is_in = 1;
        if (vertexx(1, 0) >= s.xmin && vertexx(0, 0) < s.xmax)
          if (vertexy(0, 1) >= s.ymin && vertexy(0, 0) < s.ymax) is_in2 = 1;
      } else if (s.geometry == cc.g_circ) {
        for (int i1 = -1; i1 <= 0; i1++)
          for (int j1 = -1; j1 <= 0; j1++) {
            radius = sqrt((cellx(i1, 0) - x_cent) * (cellx(i1, 0) - x_cent) +
                          (celly(0, j1) - y_cent) * (celly(0, j1) - y_cent));
            if (radius <= s.radius) is_in = 1;
          }
        if (radius <= s.radius) is_in2 = 1;
      } else if (s.geometry == cc.g_point) {
        for (int i1 = -1; i1 <= 0; i1++)
          for (int j1 = -1; j1 <= 0; j1++)
            if (vertexx(i1, 0) == x_cent && vertexy(0, j1) == y_cent) is_in = 1;
        if (vertexx(0, 0) == x_cent && vertexy(0, 0) == y_cent) is_in2 = 1;
      } else {
        continue;
      }
      if (is_in2) {
        energy0(0, 0) = s.energy;
        density0(0, 0) = s.density;
      }
      if (is_in) {
        xvel0(0, 0) = s.xvel;
        yvel0(0, 0) = s.yvel;
      }
    }
  }
};

// ---- ideal_gas_kernel.h:4 ----------------------------------------------------
struct ideal_gas_kernel {
  CL_LOOP(ideal_gas_kernel);
  static constexpr bool touch_next_row = true;
  __device__ void operator()(const D &density, const D &energy, D &pressure, D &soundspeed) const {
    double v = 1.0 / density(0, 0);
    pressure(0, 0) = (1.4 - 1.0) * density(0, 0) * energy(0, 0);
    double pressurebyenergy = (1.4 - 1.0) * density(0, 0);
    double pressurebyvolume = -1 * density(0, 0) * pressure(0, 0);
    double sound_speed_squared = v * v * (pressure(0, 0) * pressurebyenergy - pressurebyvolume);
    soundspeed(0, 0) = sqrt(sound_speed_squared);
  }
};

// ---- update_halo_kernel.h: reflective boundary copies ------------------------
// kernel1_{b2,b1,t2,t1,l2,l1,r2,r1} (:6-119): the seven cell-centred fields
// copy from (OX, OY) when their flag is set.
template <int OX, int OY>
struct uh_cells {
  static CopyLoopSpec copy_spec() {
    CopyLoopSpec c;
    c.nfields = 7;
    for (int f = 0; f < 7; f++) c.arg[f] = f, c.flag[f] = FIELD_DENSITY0 + f;
    c.flags_arg = 7;
    c.off[0] = OX; c.off[1] = OY;
    return c;
  }
  __device__ void operator()(D &density0, D &density1, D &energy0, D &energy1, D &pressure, D &viscosity,
                             D &soundspeed, const int *fields) const {
    if (fields[FIELD_DENSITY0] == 1) density0(0, 0) = density0(OX, OY);
    if (fields[FIELD_DENSITY1] == 1) density1(0, 0) = density1(OX, OY);
    if (fields[FIELD_ENERGY0] == 1) energy0(0, 0) = energy0(OX, OY);
    if (fields[FIELD_ENERGY1] == 1) energy1(0, 0) = energy1(OX, OY);
    if (fields[FIELD_PRESSURE] == 1) pressure(0, 0) = pressure(OX, OY);
    if (fields[FIELD_VISCOSITY] == 1) viscosity(0, 0) = viscosity(OX, OY);
    if (fields[FIELD_SOUNDSPEED] == 1) soundspeed(0, 0) = soundspeed(OX, OY);
  }
};
// kernel2/3/4 (:121-305): a pair of face/vertex fields copies (or negates)
// from (OX, OY) when flag F0 / F1 is set.
template <int OX, int OY, int NEG, int F0, int F1>
struct uh_pair {
  static CopyLoopSpec copy_spec() {
    CopyLoopSpec c;
    c.nfields = 2;
    c.arg[0] = 0; c.arg[1] = 1; c.flag[0] = F0; c.flag[1] = F1;
    c.flags_arg = 2;
    c.neg = NEG;
    c.off[0] = OX; c.off[1] = OY;
    return c;
  }
  __device__ void operator()(D &a, D &b, const int *fields) const {
    if (fields[F0] == 1) a(0, 0) = NEG ? -a(OX, OY) : a(OX, OY);
    if (fields[F1] == 1) b(0, 0) = NEG ? -b(OX, OY) : b(OX, OY);
  }
};

#define UH_CELLS(NAME, OX, OY)                     \
  struct NAME : uh_cells<OX, OY> { CL_LOOP(NAME); }; \
  OPSB_REGISTER_COPY_LOOP(NAME);
#define UH_PAIR(NAME, OX, OY, NEG, F0, F1)                     \
  struct NAME : uh_pair<OX, OY, NEG, F0, F1> { CL_LOOP(NAME); }; \
  OPSB_REGISTER_COPY_LOOP(NAME);

UH_CELLS(update_halo_kernel1_b2, 0, 3)
UH_CELLS(update_halo_kernel1_b1, 0, 1)
UH_CELLS(update_halo_kernel1_t2, 0, -3)
UH_CELLS(update_halo_kernel1_t1, 0, -1)
UH_CELLS(update_halo_kernel1_l2, 3, 0)
UH_CELLS(update_halo_kernel1_l1, 1, 0)
UH_CELLS(update_halo_kernel1_r2, -3, 0)
UH_CELLS(update_halo_kernel1_r1, -1, 0)

UH_PAIR(update_halo_kernel2_xvel_plus_4_a, 0, 4, 0, FIELD_XVEL0, FIELD_XVEL1)
UH_PAIR(update_halo_kernel2_xvel_plus_2_a, 0, 2, 0, FIELD_XVEL0, FIELD_XVEL1)
UH_PAIR(update_halo_kernel2_xvel_plus_4_b, 0, -4, 0, FIELD_XVEL0, FIELD_XVEL1)
UH_PAIR(update_halo_kernel2_xvel_plus_2_b, 0, -2, 0, FIELD_XVEL0, FIELD_XVEL1)
UH_PAIR(update_halo_kernel2_xvel_minus_4_a, 4, 0, 1, FIELD_XVEL0, FIELD_XVEL1)
UH_PAIR(update_halo_kernel2_xvel_minus_2_a, 2, 0, 1, FIELD_XVEL0, FIELD_XVEL1)
UH_PAIR(update_halo_kernel2_xvel_minus_4_b, -4, 0, 1, FIELD_XVEL0, FIELD_XVEL1)
UH_PAIR(update_halo_kernel2_xvel_minus_2_b, -2, 0, 1, FIELD_XVEL0, FIELD_XVEL1)

UH_PAIR(update_halo_kernel2_yvel_plus_4_a, 4, 0, 0, FIELD_YVEL0, FIELD_YVEL1)
UH_PAIR(update_halo_kernel2_yvel_plus_2_a, 2, 0, 0, FIELD_YVEL0, FIELD_YVEL1)
UH_PAIR(update_halo_kernel2_yvel_plus_4_b, -4, 0, 0, FIELD_YVEL0, FIELD_YVEL1)
UH_PAIR(update_halo_kernel2_yvel_plus_2_b, -2, 0, 0, FIELD_YVEL0, FIELD_YVEL1)
UH_PAIR(update_halo_kernel2_yvel_minus_4_a, 0, 4, 1, FIELD_YVEL0, FIELD_YVEL1)
UH_PAIR(update_halo_kernel2_yvel_minus_2_a, 0, 2, 1, FIELD_YVEL0, FIELD_YVEL1)
UH_PAIR(update_halo_kernel2_yvel_minus_4_b, 0, -4, 1, FIELD_YVEL0, FIELD_YVEL1)
UH_PAIR(update_halo_kernel2_yvel_minus_2_b, 0, -2, 1, FIELD_YVEL0, FIELD_YVEL1)

UH_PAIR(update_halo_kernel3_plus_4_a, 0, 4, 0, FIELD_VOL_FLUX_X, FIELD_MASS_FLUX_X)
UH_PAIR(update_halo_kernel3_plus_2_a, 0, 2, 0, FIELD_VOL_FLUX_X, FIELD_MASS_FLUX_X)
UH_PAIR(update_halo_kernel3_plus_4_b, 0, -4, 0, FIELD_VOL_FLUX_X, FIELD_MASS_FLUX_X)
UH_PAIR(update_halo_kernel3_plus_2_b, 0, -2, 0, FIELD_VOL_FLUX_X, FIELD_MASS_FLUX_X)
UH_PAIR(update_halo_kernel3_minus_4_a, 4, 0, 1, FIELD_VOL_FLUX_X, FIELD_MASS_FLUX_X)
UH_PAIR(update_halo_kernel3_minus_2_a, 2, 0, 1, FIELD_VOL_FLUX_X, FIELD_MASS_FLUX_X)
UH_PAIR(update_halo_kernel3_minus_4_b, -4, 0, 1, FIELD_VOL_FLUX_X, FIELD_MASS_FLUX_X)
UH_PAIR(update_halo_kernel3_minus_2_b, -2, 0, 1, FIELD_VOL_FLUX_X, FIELD_MASS_FLUX_X)

UH_PAIR(update_halo_kernel4_plus_4_a, 4, 0, 0, FIELD_VOL_FLUX_Y, FIELD_MASS_FLUX_Y)
UH_PAIR(update_halo_kernel4_plus_2_a, 2, 0, 0, FIELD_VOL_FLUX_Y, FIELD_MASS_FLUX_Y)
UH_PAIR(update_halo_kernel4_plus_4_b, -4, 0, 0, FIELD_VOL_FLUX_Y, FIELD_MASS_FLUX_Y)
UH_PAIR(update_halo_kernel4_plus_2_b, -2, 0, 0, FIELD_VOL_FLUX_Y, FIELD_MASS_FLUX_Y)
UH_PAIR(update_halo_kernel4_minus_4_a, 0, 4, 1, FIELD_VOL_FLUX_Y, FIELD_MASS_FLUX_Y)
UH_PAIR(update_halo_kernel4_minus_2_a, 0, 2, 1, FIELD_VOL_FLUX_Y, FIELD_MASS_FLUX_Y)
UH_PAIR(update_halo_kernel4_minus_4_b, 0, -4, 1, FIELD_VOL_FLUX_Y, FIELD_MASS_FLUX_Y)
UH_PAIR(update_halo_kernel4_minus_2_b, 0, -2, 1, FIELD_VOL_FLUX_Y, FIELD_MASS_FLUX_Y)

// ---- viscosity_kernel.h:5 ----------------------------------------------------
struct viscosity_kernel {
  CL_LOOP(viscosity_kernel);
  __device__ void operator()(const D &xvel0, const D &yvel0, const D &celldx, const D &celldy, const D &pressure,
                             const D &density0, D &viscosity) const {
    double ugrad = (xvel0(1, 0) + xvel0(1, 1)) - (xvel0(0, 0) + xvel0(0, 1));
    double vgrad = (yvel0(0, 1) + yvel0(1, 1)) - (yvel0(0, 0) + yvel0(1, 0));
    double div = (celldx(0, 0)) * (ugrad) + (celldy(0, 0)) * (vgrad);
    // qdiv: the same quotients; exactly zero numerators (uniform regions)
    // take the product path
    double strain2 = qdiv(0.5 * (xvel0(0, 1) + xvel0(1, 1) - xvel0(0, 0) - xvel0(1, 0)), (celldy(0, 0))) +
                     qdiv(0.5 * (yvel0(1, 0) + yvel0(1, 1) - yvel0(0, 0) - yvel0(0, 1)), (celldx(0, 0)));
    double pgradx = qdiv(pressure(1, 0) - pressure(-1, 0), celldx(0, 0) + celldx(1, 0));
    double pgrady = qdiv(pressure(0, 1) - pressure(0, -1), celldy(0, 0) + celldy(0, 1));
    double pgradx2 = pgradx * pgradx;
    double pgrady2 = pgrady * pgrady;
    double limiter = qdiv(qdiv(0.5 * (ugrad), celldx(0, 0)) * pgradx2 + qdiv(0.5 * (vgrad), celldy(0, 0)) * pgrady2 +
                              strain2 * pgradx * pgrady,
                          op_max(pgradx2 + pgrady2, 1.0e-16));
    if ((limiter > 0.0) || (div >= 0.0)) {
      viscosity(0, 0) = 0.0;
    } else {
      pgradx = op_sign(op_max(1.0e-16, fabs(pgradx)), pgradx);
      pgrady = op_sign(op_max(1.0e-16, fabs(pgrady)), pgrady);
      double pgrad = sqrt(pgradx * pgradx + pgrady * pgrady);
      double xgrad = fabs(celldx(0, 0) * pgrad / pgradx);
      double ygrad = fabs(celldy(0, 0) * pgrad / pgrady);
      double grad = op_min(xgrad, ygrad);
      double grad2 = grad * grad;
      viscosity(0, 0) = 2.0 * (density0(0, 0)) * grad2 * limiter * limiter;
    }
  }
};

// ---- calc_dt_kernel.h --------------------------------------------------------
struct calc_dt_kernel {  // :7
  CL_LOOP(calc_dt_kernel);
  __device__ void operator()(const D &celldx, const D &celldy, const D &soundspeed, const D &viscosity,
                             const D &density0, const D &xvel0, const D &xarea, const D &volume, const D &yvel0,
                             const D &yarea, D &dt_min) const {
    double dsx = celldx(0, 0);
    double dsy = celldy(0, 0);
    double cc2 = soundspeed(0, 0) * soundspeed(0, 0);
    cc2 = cc2 + qdiv(2.0 * viscosity(0, 0), density0(0, 0));
    cc2 = op_max(sqrt(cc2), cc.g_small);
    double dtct = cc.dtc_safe * op_min(dsx, dsy) / cc2;
    double div = 0.0;
    double dv1 = (xvel0(0, 0) + xvel0(0, 1)) * xarea(0, 0);
    double dv2 = (xvel0(1, 0) + xvel0(1, 1)) * xarea(1, 0);
    div = div + dv2 - dv1;
    double dtut = cc.dtu_safe * 2.0 * volume(0, 0) / op_max(op_max(fabs(dv1), fabs(dv2)), cc.g_small * volume(0, 0));
    dv1 = (yvel0(0, 0) + yvel0(1, 0)) * yarea(0, 0);
    dv2 = (yvel0(0, 1) + yvel0(1, 1)) * yarea(0, 1);
    div = div + dv2 - dv1;
    double dtvt = cc.dtv_safe * 2.0 * volume(0, 0) / op_max(op_max(fabs(dv1), fabs(dv2)), cc.g_small * volume(0, 0));
    div = qdiv(div, 2.0 * volume(0, 0));
    double dtdivt;
    if (div < -cc.g_small)
      dtdivt = cc.dtdiv_safe * (-1.0 / div);
    else
      dtdivt = cc.g_big;
    dt_min(0, 0) = op_min(op_min(dtct, dtut), op_min(dtvt, dtdivt));
  }
};
struct calc_dt_kernel_min {  // :55
  CL_LOOP(calc_dt_kernel_min);
  __device__ void operator()(const D &dt_min, RED<double> &dt_min_val) const {
    *dt_min_val = op_min(*dt_min_val, dt_min(0, 0));
  }
};
struct calc_dt_kernel_get {  // :61
  CL_LOOP(calc_dt_kernel_get);
  __device__ void operator()(const D &cellx, const D &celly, RED<double> &xl_pos, RED<double> &yl_pos) const {
    *xl_pos = cellx(0, 0);
    *yl_pos = celly(0, 0);
  }
};
struct calc_dt_kernel_print {  // :74
  CL_LOOP(calc_dt_kernel_print);
  __device__ void operator()(const D &xvel0, const D &yvel0, const D &density0, const D &energy0, const D &pressure,
                             const D &soundspeed, RED<double, 12> &output) const {
    output[0] = xvel0(1, 0);
    output[1] = yvel0(1, 0);
    output[2] = xvel0(-1, 0);
    output[3] = yvel0(-1, 0);
    output[4] = xvel0(0, 1);
    output[5] = yvel0(0, 1);
    output[6] = xvel0(0, -1);
    output[7] = yvel0(0, -1);
    output[8] = density0(0, 0);
    output[9] = energy0(0, 0);
    output[10] = pressure(0, 0);
    output[11] = soundspeed(0, 0);
  }
};

// ---- PdV_kernel.h ------------------------------------------------------------
struct PdV_kernel_predict {  // :7
  CL_LOOP(PdV_kernel_predict);
  __device__ void operator()(const D &xarea, const D &xvel0, const D &yarea, const D &yvel0, D &volume_change,
                             const D &volume, const D &pressure, const D &density0, D &density1,
                             const D &viscosity, const D &energy0, D &energy1) const {
    const double dt = cc.dt;
    double left_flux = (xarea(0, 0) * (xvel0(0, 0) + xvel0(0, 1) + xvel0(0, 0) + xvel0(0, 1))) * 0.25 * dt * 0.5;
    double right_flux = (xarea(1, 0) * (xvel0(1, 0) + xvel0(1, 1) + xvel0(1, 0) + xvel0(1, 1))) * 0.25 * dt * 0.5;
    double bottom_flux = (yarea(0, 0) * (yvel0(0, 0) + yvel0(1, 0) + yvel0(0, 0) + yvel0(1, 0))) * 0.25 * dt * 0.5;
    double top_flux = (yarea(0, 1) * (yvel0(0, 1) + yvel0(1, 1) + yvel0(0, 1) + yvel0(1, 1))) * 0.25 * dt * 0.5;
    double total_flux = right_flux - left_flux + top_flux - bottom_flux;
    volume_change(0, 0) = (volume(0, 0)) / (volume(0, 0) + total_flux);
    double recip_volume = 1.0 / volume(0, 0);
    double energy_change = (pressure(0, 0) / density0(0, 0) + qdiv(viscosity(0, 0), density0(0, 0))) * total_flux * recip_volume;
    energy1(0, 0) = energy0(0, 0) - energy_change;
    density1(0, 0) = density0(0, 0) * volume_change(0, 0);
  }
};
struct PdV_kernel_nopredict {  // :45
  CL_LOOP(PdV_kernel_nopredict);
  static constexpr int min_blocks = 6;
  __device__ void operator()(const D &xarea, const D &xvel0, const D &xvel1, const D &yarea, const D &yvel0,
                             const D &yvel1, D &volume_change, const D &volume, const D &pressure,
                             const D &density0, D &density1, const D &viscosity, const D &energy0,
                             D &energy1) const {
    const double dt = cc.dt;
    double left_flux = (xarea(0, 0) * (xvel0(0, 0) + xvel0(0, 1) + xvel1(0, 0) + xvel1(0, 1))) * 0.25 * dt;
    double right_flux = (xarea(1, 0) * (xvel0(1, 0) + xvel0(1, 1) + xvel1(1, 0) + xvel1(1, 1))) * 0.25 * dt;
    double bottom_flux = (yarea(0, 0) * (yvel0(0, 0) + yvel0(1, 0) + yvel1(0, 0) + yvel1(1, 0))) * 0.25 * dt;
    double top_flux = (yarea(0, 1) * (yvel0(0, 1) + yvel0(1, 1) + yvel1(0, 1) + yvel1(1, 1))) * 0.25 * dt;
    double total_flux = right_flux - left_flux + top_flux - bottom_flux;
    volume_change(0, 0) = (volume(0, 0)) / (volume(0, 0) + total_flux);
    double recip_volume = 1.0 / volume(0, 0);
    double energy_change = (pressure(0, 0) / density0(0, 0) + qdiv(viscosity(0, 0), density0(0, 0))) * total_flux * recip_volume;
    energy1(0, 0) = energy0(0, 0) - energy_change;
    density1(0, 0) = density0(0, 0) * volume_change(0, 0);
  }
};

// ---- revert_kernel.h:5 -------------------------------------------------------
struct revert_kernel {
  CL_LOOP(revert_kernel);
  __device__ void operator()(const D &density0, D &density1, const D &energy0, D &energy1) const {
    density1(0, 0) = density0(0, 0);
    energy1(0, 0) = energy0(0, 0);
  }
};

// ---- accelerate_kernel.h:8 ---------------------------------------------------
struct accelerate_kernel {
  CL_LOOP(accelerate_kernel);
  static constexpr bool touch_next_row = true;
  static constexpr int min_blocks = 4;
  __device__ void operator()(const D &density0, const D &volume, D &stepbymass, const D &xvel0, D &xvel1,
                             const D &xarea, const D &pressure, const D &yvel0, D &yvel1, const D &yarea,
                             const D &viscosity) const {
    double nodal_mass = (density0(-1, -1) * volume(-1, -1) + density0(0, -1) * volume(0, -1) +
                         density0(0, 0) * volume(0, 0) + density0(-1, 0) * volume(-1, 0)) *
                        0.25;
    stepbymass(0, 0) = 0.5 * cc.dt / nodal_mass;
    xvel1(0, 0) = xvel0(0, 0) - stepbymass(0, 0) * (xarea(0, 0) * (pressure(0, 0) - pressure(-1, 0)) +
                                                    xarea(0, -1) * (pressure(0, -1) - pressure(-1, -1)));
    yvel1(0, 0) = yvel0(0, 0) - stepbymass(0, 0) * (yarea(0, 0) * (pressure(0, 0) - pressure(0, -1)) +
                                                    yarea(-1, 0) * (pressure(-1, 0) - pressure(-1, -1)));
    xvel1(0, 0) = xvel1(0, 0) - stepbymass(0, 0) * (xarea(0, 0) * (viscosity(0, 0) - viscosity(-1, 0)) +
                                                    xarea(0, -1) * (viscosity(0, -1) - viscosity(-1, -1)));
    yvel1(0, 0) = yvel1(0, 0) - stepbymass(0, 0) * (yarea(0, 0) * (viscosity(0, 0) - viscosity(0, -1)) +
                                                    yarea(-1, 0) * (viscosity(-1, 0) - viscosity(-1, -1)));
  }
};

// ---- flux_calc_kernel.h ------------------------------------------------------
struct flux_calc_kernelx {  // :4
  CL_LOOP(flux_calc_kernelx);
  __device__ void operator()(D &vol_flux_x, const D &xarea, const D &xvel0, const D &xvel1) const {
    vol_flux_x(0, 0) = 0.25 * cc.dt * (xarea(0, 0)) * ((xvel0(0, 0)) + (xvel0(0, 1)) + (xvel1(0, 0)) + (xvel1(0, 1)));
  }
};
struct flux_calc_kernely {  // :12
  CL_LOOP(flux_calc_kernely);
  __device__ void operator()(D &vol_flux_y, const D &yarea, const D &yvel0, const D &yvel1) const {
    vol_flux_y(0, 0) = 0.25 * cc.dt * (yarea(0, 0)) * ((yvel0(0, 0)) + (yvel0(1, 0)) + (yvel1(0, 0)) + (yvel1(1, 0)));
  }
};

// ---- advec_cell_kernel.h -----------------------------------------------------
struct advec_cell_kernel1_xdir {  // :7
  CL_LOOP(advec_cell_kernel1_xdir);
  __device__ void operator()(D &pre_vol, D &post_vol, const D &volume, const D &vol_flux_x, const D &vol_flux_y) const {
    pre_vol(0, 0) = volume(0, 0) + (vol_flux_x(1, 0) - vol_flux_x(0, 0) + vol_flux_y(0, 1) - vol_flux_y(0, 0));
    post_vol(0, 0) = pre_vol(0, 0) - (vol_flux_x(1, 0) - vol_flux_x(0, 0));
  }
};
struct advec_cell_kernel2_xdir {  // :19
  CL_LOOP(advec_cell_kernel2_xdir);
  __device__ void operator()(D &pre_vol, D &post_vol, const D &volume, const D &vol_flux_x) const {
    pre_vol(0, 0) = volume(0, 0) + vol_flux_x(1, 0) - vol_flux_x(0, 0);
    post_vol(0, 0) = volume(0, 0);
  }
};

// The donor-cell / van Leer flux of advec_cell_kernel3_{x,y}dir (:28, :133),
// written once over a 1D view along the sweep direction: V(k) is the value k
// cells away along the sweep.
template <class View>
__device__ __forceinline__ void advec_cell_flux(double vol_flux, const View &pre_vol, int cell_max_test,
                                                const View &vertexd, const View &density1, const View &energy1,
                                                double &mass_flux, double &ener_flux) {
  const double one_by_six = 1.0 / 6.0;
  int upwind, donor, downwind, dif;
  if (vol_flux > 0.0) {
    upwind = -2; donor = -1; downwind = 0; dif = donor;
  } else if (cell_max_test) {
    upwind = 1; donor = 0; downwind = -1; dif = upwind;
  } else {
    upwind = 0; donor = 0; downwind = -1; dif = upwind;
  }
  double sigmat = qdiv(fabs(vol_flux), pre_vol(donor));
  double sigma3 = (1.0 + sigmat) * qratio(vertexd(0), vertexd(dif));
  double sigma4 = 2.0 - sigmat;
  double sigmav = sigmat;
  double diffuw = density1(donor) - density1(upwind);
  double diffdw = density1(downwind) - density1(donor);
  double limiter;
  if ((diffuw * diffdw) > 0.0)
    limiter = (1.0 - sigmav) * op_sign(1.0, diffdw) *
              op_min(op_min(fabs(diffuw), fabs(diffdw)), one_by_six * (sigma3 * fabs(diffuw) + sigma4 * fabs(diffdw)));
  else
    limiter = 0.0;
  mass_flux = (vol_flux) * (density1(donor) + limiter);
  double sigmam = qdiv(fabs(mass_flux), density1(donor) * pre_vol(donor));
  diffuw = energy1(donor) - energy1(upwind);
  diffdw = energy1(downwind) - energy1(donor);
  if ((diffuw * diffdw) > 0.0)
    limiter = (1.0 - sigmam) * op_sign(1.0, diffdw) *
              op_min(op_min(fabs(diffuw), fabs(diffdw)), one_by_six * (sigma3 * fabs(diffuw) + sigma4 * fabs(diffdw)));
  else
    limiter = 0.0;
  ener_flux = mass_flux * (energy1(donor) + limiter);
}

struct XView {
  const D &a;
  __device__ double operator()(int k) const { return a(k, 0); }
};
struct YView {
  const D &a;
  __device__ double operator()(int k) const { return a(0, k); }
};

struct advec_cell_kernel3_xdir {  // :28
  CL_LOOP(advec_cell_kernel3_xdir);
  static constexpr bool touch_next_row = true;
  __device__ void operator()(const D &vol_flux_x, const D &pre_vol, const I &xx, const D &vertexdx, const D &density1,
                             const D &energy1, D &mass_flux_x, D &ener_flux) const {
    double mf, ef;
    advec_cell_flux(vol_flux_x(0, 0), XView{pre_vol}, xx(1, 0) < cc.field.x_max + 2 - 2, XView{vertexdx},
                    XView{density1}, XView{energy1}, mf, ef);
    mass_flux_x(0, 0) = mf;
    ener_flux(0, 0) = ef;
  }
};
struct advec_cell_kernel4_xdir {  // :106
  CL_LOOP(advec_cell_kernel4_xdir);
  static constexpr bool touch_next_row = true;
  static constexpr int min_blocks = 4;
  __device__ void operator()(D &density1, D &energy1, const D &mass_flux_x, const D &vol_flux_x, const D &pre_vol,
                             const D &post_vol, D &pre_mass, D &post_mass, D &advec_vol, D &post_ener,
                             const D &ener_flux) const {
    pre_mass(0, 0) = density1(0, 0) * pre_vol(0, 0);
    post_mass(0, 0) = pre_mass(0, 0) + mass_flux_x(0, 0) - mass_flux_x(1, 0);
    post_ener(0, 0) = (energy1(0, 0) * pre_mass(0, 0) + ener_flux(0, 0) - ener_flux(1, 0)) / post_mass(0, 0);
    advec_vol(0, 0) = pre_vol(0, 0) + vol_flux_x(0, 0) - vol_flux_x(1, 0);
    density1(0, 0) = post_mass(0, 0) / advec_vol(0, 0);
    energy1(0, 0) = post_ener(0, 0);
  }
};
struct advec_cell_kernel1_ydir {  // :123
  CL_LOOP(advec_cell_kernel1_ydir);
  __device__ void operator()(D &pre_vol, D &post_vol, const D &volume, const D &vol_flux_x, const D &vol_flux_y) const {
    pre_vol(0, 0) = volume(0, 0) + (vol_flux_y(0, 1) - vol_flux_y(0, 0) + vol_flux_x(1, 0) - vol_flux_x(0, 0));
    post_vol(0, 0) = pre_vol(0, 0) - (vol_flux_y(0, 1) - vol_flux_y(0, 0));
  }
};
struct advec_cell_kernel2_ydir {  // :133
  CL_LOOP(advec_cell_kernel2_ydir);
  __device__ void operator()(D &pre_vol, D &post_vol, const D &volume, const D &vol_flux_y) const {
    pre_vol(0, 0) = volume(0, 0) + vol_flux_y(0, 1) - vol_flux_y(0, 0);
    post_vol(0, 0) = volume(0, 0);
  }
};
struct advec_cell_kernel3_ydir {  // :142
  CL_LOOP(advec_cell_kernel3_ydir);
  static constexpr bool touch_next_row = true;
  __device__ void operator()(const D &vol_flux_y, const D &pre_vol, const I &yy, const D &vertexdy, const D &density1,
                             const D &energy1, D &mass_flux_y, D &ener_flux) const {
    double mf, ef;
    advec_cell_flux(vol_flux_y(0, 0), YView{pre_vol}, yy(0, 1) < cc.field.y_max + 2 - 2, YView{vertexdy},
                    YView{density1}, YView{energy1}, mf, ef);
    mass_flux_y(0, 0) = mf;
    ener_flux(0, 0) = ef;
  }
};
struct advec_cell_kernel4_ydir {  // :205
  CL_LOOP(advec_cell_kernel4_ydir);
  static constexpr int min_blocks = 4;
  __device__ void operator()(D &density1, D &energy1, const D &mass_flux_y, const D &vol_flux_y, const D &pre_vol,
                             const D &post_vol, D &pre_mass, D &post_mass, D &advec_vol, D &post_ener,
                             const D &ener_flux) const {
    pre_mass(0, 0) = density1(0, 0) * pre_vol(0, 0);
    post_mass(0, 0) = pre_mass(0, 0) + mass_flux_y(0, 0) - mass_flux_y(0, 1);
    post_ener(0, 0) = (energy1(0, 0) * pre_mass(0, 0) + ener_flux(0, 0) - ener_flux(0, 1)) / post_mass(0, 0);
    advec_vol(0, 0) = pre_vol(0, 0) + vol_flux_y(0, 0) - vol_flux_y(0, 1);
    density1(0, 0) = post_mass(0, 0) / advec_vol(0, 0);
    energy1(0, 0) = post_ener(0, 0);
  }
};

// ---- advec_mom_kernel.h ------------------------------------------------------
struct advec_mom_kernel_x1 {  // :4
  CL_LOOP(advec_mom_kernel_x1);
  __device__ void operator()(D &pre_vol, D &post_vol, const D &volume, const D &vol_flux_x, const D &vol_flux_y) const {
    post_vol(0, 0) = volume(0, 0) + vol_flux_y(0, 1) - vol_flux_y(0, 0);
    pre_vol(0, 0) = post_vol(0, 0) + vol_flux_x(1, 0) - vol_flux_x(0, 0);
  }
};
struct advec_mom_kernel_y1 {  // :13
  CL_LOOP(advec_mom_kernel_y1);
  __device__ void operator()(D &pre_vol, D &post_vol, const D &volume, const D &vol_flux_x, const D &vol_flux_y) const {
    post_vol(0, 0) = volume(0, 0) + vol_flux_x(1, 0) - vol_flux_x(0, 0);
    pre_vol(0, 0) = post_vol(0, 0) + vol_flux_y(0, 1) - vol_flux_y(0, 0);
  }
};
struct advec_mom_kernel_x2 {  // :22
  CL_LOOP(advec_mom_kernel_x2);
  __device__ void operator()(D &pre_vol, D &post_vol, const D &volume, const D &vol_flux_y) const {
    post_vol(0, 0) = volume(0, 0);
    pre_vol(0, 0) = post_vol(0, 0) + vol_flux_y(0, 1) - vol_flux_y(0, 0);
  }
};
struct advec_mom_kernel_y2 {  // :31
  CL_LOOP(advec_mom_kernel_y2);
  __device__ void operator()(D &pre_vol, D &post_vol, const D &volume, const D &vol_flux_x) const {
    post_vol(0, 0) = volume(0, 0);
    pre_vol(0, 0) = post_vol(0, 0) + vol_flux_x(1, 0) - vol_flux_x(0, 0);
  }
};
struct advec_mom_kernel_mass_flux_x {  // :40
  CL_LOOP(advec_mom_kernel_mass_flux_x);
  __device__ void operator()(D &node_flux, const D &mass_flux_x) const {
    node_flux(0, 0) = 0.25 * (mass_flux_x(0, -1) + mass_flux_x(0, 0) + mass_flux_x(1, -1) + mass_flux_x(1, 0));
  }
};
struct advec_mom_kernel_mass_flux_y {  // :49
  CL_LOOP(advec_mom_kernel_mass_flux_y);
  __device__ void operator()(D &node_flux, const D &mass_flux_y) const {
    node_flux(0, 0) = 0.25 * (mass_flux_y(-1, 0) + mass_flux_y(0, 0) + mass_flux_y(-1, 1) + mass_flux_y(0, 1));
  }
};
struct advec_mom_kernel_post_pre_advec_x {  // :58
  CL_LOOP(advec_mom_kernel_post_pre_advec_x);
  __device__ void operator()(D &node_mass_post, const D &post_vol, const D &density1, D &node_mass_pre,
                             const D &node_flux) const {
    node_mass_post(0, 0) = 0.25 * (density1(0, -1) * post_vol(0, -1) + density1(0, 0) * post_vol(0, 0) +
                                   density1(-1, -1) * post_vol(-1, -1) + density1(-1, 0) * post_vol(-1, 0));
    node_mass_pre(0, 0) = node_mass_post(0, 0) - node_flux(-1, 0) + node_flux(0, 0);
  }
};
struct advec_mom_kernel_post_pre_advec_y {  // :75
  CL_LOOP(advec_mom_kernel_post_pre_advec_y);
  __device__ void operator()(D &node_mass_post, const D &post_vol, const D &density1, D &node_mass_pre,
                             const D &node_flux) const {
    node_mass_post(0, 0) = 0.25 * (density1(0, -1) * post_vol(0, -1) + density1(0, 0) * post_vol(0, 0) +
                                   density1(-1, -1) * post_vol(-1, -1) + density1(-1, 0) * post_vol(-1, 0));
    node_mass_pre(0, 0) = node_mass_post(0, 0) - node_flux(0, -1) + node_flux(0, 0);
  }
};

// Momentum flux of advec_mom_kernel1_{x,y}_nonvector (:139, :242) over a 1D
// view along the sweep.
template <class View>
__device__ __forceinline__ double advec_mom_flux(double node_flux, const View &node_mass_pre, const View &celld,
                                                 const View &vel1) {
  int upwind, donor, downwind, dif;
  if ((node_flux) < 0.0) {
    upwind = 2; donor = 1; downwind = 0; dif = donor;
  } else {
    upwind = -1; donor = 0; downwind = 1; dif = upwind;
  }
  double sigma = qdiv(fabs(node_flux), node_mass_pre(donor));
  double width = celld(0);
  double vdiffuw = vel1(donor) - vel1(upwind);
  double vdiffdw = vel1(downwind) - vel1(donor);
  double limiter = 0.0;
  if (vdiffuw * vdiffdw > 0.0) {
    double auw = fabs(vdiffuw);
    double adw = fabs(vdiffdw);
    double wind = 1.0;
    if (vdiffdw <= 0.0) wind = -1.0;
    limiter = wind * op_min(width * ((2.0 - sigma) * adw / width + (1.0 + sigma) * auw / celld(dif)) / 6.0,
                            op_min(auw, adw));
  }
  double advec_vel_temp = vel1(donor) + (1.0 - sigma) * limiter;
  return advec_vel_temp * node_flux;
}

struct advec_mom_kernel1_x_nonvector {  // :139
  CL_LOOP(advec_mom_kernel1_x_nonvector);
  __device__ void operator()(const D &node_flux, const D &node_mass_pre, D &mom_flux, const D &celldx,
                             const D &vel1) const {
    mom_flux(0, 0) = advec_mom_flux(node_flux(0, 0), XView{node_mass_pre}, XView{celldx}, XView{vel1});
  }
};
struct advec_mom_kernel1_y_nonvector {  // :242
  CL_LOOP(advec_mom_kernel1_y_nonvector);
  __device__ void operator()(const D &node_flux, const D &node_mass_pre, D &mom_flux, const D &celldy,
                             const D &vel1) const {
    mom_flux(0, 0) = advec_mom_flux(node_flux(0, 0), YView{node_mass_pre}, YView{celldy}, YView{vel1});
  }
};
struct advec_mom_kernel2_x {  // :284
  CL_LOOP(advec_mom_kernel2_x);
  __device__ void operator()(D &vel1, const D &node_mass_post, const D &node_mass_pre, const D &mom_flux) const {
    vel1(0, 0) = qdiv(vel1(0, 0) * node_mass_pre(0, 0) + mom_flux(-1, 0) - mom_flux(0, 0), node_mass_post(0, 0));
  }
};
struct advec_mom_kernel2_y {  // :293
  CL_LOOP(advec_mom_kernel2_y);
  __device__ void operator()(D &vel1, const D &node_mass_post, const D &node_mass_pre, const D &mom_flux) const {
    vel1(0, 0) = qdiv(vel1(0, 0) * node_mass_pre(0, 0) + mom_flux(0, -1) - mom_flux(0, 0), node_mass_post(0, 0));
  }
};

// ---- reset_field_kernel.h ----------------------------------------------------
struct reset_field_kernel1 {  // :5
  CL_LOOP(reset_field_kernel1);
  __device__ void operator()(D &density0, const D &density1, D &energy0, const D &energy1) const {
    density0(0, 0) = density1(0, 0);
    energy0(0, 0) = energy1(0, 0);
  }
};
struct reset_field_kernel2 {  // :13
  CL_LOOP(reset_field_kernel2);
  __device__ void operator()(D &xvel0, const D &xvel1, D &yvel0, const D &yvel1) const {
    xvel0(0, 0) = xvel1(0, 0);
    yvel0(0, 0) = yvel1(0, 0);
  }
};

// ---- field_summary_kernel.h:4 -------------------------------------------------
struct field_summary_kernel {
  CL_LOOP(field_summary_kernel);
  static constexpr bool touch_next_row = true;
  static constexpr int min_blocks = 6;
  __device__ void operator()(const D &volume, const D &density0, const D &energy0, const D &pressure, const D &xvel0,
                             const D &yvel0, RED<double> &vol, RED<double> &mass, RED<double> &ie, RED<double> &ke,
                             RED<double> &press) const {
    double vsqrd = 0.0;
    vsqrd = vsqrd + 0.25 * (xvel0(0, 0) * xvel0(0, 0) + yvel0(0, 0) * yvel0(0, 0));
    vsqrd = vsqrd + 0.25 * (xvel0(1, 0) * xvel0(1, 0) + yvel0(1, 0) * yvel0(1, 0));
    vsqrd = vsqrd + 0.25 * (xvel0(0, 1) * xvel0(0, 1) + yvel0(0, 1) * yvel0(0, 1));
    vsqrd = vsqrd + 0.25 * (xvel0(1, 1) * xvel0(1, 1) + yvel0(1, 1) * yvel0(1, 1));
    double cell_vol = volume(0, 0);
    double cell_mass = cell_vol * density0(0, 0);
    *vol = *vol + cell_vol;
    *mass = *mass + cell_mass;
    *ie = *ie + cell_mass * energy0(0, 0);
    *ke = *ke + cell_mass * 0.5 * vsqrd;
    *press = *press + cell_vol * pressure(0, 0);
  }
};

// ---- registration ------------------------------------------------------------
#define REG(K) OPSB_REGISTER_LOOP(K);
REG(initialise_chunk_kernel_xx) REG(initialise_chunk_kernel_yy) REG(initialise_chunk_kernel_x)
REG(initialise_chunk_kernel_y) REG(initialise_chunk_kernel_cellx) REG(initialise_chunk_kernel_celly)
REG(initialise_chunk_kernel_volume) REG(generate_chunk_kernel) REG(ideal_gas_kernel)
REG(update_halo_kernel1_b2) REG(update_halo_kernel1_b1) REG(update_halo_kernel1_t2) REG(update_halo_kernel1_t1)
REG(update_halo_kernel1_l2) REG(update_halo_kernel1_l1) REG(update_halo_kernel1_r2) REG(update_halo_kernel1_r1)
REG(update_halo_kernel2_xvel_plus_4_a) REG(update_halo_kernel2_xvel_plus_2_a) REG(update_halo_kernel2_xvel_plus_4_b)
REG(update_halo_kernel2_xvel_plus_2_b) REG(update_halo_kernel2_xvel_minus_4_a) REG(update_halo_kernel2_xvel_minus_2_a)
REG(update_halo_kernel2_xvel_minus_4_b) REG(update_halo_kernel2_xvel_minus_2_b)
REG(update_halo_kernel2_yvel_plus_4_a) REG(update_halo_kernel2_yvel_plus_2_a) REG(update_halo_kernel2_yvel_plus_4_b)
REG(update_halo_kernel2_yvel_plus_2_b) REG(update_halo_kernel2_yvel_minus_4_a) REG(update_halo_kernel2_yvel_minus_2_a)
REG(update_halo_kernel2_yvel_minus_4_b) REG(update_halo_kernel2_yvel_minus_2_b)
REG(update_halo_kernel3_plus_4_a) REG(update_halo_kernel3_plus_2_a) REG(update_halo_kernel3_plus_4_b)
REG(update_halo_kernel3_plus_2_b) REG(update_halo_kernel3_minus_4_a) REG(update_halo_kernel3_minus_2_a)
REG(update_halo_kernel3_minus_4_b) REG(update_halo_kernel3_minus_2_b)
REG(update_halo_kernel4_plus_4_a) REG(update_halo_kernel4_plus_2_a) REG(update_halo_kernel4_plus_4_b)
REG(update_halo_kernel4_plus_2_b) REG(update_halo_kernel4_minus_4_a) REG(update_halo_kernel4_minus_2_a)
REG(update_halo_kernel4_minus_4_b) REG(update_halo_kernel4_minus_2_b)
REG(viscosity_kernel) REG(calc_dt_kernel) REG(calc_dt_kernel_min) REG(calc_dt_kernel_get) REG(calc_dt_kernel_print)
REG(PdV_kernel_predict) REG(PdV_kernel_nopredict) REG(revert_kernel) REG(accelerate_kernel)
REG(flux_calc_kernelx) REG(flux_calc_kernely)
REG(advec_cell_kernel1_xdir) REG(advec_cell_kernel2_xdir) REG(advec_cell_kernel3_xdir) REG(advec_cell_kernel4_xdir)
REG(advec_cell_kernel1_ydir) REG(advec_cell_kernel2_ydir) REG(advec_cell_kernel3_ydir) REG(advec_cell_kernel4_ydir)
REG(advec_mom_kernel_x1) REG(advec_mom_kernel_y1) REG(advec_mom_kernel_x2) REG(advec_mom_kernel_y2)
REG(advec_mom_kernel_mass_flux_x) REG(advec_mom_kernel_mass_flux_y)
REG(advec_mom_kernel_post_pre_advec_x) REG(advec_mom_kernel_post_pre_advec_y)
REG(advec_mom_kernel1_x_nonvector) REG(advec_mom_kernel1_y_nonvector) REG(advec_mom_kernel2_x) REG(advec_mom_kernel2_y)
REG(reset_field_kernel1) REG(reset_field_kernel2) REG(field_summary_kernel)

// The hydro cycle's loop kernels as two fusion groups: the lazy queue's
// planner (fusion.cpp) may run any chain of one group's kernels, with the
// boundary copies between them, as one tiled kernel. The timestep and
// Lagrangian loops compile leaner than the advection loops, so they get a
// group (and register budget) of their own.
static fuse::GroupRegistrar<2, ideal_gas_kernel, viscosity_kernel, calc_dt_kernel, calc_dt_kernel_min,
                            PdV_kernel_predict, PdV_kernel_nopredict, revert_kernel, accelerate_kernel,
                            flux_calc_kernelx, flux_calc_kernely, reset_field_kernel1, reset_field_kernel2>
    fused_lagrange("cloverleaf2d_lagrange");
static fuse::GroupRegistrar<2, advec_cell_kernel1_xdir, advec_cell_kernel2_xdir, advec_cell_kernel3_xdir,
                            advec_cell_kernel4_xdir, advec_cell_kernel1_ydir, advec_cell_kernel2_ydir,
                            advec_cell_kernel3_ydir, advec_cell_kernel4_ydir, advec_mom_kernel_x1,
                            advec_mom_kernel_y1, advec_mom_kernel_x2, advec_mom_kernel_y2,
                            advec_mom_kernel_mass_flux_x, advec_mom_kernel_mass_flux_y,
                            advec_mom_kernel_post_pre_advec_x, advec_mom_kernel_post_pre_advec_y,
                            advec_mom_kernel1_x_nonvector, advec_mom_kernel1_y_nonvector, advec_mom_kernel2_x,
                            advec_mom_kernel2_y>
    fused_advect("cloverleaf2d_advect");

// Named constants (ops_decl_const in clover_leaf.cpp:147-160).
struct ConstReg {
  ConstReg() {
#define C(name, member) Runtime::register_const("cloverleaf/" name, &cc, offsetof(Consts, member), sizeof(Consts::member))
    C("g_small", g_small); C("g_big", g_big); C("dtc_safe", dtc_safe); C("dtu_safe", dtu_safe);
    C("dtv_safe", dtv_safe); C("dtdiv_safe", dtdiv_safe); C("dt", dt); C("field", field); C("grid", grid);
    C("number_of_states", number_of_states); C("g_circ", g_circ); C("g_point", g_point); C("g_rect", g_rect);
    C("states", states);
#undef C
  }
};
static ConstReg const_reg;

}  // namespace clover
}  // namespace opsb
