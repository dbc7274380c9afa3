// CloverLeaf 3D hydro loop kernels (compressible Euler, Lagrangian step plus
// directionally split advective remap; ideal gas, gamma = 1.4).
//
// Each functor restates one reference kernel with the same operation order
// (apps/c/CloverLeaf_3D/*_kernel.h, cited per functor); with --fmad=false the
// cell updates round exactly like the reference's x86-64 CPU build. Kernels
// that differ only in the axis they work along are one template over the
// axis, which keeps every expression as the reference writes it. Divisions
// whose numerator is often exactly zero go through qdiv (same IEEE quotient,
// no division for a zero numerator), the advection limiter's cell-width
// ratio through qratio (exactly 1 for equal widths). Loop names are
// "cloverleaf3d/<reference kernel name>".
#include <cstddef>

#include "clover3d_common.h"
#include "runtime.h"

namespace opsb {
namespace clover3d {

__constant__ Consts c3;

using D = ACC3<double>;
using I = ACC3<int>;

#define C3_LOOP(NAME) static constexpr const char *kname = "cloverleaf3d/" #NAME
// Kernels with many live values (the 8-point velocity gathers, the limiter
// arithmetic) get a larger register budget: C3_HEAVY_MINB resident CTAs of
// 256 threads per SM instead of the default 4.
#ifndef C3_HEAVY_MINB
#define C3_HEAVY_MINB 4
#endif
#define C3_HEAVY static constexpr int min_blocks = C3_HEAVY_MINB

// Offset `o` along axis AX (0 = x, 1 = y, 2 = z).
template <int AX, class A>
__device__ __forceinline__ auto ax(const A &a, int o) {
  if constexpr (AX == 0) return a(o, 0, 0);
  else if constexpr (AX == 1) return a(0, o, 0);
  else return a(0, 0, o);
}

// ---- initialise_chunk_kernel.h -------------------------------------------
struct initialise_chunk_kernel_xx {  // :64
  C3_LOOP(initialise_chunk_kernel_xx);
  __device__ void operator()(I &xx, const IDX &idx) const { xx(0, 0, 0) = idx[0] - 2; }
};
struct initialise_chunk_kernel_yy {  // :68
  C3_LOOP(initialise_chunk_kernel_yy);
  __device__ void operator()(I &yy, const IDX &idx) const { yy(0, 0, 0) = idx[1] - 2; }
};
struct initialise_chunk_kernel_zz {  // :72
  C3_LOOP(initialise_chunk_kernel_zz);
  __device__ void operator()(I &zz, const IDX &idx) const { zz(0, 0, 0) = idx[2] - 2; }
};
struct initialise_chunk_kernel_x {  // :7
  C3_LOOP(initialise_chunk_kernel_x);
  __device__ void operator()(D &vertexx, const I &xx, D &vertexdx) const {
    int x_min = c3.field.x_min - 2;
    double min_x, d_x;
    d_x = (c3.grid.xmax - c3.grid.xmin) / (double)c3.grid.x_cells;
    min_x = c3.grid.xmin + d_x * c3.field.left;
    vertexx(0, 0, 0) = min_x + d_x * (xx(0, 0, 0) - x_min);
    vertexdx(0, 0, 0) = (double)d_x;
  }
};
struct initialise_chunk_kernel_y {  // :25
  C3_LOOP(initialise_chunk_kernel_y);
  __device__ void operator()(D &vertexy, const I &yy, D &vertexdy) const {
    int y_min = c3.field.y_min - 2;
    double min_y, d_y;
    d_y = (c3.grid.ymax - c3.grid.ymin) / (double)c3.grid.y_cells;
    min_y = c3.grid.ymin + d_y * c3.field.bottom;
    vertexy(0, 0, 0) = min_y + d_y * (yy(0, 0, 0) - y_min);
    vertexdy(0, 0, 0) = (double)d_y;
  }
};
struct initialise_chunk_kernel_z {  // :39
  C3_LOOP(initialise_chunk_kernel_z);
  __device__ void operator()(D &vertexz, const I &zz, D &vertexdz) const {
    int z_min = c3.field.z_min - 2;
    double min_z, d_z;
    d_z = (c3.grid.zmax - c3.grid.zmin) / (double)c3.grid.z_cells;
    min_z = c3.grid.zmin + d_z * c3.field.back;
    vertexz(0, 0, 0) = min_z + d_z * (zz(0, 0, 0) - z_min);
    vertexdz(0, 0, 0) = (double)d_z;
  }
};
struct initialise_chunk_kernel_cellx {  // :77
  C3_LOOP(initialise_chunk_kernel_cellx);
  __device__ void operator()(const D &vertexx, D &cellx, D &celldx) const {
    double d_x = (c3.grid.xmax - c3.grid.xmin) / (double)c3.grid.x_cells;
    cellx(0, 0, 0) = 0.5 * (vertexx(0, 0, 0) + vertexx(1, 0, 0));
    celldx(0, 0, 0) = d_x;
  }
};
struct initialise_chunk_kernel_celly {  // :91
  C3_LOOP(initialise_chunk_kernel_celly);
  __device__ void operator()(const D &vertexy, D &celly, D &celldy) const {
    double d_y = (c3.grid.ymax - c3.grid.ymin) / (double)c3.grid.y_cells;
    celly(0, 0, 0) = 0.5 * (vertexy(0, 0, 0) + vertexy(0, 1, 0));
    celldy(0, 0, 0) = d_y;
  }
};
struct initialise_chunk_kernel_cellz {  // :104
  C3_LOOP(initialise_chunk_kernel_cellz);
  __device__ void operator()(const D &vertexz, D &cellz, D &celldz) const {
    double d_z = (c3.grid.zmax - c3.grid.zmin) / (double)c3.grid.z_cells;
    cellz(0, 0, 0) = 0.5 * (vertexz(0, 0, 0) + vertexz(0, 0, 1));
    celldz(0, 0, 0) = d_z;
  }
};
struct initialise_chunk_kernel_volume {  // :118
  C3_LOOP(initialise_chunk_kernel_volume);
  __device__ void operator()(D &volume, const D &celldy, D &xarea, const D &celldx, D &yarea, const D &celldz,
                             D &zarea) const {
    double d_x, d_y, d_z;
    d_x = (c3.grid.xmax - c3.grid.xmin) / (double)c3.grid.x_cells;
    d_y = (c3.grid.ymax - c3.grid.ymin) / (double)c3.grid.y_cells;
    d_z = (c3.grid.zmax - c3.grid.zmin) / (double)c3.grid.z_cells;
    volume(0, 0, 0) = d_x * d_y * d_z;
    xarea(0, 0, 0) = celldy(0, 0, 0) * celldz(0, 0, 0);
    yarea(0, 0, 0) = celldx(0, 0, 0) * celldz(0, 0, 0);
    zarea(0, 0, 0) = celldx(0, 0, 0) * celldy(0, 0, 0);
  }
};

// ---- generate_chunk_kernel.h:9 (cuboids, spheres, points) -------------------
// is_in is set once per cell and never cleared between states, as in the
// reference: a later state then takes over the velocities too.
struct generate_chunk_kernel {
  C3_LOOP(generate_chunk_kernel);
  __device__ void operator()(const D &vertexx, const D &vertexy, const D &vertexz, D &energy0, D &density0, D &xvel0,
                             D &yvel0, D &zvel0, const D &cellx, const D &celly, const D &cellz) const {
    double radius = 0.0, x_cent, y_cent, z_cent;
    int is_in = 0;
    energy0(0, 0, 0) = c3.states[0].energy;
    density0(0, 0, 0) = c3.states[0].density;
    xvel0(0, 0, 0) = c3.states[0].xvel;
    yvel0(0, 0, 0) = c3.states[0].yvel;
    zvel0(0, 0, 0) = c3.states[0].zvel;
    for (int i = 1; i < c3.number_of_states; i++) {
      const state_type &s = c3.states[i];
      x_cent = s.xmin;
      y_cent = s.ymin;
      z_cent = s.zmin;
      if (s.geometry == c3.g_cube) {
        for (int i1 = -1; i1 <= 0; i1++)
          for (int j1 = -1; j1 <= 0; j1++)
            for (int k1 = -1; k1 <= 0; k1++)
              if (vertexx(1 + i1, 0, 0) >= s.xmin && vertexx(0 + i1, 0, 0) < s.xmax)
                if (vertexy(0, 1 + j1, 0) >= s.ymin && vertexy(0, 0 + j1, 0) < s.ymax)
                  if (vertexz(0, 0, 1 + k1) >= s.zmin && vertexz(0, 0, 0 + k1) < s.zmax) is_in = 1;
        if (vertexx(1, 0, 0) >= s.xmin && vertexx(0, 0, 0) < s.xmax)
          if (vertexy(0, 1, 0) >= s.ymin && vertexy(0, 0, 0) < s.ymax)
            if (vertexz(0, 0, 1) >= s.zmin && vertexz(0, 0, 0) < s.zmax) {
              energy0(0, 0, 0) = s.energy;
              density0(0, 0, 0) = s.density;
            }
        if (is_in) {
          xvel0(0, 0, 0) = s.xvel;
          yvel0(0, 0, 0) = s.yvel;
          zvel0(0, 0, 0) = s.zvel;
        }
      } else if (s.geometry == c3.g_sphe) {
        for (int i1 = -1; i1 <= 0; i1++)
          for (int j1 = -1; j1 <= 0; j1++)
            for (int k1 = -1; k1 <= 0; k1++) {
              radius = sqrt((cellx(0, 0, 0) - x_cent) * (cellx(0, 0, 0) - x_cent) +
                            (celly(0, 0, 0) - y_cent) * (celly(0, 0, 0) - y_cent) +
                            (cellz(0, 0, 0) - z_cent) * (cellz(0, 0, 0) - z_cent));
              if (radius <= s.radius) is_in = 1;
            }
        if (radius <= s.radius) {
          energy0(0, 0, 0) = s.energy;
          density0(0, 0, 0) = s.density;
        }
        if (is_in) {
          xvel0(0, 0, 0) = s.xvel;
          yvel0(0, 0, 0) = s.yvel;
          zvel0(0, 0, 0) = s.zvel;
        }
      } else if (s.geometry == c3.g_point) {
        for (int i1 = -1; i1 <= 0; i1++)
          for (int j1 = -1; j1 <= 0; j1++)
            for (int k1 = -1; k1 <= 0; k1++)
              if (vertexx(0 + i1, 0, 0) == x_cent && vertexy(0, 0 + j1, 0) == y_cent &&
                  vertexz(0, 0, 0 + k1) == z_cent)
                is_in = 1;
        if (vertexx(0, 0, 0) == x_cent && vertexy(0, 0, 0) == y_cent && vertexz(0, 0, 0) == z_cent) {
          energy0(0, 0, 0) = s.energy;
          density0(0, 0, 0) = s.density;
        }
        if (is_in) {
          xvel0(0, 0, 0) = s.xvel;
          yvel0(0, 0, 0) = s.yvel;
          zvel0(0, 0, 0) = s.zvel;
        }
      }
    }
  }
};

// ---- ideal_gas_kernel.h:7 ------------------------------------------------------
struct ideal_gas_kernel {
  C3_LOOP(ideal_gas_kernel);
  __device__ void operator()(const D &density, const D &energy, D &pressure, D &soundspeed) const {
    double sound_speed_squared, v, pressurebyenergy, pressurebyvolume;
    v = 1.0 / density(0, 0, 0);
    pressure(0, 0, 0) = (1.4 - 1.0) * density(0, 0, 0) * energy(0, 0, 0);
    pressurebyenergy = (1.4 - 1.0) * density(0, 0, 0);
    pressurebyvolume = -1.0 * density(0, 0, 0) * pressure(0, 0, 0);
    sound_speed_squared = v * v * (pressure(0, 0, 0) * pressurebyenergy - pressurebyvolume);
    soundspeed(0, 0, 0) = sqrt(sound_speed_squared);
  }
};

// ---- update_halo_kernel.h: reflective boundary copies ------------------------
// The seven cell-centred fields, copied from the mirror point (OX, OY, OZ).
template <int OX, int OY, int OZ>
struct uh1 {
  static CopyLoopSpec copy_spec() {
    CopyLoopSpec c;
    c.nfields = 7;
    for (int f = 0; f < 7; f++) c.arg[f] = f, c.flag[f] = FIELD_DENSITY0 + f;
    c.flags_arg = 7;
    c.off[0] = OX; c.off[1] = OY; c.off[2] = OZ;
    return c;
  }
  __device__ void operator()(D &density0, D &density1, D &energy0, D &energy1, D &pressure, D &viscosity,
                             D &soundspeed, const int *fields) const {
    if (fields[FIELD_DENSITY0] == 1) density0(0, 0, 0) = density0(OX, OY, OZ);
    if (fields[FIELD_DENSITY1] == 1) density1(0, 0, 0) = density1(OX, OY, OZ);
    if (fields[FIELD_ENERGY0] == 1) energy0(0, 0, 0) = energy0(OX, OY, OZ);
    if (fields[FIELD_ENERGY1] == 1) energy1(0, 0, 0) = energy1(OX, OY, OZ);
    if (fields[FIELD_PRESSURE] == 1) pressure(0, 0, 0) = pressure(OX, OY, OZ);
    if (fields[FIELD_VISCOSITY] == 1) viscosity(0, 0, 0) = viscosity(OX, OY, OZ);
    if (fields[FIELD_SOUNDSPEED] == 1) soundspeed(0, 0, 0) = soundspeed(OX, OY, OZ);
  }
};
// A pair of face or node fields (F0, F1), copied (NEG = 0) or reflected
// (NEG = 1, the velocity or flux normal to the face) from (OX, OY, OZ).
template <int OX, int OY, int OZ, int NEG, int F0, int F1>
struct uh2 {
  static CopyLoopSpec copy_spec() {
    CopyLoopSpec c;
    c.nfields = 2;
    c.arg[0] = 0; c.arg[1] = 1; c.flag[0] = F0; c.flag[1] = F1;
    c.flags_arg = 2;
    c.neg = NEG;
    c.off[0] = OX; c.off[1] = OY; c.off[2] = OZ;
    return c;
  }
  __device__ void operator()(D &a, D &b, const int *fields) const {
    if (fields[F0] == 1) a(0, 0, 0) = NEG ? -(a(OX, OY, OZ)) : a(OX, OY, OZ);
    if (fields[F1] == 1) b(0, 0, 0) = NEG ? -(b(OX, OY, OZ)) : b(OX, OY, OZ);
  }
};
#define UH1(NAME, OX, OY, OZ)                     \
  struct NAME : uh1<OX, OY, OZ> { C3_LOOP(NAME); }; \
  OPSB_REGISTER_COPY_LOOP(NAME);
#define UH2(NAME, OX, OY, OZ, NEG, ...)                               \
  struct NAME : uh2<OX, OY, OZ, NEG, __VA_ARGS__> { C3_LOOP(NAME); }; \
  OPSB_REGISTER_COPY_LOOP(NAME);
UH1(update_halo_kernel1_b2, 0, 3, 0)
UH1(update_halo_kernel1_b1, 0, 1, 0)
UH1(update_halo_kernel1_t2, 0, -3, 0)
UH1(update_halo_kernel1_t1, 0, -1, 0)
UH1(update_halo_kernel1_l2, 3, 0, 0)
UH1(update_halo_kernel1_l1, 1, 0, 0)
UH1(update_halo_kernel1_r2, -3, 0, 0)
UH1(update_halo_kernel1_r1, -1, 0, 0)
UH1(update_halo_kernel1_ba2, 0, 0, 3)
UH1(update_halo_kernel1_ba1, 0, 0, 1)
UH1(update_halo_kernel1_fr2, 0, 0, -3)
UH1(update_halo_kernel1_fr1, 0, 0, -1)
#define XV FIELD_XVEL0, FIELD_XVEL1
#define YV FIELD_YVEL0, FIELD_YVEL1
#define ZV FIELD_ZVEL0, FIELD_ZVEL1
#define FX FIELD_VOL_FLUX_X, FIELD_MASS_FLUX_X
#define FY FIELD_VOL_FLUX_Y, FIELD_MASS_FLUX_Y
#define FZ FIELD_VOL_FLUX_Z, FIELD_MASS_FLUX_Z
UH2(update_halo_kernel2_xvel_plus_4_bot, 0, 4, 0, 0, XV)
UH2(update_halo_kernel2_xvel_plus_2_bot, 0, 2, 0, 0, XV)
UH2(update_halo_kernel2_xvel_plus_4_top, 0, -4, 0, 0, XV)
UH2(update_halo_kernel2_xvel_plus_2_top, 0, -2, 0, 0, XV)
UH2(update_halo_kernel2_xvel_minus_4_left, 4, 0, 0, 1, XV)
UH2(update_halo_kernel2_xvel_minus_2_left, 2, 0, 0, 1, XV)
UH2(update_halo_kernel2_xvel_minus_4_right, -4, 0, 0, 1, XV)
UH2(update_halo_kernel2_xvel_minus_2_right, -2, 0, 0, 1, XV)
UH2(update_halo_kernel2_xvel_plus_4_back, 0, 0, 4, 0, XV)
UH2(update_halo_kernel2_xvel_plus_2_back, 0, 0, 2, 0, XV)
UH2(update_halo_kernel2_xvel_plus_4_front, 0, 0, -4, 0, XV)
UH2(update_halo_kernel2_xvel_plus_2_front, 0, 0, -2, 0, XV)
UH2(update_halo_kernel2_yvel_minus_4_bot, 0, 4, 0, 1, YV)
UH2(update_halo_kernel2_yvel_minus_2_bot, 0, 2, 0, 1, YV)
UH2(update_halo_kernel2_yvel_minus_4_top, 0, -4, 0, 1, YV)
UH2(update_halo_kernel2_yvel_minus_2_top, 0, -2, 0, 1, YV)
UH2(update_halo_kernel2_yvel_plus_4_left, 4, 0, 0, 0, YV)
UH2(update_halo_kernel2_yvel_plus_2_left, 2, 0, 0, 0, YV)
UH2(update_halo_kernel2_yvel_plus_4_right, -4, 0, 0, 0, YV)
UH2(update_halo_kernel2_yvel_plus_2_right, -2, 0, 0, 0, YV)
UH2(update_halo_kernel2_yvel_plus_4_back, 0, 0, 4, 0, YV)
UH2(update_halo_kernel2_yvel_plus_2_back, 0, 0, 2, 0, YV)
UH2(update_halo_kernel2_yvel_plus_4_front, 0, 0, -4, 0, YV)
UH2(update_halo_kernel2_yvel_plus_2_front, 0, 0, -2, 0, YV)
UH2(update_halo_kernel2_zvel_plus_4_bot, 0, 4, 0, 0, ZV)
UH2(update_halo_kernel2_zvel_plus_2_bot, 0, 2, 0, 0, ZV)
UH2(update_halo_kernel2_zvel_plus_4_top, 0, -4, 0, 0, ZV)
UH2(update_halo_kernel2_zvel_plus_2_top, 0, -2, 0, 0, ZV)
UH2(update_halo_kernel2_zvel_plus_4_left, 4, 0, 0, 0, ZV)
UH2(update_halo_kernel2_zvel_plus_2_left, 2, 0, 0, 0, ZV)
UH2(update_halo_kernel2_zvel_plus_4_right, -4, 0, 0, 0, ZV)
UH2(update_halo_kernel2_zvel_plus_2_right, -2, 0, 0, 0, ZV)
UH2(update_halo_kernel2_zvel_minus_4_back, 0, 0, 4, 1, ZV)
UH2(update_halo_kernel2_zvel_minus_2_back, 0, 0, 2, 1, ZV)
UH2(update_halo_kernel2_zvel_minus_4_front, 0, 0, -4, 1, ZV)
UH2(update_halo_kernel2_zvel_minus_2_front, 0, 0, -2, 1, ZV)
UH2(update_halo_kernel3_plus_4_a, 0, 4, 0, 0, FX)
UH2(update_halo_kernel3_plus_2_a, 0, 2, 0, 0, FX)
UH2(update_halo_kernel3_plus_4_b, 0, -4, 0, 0, FX)
UH2(update_halo_kernel3_plus_2_b, 0, -2, 0, 0, FX)
UH2(update_halo_kernel3_minus_4_a, 4, 0, 0, 1, FX)
UH2(update_halo_kernel3_minus_2_a, 2, 0, 0, 1, FX)
UH2(update_halo_kernel3_minus_4_b, -4, 0, 0, 1, FX)
UH2(update_halo_kernel3_minus_2_b, -2, 0, 0, 1, FX)
UH2(update_halo_kernel3_plus_4_back, 0, 0, 4, 0, FX)
UH2(update_halo_kernel3_plus_2_back, 0, 0, 2, 0, FX)
UH2(update_halo_kernel3_plus_4_front, 0, 0, -4, 0, FX)
UH2(update_halo_kernel3_plus_2_front, 0, 0, -2, 0, FX)
UH2(update_halo_kernel4_minus_4_a, 0, 4, 0, 1, FY)
UH2(update_halo_kernel4_minus_2_a, 0, 2, 0, 1, FY)
UH2(update_halo_kernel4_minus_4_b, 0, -4, 0, 1, FY)
UH2(update_halo_kernel4_minus_2_b, 0, -2, 0, 1, FY)
UH2(update_halo_kernel4_plus_4_a, 4, 0, 0, 0, FY)
UH2(update_halo_kernel4_plus_2_a, 2, 0, 0, 0, FY)
UH2(update_halo_kernel4_plus_4_b, -4, 0, 0, 0, FY)
UH2(update_halo_kernel4_plus_2_b, -2, 0, 0, 0, FY)
UH2(update_halo_kernel4_plus_4_back, 0, 0, 4, 0, FY)
UH2(update_halo_kernel4_plus_2_back, 0, 0, 2, 0, FY)
UH2(update_halo_kernel4_plus_4_front, 0, 0, -4, 0, FY)
UH2(update_halo_kernel4_plus_2_front, 0, 0, -2, 0, FY)
UH2(update_halo_kernel5_plus_4_a, 0, 4, 0, 0, FZ)
UH2(update_halo_kernel5_plus_2_a, 0, 2, 0, 0, FZ)
UH2(update_halo_kernel5_plus_4_b, 0, -4, 0, 0, FZ)
UH2(update_halo_kernel5_plus_2_b, 0, -2, 0, 0, FZ)
UH2(update_halo_kernel5_plus_4_left, 4, 0, 0, 0, FZ)
UH2(update_halo_kernel5_plus_2_left, 2, 0, 0, 0, FZ)
UH2(update_halo_kernel5_plus_4_right, -4, 0, 0, 0, FZ)
UH2(update_halo_kernel5_plus_2_right, -2, 0, 0, 0, FZ)
UH2(update_halo_kernel5_minus_4_back, 0, 0, 4, 1, FZ)
UH2(update_halo_kernel5_minus_2_back, 0, 0, 2, 1, FZ)
UH2(update_halo_kernel5_minus_4_front, 0, 0, -4, 1, FZ)
UH2(update_halo_kernel5_minus_2_front, 0, 0, -2, 1, FZ)
#undef XV
#undef YV
#undef ZV
#undef FX
#undef FY
#undef FZ

// ---- viscosity_kernel.h:7 --------------------------------------------------------
struct viscosity_kernel {
  C3_LOOP(viscosity_kernel);
  C3_HEAVY;
  __device__ void operator()(const D &xvel0, const D &yvel0, const D &celldx, const D &celldy, const D &pressure,
                             const D &density0, D &viscosity, const D &zvel0, const D &celldz, const D &xarea,
                             const D &yarea, const D &zarea) const {
    double grad2, pgradx, pgrady, pgradz, pgradx2, pgrady2, pgradz2, grad, ygrad, xgrad, zgrad, div, limiter, pgrad;
    double ugradx1 = xvel0(0, 0, 0) + xvel0(0, 1, 0) + xvel0(0, 0, 1) + xvel0(0, 1, 1);
    double ugradx2 = xvel0(1, 0, 0) + xvel0(1, 1, 0) + xvel0(1, 0, 1) + xvel0(1, 1, 1);
    double ugrady1 = xvel0(0, 0, 0) + xvel0(1, 0, 0) + xvel0(0, 0, 1) + xvel0(1, 0, 1);
    double ugrady2 = xvel0(0, 1, 0) + xvel0(1, 1, 0) + xvel0(0, 1, 1) + xvel0(1, 1, 1);
    double ugradz1 = xvel0(0, 0, 0) + xvel0(1, 0, 0) + xvel0(0, 1, 0) + xvel0(1, 1, 0);
    double ugradz2 = xvel0(0, 0, 1) + xvel0(1, 0, 1) + xvel0(0, 1, 1) + xvel0(1, 1, 1);
    double vgradx1 = yvel0(0, 0, 0) + yvel0(0, 1, 0) + yvel0(0, 0, 1) + yvel0(0, 1, 1);
    double vgradx2 = yvel0(1, 0, 0) + yvel0(1, 1, 0) + yvel0(1, 0, 1) + yvel0(1, 1, 1);
    double vgrady1 = yvel0(0, 0, 0) + yvel0(1, 0, 0) + yvel0(0, 0, 1) + yvel0(1, 0, 1);
    double vgrady2 = yvel0(0, 1, 0) + yvel0(1, 1, 0) + yvel0(0, 1, 1) + yvel0(1, 1, 1);
    double vgradz1 = yvel0(0, 0, 0) + yvel0(1, 0, 0) + yvel0(0, 1, 0) + yvel0(1, 1, 0);
    double vgradz2 = yvel0(0, 0, 1) + yvel0(1, 0, 1) + yvel0(0, 1, 1) + yvel0(1, 1, 1);
    double wgradx1 = zvel0(0, 0, 0) + zvel0(0, 1, 0) + zvel0(0, 0, 1) + zvel0(0, 1, 1);
    double wgradx2 = zvel0(1, 0, 0) + zvel0(1, 1, 0) + zvel0(1, 0, 1) + zvel0(1, 1, 1);
    double wgrady1 = zvel0(0, 0, 0) + zvel0(1, 0, 0) + zvel0(0, 0, 1) + zvel0(1, 0, 1);
    double wgrady2 = zvel0(0, 1, 0) + zvel0(1, 1, 0) + zvel0(0, 1, 1) + zvel0(1, 1, 1);
    double wgradz1 = zvel0(0, 0, 0) + zvel0(1, 0, 0) + zvel0(0, 1, 0) + zvel0(1, 1, 0);
    double wgradz2 = zvel0(0, 0, 1) + zvel0(1, 0, 1) + zvel0(0, 1, 1) + zvel0(1, 1, 1);
    div = xarea(0, 0, 0) * (ugradx2 - ugradx1) + yarea(0, 0, 0) * (vgrady2 - vgrady1) +
          zarea(0, 0, 0) * (wgradz2 - wgradz1);
    // qdiv: the same quotients; exactly zero numerators (uniform regions)
    // take the product path
    double xx = qdiv(0.25 * (ugradx2 - ugradx1), (celldx(0, 0, 0)));
    double yy = qdiv(0.25 * (vgrady2 - vgrady1), (celldy(0, 0, 0)));
    double zz = qdiv(0.25 * (wgradz2 - wgradz1), (celldz(0, 0, 0)));
    double xy = qdiv(0.25 * (ugrady2 - ugrady1), (celldy(0, 0, 0))) + qdiv(0.25 * (vgradx2 - vgradx1), (celldx(0, 0, 0)));
    double xz = qdiv(0.25 * (ugradz2 - ugradz1), (celldz(0, 0, 0))) + qdiv(0.25 * (wgradx2 - wgradx1), (celldx(0, 0, 0)));
    double yz = qdiv(0.25 * (vgradz2 - vgradz1), (celldz(0, 0, 0))) + qdiv(0.25 * (wgrady2 - wgrady1), (celldy(0, 0, 0)));
    pgradx = qdiv(pressure(1, 0, 0) - pressure(-1, 0, 0), celldx(0, 0, 0) + celldx(1, 0, 0));
    pgrady = qdiv(pressure(0, 1, 0) - pressure(0, -1, 0), celldy(0, 0, 0) + celldy(0, 1, 0));
    pgradz = qdiv(pressure(0, 0, 1) - pressure(0, 0, -1), celldz(0, 0, 0) + celldz(0, 0, 1));
    pgradx2 = pgradx * pgradx;
    pgrady2 = pgrady * pgrady;
    pgradz2 = pgradz * pgradz;
    limiter = qdiv(xx * pgradx2 + yy * pgrady2 + zz * pgradz2 + xy * pgradx * pgrady + xz * pgradx * pgradz +
                       yz * pgrady * pgradz,
                   op_max(pgradx2 + pgrady2 + pgradz2, 1.0e-16));
    if ((limiter > 0.0) || (div >= 0.0)) {
      viscosity(0, 0, 0) = 0.0;
    } else {
      pgradx = op_sign(op_max(1.0e-16, fabs(pgradx)), pgradx);
      pgrady = op_sign(op_max(1.0e-16, fabs(pgrady)), pgrady);
      pgradz = op_sign(op_max(1.0e-16, fabs(pgradz)), pgradz);
      pgrad = sqrt(pgradx * pgradx + pgrady * pgrady + pgradz * pgradz);
      xgrad = fabs(celldx(0, 0, 0) * pgrad / pgradx);
      ygrad = fabs(celldy(0, 0, 0) * pgrad / pgrady);
      zgrad = fabs(celldz(0, 0, 0) * pgrad / pgradz);
      grad = op_min(xgrad, op_min(ygrad, zgrad));
      grad2 = grad * grad;
      viscosity(0, 0, 0) = 2.0 * (density0(0, 0, 0)) * grad2 * limiter * limiter;
    }
  }
};

// ---- calc_dt_kernel.h -------------------------------------------------------------
struct calc_dt_kernel {  // :7
  C3_LOOP(calc_dt_kernel);
  C3_HEAVY;
  __device__ void operator()(const D &celldx, const D &celldy, const D &soundspeed, const D &viscosity,
                             const D &density0, const D &xvel0, const D &xarea, const D &volume, const D &yvel0,
                             const D &yarea, D &dt_min, const D &celldz, const D &zvel0, const D &zarea) const {
    double div, ds, dtut, dtvt, dtct, dtwt, dtdivt, cc, dv1, dv2, du1, du2, dw1, dw2;
    ds = op_min(op_min(celldx(0, 0, 0), celldy(0, 0, 0)), celldz(0, 0, 0));
    ds = 1.0 / (ds * ds);
    cc = soundspeed(0, 0, 0) * soundspeed(0, 0, 0);
    cc = cc + qdiv(2.0 * viscosity(0, 0, 0), density0(0, 0, 0));
    dtct = ds * cc;
    dtct = c3.dtc_safe * 1.0 / op_max(sqrt(dtct), c3.g_small);
    du1 = (xvel0(0, 0, 0) + xvel0(0, 1, 0) + xvel0(0, 0, 1) + xvel0(0, 1, 1)) * xarea(0, 0, 0);
    du2 = (xvel0(1, 0, 0) + xvel0(1, 1, 0) + xvel0(1, 0, 1) + xvel0(1, 1, 1)) * xarea(0, 0, 0);
    dtut = c3.dtu_safe * 4.0 * volume(0, 0, 0) / op_max(op_max(fabs(du1), fabs(du2)), 1.0e-5 * volume(0, 0, 0));
    dv1 = (yvel0(0, 0, 0) + yvel0(1, 0, 0) + yvel0(0, 0, 1) + yvel0(1, 0, 1)) * yarea(0, 0, 0);
    dv2 = (yvel0(0, 1, 0) + yvel0(1, 1, 0) + yvel0(0, 1, 1) + yvel0(1, 1, 1)) * yarea(0, 0, 0);
    dtvt = c3.dtv_safe * 4.0 * volume(0, 0, 0) / op_max(op_max(fabs(dv1), fabs(dv2)), 1.0e-5 * volume(0, 0, 0));
    dw1 = (zvel0(0, 0, 0) + zvel0(0, 1, 0) + zvel0(1, 0, 0) + zvel0(1, 1, 0)) * zarea(0, 0, 0);
    dw2 = (zvel0(0, 0, 1) + zvel0(0, 1, 1) + zvel0(1, 0, 1) + zvel0(1, 1, 1)) * zarea(0, 0, 0);
    dtwt = c3.dtw_safe * 4.0 * volume(0, 0, 0) / op_max(op_max(fabs(dw1), fabs(dw2)), 1.0e-5 * volume(0, 0, 0));
    div = du2 - du1 + dv2 - dv1 + dw2 - dw1;
    dtdivt = c3.dtdiv_safe * 4.0 * (volume(0, 0, 0)) / op_max(volume(0, 0, 0) * 1.0e-05, fabs(div));
    dt_min(0, 0, 0) = op_min(op_min(op_min(dtct, dtut), op_min(dtvt, dtdivt)), dtwt);
  }
};
struct calc_dt_kernel_min {  // :49
  C3_LOOP(calc_dt_kernel_min);
  __device__ void operator()(const D &dt_min, RED<double> &dt_min_val) const {
    *dt_min_val = op_min(*dt_min_val, dt_min(0, 0, 0));
  }
};
struct calc_dt_kernel_get {  // :54
  C3_LOOP(calc_dt_kernel_get);
  __device__ void operator()(const D &cellx, const D &celly, RED<double> &xl_pos, RED<double> &yl_pos, const D &cellz,
                             RED<double> &zl_pos) const {
    *xl_pos = cellx(0, 0, 0);
    *yl_pos = celly(0, 0, 0);
    *zl_pos = cellz(0, 0, 0);
  }
};
struct calc_dt_kernel_print {  // :61
  C3_LOOP(calc_dt_kernel_print);
  __device__ void operator()(const D &xvel0, const D &yvel0, const D &zvel0, const D &density0, const D &energy0,
                             const D &pressure, const D &soundspeed, RED<double, 28> &output) const {
    output[0] = xvel0(0, 0, 0);
    output[1] = yvel0(0, 0, 0);
    output[2] = zvel0(0, 0, 0);
    output[3] = xvel0(1, 0, 0);
    output[4] = yvel0(1, 0, 0);
    output[5] = zvel0(0, 0, 0);
    output[6] = xvel0(1, 1, 0);
    output[7] = yvel0(1, 1, 0);
    output[8] = zvel0(0, 0, 0);
    output[9] = xvel0(0, 1, 0);
    output[10] = yvel0(0, 1, 0);
    output[11] = zvel0(0, 0, 0);
    output[12] = xvel0(0, 0, 1);
    output[13] = yvel0(0, 0, 1);
    output[14] = zvel0(0, 0, 1);
    output[15] = xvel0(1, 0, 1);
    output[16] = yvel0(1, 0, 1);
    output[17] = zvel0(0, 0, 1);
    output[18] = xvel0(1, 1, 1);
    output[19] = yvel0(1, 1, 1);
    output[20] = zvel0(0, 0, 1);
    output[21] = xvel0(0, 1, 1);
    output[22] = yvel0(0, 1, 1);
    output[23] = zvel0(0, 0, 1);
    output[24] = density0(0, 0, 0);
    output[25] = energy0(0, 0, 0);
    output[26] = pressure(0, 0, 0);
    output[27] = soundspeed(0, 0, 0);
  }
};

// ---- PdV_kernel.h ------------------------------------------------------------------
// The face fluxes of the predictor (velocities at the old time twice, half
// the timestep, :7) and the corrector (old and new velocities, :70).
struct PdV_kernel_predict {
  C3_LOOP(PdV_kernel_predict);
  C3_HEAVY;
  __device__ void operator()(const D &xarea, const D &xvel0, const D &yarea, const D &yvel0, D &volume_change,
                             const D &volume, const D &pressure, const D &density0, D &density1,
                             const D &viscosity, const D &energy0, D &energy1, const D &zarea,
                             const D &zvel0) const {
    double recip_volume, energy_change;
    double right_flux, left_flux, top_flux, bottom_flux, back_flux, front_flux, total_flux;
    const double dt = c3.dt;
    left_flux = (xarea(0, 0, 0) * (xvel0(0, 0, 0) + xvel0(0, 1, 0) + xvel0(0, 0, 1) + xvel0(0, 1, 1) +
                                   xvel0(0, 0, 0) + xvel0(0, 1, 0) + xvel0(0, 0, 1) + xvel0(0, 1, 1))) *
                0.125 * dt * 0.5;
    right_flux = (xarea(1, 0, 0) * (xvel0(1, 0, 0) + xvel0(1, 1, 0) + xvel0(1, 0, 1) + xvel0(1, 1, 1) +
                                    xvel0(1, 0, 0) + xvel0(1, 1, 0) + xvel0(1, 0, 1) + xvel0(1, 1, 1))) *
                 0.125 * dt * 0.5;
    bottom_flux = (yarea(0, 0, 0) * (yvel0(0, 0, 0) + yvel0(1, 0, 0) + yvel0(0, 0, 1) + yvel0(1, 0, 1) +
                                     yvel0(0, 0, 0) + yvel0(1, 0, 0) + yvel0(0, 0, 1) + yvel0(1, 0, 1))) *
                  0.125 * dt * 0.5;
    top_flux = (yarea(0, 1, 0) * (yvel0(0, 1, 0) + yvel0(1, 1, 0) + yvel0(0, 1, 1) + yvel0(1, 1, 1) +
                                  yvel0(0, 1, 0) + yvel0(1, 1, 0) + yvel0(0, 1, 1) + yvel0(1, 1, 1))) *
               0.125 * dt * 0.5;
    back_flux = (zarea(0, 0, 0) * (zvel0(0, 0, 0) + zvel0(1, 0, 0) + zvel0(0, 1, 0) + zvel0(1, 1, 0) +
                                   zvel0(0, 0, 0) + zvel0(1, 0, 0) + zvel0(0, 1, 0) + zvel0(1, 1, 0))) *
                0.125 * dt * 0.5;
    front_flux = (zarea(0, 0, 1) * (zvel0(0, 0, 1) + zvel0(1, 0, 1) + zvel0(0, 1, 1) + zvel0(1, 1, 1) +
                                    zvel0(0, 0, 1) + zvel0(1, 0, 1) + zvel0(0, 1, 1) + zvel0(1, 1, 1))) *
                 0.125 * dt * 0.5;
    total_flux = right_flux - left_flux + top_flux - bottom_flux + front_flux - back_flux;
    volume_change(0, 0, 0) = (volume(0, 0, 0)) / (volume(0, 0, 0) + total_flux);
    recip_volume = 1.0 / volume(0, 0, 0);
    energy_change =
        (pressure(0, 0, 0) / density0(0, 0, 0) + qdiv(viscosity(0, 0, 0), density0(0, 0, 0))) * total_flux * recip_volume;
    energy1(0, 0, 0) = energy0(0, 0, 0) - energy_change;
    density1(0, 0, 0) = density0(0, 0, 0) * volume_change(0, 0, 0);
  }
};
struct PdV_kernel_nopredict {
  C3_LOOP(PdV_kernel_nopredict);
  C3_HEAVY;
  __device__ void operator()(const D &xarea, const D &xvel0, const D &xvel1, const D &yarea, const D &yvel0,
                             const D &yvel1, D &volume_change, const D &volume, const D &pressure,
                             const D &density0, D &density1, const D &viscosity, const D &energy0, D &energy1,
                             const D &zarea, const D &zvel0, const D &zvel1) const {
    double recip_volume, energy_change;
    double right_flux, left_flux, top_flux, bottom_flux, back_flux, front_flux, total_flux;
    const double dt = c3.dt;
    left_flux = (xarea(0, 0, 0) * (xvel0(0, 0, 0) + xvel0(0, 1, 0) + xvel0(0, 0, 1) + xvel0(0, 1, 1) +
                                   xvel1(0, 0, 0) + xvel1(0, 1, 0) + xvel1(0, 0, 1) + xvel1(0, 1, 1))) *
                0.125 * dt;
    right_flux = (xarea(1, 0, 0) * (xvel0(1, 0, 0) + xvel0(1, 1, 0) + xvel0(1, 0, 1) + xvel0(1, 1, 1) +
                                    xvel1(1, 0, 0) + xvel1(1, 1, 0) + xvel1(1, 0, 1) + xvel1(1, 1, 1))) *
                 0.125 * dt;
    bottom_flux = (yarea(0, 0, 0) * (yvel0(0, 0, 0) + yvel0(1, 0, 0) + yvel0(0, 0, 1) + yvel0(1, 0, 1) +
                                     yvel1(0, 0, 0) + yvel1(1, 0, 0) + yvel1(0, 0, 1) + yvel1(1, 0, 1))) *
                  0.125 * dt;
    top_flux = (yarea(0, 1, 0) * (yvel0(0, 1, 0) + yvel0(1, 1, 0) + yvel0(0, 1, 1) + yvel0(1, 1, 1) +
                                  yvel1(0, 1, 0) + yvel1(1, 1, 0) + yvel1(0, 1, 1) + yvel1(1, 1, 1))) *
               0.125 * dt;
    back_flux = (zarea(0, 0, 0) * (zvel0(0, 0, 0) + zvel0(1, 0, 0) + zvel0(0, 1, 0) + zvel0(1, 1, 0) +
                                   zvel1(0, 0, 0) + zvel1(1, 0, 0) + zvel1(0, 1, 0) + zvel1(1, 1, 0))) *
                0.125 * dt;
    front_flux = (zarea(0, 0, 1) * (zvel0(0, 0, 1) + zvel0(1, 0, 1) + zvel0(0, 1, 1) + zvel0(1, 1, 1) +
                                    zvel1(0, 0, 1) + zvel1(1, 0, 1) + zvel1(0, 1, 1) + zvel1(1, 1, 1))) *
                 0.125 * dt;
    total_flux = right_flux - left_flux + top_flux - bottom_flux + front_flux - back_flux;
    volume_change(0, 0, 0) = (volume(0, 0, 0)) / (volume(0, 0, 0) + total_flux);
    recip_volume = 1.0 / volume(0, 0, 0);
    energy_change =
        (pressure(0, 0, 0) / density0(0, 0, 0) + qdiv(viscosity(0, 0, 0), density0(0, 0, 0))) * total_flux * recip_volume;
    energy1(0, 0, 0) = energy0(0, 0, 0) - energy_change;
    density1(0, 0, 0) = density0(0, 0, 0) * volume_change(0, 0, 0);
  }
};

// ---- revert_kernel.h:7 ----------------------------------------------------------------
struct revert_kernel {
  C3_LOOP(revert_kernel);
  __device__ void operator()(const D &density0, D &density1, const D &energy0, D &energy1) const {
    density1(0, 0, 0) = density0(0, 0, 0);
    energy1(0, 0, 0) = energy0(0, 0, 0);
  }
};

// ---- accelerate_kernel.h:7 --------------------------------------------------------------
struct accelerate_kernel {
  C3_LOOP(accelerate_kernel);
  C3_HEAVY;
  __device__ void operator()(const D &density0, const D &volume, D &stepbymass, const D &xvel0, D &xvel1,
                             const D &xarea, const D &pressure, const D &yvel0, D &yvel1, const D &yarea,
                             const D &viscosity, const D &zvel0, D &zvel1, const D &zarea) const {
    double nodal_mass = 0.0;
    nodal_mass = (density0(-1, -1, 0) * volume(-1, -1, 0) + density0(0, -1, 0) * volume(0, -1, 0) +
                  density0(0, 0, 0) * volume(0, 0, 0) + density0(-1, 0, 0) * volume(-1, 0, 0) +
                  density0(-1, -1, -1) * volume(-1, -1, -1) + density0(0, -1, -1) * volume(0, -1, -1) +
                  density0(0, 0, -1) * volume(0, 0, -1) + density0(-1, 0, -1) * volume(-1, 0, -1)) *
                 0.125;
    stepbymass(0, 0, 0) = 0.25 * c3.dt / nodal_mass;
    xvel1(0, 0, 0) = xvel0(0, 0, 0) - stepbymass(0, 0, 0) *
                                          (xarea(0, 0, 0) * (pressure(0, 0, 0) - pressure(-1, 0, 0)) +
                                           xarea(0, -1, 0) * (pressure(0, -1, 0) - pressure(-1, -1, 0)) +
                                           xarea(0, 0, -1) * (pressure(0, 0, -1) - pressure(-1, 0, -1)) +
                                           xarea(0, -1, -1) * (pressure(0, -1, -1) - pressure(-1, -1, -1)));
    yvel1(0, 0, 0) = yvel0(0, 0, 0) - stepbymass(0, 0, 0) *
                                          (yarea(0, 0, 0) * (pressure(0, 0, 0) - pressure(0, -1, 0)) +
                                           yarea(-1, 0, 0) * (pressure(-1, 0, 0) - pressure(-1, -1, 0)) +
                                           yarea(0, 0, -1) * (pressure(0, 0, -1) - pressure(0, -1, -1)) +
                                           yarea(-1, 0, -1) * (pressure(-1, 0, -1) - pressure(-1, -1, -1)));
    zvel1(0, 0, 0) = zvel0(0, 0, 0) - stepbymass(0, 0, 0) *
                                          (zarea(0, 0, 0) * (pressure(0, 0, 0) - pressure(0, 0, -1)) +
                                           zarea(0, -1, 0) * (pressure(0, -1, 0) - pressure(0, -1, -1)) +
                                           zarea(-1, 0, 0) * (pressure(-1, 0, 0) - pressure(-1, 0, -1)) +
                                           zarea(-1, -1, 0) * (pressure(-1, -1, 0) - pressure(-1, -1, -1)));
    xvel1(0, 0, 0) = xvel1(0, 0, 0) - stepbymass(0, 0, 0) *
                                          (xarea(0, 0, 0) * (viscosity(0, 0, 0) - viscosity(-1, 0, 0)) +
                                           xarea(0, -1, 0) * (viscosity(0, -1, 0) - viscosity(-1, -1, 0)) +
                                           xarea(0, 0, -1) * (viscosity(0, 0, -1) - viscosity(-1, 0, -1)) +
                                           xarea(0, -1, -1) * (viscosity(0, -1, -1) - viscosity(-1, -1, -1)));
    yvel1(0, 0, 0) = yvel1(0, 0, 0) - stepbymass(0, 0, 0) *
                                          (yarea(0, 0, 0) * (viscosity(0, 0, 0) - viscosity(0, -1, 0)) +
                                           yarea(-1, 0, 0) * (viscosity(-1, 0, 0) - viscosity(-1, -1, 0)) +
                                           yarea(0, 0, -1) * (viscosity(0, 0, -1) - viscosity(0, -1, -1)) +
                                           yarea(-1, 0, -1) * (viscosity(-1, 0, -1) - viscosity(-1, -1, -1)));
    zvel1(0, 0, 0) = zvel1(0, 0, 0) - stepbymass(0, 0, 0) *
                                          (zarea(0, 0, 0) * (viscosity(0, 0, 0) - viscosity(0, 0, -1)) +
                                           zarea(0, -1, 0) * (viscosity(0, -1, 0) - viscosity(0, -1, -1)) +
                                           zarea(-1, 0, 0) * (viscosity(-1, 0, 0) - viscosity(-1, 0, -1)) +
                                           zarea(-1, -1, 0) * (viscosity(-1, -1, 0) - viscosity(-1, -1, -1)));
  }
};

// ---- flux_calc_kernel.h -----------------------------------------------------------------
struct flux_calc_kernelx {  // :7
  C3_LOOP(flux_calc_kernelx);
  __device__ void operator()(D &vol_flux_x, const D &xarea, const D &xvel0, const D &xvel1) const {
    vol_flux_x(0, 0, 0) = 0.125 * c3.dt * (xarea(0, 0, 0)) *
                          (xvel0(0, 0, 0) + xvel0(0, 1, 0) + xvel0(0, 0, 1) + xvel0(0, 1, 1) + xvel1(0, 0, 0) +
                           xvel1(0, 1, 0) + xvel1(0, 0, 1) + xvel1(0, 1, 1));
  }
};
struct flux_calc_kernely {  // :14
  C3_LOOP(flux_calc_kernely);
  __device__ void operator()(D &vol_flux_y, const D &yarea, const D &yvel0, const D &yvel1) const {
    vol_flux_y(0, 0, 0) = 0.125 * c3.dt * (yarea(0, 0, 0)) *
                          (yvel0(0, 0, 0) + yvel0(1, 0, 0) + yvel0(0, 0, 1) + yvel0(1, 0, 1) + yvel1(0, 0, 0) +
                           yvel1(1, 0, 0) + yvel1(0, 0, 1) + yvel1(1, 0, 1));
  }
};
// The reference reads zvel0(1,0,0) twice and zvel0(0,1,0) not at all; kept.
struct flux_calc_kernelz {  // :21
  C3_LOOP(flux_calc_kernelz);
  __device__ void operator()(D &vol_flux_z, const D &zarea, const D &zvel0, const D &zvel1) const {
    vol_flux_z(0, 0, 0) = 0.125 * c3.dt * (zarea(0, 0, 0)) *
                          (zvel0(0, 0, 0) + zvel0(1, 0, 0) + zvel0(1, 0, 0) + zvel0(1, 1, 0) + zvel1(0, 0, 0) +
                           zvel1(1, 0, 0) + zvel1(0, 1, 0) + zvel1(1, 1, 0));
  }
};

// ---- advec_cell_kernel.h ------------------------------------------------------------------
struct advec_cell_kernel1_xdir {  // :7
  C3_LOOP(advec_cell_kernel1_xdir);
  __device__ void operator()(D &pre_vol, D &post_vol, const D &volume, const D &vol_flux_x, const D &vol_flux_y,
                             const D &vol_flux_z) const {
    pre_vol(0, 0, 0) = volume(0, 0, 0) + (vol_flux_x(1, 0, 0) - vol_flux_x(0, 0, 0) + vol_flux_y(0, 1, 0) -
                                          vol_flux_y(0, 0, 0) + vol_flux_z(0, 0, 1) - vol_flux_z(0, 0, 0));
    post_vol(0, 0, 0) = pre_vol(0, 0, 0) - (vol_flux_x(1, 0, 0) - vol_flux_x(0, 0, 0));
  }
};
struct advec_cell_kernel2_xdir {  // :18
  C3_LOOP(advec_cell_kernel2_xdir);
  __device__ void operator()(D &pre_vol, D &post_vol, const D &volume, const D &vol_flux_x) const {
    pre_vol(0, 0, 0) = volume(0, 0, 0) + vol_flux_x(1, 0, 0) - vol_flux_x(0, 0, 0);
    post_vol(0, 0, 0) = volume(0, 0, 0);
  }
};
struct advec_cell_kernel1_ydir {  // :105
  C3_LOOP(advec_cell_kernel1_ydir);
  __device__ void operator()(D &pre_vol, D &post_vol, const D &volume, const D &vol_flux_z,
                             const D &vol_flux_y) const {
    pre_vol(0, 0, 0) = volume(0, 0, 0) + vol_flux_y(0, 1, 0) - vol_flux_y(0, 0, 0) + vol_flux_z(0, 0, 1) -
                       vol_flux_z(0, 0, 0);
    post_vol(0, 0, 0) = pre_vol(0, 0, 0) - (vol_flux_y(0, 1, 0) - vol_flux_y(0, 0, 0));
  }
};
struct advec_cell_kernel2_ydir {  // :113
  C3_LOOP(advec_cell_kernel2_ydir);
  __device__ void operator()(D &pre_vol, D &post_vol, const D &volume, const D &vol_flux_y,
                             const D &vol_flux_x) const {
    pre_vol(0, 0, 0) = volume(0, 0, 0) + vol_flux_y(0, 1, 0) - vol_flux_y(0, 0, 0) + vol_flux_x(1, 0, 0) -
                       vol_flux_x(0, 0, 0);
    post_vol(0, 0, 0) = pre_vol(0, 0, 0) - (vol_flux_y(0, 1, 0) - vol_flux_y(0, 0, 0));
  }
};
struct advec_cell_kernel1_zdir {  // :201
  C3_LOOP(advec_cell_kernel1_zdir);
  __device__ void operator()(D &pre_vol, D &post_vol, const D &volume, const D &vol_flux_x, const D &vol_flux_y,
                             const D &vol_flux_z) const {
    pre_vol(0, 0, 0) = volume(0, 0, 0) + (vol_flux_x(1, 0, 0) - vol_flux_x(0, 0, 0) + vol_flux_y(0, 1, 0) -
                                          vol_flux_y(0, 0, 0) + vol_flux_z(0, 0, 1) - vol_flux_z(0, 0, 0));
    post_vol(0, 0, 0) = pre_vol(0, 0, 0) - (vol_flux_z(0, 0, 1) - vol_flux_z(0, 0, 0));
  }
};
struct advec_cell_kernel2_zdir {  // :212
  C3_LOOP(advec_cell_kernel2_zdir);
  __device__ void operator()(D &pre_vol, D &post_vol, const D &volume, const D &vol_flux_z) const {
    pre_vol(0, 0, 0) = volume(0, 0, 0) + vol_flux_z(0, 0, 1) - vol_flux_z(0, 0, 0);
    post_vol(0, 0, 0) = volume(0, 0, 0);
  }
};

// Van Leer limited mass and energy fluxes through the low face of the cell
// along AX (advec_cell_kernel3_{x,y,z}dir, :24, :121, :218). `cmax` is the
// reference's x_max / y_max / z_max.
template <int AX>
__device__ __forceinline__ void advec_cell_flux(const D &vol_flux, const D &pre_vol, const I &cc, const D &vertexd,
                                                const D &density1, const D &energy1, D &mass_flux, D &ener_flux,
                                                int cmax) {
  double sigmat, sigmav, sigmam, sigma3, sigma4;
  double diffuw, diffdw, limiter;
  double one_by_six = 1.0 / 6.0;
  int upwind, donor, downwind, dif;
  if (vol_flux(0, 0, 0) > 0.0) {
    upwind = -2;
    donor = -1;
    downwind = 0;
    dif = donor;
  } else if (ax<AX>(cc, 1) < cmax + 2 - 2) {
    upwind = 1;
    donor = 0;
    downwind = -1;
    dif = upwind;
  } else {
    upwind = 0;
    donor = 0;
    downwind = -1;
    dif = upwind;
  }
  sigmat = qdiv(fabs(vol_flux(0, 0, 0)), ax<AX>(pre_vol, donor));
  sigma3 = (1.0 + sigmat) * qratio(vertexd(0, 0, 0), ax<AX>(vertexd, dif));
  sigma4 = 2.0 - sigmat;
  sigmav = sigmat;
  diffuw = ax<AX>(density1, donor) - ax<AX>(density1, upwind);
  diffdw = ax<AX>(density1, downwind) - ax<AX>(density1, donor);
  if ((diffuw * diffdw) > 0.0)
    limiter = (1.0 - sigmav) * op_sign(1.0, diffdw) *
              op_min(op_min(fabs(diffuw), fabs(diffdw)), one_by_six * (sigma3 * fabs(diffuw) + sigma4 * fabs(diffdw)));
  else
    limiter = 0.0;
  mass_flux(0, 0, 0) = (vol_flux(0, 0, 0)) * (ax<AX>(density1, donor) + limiter);
  sigmam = qdiv(fabs(mass_flux(0, 0, 0)), ax<AX>(density1, donor) * ax<AX>(pre_vol, donor));
  diffuw = ax<AX>(energy1, donor) - ax<AX>(energy1, upwind);
  diffdw = ax<AX>(energy1, downwind) - ax<AX>(energy1, donor);
  if ((diffuw * diffdw) > 0.0)
    limiter = (1.0 - sigmam) * op_sign(1.0, diffdw) *
              op_min(op_min(fabs(diffuw), fabs(diffdw)), one_by_six * (sigma3 * fabs(diffuw) + sigma4 * fabs(diffdw)));
  else
    limiter = 0.0;
  ener_flux(0, 0, 0) = mass_flux(0, 0, 0) * (ax<AX>(energy1, donor) + limiter);
}
struct advec_cell_kernel3_xdir {
  C3_LOOP(advec_cell_kernel3_xdir);
  C3_HEAVY;
  __device__ void operator()(const D &vol_flux_x, const D &pre_vol, const I &xx, const D &vertexdx,
                             const D &density1, const D &energy1, D &mass_flux_x, D &ener_flux) const {
    advec_cell_flux<0>(vol_flux_x, pre_vol, xx, vertexdx, density1, energy1, mass_flux_x, ener_flux, c3.field.x_max);
  }
};
struct advec_cell_kernel3_ydir {
  C3_LOOP(advec_cell_kernel3_ydir);
  C3_HEAVY;
  __device__ void operator()(const D &vol_flux_y, const D &pre_vol, const I &yy, const D &vertexdy,
                             const D &density1, const D &energy1, D &mass_flux_y, D &ener_flux) const {
    advec_cell_flux<1>(vol_flux_y, pre_vol, yy, vertexdy, density1, energy1, mass_flux_y, ener_flux, c3.field.y_max);
  }
};
struct advec_cell_kernel3_zdir {
  C3_LOOP(advec_cell_kernel3_zdir);
  C3_HEAVY;
  __device__ void operator()(const D &vol_flux_z, const D &pre_vol, const I &zz, const D &vertexdz,
                             const D &density1, const D &energy1, D &mass_flux_z, D &ener_flux) const {
    advec_cell_flux<2>(vol_flux_z, pre_vol, zz, vertexdz, density1, energy1, mass_flux_z, ener_flux, c3.field.z_max);
  }
};

// Density and energy after the remap along AX (advec_cell_kernel4_*, :87,
// :185, :282).
template <int AX>
__device__ __forceinline__ void advec_cell_update(D &density1, D &energy1, const D &mass_flux, const D &vol_flux,
                                                  const D &pre_vol, D &pre_mass, D &post_mass, D &advec_vol,
                                                  D &post_ener, const D &ener_flux) {
  pre_mass(0, 0, 0) = density1(0, 0, 0) * pre_vol(0, 0, 0);
  post_mass(0, 0, 0) = pre_mass(0, 0, 0) + mass_flux(0, 0, 0) - ax<AX>(mass_flux, 1);
  post_ener(0, 0, 0) =
      (energy1(0, 0, 0) * pre_mass(0, 0, 0) + ener_flux(0, 0, 0) - ax<AX>(ener_flux, 1)) / post_mass(0, 0, 0);
  advec_vol(0, 0, 0) = pre_vol(0, 0, 0) + vol_flux(0, 0, 0) - ax<AX>(vol_flux, 1);
  density1(0, 0, 0) = post_mass(0, 0, 0) / advec_vol(0, 0, 0);
  energy1(0, 0, 0) = post_ener(0, 0, 0);
}
#define ADVEC_CELL4(NAME, AX)                                                                                     \
  struct NAME {                                                                                                   \
    C3_LOOP(NAME);                                                                                                \
    __device__ void operator()(D &density1, D &energy1, const D &mass_flux, const D &vol_flux, const D &pre_vol, \
                               const D &post_vol, D &pre_mass, D &post_mass, D &advec_vol, D &post_ener,          \
                               const D &ener_flux) const {                                                        \
      advec_cell_update<AX>(density1, energy1, mass_flux, vol_flux, pre_vol, pre_mass, post_mass, advec_vol,     \
                            post_ener, ener_flux);                                                                \
    }                                                                                                             \
  };
ADVEC_CELL4(advec_cell_kernel4_xdir, 0)
ADVEC_CELL4(advec_cell_kernel4_ydir, 1)
ADVEC_CELL4(advec_cell_kernel4_zdir, 2)

// ---- advec_mom_kernel.h -------------------------------------------------------------------
struct advec_mom_kernel_x1 {  // :7
  C3_LOOP(advec_mom_kernel_x1);
  __device__ void operator()(D &pre_vol, D &post_vol, const D &volume, const D &vol_flux_x, const D &vol_flux_y,
                             const D &vol_flux_z) const {
    post_vol(0, 0, 0) = volume(0, 0, 0) + vol_flux_y(0, 1, 0) - vol_flux_y(0, 0, 0) + vol_flux_z(0, 0, 1) -
                        vol_flux_z(0, 0, 0);
    pre_vol(0, 0, 0) = post_vol(0, 0, 0) + vol_flux_x(1, 0, 0) - vol_flux_x(0, 0, 0);
  }
};
struct advec_mom_kernel_z1 {  // :16
  C3_LOOP(advec_mom_kernel_z1);
  __device__ void operator()(D &pre_vol, D &post_vol, const D &volume, const D &vol_flux_x, const D &vol_flux_y,
                             const D &vol_flux_z) const {
    post_vol(0, 0, 0) = volume(0, 0, 0) + vol_flux_x(1, 0, 0) - vol_flux_x(0, 0, 0) + vol_flux_y(0, 1, 0) -
                        vol_flux_y(0, 0, 0);
    pre_vol(0, 0, 0) = post_vol(0, 0, 0) + vol_flux_z(0, 0, 1) - vol_flux_z(0, 0, 0);
  }
};
struct advec_mom_kernel_x2 {  // :25
  C3_LOOP(advec_mom_kernel_x2);
  __device__ void operator()(D &pre_vol, D &post_vol, const D &volume, const D &vol_flux_y,
                             const D &vol_flux_z) const {
    post_vol(0, 0, 0) = volume(0, 0, 0) + vol_flux_z(0, 0, 1) - vol_flux_z(0, 0, 0);
    pre_vol(0, 0, 0) = post_vol(0, 0, 0) + vol_flux_y(0, 1, 0) - vol_flux_y(0, 0, 0);
  }
};
struct advec_mom_kernel_y2 {  // :33
  C3_LOOP(advec_mom_kernel_y2);
  __device__ void operator()(D &pre_vol, D &post_vol, const D &volume, const D &vol_flux_x,
                             const D &vol_flux_y) const {
    post_vol(0, 0, 0) = volume(0, 0, 0) + vol_flux_x(1, 0, 0) - vol_flux_x(0, 0, 0);
    pre_vol(0, 0, 0) = post_vol(0, 0, 0) + vol_flux_y(0, 1, 0) - vol_flux_y(0, 0, 0);
  }
};
struct advec_mom_kernel_x3 {  // :41
  C3_LOOP(advec_mom_kernel_x3);
  __device__ void operator()(D &pre_vol, D &post_vol, const D &volume, const D &vol_flux_x) const {
    post_vol(0, 0, 0) = volume(0, 0, 0);
    pre_vol(0, 0, 0) = post_vol(0, 0, 0) + vol_flux_x(1, 0, 0) - vol_flux_x(0, 0, 0);
  }
};
struct advec_mom_kernel_z3 {  // :48
  C3_LOOP(advec_mom_kernel_z3);
  __device__ void operator()(D &pre_vol, D &post_vol, const D &volume, const D &vol_flux_z) const {
    post_vol(0, 0, 0) = volume(0, 0, 0);
    pre_vol(0, 0, 0) = post_vol(0, 0, 0) + vol_flux_z(0, 0, 1) - vol_flux_z(0, 0, 0);
  }
};
struct advec_mom_kernel_mass_flux_x {  // :55
  C3_LOOP(advec_mom_kernel_mass_flux_x);
  __device__ void operator()(D &node_flux, const D &mass_flux_x) const {
    node_flux(0, 0, 0) = 0.125 * (mass_flux_x(0, -1, 0) + mass_flux_x(0, 0, 0) + mass_flux_x(1, -1, 0) +
                                  mass_flux_x(1, 0, 0) + mass_flux_x(0, -1, -1) + mass_flux_x(0, 0, -1) +
                                  mass_flux_x(1, -1, -1) + mass_flux_x(1, 0, -1));
  }
};
struct advec_mom_kernel_mass_flux_y {  // :63
  C3_LOOP(advec_mom_kernel_mass_flux_y);
  __device__ void operator()(D &node_flux, const D &mass_flux_y) const {
    node_flux(0, 0, 0) = 0.125 * (mass_flux_y(-1, 0, 0) + mass_flux_y(0, 0, 0) + mass_flux_y(-1, 1, 0) +
                                  mass_flux_y(0, 1, 0) + mass_flux_y(-1, 0, -1) + mass_flux_y(0, 0, -1) +
                                  mass_flux_y(-1, 1, -1) + mass_flux_y(0, 1, -1));
  }
};
struct advec_mom_kernel_mass_flux_z {  // :71
  C3_LOOP(advec_mom_kernel_mass_flux_z);
  __device__ void operator()(D &node_flux, const D &mass_flux_z) const {
    node_flux(0, 0, 0) = 0.125 * (mass_flux_z(-1, 0, 0) + mass_flux_z(0, 0, 0) + mass_flux_z(-1, 0, 1) +
                                  mass_flux_z(0, 0, 1) + mass_flux_z(-1, -1, 0) + mass_flux_z(0, -1, 0) +
                                  mass_flux_z(-1, -1, 1) + mass_flux_z(0, -1, 1));
  }
};
// Nodal masses after and before the sweep along AX (:79, :93, :107): the
// same post-remap mass in every direction, the pre mass adds back the
// nodal flux through the low face of AX.
template <int AX>
__device__ __forceinline__ void advec_mom_post_pre(D &node_mass_post, const D &post_vol, const D &density1,
                                                   D &node_mass_pre, const D &node_flux) {
  node_mass_post(0, 0, 0) =
      0.125 * (density1(0, -1, 0) * post_vol(0, -1, 0) + density1(0, 0, 0) * post_vol(0, 0, 0) +
               density1(-1, -1, 0) * post_vol(-1, -1, 0) + density1(-1, 0, 0) * post_vol(-1, 0, 0) +
               density1(0, -1, -1) * post_vol(0, -1, -1) + density1(0, 0, -1) * post_vol(0, 0, -1) +
               density1(-1, -1, -1) * post_vol(-1, -1, -1) + density1(-1, 0, -1) * post_vol(-1, 0, -1));
  node_mass_pre(0, 0, 0) = node_mass_post(0, 0, 0) - ax<AX>(node_flux, -1) + node_flux(0, 0, 0);
}
#define ADVEC_MOM_PP(NAME, AX)                                                                                   \
  struct NAME {                                                                                                  \
    C3_LOOP(NAME);                                                                                               \
    __device__ void operator()(D &node_mass_post, const D &post_vol, const D &density1, D &node_mass_pre,       \
                               const D &node_flux) const {                                                       \
      advec_mom_post_pre<AX>(node_mass_post, post_vol, density1, node_mass_pre, node_flux);                     \
    }                                                                                                            \
  };
ADVEC_MOM_PP(advec_mom_kernel_post_pre_advec_x, 0)
ADVEC_MOM_PP(advec_mom_kernel_post_pre_advec_y, 1)
ADVEC_MOM_PP(advec_mom_kernel_post_pre_advec_z, 2)

// Limited momentum flux through the node face along AX
// (advec_mom_kernel1_{x,y,z}_nonvector, :121, :154, :186).
template <int AX>
__device__ __forceinline__ void advec_mom_flux(const D &node_flux, const D &node_mass_pre, D &mom_flux,
                                               const D &celld, const D &vel1) {
  double sigma, wind, width;
  double vdiffuw, vdiffdw, auw, adw, limiter;
  int upwind, donor, downwind, dif;
  double advec_vel_temp;
  if ((node_flux(0, 0, 0)) < 0.0) {
    upwind = 2;
    donor = 1;
    downwind = 0;
    dif = donor;
  } else {
    upwind = -1;
    donor = 0;
    downwind = 1;
    dif = upwind;
  }
  sigma = qdiv(fabs(node_flux(0, 0, 0)), ax<AX>(node_mass_pre, donor));
  width = celld(0, 0, 0);
  vdiffuw = ax<AX>(vel1, donor) - ax<AX>(vel1, upwind);
  vdiffdw = ax<AX>(vel1, downwind) - ax<AX>(vel1, donor);
  limiter = 0.0;
  if (vdiffuw * vdiffdw > 0.0) {
    auw = fabs(vdiffuw);
    adw = fabs(vdiffdw);
    wind = 1.0;
    if (vdiffdw <= 0.0) wind = -1.0;
    limiter = wind * op_min(width * ((2.0 - sigma) * adw / width + (1.0 + sigma) * auw / ax<AX>(celld, dif)) / 6.0,
                            op_min(auw, adw));
  }
  advec_vel_temp = ax<AX>(vel1, donor) + (1.0 - sigma) * limiter;
  mom_flux(0, 0, 0) = advec_vel_temp * node_flux(0, 0, 0);
}
#define ADVEC_MOM1(NAME, AX)                                                                                     \
  struct NAME {                                                                                                  \
    C3_LOOP(NAME);                                                                                               \
    __device__ void operator()(const D &node_flux, const D &node_mass_pre, D &mom_flux, const D &celld,         \
                               const D &vel1) const {                                                            \
      advec_mom_flux<AX>(node_flux, node_mass_pre, mom_flux, celld, vel1);                                      \
    }                                                                                                            \
  };
ADVEC_MOM1(advec_mom_kernel1_x_nonvector, 0)
ADVEC_MOM1(advec_mom_kernel1_y_nonvector, 1)
ADVEC_MOM1(advec_mom_kernel1_z_nonvector, 2)

// Velocity after the momentum remap along AX (advec_mom_kernel2_*, :219).
template <int AX>
struct advec_mom_vel {
  __device__ void operator()(D &vel1, const D &node_mass_post, const D &node_mass_pre, const D &mom_flux) const {
    vel1(0, 0, 0) = qdiv(vel1(0, 0, 0) * node_mass_pre(0, 0, 0) + ax<AX>(mom_flux, -1) - mom_flux(0, 0, 0),
                         node_mass_post(0, 0, 0));
  }
};
struct advec_mom_kernel2_x : advec_mom_vel<0> { C3_LOOP(advec_mom_kernel2_x); };
struct advec_mom_kernel2_y : advec_mom_vel<1> { C3_LOOP(advec_mom_kernel2_y); };
struct advec_mom_kernel2_z : advec_mom_vel<2> { C3_LOOP(advec_mom_kernel2_z); };

// ---- reset_field_kernel.h --------------------------------------------------------------
struct reset_field_kernel1 {  // :7
  C3_LOOP(reset_field_kernel1);
  __device__ void operator()(D &density0, const D &density1, D &energy0, const D &energy1) const {
    density0(0, 0, 0) = density1(0, 0, 0);
    energy0(0, 0, 0) = energy1(0, 0, 0);
  }
};
struct reset_field_kernel2 {  // :13
  C3_LOOP(reset_field_kernel2);
  __device__ void operator()(D &xvel0, const D &xvel1, D &yvel0, const D &yvel1, D &zvel0, const D &zvel1) const {
    xvel0(0, 0, 0) = xvel1(0, 0, 0);
    yvel0(0, 0, 0) = yvel1(0, 0, 0);
    zvel0(0, 0, 0) = zvel1(0, 0, 0);
  }
};

// ---- field_summary_kernel.h:4 -------------------------------------------------------------
struct field_summary_kernel {
  C3_LOOP(field_summary_kernel);
  C3_HEAVY;
  __device__ void operator()(const D &volume, const D &density0, const D &energy0, const D &pressure, const D &xvel0,
                             const D &yvel0, const D &zvel0, RED<double> &vol, RED<double> &mass, RED<double> &ie,
                             RED<double> &ke, RED<double> &press) const {
    double vsqrd, cell_vol, cell_mass;
    vsqrd = 0.0;
    vsqrd += 0.125 * (xvel0(0, 0, 0) * xvel0(0, 0, 0) + yvel0(0, 0, 0) * yvel0(0, 0, 0) +
                      zvel0(0, 0, 0) * zvel0(0, 0, 0));
    vsqrd += 0.125 * (xvel0(1, 0, 0) * xvel0(1, 0, 0) + yvel0(1, 0, 0) * yvel0(1, 0, 0) +
                      zvel0(1, 0, 0) * zvel0(1, 0, 0));
    vsqrd += 0.125 * (xvel0(0, 1, 0) * xvel0(0, 1, 0) + yvel0(0, 1, 0) * yvel0(0, 1, 0) +
                      zvel0(0, 1, 0) * zvel0(0, 1, 0));
    vsqrd += 0.125 * (xvel0(1, 1, 0) * xvel0(1, 1, 0) + yvel0(1, 1, 0) * yvel0(1, 1, 0) +
                      zvel0(1, 1, 0) * zvel0(1, 1, 0));
    vsqrd += 0.125 * (xvel0(0, 0, 1) * xvel0(0, 0, 1) + yvel0(0, 0, 1) * yvel0(0, 0, 1) +
                      zvel0(0, 0, 1) * zvel0(0, 0, 1));
    vsqrd += 0.125 * (xvel0(1, 0, 1) * xvel0(1, 0, 1) + yvel0(1, 0, 1) * yvel0(1, 0, 1) +
                      zvel0(1, 0, 1) * zvel0(1, 0, 1));
    vsqrd += 0.125 * (xvel0(0, 1, 1) * xvel0(0, 1, 1) + yvel0(0, 1, 1) * yvel0(0, 1, 1) +
                      zvel0(0, 1, 1) * zvel0(0, 1, 1));
    vsqrd += 0.125 * (xvel0(1, 1, 1) * xvel0(1, 1, 1) + yvel0(1, 1, 1) * yvel0(1, 1, 1) +
                      zvel0(1, 1, 1) * zvel0(1, 1, 1));
    cell_vol = volume(0, 0, 0);
    cell_mass = cell_vol * density0(0, 0, 0);
    *vol = *vol + cell_vol;
    *mass = *mass + cell_mass;
    *ie = *ie + cell_mass * energy0(0, 0, 0);
    *ke = *ke + cell_mass * 0.5 * vsqrd;
    *press = *press + cell_vol * pressure(0, 0, 0);
  }
};

// ---- registration ------------------------------------------------------------
#define REG(K) OPSB_REGISTER_LOOP(K);
REG(initialise_chunk_kernel_xx) REG(initialise_chunk_kernel_yy) REG(initialise_chunk_kernel_zz)
REG(initialise_chunk_kernel_x) REG(initialise_chunk_kernel_y) REG(initialise_chunk_kernel_z)
REG(initialise_chunk_kernel_cellx) REG(initialise_chunk_kernel_celly) REG(initialise_chunk_kernel_cellz)
REG(initialise_chunk_kernel_volume) REG(generate_chunk_kernel) REG(ideal_gas_kernel)
REG(update_halo_kernel1_b2) REG(update_halo_kernel1_b1) REG(update_halo_kernel1_t2) REG(update_halo_kernel1_t1)
REG(update_halo_kernel1_l2) REG(update_halo_kernel1_l1) REG(update_halo_kernel1_r2) REG(update_halo_kernel1_r1)
REG(update_halo_kernel1_ba2) REG(update_halo_kernel1_ba1) REG(update_halo_kernel1_fr2) REG(update_halo_kernel1_fr1)
REG(update_halo_kernel2_xvel_plus_4_bot) REG(update_halo_kernel2_xvel_plus_2_bot)
REG(update_halo_kernel2_xvel_plus_4_top) REG(update_halo_kernel2_xvel_plus_2_top)
REG(update_halo_kernel2_xvel_minus_4_left) REG(update_halo_kernel2_xvel_minus_2_left)
REG(update_halo_kernel2_xvel_minus_4_right) REG(update_halo_kernel2_xvel_minus_2_right)
REG(update_halo_kernel2_xvel_plus_4_back) REG(update_halo_kernel2_xvel_plus_2_back)
REG(update_halo_kernel2_xvel_plus_4_front) REG(update_halo_kernel2_xvel_plus_2_front)
REG(update_halo_kernel2_yvel_minus_4_bot) REG(update_halo_kernel2_yvel_minus_2_bot)
REG(update_halo_kernel2_yvel_minus_4_top) REG(update_halo_kernel2_yvel_minus_2_top)
REG(update_halo_kernel2_yvel_plus_4_left) REG(update_halo_kernel2_yvel_plus_2_left)
REG(update_halo_kernel2_yvel_plus_4_right) REG(update_halo_kernel2_yvel_plus_2_right)
REG(update_halo_kernel2_yvel_plus_4_back) REG(update_halo_kernel2_yvel_plus_2_back)
REG(update_halo_kernel2_yvel_plus_4_front) REG(update_halo_kernel2_yvel_plus_2_front)
REG(update_halo_kernel2_zvel_plus_4_bot) REG(update_halo_kernel2_zvel_plus_2_bot)
REG(update_halo_kernel2_zvel_plus_4_top) REG(update_halo_kernel2_zvel_plus_2_top)
REG(update_halo_kernel2_zvel_plus_4_left) REG(update_halo_kernel2_zvel_plus_2_left)
REG(update_halo_kernel2_zvel_plus_4_right) REG(update_halo_kernel2_zvel_plus_2_right)
REG(update_halo_kernel2_zvel_minus_4_back) REG(update_halo_kernel2_zvel_minus_2_back)
REG(update_halo_kernel2_zvel_minus_4_front) REG(update_halo_kernel2_zvel_minus_2_front)
REG(update_halo_kernel3_plus_4_a) REG(update_halo_kernel3_plus_2_a) REG(update_halo_kernel3_plus_4_b)
REG(update_halo_kernel3_plus_2_b) REG(update_halo_kernel3_minus_4_a) REG(update_halo_kernel3_minus_2_a)
REG(update_halo_kernel3_minus_4_b) REG(update_halo_kernel3_minus_2_b) REG(update_halo_kernel3_plus_4_back)
REG(update_halo_kernel3_plus_2_back) REG(update_halo_kernel3_plus_4_front) REG(update_halo_kernel3_plus_2_front)
REG(update_halo_kernel4_minus_4_a) REG(update_halo_kernel4_minus_2_a) REG(update_halo_kernel4_minus_4_b)
REG(update_halo_kernel4_minus_2_b) REG(update_halo_kernel4_plus_4_a) REG(update_halo_kernel4_plus_2_a)
REG(update_halo_kernel4_plus_4_b) REG(update_halo_kernel4_plus_2_b) REG(update_halo_kernel4_plus_4_back)
REG(update_halo_kernel4_plus_2_back) REG(update_halo_kernel4_plus_4_front) REG(update_halo_kernel4_plus_2_front)
REG(update_halo_kernel5_plus_4_a) REG(update_halo_kernel5_plus_2_a) REG(update_halo_kernel5_plus_4_b)
REG(update_halo_kernel5_plus_2_b) REG(update_halo_kernel5_plus_4_left) REG(update_halo_kernel5_plus_2_left)
REG(update_halo_kernel5_plus_4_right) REG(update_halo_kernel5_plus_2_right) REG(update_halo_kernel5_minus_4_back)
REG(update_halo_kernel5_minus_2_back) REG(update_halo_kernel5_minus_4_front) REG(update_halo_kernel5_minus_2_front)
REG(viscosity_kernel) REG(calc_dt_kernel) REG(calc_dt_kernel_min) REG(calc_dt_kernel_get) REG(calc_dt_kernel_print)
REG(PdV_kernel_predict) REG(PdV_kernel_nopredict) REG(revert_kernel) REG(accelerate_kernel)
REG(flux_calc_kernelx) REG(flux_calc_kernely) REG(flux_calc_kernelz)
REG(advec_cell_kernel1_xdir) REG(advec_cell_kernel2_xdir) REG(advec_cell_kernel3_xdir) REG(advec_cell_kernel4_xdir)
REG(advec_cell_kernel1_ydir) REG(advec_cell_kernel2_ydir) REG(advec_cell_kernel3_ydir) REG(advec_cell_kernel4_ydir)
REG(advec_cell_kernel1_zdir) REG(advec_cell_kernel2_zdir) REG(advec_cell_kernel3_zdir) REG(advec_cell_kernel4_zdir)
REG(advec_mom_kernel_x1) REG(advec_mom_kernel_z1) REG(advec_mom_kernel_x2) REG(advec_mom_kernel_y2)
REG(advec_mom_kernel_x3) REG(advec_mom_kernel_z3)
REG(advec_mom_kernel_mass_flux_x) REG(advec_mom_kernel_mass_flux_y) REG(advec_mom_kernel_mass_flux_z)
REG(advec_mom_kernel_post_pre_advec_x) REG(advec_mom_kernel_post_pre_advec_y) REG(advec_mom_kernel_post_pre_advec_z)
REG(advec_mom_kernel1_x_nonvector) REG(advec_mom_kernel1_y_nonvector) REG(advec_mom_kernel1_z_nonvector)
REG(advec_mom_kernel2_x) REG(advec_mom_kernel2_y) REG(advec_mom_kernel2_z)
REG(reset_field_kernel1) REG(reset_field_kernel2) REG(field_summary_kernel)

// Named constants (ops_decl_const in clover_leaf.cpp:150-169).
struct ConstReg {
  ConstReg() {
#define C(name, member) \
  Runtime::register_const("cloverleaf3d/" name, &c3, offsetof(Consts, member), sizeof(Consts::member))
    C("g_small", g_small); C("g_big", g_big); C("dtc_safe", dtc_safe); C("dtu_safe", dtu_safe);
    C("dtv_safe", dtv_safe); C("dtw_safe", dtw_safe); C("dtdiv_safe", dtdiv_safe); C("dt", dt);
    C("field", field); C("grid", grid); C("number_of_states", number_of_states); C("g_sphe", g_sphe);
    C("g_point", g_point); C("g_cube", g_cube); C("states", states);
#undef C
  }
};
static ConstReg const_reg;

}  // namespace clover3d
}  // namespace opsb
